"""Host-side mirror of the reference's call surface over the C-ABI.

``Context`` owns one he_ctx_t.  Its methods carry the names of the Fortran routines they replace
(poten, potenimp, forceimp, steprk, steppc, energy, steprkr, steppcr, varmu, derden) and keep
their argument meaning; module arrays move with ``upload``/``download`` in the reference's
column-major layout.  Errors raise ``HeError`` with the library's message (the reference STOPs).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import FIELDS, HeError, dptr
from .config import MP_U, KTOPS, Workload, potion_table

COMPLEX_DYN = {"psi", "pc", "q", "psiold1", "psiold2", "psiold3", "hpsiold1", "hpsiold2"}
COMPLEX_Q = {"psix", "pcx", "qx", "psixold", "hpsixold"}
MODES = {"dynamics": _lib.HE_MODE_DYNAMICS, "statics": _lib.HE_MODE_STATICS,
         "quantum": _lib.HE_MODE_QUANTUM}


class Context:
    def __init__(self, w: Workload, mode="dynamics", compute_kernels=True, precision="f64"):
        self.L = _lib.load()
        self.w = w
        self.mode = MODES[mode]
        self.precision = {"f64": _lib.HE_PREC_F64, "mixed": _lib.HE_PREC_MIXED}[precision]
        g = _lib.HeGrid(w.nx, w.ny, w.nz, w.xmax, w.ymax, w.zmax, w.npd, w.icon)
        core = {"OT": b"OT ", "OP": b"OP ", "OTC": b"OTC"}[w.core]
        f = _lib.HeFunctional(core, w.h4, w.eps4, w.sigma4, w.cp4, w.cpp4, w.den4c, w.alphas,
                              w.l, w.den0s, w.h2o2m4, w.lsolid, w.C, w.beta, w.den_m)
        h = ctypes.c_void_p()
        st = self.L.he_ctx_create(ctypes.byref(g), ctypes.byref(f), self.mode, self.precision,
                                  ctypes.byref(h))
        self.h = h.value
        if st != 0:
            msg = self.L.he_last_error(self.h).decode() if self.h else "no context"
            self.close()
            raise HeError(st, msg)
        if compute_kernels:
            self._ck(self.L.he_compute_kernels(self.h))
        if self.mode != _lib.HE_MODE_STATICS:
            ab = _lib.HeAbsorber(w.lambdah, w.txmean, w.txsurf, w.tymean, w.tysurf, w.tzmean,
                                 w.tzsurf)
            self._ck(self.L.he_set_absorber(self.h, ctypes.byref(ab)))
        if self.mode == _lib.HE_MODE_DYNAMICS and w.n_imp > 0:
            self.set_impurities(w)
        if self.mode == _lib.HE_MODE_QUANTUM and w.nq_imp > 0:
            self.set_quantum_impurities(w)

    # ---- plumbing -------------------------------------------------------------------------------
    def _ck(self, st):
        if st != 0:
            raise HeError(st, self.L.he_last_error(self.h).decode())
        return st

    def close(self):
        if getattr(self, "h", None):
            self.L.he_ctx_destroy(self.h)
            self.h = None
        for m in getattr(self, "_members", ()):
            m.close()
        self._members = []

    # ---- groups (he_ctx_group): several statics droplets per launch ----------------------------
    def group(self, members):
        """Make this context the leader of itself plus `members` (contexts created alike and set
        up on their own, in the same ring state).  The leader takes the members over: it closes
        them when it closes, and they must not be called directly any more."""
        hs = (ctypes.c_void_p * (1 + len(members)))(self.h, *[m.h for m in members])
        self._ck(self.L.he_ctx_group(hs, 1 + len(members)))
        self._members = list(members)

    @property
    def members(self):
        return self.L.he_group_size(self.h)

    def upload_member(self, m, name, arr):
        dt = np.complex128 if self._is_complex(name) else np.float64
        a = np.asarray(arr, dtype=dt).reshape(self._shape(name), order="F")
        buf = np.ascontiguousarray(a.ravel(order="F"))
        self._ck(self.L.he_upload_member(self.h, m, FIELDS[name], buf.ctypes.data_as(ctypes.c_void_p),
                                         buf.nbytes))

    def download_member(self, m, name):
        dt = np.complex128 if self._is_complex(name) else np.float64
        shape = self._shape(name)
        buf = np.empty(int(np.prod(shape)), dtype=dt)
        self._ck(self.L.he_download_member(self.h, m, FIELDS[name], buf.ctypes.data_as(ctypes.c_void_p),
                                           buf.nbytes))
        return buf.reshape(shape, order="F")

    def member_mu(self, n4, after_rk=False):
        out = np.zeros(self.members)
        self._ck(self.L.he_member_mu(self.h, n4, 1 if after_rk else 0, dptr(out)))
        return out

    def statics_iterations_members(self, niter, deltat, mu4, n4):
        """he_statics_iterations_members: (mu4, mu4err, errpc) arrays over the members."""
        mu = np.ascontiguousarray(np.asarray(mu4, np.float64).copy())
        err, pc = np.zeros(self.members), np.zeros(self.members)
        self._ck(self.L.he_statics_iterations_members(self.h, niter, deltat, n4, dptr(mu), dptr(err),
                                                      dptr(pc)))
        return mu, err, pc

    def qimp_moments_members(self):
        """(members, nq, 4) array of norm, <x>, <y>, <z> per member and impurity."""
        nq = self.w.nq_imp
        out = np.zeros(self.members * nq * 4)
        self._ck(self.L.he_qimp_moments_members(self.h, dptr(out)))
        return out.reshape(self.members, nq, 4)

    def energy_members(self):
        out = (_lib.HeEnergies * self.members)()
        self._ck(self.L.he_energy_members(self.h, out))
        return [{k: getattr(e, k) for k, _ in _lib.HeEnergies._fields_} for e in out]

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def launches(self):
        return int(self.L.he_launch_count(self.h))

    @property
    def device_bytes(self):
        return int(self.L.he_device_bytes(self.h))

    def timing(self, enable=True):
        self._ck(self.L.he_timing(self.h, 1 if enable else 0))

    def timing_report(self):
        """{kernel name: (launches, total ms)} of the launches recorded since timing(True)."""
        buf = (_lib.HeKernelTime * 64)()
        n = ctypes.c_int(0)
        self._ck(self.L.he_timing_report(self.h, buf, 64, ctypes.byref(n)))
        return {buf[i].name.decode(): (int(buf[i].launches), float(buf[i].ms))
                for i in range(min(n.value, 64))}

    def tuned_tiles(self):
        """FFT tile sizes (x, y, z) chosen by the context's autotuner."""
        v = [ctypes.c_int(0) for _ in range(3)]
        self._ck(self.L.he_tuned_tiles(self.h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def set_fft_variant(self, pass_, variant, tile):
        """Override the autotuner for one pass family: pass_ 'x' (every mode), 'x0'..'x5' (one
        x mode), 'y', 'z', 'xy' (fused plane passes of the classical field evaluation) or 'yz'
        (64^3: convolutions with fused y-z passes over a thread-block cluster);
        variant 0/1 (x: one-shot / pipelined, y: register only, z: shared memory / register,
        xy: off / on); tile 8 or 16."""
        code = {"x": 0, "y": 1, "z": 2, "xy": 9, "yz": 10}.get(pass_)
        if code is None:
            code = 3 + int(pass_[1:])
        self._ck(self.L.he_set_fft_variant(self.h, code, variant, tile))

    def state_fingerprint(self):
        """Hash of the buffer relabelling, ring indices and lazy flags (he_state_fingerprint)."""
        v = ctypes.c_ulonglong(0)
        self._ck(self.L.he_state_fingerprint(self.h, ctypes.byref(v)))
        return int(v.value)

    def autotune_report(self):
        """The FFT autotuner's trial times, one line per variant, and the x-pass variant chosen."""
        buf = ctypes.create_string_buffer(4096)
        self._ck(self.L.he_autotune_report(self.h, buf, len(buf)))
        return buf.value.decode()

    def synchronize(self):
        self._ck(self.L.he_synchronize(self.h))

    def join(self):
        """Join the side stream's queued work into the context's stream (no host wait)."""
        self._ck(self.L.he_join(self.h))

    def set_stream(self, stream_ptr):
        self._ck(self.L.he_set_stream(self.h, ctypes.c_void_p(stream_ptr)))

    def _shape(self, name):
        w = self.w
        if name in ("fden", "fvlj4", "wcgk", "kalfs"):
            return (w.nx // 2 + 1, w.ny, w.nz)
        if name in ("rimp", "vimp", "aimp", "F", "pcr", "pcv", "qr", "qv"):
            return (w.n_imp, 3)
        if name in ("rimpold", "vimpold"):
            return (w.n_imp, 3, 3)
        if name == "aimpold":
            return (w.n_imp, 3, 2)
        if name == "ring":
            return (13,)
        n = w.nq_imp
        if name in ("psix", "upotx", "pcx", "qx"):
            return (w.nx, w.ny, w.nz, n)
        if name == "psixold":
            return (w.nx, w.ny, w.nz, 3, n)
        if name == "hpsixold":
            return (w.nx, w.ny, w.nz, 2, n)
        if name == "uimpk":
            return (w.nx // 2 + 1, w.ny, w.nz, n)
        if name == "uimpkk":
            return (w.nx // 2 + 1, w.ny, w.nz, n, n)
        return (w.nx, w.ny, w.nz)

    def _is_complex(self, name):
        return (name == "fden" or name in COMPLEX_Q or
                (self.mode != _lib.HE_MODE_STATICS and name in COMPLEX_DYN))

    def upload(self, name, arr):
        dt = np.complex128 if self._is_complex(name) else np.float64
        a = np.asarray(arr, dtype=dt).reshape(self._shape(name), order="F")
        buf = np.ascontiguousarray(a.ravel(order="F"))
        self._ck(self.L.he_upload(self.h, FIELDS[name], buf.ctypes.data_as(ctypes.c_void_p),
                                  buf.nbytes))

    def download(self, name):
        dt = np.complex128 if self._is_complex(name) else np.float64
        shape = self._shape(name)
        buf = np.empty(int(np.prod(shape)), dtype=dt)
        self._ck(self.L.he_download(self.h, FIELDS[name], buf.ctypes.data_as(ctypes.c_void_p),
                                    buf.nbytes))
        return buf.reshape(shape, order="F")

    # ---- set-up ---------------------------------------------------------------------------------
    def set_kernels(self, fvlj4, wcgk, kalfs=None):
        a = np.ascontiguousarray(np.asarray(fvlj4, np.float64).ravel(order="F"))
        b = np.ascontiguousarray(np.asarray(wcgk, np.float64).ravel(order="F"))
        k = None if kalfs is None else np.ascontiguousarray(np.asarray(kalfs, np.float64).ravel(order="F"))
        self._ck(self.L.he_set_kernels(self.h, dptr(a), dptr(b), None if k is None else dptr(k)))

    def set_impurities(self, w: Workload):
        potion, npot, delinter, rmax = potion_table(w)
        self._potion = np.ascontiguousarray(potion.ravel(order="F"))
        self._m = np.ascontiguousarray(np.asarray(w.m_imp_u, np.float64))
        im = _lib.HeImpurities(w.n_imp, dptr(self._m), dptr(self._potion), npot, delinter, rmax,
                               w.ii_kind, w.ii_D, w.ii_re, w.ii_a, w.ii_rcut, w.ii_umax)
        self._ck(self.L.he_set_impurities(self.h, ctypes.byref(im)))
        if w.rimp0:
            self.upload("rimp", np.array(w.rimp0, dtype=np.float64))
        if w.vimp0_aps:
            # imp.input gives A/ps; the driver converts to A K (DFT4He3d.f90:313)
            self.upload("vimp", np.array(w.vimp0_aps, dtype=np.float64) * KTOPS)

    def set_quantum_impurities(self, w: Workload, uimp_k=None, uimp_k_k=None):
        """he_set_quantum_impurities: masses, mu4 and the He-X / X-X pair potentials of the
        workload; uimp_k / uimp_k_k host tables replace the device FT_V_spline when given."""
        from .config import pair_rows
        n = w.nq_imp
        hex_, xx = pair_rows(w)
        q = _lib.HeQImpurities()
        q.n_imp = n
        self._mq = np.ascontiguousarray(np.asarray(w.mq_imp_u, np.float64))
        q.m_imp_u = dptr(self._mq)
        q.mu4 = w.mu4
        for i in range(n):
            q.he_x[i] = _lib.HePairPot(int(hex_[i, 0]), *hex_[i, 1:])
            for j in range(n):
                r = xx[i + n * j]
                q.x_x[i + n * j] = _lib.HePairPot(int(r[0]), *r[1:])
        self._uk = self._ukk = None
        if uimp_k is not None:
            self._uk = np.ascontiguousarray(np.asarray(uimp_k, np.float64).ravel(order="F"))
            q.uimp_k = dptr(self._uk)
        if uimp_k_k is not None:
            self._ukk = np.ascontiguousarray(np.asarray(uimp_k_k, np.float64).ravel(order="F"))
            q.uimp_k_k = dptr(self._ukk)
        q.n_spline, q.nq, q.parabolic = w.n_spline, w.nq, w.parabolic
        self._ck(self.L.he_set_quantum_impurities(self.h, ctypes.byref(q)))

    OBSERVABLES = ("n", "xcm", "ycm", "zcm", "lx", "ly", "lz", "vcomx", "vcomy", "vcomz",
                   "r2x", "r2y", "r2z")

    def observables(self, npart):
        """Droplet observables of the dynamics drivers (N, r_cm, <L>, <Vcom>, <r^2>)."""
        out = np.zeros(13)
        self._ck(self.L.he_observables(self.h, int(npart), dptr(out)))
        return dict(zip(self.OBSERVABLES, out))

    def qimp_moments(self):
        """(N_imp, 4): norm, <x>, <y>, <z> of each impurity density."""
        n = self.w.nq_imp
        out = np.zeros(4 * n)
        self._ck(self.L.he_qimp_moments(self.h, dptr(out)))
        return out.reshape(n, 4)

    # ---- Dynamics_TDDFT routines ----------------------------------------------------------------
    def poten(self):
        self._ck(self.L.he_poten(self.h))

    def potenimp(self):
        self._ck(self.L.he_potenimp(self.h))

    def forceimp(self, want=False):
        if want:
            F = np.zeros(3 * max(self.w.n_imp, 1))
            self._ck(self.L.he_forceimp(self.h, dptr(F)))
            return F[: 3 * self.w.n_imp].reshape((self.w.n_imp, 3), order="F")
        self._ck(self.L.he_forceimp(self.h, None))
        return None

    def set_accel(self):
        self._ck(self.L.he_set_accel(self.h))

    def lstopimp(self):
        f = ctypes.c_int(0)
        self._ck(self.L.he_lstopimp(self.h, ctypes.byref(f)))
        return bool(f.value)

    def steprk(self, deltat):
        self._ck(self.L.he_steprk(self.h, deltat))

    def steppc(self, deltat, errors=True):
        if not errors:
            self._ck(self.L.he_steppc(self.h, deltat, None, None, None))
            return None
        e = [ctypes.c_double(0.0) for _ in range(3)]
        self._ck(self.L.he_steppc(self.h, deltat, *[ctypes.byref(x) for x in e]))
        return tuple(x.value for x in e)

    def energy(self):
        e = _lib.HeEnergies()
        self._ck(self.L.he_energy(self.h, ctypes.byref(e)))
        return {k: getattr(e, k) for k, _ in _lib.HeEnergies._fields_}

    def derden(self):
        self._ck(self.L.he_derden(self.h))

    # ---- He_statics routines --------------------------------------------------------------------
    def refresh_density(self):
        self._ck(self.L.he_refresh_density(self.h))

    def evolo0(self, mu4, n4):
        m, e = ctypes.c_double(mu4), ctypes.c_double(0.0)
        self._ck(self.L.he_evolo0(self.h, ctypes.byref(m), ctypes.byref(e), n4))
        return m.value, e.value

    def steprkr(self, deltat, mu4, n4):
        m, e = ctypes.c_double(mu4), ctypes.c_double(0.0)
        self._ck(self.L.he_steprkr(self.h, deltat, ctypes.byref(m), ctypes.byref(e), n4))
        return m.value, e.value

    def steppcr(self, deltat, mu4, n4):
        m, e, p = ctypes.c_double(mu4), ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._ck(self.L.he_steppcr(self.h, deltat, ctypes.byref(m), ctypes.byref(e), n4,
                                   ctypes.byref(p)))
        self.errpc = p.value
        return m.value, e.value

    def statics_iterations(self, niter, deltat, mu4, n4):
        """niter passes of steppcr + refresh_density + poten with one host read at the end
        (he_statics_iterations); returns (mu4, mu4err) of the last pass, errpc in self.errpc."""
        m, e, p = ctypes.c_double(mu4), ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._ck(self.L.he_statics_iterations(self.h, niter, deltat, ctypes.byref(m),
                                              ctypes.byref(e), n4, ctypes.byref(p)))
        self.errpc = p.value
        return m.value, e.value

    def varmu(self, npart, mu):
        e = ctypes.c_double(0.0)
        self._ck(self.L.he_varmu(self.h, npart, mu, ctypes.byref(e)))
        return e.value


def mass_of(w: Workload):
    return np.asarray(w.m_imp_u, np.float64) * MP_U


def ft_v_spline_table(pot, pmax, hp, n_spline=100001, parabolic=0):
    """FT_V_spline's momentum table V(i*hp), i < int(pmax/hp + 1.5), computed on the device."""
    L = _lib.load()
    n_p = int(pmax / hp + 1.5)
    out = np.zeros(n_p)
    err = ctypes.create_string_buffer(256)
    pp = _lib.HePairPot(int(pot[0]), *[float(v) for v in pot[1:6]])
    st = L.he_ft_v_spline_table(ctypes.byref(pp), pmax, hp, n_spline, parabolic, dptr(out), n_p,
                                err, 256)
    if st != 0:
        raise HeError(st, err.value.decode())
    return out

