"""ctypes front end of the CPU oracle (oracle/he_oracle.cpp).

TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.  Only tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference legs may import this.
Parity of the full step is unpinned by the reference (it cannot be built here); the pinned parts
are listed in he_oracle.cpp's header.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class HoParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("zmax", ctypes.c_double),
        ("npd", ctypes.c_int), ("icon", ctypes.c_int),
        ("core", ctypes.c_int),
        ("h4", ctypes.c_double), ("eps4", ctypes.c_double), ("sigma4", ctypes.c_double),
        ("cp4", ctypes.c_double), ("cpp4", ctypes.c_double), ("den4c", ctypes.c_double),
        ("alphas", ctypes.c_double), ("l", ctypes.c_double), ("den0s", ctypes.c_double),
        ("h2o2m4", ctypes.c_double),
        ("lsolid", ctypes.c_int),
        ("C", ctypes.c_double), ("beta", ctypes.c_double), ("den_m", ctypes.c_double),
        ("lambdah", ctypes.c_double), ("txmean", ctypes.c_double), ("txsurf", ctypes.c_double),
        ("tymean", ctypes.c_double), ("tysurf", ctypes.c_double),
        ("tzmean", ctypes.c_double), ("tzsurf", ctypes.c_double),
        ("n_imp", ctypes.c_int),
        ("pot_kind", ctypes.c_int),
        ("pot_D", ctypes.c_double), ("pot_re", ctypes.c_double), ("pot_a", ctypes.c_double),
        ("pot_rcut", ctypes.c_double), ("pot_umax", ctypes.c_double),
        ("ii_kind", ctypes.c_int),
        ("ii_D", ctypes.c_double), ("ii_re", ctypes.c_double), ("ii_a", ctypes.c_double),
        ("ii_rcut", ctypes.c_double), ("ii_umax", ctypes.c_double),
        ("dtmin", ctypes.c_double), ("sdmu", ctypes.c_double), ("dmumax", ctypes.c_double),
        ("nthreads", ctypes.c_int),
    ]


CORES = {"OT": 0, "OP": 1, "OTC": 2}


def make_params(cfg, nthreads=0):
    """HoParams from a workload dict (keys as in he_dft_2024_b200.config.Workload.as_dict())."""
    p = HoParams()
    for name, _ in HoParams._fields_:
        if name == "core":
            p.core = CORES[cfg["core"]]
        elif name == "nthreads":
            p.nthreads = nthreads
        elif name in cfg:
            setattr(p, name, cfg[name])
    return p


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(HoParams)
        dp = ctypes.POINTER(ctypes.c_double)
        vp = ctypes.c_void_p
        L.ho_sine_integral.restype = ctypes.c_double
        L.ho_sine_integral.argtypes = [ctypes.c_double]
        L.ho_bforce.restype = ctypes.c_double
        L.ho_bforce.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ho_bickley13.argtypes = [dp, dp]
        L.ho_fforma.argtypes = [P, dp]
        L.ho_initcg.argtypes = [P, ctypes.c_double, dp]
        L.ho_r2c.argtypes = [P, dp, dp]
        L.ho_c2r.argtypes = [P, dp, dp]
        L.ho_deriv.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
        L.ho_dyn_create.restype = vp
        L.ho_dyn_create.argtypes = [P, dp]
        L.ho_dyn_destroy.argtypes = [vp]
        L.ho_dyn_field.restype = dp
        L.ho_dyn_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)]
        for f in ("potenimp", "poten", "forceimp", "set_accel"):
            getattr(L, "ho_dyn_" + f).argtypes = [vp]
        L.ho_dyn_steprk.argtypes = [vp, ctypes.c_double]
        L.ho_dyn_steppc.argtypes = [vp, ctypes.c_double, dp]
        L.ho_dyn_energy.argtypes = [vp, dp]
        L.ho_dyn_lstopimp.restype = ctypes.c_int
        L.ho_dyn_lstopimp.argtypes = [vp]
        L.ho_dyn_ring.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        L.ho_stat_create.restype = vp
        L.ho_stat_create.argtypes = [P]
        L.ho_stat_destroy.argtypes = [vp]
        L.ho_stat_field.restype = dp
        L.ho_stat_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)]
        L.ho_stat_refresh.argtypes = [vp]
        L.ho_stat_poten.argtypes = [vp]
        for f in ("evolo0", "steprkr", "steppcr"):
            getattr(L, "ho_stat_" + f).argtypes = (
                [vp, dp, dp, ctypes.c_int] if f == "evolo0" else [vp, ctypes.c_double, dp, dp, ctypes.c_int])
        L.ho_stat_errpc.restype = ctypes.c_double
        L.ho_stat_errpc.argtypes = [vp]
        L.ho_stat_energy.argtypes = [vp, dp]
        L.ho_stat_varmu.restype = ctypes.c_double
        L.ho_stat_varmu.argtypes = [vp, ctypes.c_int, ctypes.c_double]
        ci, cd = ctypes.c_int, ctypes.c_double
        L.ho_qdyn_create.restype = vp
        L.ho_qdyn_create.argtypes = [P, ci, dp, cd, dp, dp, ci, ci, ci]
        L.ho_qdyn_destroy.argtypes = [vp]
        L.ho_qdyn_field.restype = dp
        L.ho_qdyn_field.argtypes = [vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_long)]
        for f in ("potenimp", "poten"):
            getattr(L, "ho_qdyn_" + f).argtypes = [vp]
        L.ho_qdyn_steprk.argtypes = [vp, cd]
        L.ho_qdyn_steppc.argtypes = [vp, cd, dp]
        L.ho_qdyn_energy.argtypes = [vp, dp]
        L.ho_qdyn_moments.argtypes = [vp, dp]
        L.ho_qdyn_ring.argtypes = [vp, ctypes.POINTER(ci), ci]
        L.ho_ft_vpp_table.restype = ci
        L.ho_ft_vpp_table.argtypes = [dp, cd, cd, ci, ci, dp, ci]
        L.ho_ft_vpp_point.restype = cd
        L.ho_ft_vpp_point.argtypes = [dp, cd, ci, ci]
        L.ho_spline.argtypes = [dp, dp, cd, cd, ci, dp, dp, dp, dp]
        L.ho_dyn_observables.argtypes = [vp, ci, dp]
        L.ho_qdyn_observables.argtypes = [vp, ci, dp]
        L.ho_findi.restype = ci
        L.ho_findi.argtypes = [dp, cd, ci]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


ENERGY_KEYS = ("etot4", "ekin4", "elj4", "ecor4", "esolid", "ealphas", "ekinx", "eHeX",
               "eimpu_impu", "eimpu", "etot")


class _Fields:
    _field_fn = None

    def _view(self, name):
        n = ctypes.c_long(0)
        ptr = self._field_fn(self.h, name.encode(), ctypes.byref(n))
        if not ptr:
            raise KeyError(name)
        return np.ctypeslib.as_array(ptr, shape=(n.value,))

    def get(self, name):
        v = self._view(name).copy()
        if name in self.COMPLEX:
            v = v.view(np.complex128)
        return v

    def set(self, name, arr):
        v = self._view(name)
        flat = np.asarray(arr).ravel(order="F")
        if name in self.COMPLEX:
            flat = np.ascontiguousarray(flat.astype(np.complex128)).view(np.float64)
        v[:] = flat


class Dynamics(_Fields):
    """Dynamics_TDDFT module state + poten/potenimp/forceimp/steprk/steppc/energy."""
    COMPLEX = {"psi", "pc", "q", "fden", "psiold1", "psiold2", "psiold3", "hpsiold1", "hpsiold2"}

    def __init__(self, cfg, m_imp_u=(), nthreads=0):
        self.L = lib()
        self.p = make_params(cfg, nthreads)
        m = np.asarray(list(m_imp_u) + [0.0], dtype=np.float64)
        self.h = self.L.ho_dyn_create(ctypes.byref(self.p), _dp(m))
        self._field_fn = self.L.ho_dyn_field
        n = int(cfg.get("n_imp", 0))
        if n and cfg.get("rimp0"):
            self.set("rimp", np.array(cfg["rimp0"], dtype=np.float64).reshape(n, 3))
        if n and cfg.get("vimp0_aps"):
            # imp.input velocities are in A/ps; the driver multiplies by 7.63822291
            # (Dynamics_TDDFT/DFT4He3d.f90:313)
            self.set("vimp", np.array(cfg["vimp0_aps"], dtype=np.float64).reshape(n, 3) * 7.63822291)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ho_dyn_destroy(self.h)
            self.h = None

    def potenimp(self): self.L.ho_dyn_potenimp(self.h)
    def poten(self): self.L.ho_dyn_poten(self.h)
    def forceimp(self): self.L.ho_dyn_forceimp(self.h)
    def set_accel(self): self.L.ho_dyn_set_accel(self.h)
    def steprk(self, dt): self.L.ho_dyn_steprk(self.h, dt)

    def steppc(self, dt):
        e = np.zeros(3)
        self.L.ho_dyn_steppc(self.h, dt, _dp(e))
        return tuple(e)

    def energy(self):
        e = np.zeros(11)
        self.L.ho_dyn_energy(self.h, _dp(e))
        return dict(zip(ENERGY_KEYS, e))

    def lstopimp(self): return bool(self.L.ho_dyn_lstopimp(self.h))

    OBSERVABLES = ("n", "xcm", "ycm", "zcm", "lx", "ly", "lz", "vcomx", "vcomy", "vcomz",
                   "r2x", "r2y", "r2z")

    def observables(self, npart):
        out = np.zeros(13)
        self.L.ho_dyn_observables(self.h, int(npart), _dp(out))
        return dict(zip(self.OBSERVABLES, out))

    def ring(self, values=None):
        """Get (or set) ioldp(3), ioldh(2), ioldr(3), ioldv(3), iolda(2)."""
        r = (ctypes.c_int * 13)()
        if values is not None:
            for i, v in enumerate(values):
                r[i] = int(v)
            self.L.ho_dyn_ring(self.h, r, 1)
            return list(values)
        self.L.ho_dyn_ring(self.h, r, 0)
        return list(r)


class Statics(_Fields):
    """He_statics module state + poten/steprkr/steppcr/energy (pure droplet)."""
    COMPLEX = {"fden"}

    def __init__(self, cfg, nthreads=0):
        self.L = lib()
        self.p = make_params(cfg, nthreads)
        self.h = self.L.ho_stat_create(ctypes.byref(self.p))
        self._field_fn = self.L.ho_stat_field

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ho_stat_destroy(self.h)
            self.h = None

    def refresh(self): self.L.ho_stat_refresh(self.h)
    def poten(self): self.L.ho_stat_poten(self.h)

    def evolo0(self, mu, n4):
        m, e = ctypes.c_double(mu), ctypes.c_double(0)
        self.L.ho_stat_evolo0(self.h, ctypes.byref(m), ctypes.byref(e), n4)
        return m.value, e.value

    def steprkr(self, dt, mu, n4):
        m, e = ctypes.c_double(mu), ctypes.c_double(0)
        self.L.ho_stat_steprkr(self.h, dt, ctypes.byref(m), ctypes.byref(e), n4)
        return m.value, e.value

    def steppcr(self, dt, mu, n4):
        m, e = ctypes.c_double(mu), ctypes.c_double(0)
        self.L.ho_stat_steppcr(self.h, dt, ctypes.byref(m), ctypes.byref(e), n4)
        return m.value, e.value

    def errpc(self): return self.L.ho_stat_errpc(self.h)

    def energy(self):
        e = np.zeros(11)
        self.L.ho_stat_energy(self.h, _dp(e))
        return dict(zip(ENERGY_KEYS, e))

    def varmu(self, npart, mu): return self.L.ho_stat_varmu(self.h, npart, mu)


def r2c(cfg, a):
    p = make_params(cfg)
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    out = np.zeros((nx // 2 + 1) * ny * nz * 2)
    src = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
    lib().ho_r2c(ctypes.byref(p), _dp(src), _dp(out))
    return out.view(np.complex128).reshape((nx // 2 + 1, ny, nz), order="F")


def c2r(cfg, c):
    p = make_params(cfg)
    nx, ny, nz = cfg["nx"], cfg["ny"], cfg["nz"]
    src = np.ascontiguousarray(np.asarray(c, dtype=np.complex128).ravel(order="F")).view(np.float64)
    out = np.zeros(nx * ny * nz)
    lib().ho_c2r(ctypes.byref(p), _dp(src), _dp(out))
    return out.reshape((nx, ny, nz), order="F")


def deriv(cfg, f, id_, axis):
    p = make_params(cfg)
    f = np.asarray(f)
    cpx = np.iscomplexobj(f)
    src = np.ascontiguousarray(f.ravel(order="F").astype(np.complex128 if cpx else np.float64))
    out = np.zeros_like(src)
    lib().ho_deriv(ctypes.byref(p), id_, axis, int(cpx), _dp(src.view(np.float64)),
                   _dp(out.view(np.float64)))
    return out.reshape(f.shape, order="F")


def bickley13():
    w1, w2 = np.zeros(13), np.zeros(13)
    lib().ho_bickley13(_dp(w1), _dp(w2))
    return w1, w2


class QDynamics(_Fields):
    """Dynamics_quantum_impurities module state + potenimp/poten/steprk/steppc/energy.
    Per-impurity fields are named "psix:0", "upotx:1", "uimpk:0", ...; "uimpkk<j>:<i>" is
    uimp_k_k(:,:,:,i,j)."""
    COMPLEX_BASE = {"psi", "pc", "q", "fden", "psiold1", "psiold2", "psiold3", "hpsiold1",
                    "hpsiold2", "psix", "pcx", "qx", "psixold1", "psixold2", "psixold3",
                    "hpsixold1", "hpsixold2"}

    class _C:
        def __contains__(self, name):
            return name.split(":")[0] in QDynamics.COMPLEX_BASE

    COMPLEX = _C()

    def __init__(self, cfg, nthreads=0):
        from he_dft_2024_b200 import config as C  # pair rows share the product's workload layout
        self.L = lib()
        self.p = make_params(cfg, nthreads)
        w = C.Workload(**{k: v for k, v in cfg.items() if k in C.Workload.__dataclass_fields__})
        hex_, xx = C.pair_rows(w)
        self.ni = w.nq_imp
        m = np.asarray(list(w.mq_imp_u) + [0.0], dtype=np.float64)
        hex_ = np.ascontiguousarray(hex_.ravel())
        xx = np.ascontiguousarray(xx.ravel()) if xx.size else np.zeros(6)
        self.h = self.L.ho_qdyn_create(ctypes.byref(self.p), self.ni, _dp(m), w.mu4, _dp(hex_),
                                       _dp(xx), w.n_spline, w.nq, w.parabolic)
        self._field_fn = self.L.ho_qdyn_field

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ho_qdyn_destroy(self.h)
            self.h = None

    def potenimp(self): self.L.ho_qdyn_potenimp(self.h)
    def poten(self): self.L.ho_qdyn_poten(self.h)
    def steprk(self, dt): self.L.ho_qdyn_steprk(self.h, dt)

    def steppc(self, dt):
        e = np.zeros(2)
        self.L.ho_qdyn_steppc(self.h, dt, _dp(e))
        return tuple(e)

    def energy(self):
        e = np.zeros(11)
        self.L.ho_qdyn_energy(self.h, _dp(e))
        return dict(zip(ENERGY_KEYS, e))

    def moments(self):
        out = np.zeros(4 * self.ni)
        self.L.ho_qdyn_moments(self.h, _dp(out))
        return out.reshape(self.ni, 4)

    def ring(self, values=None):
        r = (ctypes.c_int * 5)()
        if values is not None:
            for i, v in enumerate(values[:5]):
                r[i] = int(v)
            self.L.ho_qdyn_ring(self.h, r, 1)
            return list(values[:5])
        self.L.ho_qdyn_ring(self.h, r, 0)
        return list(r)


def ft_vpp_table(pot, pmax, hp, nspline=100001, parabolic=0):
    """FT_V_spline's Vpp table (after the small-q redefinition) for pot = {kind,D,re,a,rcut,umax}."""
    pot = np.ascontiguousarray(pot, dtype=np.float64)
    n_p = int(pmax / hp + 1.5)
    out = np.zeros(n_p)
    got = lib().ho_ft_vpp_table(_dp(pot), pmax, hp, nspline, parabolic, _dp(out), n_p)
    assert got == n_p, (got, n_p)
    return out


def ft_vpp_point(pot, p, nspline=100001, parabolic=0):
    pot = np.ascontiguousarray(pot, dtype=np.float64)
    return lib().ho_ft_vpp_point(_dp(pot), p, nspline, parabolic)


def spline(x, y, s1, sn):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = len(x)
    a, b, c, d = (np.zeros(n) for _ in range(4))
    lib().ho_spline(_dp(x), _dp(y), s1, sn, n, _dp(a), _dp(b), _dp(c), _dp(d))
    return a, b, c, d


def findi(x, xc):
    x = np.ascontiguousarray(x, dtype=np.float64)
    return lib().ho_findi(_dp(x), float(xc), len(x))

