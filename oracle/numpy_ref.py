"""A second, independent CPU restatement of the real-time step: numpy / numpy.fft, binary64.

TEST INFRASTRUCTURE ONLY, like the rest of oracle/: it cross-checks the C++ oracle
(he_oracle.cpp) and serves as a second timed CPU point.  It was written from the reference's
Fortran, routine by routine, and shares no code with the C++ oracle or with the device path.  It
covers the classical-impurity dynamics path with core4 = 'OT '/'OP ' and icon = 13:

    derivnD / Deriv3D_pc   Dynamics_TDDFT/init_deriv_parallel.f90:933-1090 (icon 13 rows of
                           Redef, redef.f:133-170, applied to the Bickley table newder.f:99-130)
    poten                  Dynamics_TDDFT/poten.f90:131-218 (ldroplet_frozen = .false.)
    potenimp/updatepoten   Dynamics_TDDFT/potenimp.f90:1-19, :83-123
    forceimp               Dynamics_TDDFT/potenimp.f90:23-67 (one impurity: F_ij = 0)
    steprk                 Dynamics_TDDFT/steprk.f90:1-144
    steppc                 Dynamics_TDDFT/steppc.f90:1-180
    energy                 Dynamics_TDDFT/energy.f90:107-178
    driver glue            DFT4He3d.f90:313 (vimp in A/ps x 7.63822291), :562-576 (set-up),
                           :592-601 (timec), :677-697 (aimp = F/m_imp)

Inputs shared with the other implementations, as the Fortran driver shares them: the k-space
kernels fvlj4 and wcgk (fforma/initcg output) and the derivative table (tests/golden/
bickley13.json, read from the reference's BLOCK DATA text).  Fields are numpy arrays of shape
(nx, ny, nz) in Fortran order; the half spectrum is (nx/2+1, ny, nz).

The object mirrors the oracle's Python surface (set/get/potenimp/poten/forceimp/set_accel/steprk/
steppc/energy), so the same driver sequence (he_dft_2024_b200.driver) runs on it.
"""
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(os.path.dirname(HERE), "tests", "golden", "bickley13.json")
KTOPS = 7.63822291   # DFT4He3d.f90:313
MP_U = 0.02061484    # modules.f90:324


def bickley(k):
    """The 13x13 matrix Cdc(K, :, :) of the table (as expanded by newder.f:99-130)."""
    g = json.load(open(GOLDEN))
    return np.array([float.fromhex(e["hex"]) for e in g[f"K{k}"]]).reshape(13, 13)


def redef13(cd):
    """Redef for icon = 13 (redef.f:151-170, then :133-150): the first KO2 rows are the row below
    shifted one place left with a zero entering on the right; the last KO2 rows the row above
    shifted right with a zero entering on the left."""
    c = cd.copy()
    for i in range(5, -1, -1):           # Fortran rows KO2..1
        c[i, :12] = c[i + 1, 1:]
        c[i, 12] = 0.0
    for i in range(7, 13):               # Fortran rows KO2+2..K
        c[i, 1:] = c[i - 1, :12]
        c[i, 0] = 0.0
    return c


# tanh element by element through the C library: 1 + tanh(beta (den - den_m)) cancels to ~1e-12 in
# the droplet (esolid, the solid penalty), so the last bit of tanh shows at the 1e-4 level there;
# the C library's tanh is the one a Fortran or C++ build of the reference calls.
_tanh = np.frompyfunc(math.tanh, 1, 1)


def libm_tanh(a):
    return _tanh(a).astype(np.float64)


class NumpyDynamics:
    COMPLEX = {"psi", "pc", "q", "fden", "psiold1", "psiold2", "psiold3", "hpsiold1", "hpsiold2"}

    def __init__(self, w, fvlj4, wcgk):
        assert w.icon == 13 and w.npd == 13 and w.core in ("OT", "OP") and w.n_imp <= 1
        self.w = w
        self.n = (w.nx, w.ny, w.nz)
        self.nk = (w.nx // 2 + 1, w.ny, w.nz)
        self.h = w.h
        self.dxyz = self.h[0] * self.h[1] * self.h[2]
        self.nxyz = w.nx * w.ny * w.nz
        self.fvlj4 = np.asarray(fvlj4, np.float64).reshape(self.nk, order="F")
        self.wcgk = np.asarray(wcgk, np.float64).reshape(self.nk, order="F")
        # derivative matrices Cd(id) = Redef(Cdc(id)) * Sto, Sto = 1/h**id, per axis
        self.cd = {(idd, a): redef13(bickley(idd)) * (1.0 / self.h[a] ** idd)
                   for idd in (1, 2) for a in range(3)}
        # grid x_i = -xmax + h (i-1) (DFT4He3d.f90:321-329)
        self.x = [-m + hh * np.arange(k) for m, hh, k in
                  zip((w.xmax, w.ymax, w.zmax), self.h, self.n)]
        # timec (DFT4He3d.f90:592-601): (Lambdah*(1+t_x + 1+t_y + 1+t_z), 1), left to right
        tx = np.tanh((np.abs(self.x[0]) - w.txmean) / w.txsurf)[:, None, None]
        ty = np.tanh((np.abs(self.x[1]) - w.tymean) / w.tysurf)[None, :, None]
        tz = np.tanh((np.abs(self.x[2]) - w.tzmean) / w.tzsurf)[None, None, :]
        self.timec = w.lambdah * ((((((1.0 + tx) + 1.0) + ty) + 1.0) + tz))
        z = lambda: np.zeros(self.n, order="F")
        zc = lambda: np.zeros(self.n, np.complex128, order="F")
        self.f = {k: zc() for k in ("psi", "pc", "q", "psiold1", "psiold2", "psiold3",
                                    "hpsiold1", "hpsiold2")}
        self.f.update({k: z() for k in ("den", "pot4", "dencg", "delj4", "uimp", "dxden",
                                        "dyden", "dzden")})
        self.f["fden"] = np.zeros(self.nk, np.complex128, order="F")
        self.ioldp, self.ioldh = [1, 2, 3], [1, 2]
        self.ioldr, self.ioldv, self.iolda = [1, 2, 3], [1, 2, 3], [1, 2]
        # classical impurity (classicimp module); potenimpini table (potenimpini.f90:31-59)
        ni = w.n_imp
        self.ni = ni
        self.m_imp = np.asarray(w.m_imp_u, np.float64) * MP_U
        self.rimp = np.array(w.rimp0, np.float64).reshape(ni, 3) if ni else np.zeros((0, 3))
        self.vimp = (np.array(w.vimp0_aps, np.float64).reshape(ni, 3) * KTOPS if ni
                     else np.zeros((0, 3)))
        self.aimp = np.zeros((ni, 3))
        self.F = np.zeros((ni, 3))
        self.rimpold = np.zeros((ni, 3, 3))
        self.vimpold = np.zeros((ni, 3, 3))
        self.aimpold = np.zeros((ni, 3, 2))
        self.pcr, self.pcv = np.zeros((ni, 3)), np.zeros((ni, 3))
        self.qr, self.qv = np.zeros((ni, 3)), np.zeros((ni, 3))
        self.uimp_k = np.zeros((max(ni, 1),) + self.n)
        self.npot = 100 * max(self.n) + 1
        rmax = 4.0 * max(w.xmax, w.ymax, w.zmax)
        self.rmaxinterpol = rmax
        self.delinter = rmax / float(self.npot - 1)
        r = np.arange(self.npot, dtype=np.float64) * self.delinter
        e = 1.0 - np.exp(-w.pot_a * (r - w.pot_re))
        v = w.pot_D * (e * e - 1.0) if w.pot_kind == 1 else np.zeros_like(r)
        self.potion = np.where(r < w.pot_rcut, w.pot_umax, v)

    # ---- module-array access (the oracle's surface) ----
    def set(self, name, arr):
        if name in ("rimp", "vimp", "aimp"):
            setattr(self, name, np.asarray(arr, np.float64).reshape(self.ni, 3).copy())
            return
        shape = self.nk if name == "fden" else self.n
        dt = np.complex128 if name in self.COMPLEX else np.float64
        self.f[name] = np.asfortranarray(np.asarray(arr, dt).reshape(shape, order="F"))

    def get(self, name):
        if name in ("rimp", "vimp", "aimp", "F"):
            return getattr(self, name).ravel(order="F").copy()
        return self.f[name].ravel(order="F").copy()

    # ---- derivnD (init_deriv_parallel.f90:933-1090 with the icon 13 matrix) ----
    def deriv(self, idd, a, f):
        cd = self.cd[(idd, a)]
        n = f.shape[a]
        if n < 13:  # init_deriv_parallel.f90:949-953
            return np.zeros_like(f)
        g = np.moveaxis(f, a, 0)
        out = np.empty_like(g)
        # interior rows: Sum(Cd(ko2p1,:)*f(i-ko2:i+ko2)), the sum taken left to right
        acc = cd[6, 0] * g[0:n - 12]
        for j in range(1, 13):
            acc = acc + cd[6, j] * g[j:n - 12 + j]
        out[6:n - 6] = acc
        # first and last KO2 rows from the first / last 13 points
        for i in range(6):
            acc = cd[i, 0] * g[0]
            for j in range(1, 13):
                acc = acc + cd[i, j] * g[j]
            out[i] = acc
        for i in range(n - 6, n):
            r = i - n + 13
            acc = cd[r, 0] * g[n - 13]
            for j in range(1, 13):
                acc = acc + cd[r, j] * g[n - 13 + j]
            out[i] = acc
        return np.moveaxis(out, 0, a)

    # ---- fft.f90: fftfw (R2C, unnormalised), fftbk (C2R times renor = 1/nxyz) ----
    def fftfw(self, f):
        return np.fft.rfftn(f, axes=(2, 1, 0))

    def fftbk(self, fk):
        return np.fft.irfftn(fk, s=(self.n[2], self.n[1], self.n[0]), axes=(2, 1, 0))

    # ---- poten (poten.f90:131-218) ----
    def poten(self):
        w, f = self.w, self.f
        den = f["den"]
        f["fden"] = self.fftfw(den)
        f["dencg"] = self.fftbk(f["fden"] * self.wcgk)
        self.derden()
        f["delj4"] = self.fftbk(f["fden"] * self.fvlj4)
        a0, a1 = w.cp4 / 2.0, w.cpp4 / 3.0
        dencg = f["dencg"]
        sto1 = den * dencg * (w.cp4 + w.cpp4 * dencg)
        sto1 = self.fftbk(self.fftfw(sto1) * self.wcgk)
        if w.lsolid:
            t = libm_tanh(w.beta * (den - w.den_m))
            penalty = w.C * (1.0 + t + w.beta * den * (1.0 - t ** 2))
        pot4 = f["delj4"] + dencg ** 2 * (a0 + a1 * dencg) + sto1
        if w.lsolid:
            pot4 = pot4 + penalty
        f["pot4"] = pot4

    def derden(self):  # derden.f90:26-28
        den = self.f["den"]
        self.f["dxden"] = self.deriv(1, 0, den)
        self.f["dyden"] = self.deriv(1, 1, den)
        self.f["dzden"] = self.deriv(1, 2, den)

    # ---- potenimp / updatepoten (potenimp.f90:83-123) ----
    def potenimp(self):
        x, y, z = self.x
        self.f["uimp"] = np.zeros(self.n)
        for k in range(self.ni):
            zt = (z - self.rimp[k, 2]) ** 2
            yt = (y - self.rimp[k, 1])[:, None] ** 2 + zt[None, :]
            r = np.sqrt((x - self.rimp[k, 0])[:, None, None] ** 2 + yt[None, :, :])
            assert np.all(r <= self.rmaxinterpol)
            ir = (r / self.delinter).astype(np.int64)       # int(r/DelInter), 0-based
            rmod = np.fmod(r, self.delinter) / self.delinter
            self.uimp_k[k] = self.potion[ir] * (1.0 - rmod) + self.potion[ir + 1] * rmod
            self.f["uimp"] = self.f["uimp"] + self.uimp_k[k]

    # ---- forceimp (potenimp.f90:23-67) ----
    def forceimp(self):
        f = self.f
        for k in range(self.ni):
            self.F[k, 0] = -np.sum(f["dxden"] * self.uimp_k[k]) * self.dxyz
            self.F[k, 1] = -np.sum(f["dyden"] * self.uimp_k[k]) * self.dxyz
            self.F[k, 2] = -np.sum(f["dzden"] * self.uimp_k[k]) * self.dxyz

    def set_accel(self):  # DFT4He3d.f90:692-694
        self.aimp = self.F / self.m_imp[:, None]

    # ---- H psi (steprk.f90:67, steppc.f90:51,118) ----
    def hpsi(self):
        f, w = self.f, self.w
        psi = f["psi"]
        lap = self.deriv(2, 0, psi) + self.deriv(2, 1, psi) + self.deriv(2, 2, psi)
        a = lap * w.h2o2m4 - f["pot4"] * psi
        # timec*a with timec = (tr, 1), minus i*uimp*psi
        return (self.timec * a.real - a.imag + f["uimp"] * psi.imag) + \
            1j * (self.timec * a.imag + a.real - f["uimp"] * psi.real)

    def _field(self):
        self.potenimp()
        self.poten()
        self.forceimp()

    # ---- steprk (steprk.f90:1-144) ----
    def steprk(self, deltat):
        f = self.f
        r2 = 1.0 / np.sqrt(2.0)
        arun = (0.5, 1.0 - r2, 1.0 + r2, 1.0 / 6.0)
        brun = (2.0, 1.0, 1.0, 2.0)
        crun = (0.5, 1.0 - r2, 1.0 + r2, 0.5)
        for jr in range(4):
            s4 = self.hpsi()
            s1 = arun[jr] * (s4 - brun[jr] * f["q"])
            f["q"] = f["q"] + 3.0 * s1 - crun[jr] * s4
            if jr == 0:
                f["hpsiold2"] = f["hpsiold1"]
                f["hpsiold1"] = s4
                f["psiold3"] = f["psiold2"]
                f["psiold2"] = f["psiold1"]
                f["psiold1"] = f["psi"]
            f["psi"] = f["psi"] + deltat * s1
            f["den"] = np.abs(f["psi"]) ** 2
            if self.ni:
                st = arun[jr] * (self.vimp - brun[jr] * self.qr)
                self.qr = self.qr + 3.0 * st - crun[jr] * self.vimp
                if jr == 0:
                    self.rimpold[:, :, 2] = self.rimpold[:, :, 1]
                    self.rimpold[:, :, 1] = self.rimpold[:, :, 0]
                    self.rimpold[:, :, 0] = self.rimp
                self.rimp = self.rimp + deltat * st
                st = arun[jr] * (self.aimp - brun[jr] * self.qv)
                self.qv = self.qv + 3.0 * st - crun[jr] * self.aimp
                if jr == 0:
                    self.aimpold[:, :, 1] = self.aimpold[:, :, 0]
                    self.aimpold[:, :, 0] = self.aimp
                    self.vimpold[:, :, 2] = self.vimpold[:, :, 1]
                    self.vimpold[:, :, 1] = self.vimpold[:, :, 0]
                    self.vimpold[:, :, 0] = self.vimp
                self.vimp = self.vimp + deltat * st
            if jr <= 2:  # steprk.f90:126-130
                self._field()
        self.ioldp, self.ioldh = [1, 2, 3], [1, 2]
        self.ioldr, self.ioldv, self.iolda = [1, 2, 3], [1, 2, 3], [1, 2]

    # ---- steppc (steppc.f90:1-180) ----
    def steppc(self, deltat):
        f = self.f
        c112, c9, c4o3 = 112.0 / 121.0, 9.0 / 121.0, 4.0 / 3.0
        po = lambda s: f"psiold{self.ioldp[s - 1]}"
        ho = lambda s: f"hpsiold{self.ioldh[s - 1]}"
        s4 = self.hpsi()
        s1 = f[po(3)] + c4o3 * deltat * (2.0 * s4 - f[ho(1)] + 2.0 * f[ho(2)])
        f[po(3)] = f["psi"]
        f["psi"] = s1 - c112 * f["pc"]
        f["pc"] = s1
        f[ho(2)] = s4
        f["den"] = np.abs(f["psi"]) ** 2
        self.ioldh = [self.ioldh[1], self.ioldh[0]]
        if self.ni:
            R, V, A = self.ioldr, self.ioldv, self.iolda
            st = (self.rimpold[:, :, R[2] - 1] + c4o3 * deltat *
                  (2.0 * self.vimp - self.vimpold[:, :, V[0] - 1] + 2.0 * self.vimpold[:, :, V[1] - 1]))
            self.rimpold[:, :, R[2] - 1] = self.rimp
            self.rimp = st - c112 * self.pcr
            self.pcr = st
            st = (self.vimpold[:, :, V[2] - 1] + c4o3 * deltat *
                  (2.0 * self.aimp - self.aimpold[:, :, A[0] - 1] + 2.0 * self.aimpold[:, :, A[1] - 1]))
            self.vimpold[:, :, V[2] - 1] = st - c112 * self.pcv
            self.pcv = st
            self.aimpold[:, :, A[1] - 1] = self.aimp
            self.iolda = [A[1], A[0]]
        self._field()  # steppc.f90:103-105, with or without impurities
        s4 = self.hpsi()
        s5 = 0.125 * (9.0 * f[po(3)] - f[po(2)] + 3.0 * deltat * (s4 + 2.0 * f[ho(1)] - f[ho(2)]))
        f["pc"] = f["pc"] - s5
        f["psi"] = s5 + c9 * f["pc"]
        errhe = c9 * np.sum(np.abs(f["pc"])) / self.nxyz
        f["den"] = np.abs(f["psi"]) ** 2
        p = self.ioldp
        self.ioldp = [p[2], p[0], p[1]]
        errimp = errvimp = 0.0
        if self.ni:
            R, V, A = self.ioldr, self.ioldv, self.iolda
            st = 0.125 * (9.0 * self.rimpold[:, :, R[2] - 1] - self.rimpold[:, :, R[1] - 1] +
                          3.0 * deltat * (self.vimpold[:, :, V[2] - 1] + 2.0 * self.vimp -
                                          self.vimpold[:, :, V[0] - 1]))
            self.pcr = self.pcr - st
            self.rimp = st + c9 * self.pcr
            errimp = np.sum(np.abs(c9 * self.pcr)) * 0.3333333333 / self.ni
            self.ioldr = [R[2], R[0], R[1]]
            st = 0.125 * (9.0 * self.vimp - self.vimpold[:, :, V[1] - 1] +
                          3.0 * deltat * (self.aimp + 2.0 * self.aimpold[:, :, A[0] - 1] -
                                          self.aimpold[:, :, A[1] - 1]))
            self.pcv = self.pcv - st
            self.vimpold[:, :, V[2] - 1] = self.vimp
            self.vimp = st + c9 * self.pcv
            errvimp = np.sum(np.abs(c9 * self.pcv)) * 0.3333333333 / self.ni
            self.ioldv = [V[2], V[0], V[1]]
        return errhe, errimp, errvimp

    # ---- energy (energy.f90:107-178, OT/OP core, uext = 0, one impurity) ----
    def energy(self):
        f, w = self.f, self.w
        psi, den, dencg = f["psi"], f["den"], f["dencg"]
        aux1, aux2 = 0.5 * w.cp4, (1.0 / 3.0) * w.cpp4
        ekin = np.sum(np.abs(self.deriv(1, 0, psi)) ** 2 + np.abs(self.deriv(1, 1, psi)) ** 2 +
                      np.abs(self.deriv(1, 2, psi)) ** 2)
        elj = np.sum(f["delj4"] * den)
        ecor = np.sum(den * dencg ** 2 * (aux1 + aux2 * dencg))
        esolid = w.C * np.sum(den * (1.0 + libm_tanh(w.beta * (den - w.den_m)))) * self.dxyz if w.lsolid else 0.0
        ekin4 = w.h2o2m4 * ekin * self.dxyz
        elj4 = 0.5 * elj * self.dxyz
        ecor4 = ecor * self.dxyz
        etot4 = ekin4 + elj4 + ecor4 + esolid
        ekinx = sum(0.5 * self.m_imp[k] * np.sum(self.vimp[k] * self.vimp[k]) for k in range(self.ni))
        ehex = np.sum(f["uimp"] * den) * self.dxyz
        eimpu = ekinx + ehex
        return {"etot4": etot4, "ekin4": ekin4, "elj4": elj4, "ecor4": ecor4, "esolid": esolid,
                "ealphas": 0.0, "ekinx": ekinx, "eHeX": ehex, "eimpu_impu": 0.0,
                "eimpu": eimpu, "etot": etot4 + eimpu}
