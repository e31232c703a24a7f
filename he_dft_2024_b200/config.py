"""Workload descriptions: grid, functional, absorber, impurities and the synthetic droplets.

Defaults are the reference's module initialisers (Dynamics_TDDFT/modules.f90, He_statics/
modules.f90) and driver defaults (DFT4He3d.f90:136-138, BCN4HeDFT.f90:90).  The named workloads
are the benchmark configurations of this project (statics 64^3, real-time 128^3 with a classical
Morse impurity, ...), built from seeded synthetic droplets because the reference ships no data.
"""
from dataclasses import asdict, dataclass, field, replace
from typing import List, Tuple

import numpy as np

KTOPS = 7.63822291       # ps -> K^-1 conversion factor (DFT4He3d.f90:71)
MP_U = 0.02061484        # proton mass, K^-1 A^-2 (modules.f90:324)
H4OT = 2.190323          # Orsay-Trento core radius (modules.f90:230)
H4OP = 2.359665          # Orsay-Paris core radius (modules.f90:229)


@dataclass
class Workload:
    name: str = "custom"
    # grid (modules.f90:88-105; deriva npd/icon :31-37)
    nx: int = 64
    ny: int = 64
    nz: int = 64
    xmax: float = 64.0
    ymax: float = 64.0
    zmax: float = 64.0
    npd: int = 13
    icon: int = 13
    # functional (he4, lenard4 modules)
    core: str = "OT"          # effective core after the Lsolid rule
    h4: float = H4OT
    eps4: float = 10.22
    sigma4: float = 2.556
    cp4: float = -2.41186e4
    cpp4: float = 1.85850e6
    den4c: float = 0.062
    alphas: float = 54.31
    l: float = 1.0
    den0s: float = 0.04
    h2o2m4: float = 6.05969638298
    lsolid: int = 1
    C: float = 3.1577504e4
    beta: float = 40.0
    den_m: float = 0.37
    # absorber (DFT4He3d.f90:136-138)
    lambdah: float = 2.0
    txmean: float = 1000.0
    txsurf: float = 2.0
    tymean: float = 1000.0
    tysurf: float = 2.0
    tzmean: float = 1000.0
    tzsurf: float = 2.0
    # classical impurities
    n_imp: int = 0
    m_imp_u: Tuple[float, ...] = ()
    pot_kind: int = 1         # 0 null, 1 Morse
    pot_D: float = 2.0
    pot_re: float = 6.5
    pot_a: float = 0.8
    pot_rcut: float = 0.0
    pot_umax: float = 0.0
    ii_kind: int = 0
    ii_D: float = 0.0
    ii_re: float = 0.0
    ii_a: float = 0.0
    ii_rcut: float = 0.0
    ii_umax: float = 0.0
    rimp0: Tuple[Tuple[float, float, float], ...] = ()
    vimp0_aps: Tuple[Tuple[float, float, float], ...] = ()   # A/ps, as in imp.input
    # quantum impurities (Dynamics_quantum_impurities): the He-X kernel is FT_V_spline of the
    # pot_* pair potential, the X-X kernel of the ii_* one ('null' = kind 0)
    nq_imp: int = 0
    mq_imp_u: Tuple[float, ...] = ()
    mu4: float = 0.0          # chemical-potential shift of H psi (0 unless Lbulk)
    nq: int = 1000            # potenimpini's Nq (modules.f90:165); effective max(10001, nq)
    n_spline: int = 100001    # N_FT_V_spline (FT_V_spline.f90:2)
    parabolic: int = 0        # Lparabolic_fit_FT_V_spline
    psix_width: float = 1.5   # Gaussian initial impurity wave function, A
    psix_center: Tuple[Tuple[float, float, float], ...] = ()
    psix_kick_aps: Tuple[Tuple[float, float, float], ...] = ()  # impurity velocity, A/ps
    # statics local time step (He_statics/modules.f90:299)
    dtmin: float = 1.0e-10
    sdmu: float = 1.0e-1
    dmumax: float = 1.0e2
    # droplet
    n4: int = 500
    rho0: float = 0.0218
    diffuseness: float = 0.5
    noise: float = 0.0
    seed: int = 1234
    # time stepping
    deltatps: float = 1.0e-4
    pafl: float = 0.10
    steps: int = 100

    def as_dict(self):
        return asdict(self)

    @property
    def n(self):
        return self.nx * self.ny * self.nz

    @property
    def h(self):
        return (2 * abs(self.xmax) / self.nx, 2 * abs(self.ymax) / self.ny, 2 * abs(self.zmax) / self.nz)

    @property
    def dxyz(self):
        hx, hy, hz = self.h
        return hx * hy * hz

    @property
    def deltat(self):
        """Real-time step in K^-1 from deltatps (DFT4He3d.f90:241-243)."""
        return self.deltatps / KTOPS

    @property
    def deltat_statics(self):
        """Imaginary-time step pafl*min(h)^2/(4 h2o2m4) (BCN4HeDFT.f90:1053-1065)."""
        return self.pafl * min(self.h) ** 2 / (4.0 * self.h2o2m4)


def grid_axes(w: Workload):
    """x_i = -xmax + h*(i-1) (DFT4He3d.f90:321-329)."""
    hx, hy, hz = w.h
    return (-w.xmax + hx * np.arange(w.nx), -w.ymax + hy * np.arange(w.ny),
            -w.zmax + hz * np.arange(w.nz))


def woods_saxon(w: Workload, n4=None, radius=None):
    """Seeded synthetic droplet density rho0/(exp((r-R)/a)+1) * (1 + noise*U(-1,1)), normalised
    to n4 atoms; R = 2.22 n4^(1/3) unless given.  The noise is drawn in column-major order from
    numpy's PCG64 generator seeded with w.seed."""
    n4 = w.n4 if n4 is None else n4
    x, y, z = grid_axes(w)
    R = 2.22 * n4 ** (1.0 / 3.0) if radius is None else radius
    r = np.sqrt(x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2)
    with np.errstate(over="ignore"):
        den = w.rho0 / (np.exp((r - R) / w.diffuseness) + 1.0)
    if w.noise:
        u = np.random.default_rng(w.seed).uniform(-1.0, 1.0, size=w.n)
        den = den * (1.0 + w.noise * u.reshape((w.nx, w.ny, w.nz), order="F"))
    den *= n4 / (den.sum() * w.dxyz)
    return np.asfortranarray(den)


def select_pot(kind, D, re, a, rcut, umax, r):
    """Select_Pot(selec,r,r_cutoff,umax) contract (V_impur.f90:90-2152): umax below the cutoff;
    kind 0 = 'null', 1 = Morse D[(1-exp(-a(r-re)))^2-1] (no reference counterpart)."""
    r = np.asarray(r, dtype=np.float64)
    if kind == 0:
        v = np.zeros_like(r)
    else:
        e = 1.0 - np.exp(-a * (r - re))
        v = D * (e * e - 1.0)
    return np.where(r < rcut, umax, v)


def potion_table(w: Workload):
    """potenimpini's interpolation table (potenimpini.f90:31-59): npot = 100*max(n)+1,
    rmax = 4*max(xmax), DelInter = rmax/(npot-1); returns (potion (N_imp,npot) F-order, npot,
    DelInter, rmax)."""
    npot = 100 * max(w.nx, w.ny, w.nz) + 1
    rmax = 4.0 * max(w.xmax, w.ymax, w.zmax)
    delinter = rmax / float(npot - 1)
    r = np.arange(npot, dtype=np.float64) * delinter
    row = select_pot(w.pot_kind, w.pot_D, w.pot_re, w.pot_a, w.pot_rcut, w.pot_umax, r)
    potion = np.asfortranarray(np.tile(row, (w.n_imp, 1)))
    return potion, npot, delinter, rmax


# ---- named workloads ---------------------------------------------------------------------------

# The Morse core is capped the way Select_Pot caps every reference potential (r < r_cutoff gives
# umax): below 2 A the potential is held at its value there, V(2 A) = 2532.5 K (the reference's
# Xe-He input uses r_cutoff = 2.55 A, umax = 2794 K).  Uncapped, V(0) = 6.5e4 K would make the
# explicit steppers unstable at dt = 0.1 fs.
MORSE_RCUT = 2.0
MORSE_UMAX = float(select_pot(1, 2.0, 6.5, 0.8, 0.0, 0.0, MORSE_RCUT))


def statics_500(hc=H4OT, **kw):
    """Pure 4He_500, 64^3, h = 0.7 A, imaginary time, OT core (lsolid), 100 iterations."""
    return replace(Workload(name="statics-4He500-64^3", nx=64, ny=64, nz=64, xmax=22.4, ymax=22.4,
                            zmax=22.4, n4=500, noise=0.01, h4=hc, steps=100, pafl=0.10), **kw)


def tddft_1000(n=128, **kw):
    """4He_1000 on 128^3 (h = 0.625 A), one classical 85 u impurity with the Morse He-X potential
    (D = 2 K, re = 6.5 A, a = 0.8 A^-1) starting 30 A out on z at 300 m/s inward, dt = 0.1 fs."""
    xm = 40.0 * n / 128
    return replace(Workload(name=f"tddft-4He1000-{n}^3-classical", nx=n, ny=n, nz=n, xmax=xm,
                            ymax=xm, zmax=xm, n4=1000, n_imp=1, m_imp_u=(85.0,),
                            pot_rcut=MORSE_RCUT, pot_umax=MORSE_UMAX,
                            rimp0=((0.0, 0.0, 30.0),), vimp0_aps=((0.0, 0.0, -3.0),),
                            deltatps=1.0e-4, steps=2000), **kw)


def tddft_5000_256(**kw):
    """4He_5000 on 256^3 (h = 0.5 A), same impurity and step as tddft_1000."""
    return replace(tddft_1000(), name="tddft-4He5000-256^3-classical", nx=256, ny=256, nz=256,
                   xmax=64.0, ymax=64.0, zmax=64.0, n4=5000, **kw)


def quantum_2000(n=192, speed_ms=200.0, direction=(0.0, 0.0, 1.0), **kw):
    """4He_2000 on 192^3 (h = 0.5 A) with one quantum impurity of 23 u (h2o2mx = h2o2m4 *
    4.002603/23) and the Morse He-X potential; the impurity starts as a normalised Gaussian of
    width 1.5 A at the droplet centre, kicked by exp(i k.r), k = v*7.63822291/(2 h2o2mx), with
    speed speed_ms (m/s) along direction."""
    xm = 48.0 * n / 192
    d = np.asarray(direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    v = tuple(float(c) for c in d * speed_ms / 100.0)  # m/s -> A/ps
    return replace(Workload(name=f"tddft-4He2000-{n}^3-quantum", nx=n, ny=n, nz=n, xmax=xm,
                            ymax=xm, zmax=xm, n4=2000, nq_imp=1, mq_imp_u=(23.0,),
                            pot_rcut=MORSE_RCUT, pot_umax=MORSE_UMAX,
                            psix_center=((0.0, 0.0, 0.0),), psix_kick_aps=(v,),
                            deltatps=1.0e-4, steps=1000), **kw)


def quantum_batch(count=16, n=192, seed=1234, **kw):
    """The batched quantum workload: count trajectories of quantum_2000 whose impurity speeds are
    U(0, 400) m/s and directions uniform on the sphere (numpy PCG64 seeded with seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        speed = rng.uniform(0.0, 400.0)
        d = rng.normal(size=3)
        out.append(quantum_2000(n=n, speed_ms=speed, direction=tuple(d / np.linalg.norm(d)), **kw))
    return out


def psix_initial(w: Workload, k: int = 0):
    """Impurity k's initial wave function: exp(-|r-c|^2/(2 width^2)) * exp(i kv.r), normalised
    to 1 (sum |psix|^2 dxyz = 1), kv = v[A/ps]*7.63822291/(2*h2o2mx)."""
    x, y, z = grid_axes(w)
    c = w.psix_center[k] if w.psix_center else (0.0, 0.0, 0.0)
    r2 = ((x[:, None, None] - c[0]) ** 2 + (y[None, :, None] - c[1]) ** 2 +
          (z[None, None, :] - c[2]) ** 2)
    f = np.exp(-r2 / (2.0 * w.psix_width ** 2)).astype(np.complex128)
    if w.psix_kick_aps:
        h2o2mx = w.h2o2m4 * 4.002603 / w.mq_imp_u[k]
        kv = np.asarray(w.psix_kick_aps[k], dtype=np.float64) * KTOPS / (2.0 * h2o2mx)
        ph = kv[0] * x[:, None, None] + kv[1] * y[None, :, None] + kv[2] * z[None, None, :]
        f = f * np.exp(1j * ph)
    f /= np.sqrt((np.abs(f) ** 2).sum() * w.dxyz)
    return np.asfortranarray(f)


def pair_rows(w: Workload):
    """FT_V_spline pair potentials as rows {kind, D, re, a, r_cutoff, umax}: He-X for each quantum
    impurity and X-X for each ordered pair (i + n*j; i == j and 'null' pairs are kind 0)."""
    n = w.nq_imp
    hex_ = np.array([[w.pot_kind, w.pot_D, w.pot_re, w.pot_a, w.pot_rcut, w.pot_umax]] * n,
                    dtype=np.float64).reshape(n, 6)
    xx = np.zeros((n * n, 6))
    for i in range(n):
        for j in range(n):
            if i != j and w.ii_kind:
                xx[i + n * j] = [w.ii_kind, w.ii_D, w.ii_re, w.ii_a, w.ii_rcut, w.ii_umax]
    return hex_, xx

