"""Odd grid sizes that tstgrid admits (tstgrid.f90:9-13: 15, 25, 27, 45, 75, 81, 125, 135, ...):
odd nx (no Nyquist term in the x transform) and odd ny*nz (the x pass pairs two real rows per
complex line, so the last row of an odd row count is transformed alone), against the oracle.

Tolerances: field evaluations 1e-12 of each field's max; driver iterations the FP64 bar, 1e-10
relative per step in E/N and the rho L2 norm."""
import numpy as np
import pytest

from oracle import oracle as O
from he_dft_2024_b200 import config as C
from he_dft_2024_b200.context import Context
from he_dft_2024_b200 import driver as D

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def small_dyn(shape, n_imp=1, **kw):
    w = C.tddft_1000(n=32)
    return C.replace(w, nx=shape[0], ny=shape[1], nz=shape[2], xmax=20.0, ymax=20.0, zmax=20.0,
                     n4=300, n_imp=n_imp, m_imp_u=(85.0,) * n_imp, rimp0=((0.5, -0.3, 8.0),) * n_imp,
                     vimp0_aps=((0.0, 0.0, -3.0),) * n_imp, deltatps=5e-4, **kw)


@pytest.mark.parametrize("shape", [(27, 27, 27), (45, 32, 30), (30, 27, 25), (75, 45, 27)])
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_poten_on_odd_grids(shape, precision):
    w = C.replace(small_dyn(shape, n_imp=0), noise=0.05)
    den = C.woods_saxon(w)
    o = O.Dynamics(w.as_dict())
    o.set("den", den)
    o.poten()
    tol = 1e-12 if precision == "f64" else 2e-6
    with Context(w, precision=precision) as ctx:
        ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"))
        ctx.upload("den", den)
        ctx.poten()
        for name in ("dencg", "delj4", "pot4", "fden"):
            assert rel(ctx.download(name).ravel(order="F"), o.get(name)) < tol, name


@pytest.mark.parametrize("shape", [(27, 27, 27), (45, 30, 32)])
def test_dynamics_on_odd_grids(shape):
    """8 driver iterations (3 RK-Gill, 5 predictor-corrector) with one impurity."""
    w = small_dyn(shape)
    o = O.Dynamics(w.as_dict(), m_imp_u=w.m_imp_u)
    with Context(w) as ctx:
        ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"))
        psi0 = D.initial_wavefunction(w, C.woods_saxon(w), kick=(0.0, 0.0, 0.05))
        for s in (o, ctx):
            D.dynamics_setup(s, psi0, w.n_imp)
        for it in range(1, 9):
            for s in (o, ctx):
                D.dynamics_iteration(s, it, w.deltat, w.n_imp)
            eo, eg = o.energy()["etot"], ctx.energy()["etot"]
            assert abs(eg - eo) <= 1e-10 * abs(eo), it
            lo, lg = np.linalg.norm(o.get("den")), np.linalg.norm(ctx.download("den"))
            assert abs(lg - lo) <= 1e-10 * lo, it
        assert rel(ctx.download("psi").ravel(order="F"), o.get("psi")) < 1e-10


def test_statics_on_an_odd_grid():
    """4He_500 statics on 45^3: the start and 8 imaginary-time iterations, mu and E/N per
    iteration."""
    w = C.replace(C.statics_500(), nx=45, ny=45, nz=45, xmax=22.0, ymax=22.0, zmax=22.0)
    o = O.Statics(w.as_dict())
    with Context(w, mode="statics") as ctx:
        ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"))
        mus = [D.statics_setup(s, C.woods_saxon(w), w.n4) for s in (o, ctx)]
        for it in range(1, 9):
            mus = [D.statics_iteration(s, it, w.deltat_statics, m, w.n4)[0] for s, m in zip((o, ctx), mus)]
            assert abs(mus[1] - mus[0]) <= 1e-10 * abs(mus[0]), it
            eo, eg = o.energy()["etot"], ctx.energy()["etot"]
            assert abs(eg - eo) <= 1e-10 * abs(eo), it
