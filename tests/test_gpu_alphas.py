"""The alpha_s term (core4 = 'OTC', term_alfa.f90) on the device against the CPU oracle, in the three
paths that call it: real-time dynamics with a classical impurity, imaginary-time statics and
real-time dynamics with a quantum impurity.  OTC runs without the solid penalty (the drivers force
core4 = 'OT ' when Lsolid is set: DFT4He3d.f90:460, BCN4HeDFT.f90:654).
"""
import numpy as np
import pytest

from oracle import oracle as O
from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200.context import Context

pytestmark = pytest.mark.gpu

RTOL_STEP = 1e-10
ALPHA_FIELDS = ("denalf", "falfs", "intxalf", "intyalf", "intzalf", "ualphas")


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def kernels(ctx, o):
    ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"), o.get("kalfs"))


def test_otc_classical_dynamics_matches_oracle():
    w = C.tddft_1000(n=32)
    w = C.replace(w, xmax=20.0, ymax=20.0, zmax=20.0, n4=300, core="OTC", lsolid=0,
                  rimp0=((0.5, -0.3, 8.0),), deltatps=5e-4, noise=0.02)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    o = O.Dynamics(w.as_dict(), m_imp_u=w.m_imp_u)
    with Context(w) as ctx:
        kalfs_dev = ctx.download("kalfs").ravel(order="F")
        assert rel(kalfs_dev, o.get("kalfs")) < 1e-14
        kernels(ctx, o)
        D.dynamics_setup(o, psi, w.n_imp)
        D.dynamics_setup(ctx, psi, w.n_imp)
        for name in ALPHA_FIELDS + ("pot4", "dencg", "delj4"):
            assert rel(ctx.download(name).ravel(order="F"), o.get(name)) < 1e-12, name
        for it in range(1, 8):
            D.dynamics_iteration(o, it, w.deltat, w.n_imp)
            D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
            assert rel(ctx.download("psi").ravel(order="F"), o.get("psi")) < RTOL_STEP, it
        eo, ed = o.energy(), ctx.energy()
        assert eo["ealphas"] != 0.0
        for k in ("ealphas", "etot4", "ekin4", "elj4", "ecor4", "etot"):
            assert abs(ed[k] - eo[k]) <= RTOL_STEP * max(abs(eo[k]), 1.0), (k, ed[k], eo[k])


def test_otc_statics_matches_oracle():
    w = C.replace(C.statics_500(), nx=32, ny=32, nz=32, xmax=11.2, ymax=11.2, zmax=11.2,
                  core="OTC", lsolid=0)
    den = C.woods_saxon(w)
    o = O.Statics(w.as_dict())
    with Context(w, mode="statics") as ctx:
        kernels(ctx, o)
        mu_o = D.statics_setup(o, den, w.n4)
        mu_d = D.statics_setup(ctx, den, w.n4)
        assert abs(mu_d - mu_o) <= 1e-11 * abs(mu_o)
        for name in ALPHA_FIELDS + ("pot4",):
            assert rel(ctx.download(name).ravel(order="F"), o.get(name)) < 1e-12, name
        for it in range(1, 8):
            mu_o, _ = D.statics_iteration(o, it, w.deltat_statics, mu_o, w.n4)
            mu_d, _ = D.statics_iteration(ctx, it, w.deltat_statics, mu_d, w.n4)
            assert abs(mu_d - mu_o) <= RTOL_STEP * abs(mu_o), it
        assert rel(ctx.download("psi").ravel(order="F"), o.get("psi")) < RTOL_STEP
        eo, ed = o.energy(), ctx.energy()
        for k in ("ealphas", "etot4", "ekin4"):
            assert abs(ed[k] - eo[k]) <= RTOL_STEP * max(abs(eo[k]), 1.0), (k, ed[k], eo[k])


def test_otc_quantum_dynamics_matches_oracle():
    w = C.quantum_2000(n=32)
    w = C.replace(w, xmax=12.0, ymax=12.0, zmax=12.0, n4=300, n_spline=4001, deltatps=5e-4,
                  core="OTC", lsolid=0)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    psix = [C.psix_initial(w, 0)]
    o = O.QDynamics(w.as_dict())
    with Context(w, mode="quantum") as ctx:
        kernels(ctx, o)
        D.quantum_setup(o, psi, psix)
        D.quantum_setup(ctx, psi, psix)
        for name in ALPHA_FIELDS + ("pot4",):
            assert rel(ctx.download(name).ravel(order="F"), o.get(name)) < 1e-12, name
        for it in range(1, 6):
            D.quantum_iteration(o, it, w.deltat)
            D.quantum_iteration(ctx, it, w.deltat)
        assert rel(ctx.download("psi").ravel(order="F"), o.get("psi")) < RTOL_STEP
        assert rel(ctx.download("psix")[..., 0].ravel(order="F"), o.get("psix:0")) < RTOL_STEP
        eo, ed = o.energy(), ctx.energy()
        for k in ("ealphas", "etot4", "etot"):
            assert abs(ed[k] - eo[k]) <= RTOL_STEP * max(abs(eo[k]), 1.0), (k, ed[k], eo[k])
