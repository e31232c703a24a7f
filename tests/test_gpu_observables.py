"""Droplet observables (he_observables) and restart files (checkpoint.snapshot / restore) on the
device: observables against the oracle's restatement of the driver's loops
(Dynamics_TDDFT/DFT4He3d.f90:720-838, r_cm.f90); a snapshot restored into a fresh context
reproduces the state it was taken from."""
import numpy as np
import pytest

from oracle import oracle as O
from he_dft_2024_b200 import checkpoint as K
from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200.context import Context

pytestmark = pytest.mark.gpu


def moving_droplet():
    w = C.tddft_1000(n=32)
    w = C.replace(w, xmax=20.0, ymax=20.0, zmax=20.0, n4=300, rimp0=((0.5, -0.3, 8.0),),
                  deltatps=5e-4, noise=0.02)
    den = C.woods_saxon(w)
    x, y, z = C.grid_axes(w)
    # a translation plus a rotation-like phase, so that <Vcom> and <L> are not zero
    ph = 0.08 * x[:, None, None] - 0.05 * z[None, None, :] + 0.004 * x[:, None, None] * y[None, :, None]
    psi = np.asfortranarray(np.sqrt(den) * np.exp(1j * ph))
    return w, psi


def test_observables_match_oracle():
    w, psi = moving_droplet()
    o = O.Dynamics(w.as_dict(), m_imp_u=w.m_imp_u)
    with Context(w) as ctx:
        ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"))
        for side in (o, ctx):
            D.dynamics_setup(side, psi, w.n_imp)
            for it in range(1, 6):
                D.dynamics_iteration(side, it, w.deltat, w.n_imp)
        got = ctx.observables(w.n4)
    ref = o.observables(w.n4)
    assert abs(ref["vcomx"]) > 1e-3 and abs(ref["lz"]) > 1e-3
    for k, r in ref.items():
        assert abs(got[k] - r) <= 1e-10 * max(abs(r), 1.0), (k, got[k], r)


def test_snapshot_restore_round_trip(tmp_path):
    w, psi = moving_droplet()
    p = tmp_path / "psi.restart"
    with Context(w) as a:
        D.dynamics_setup(a, psi, w.n_imp)
        for it in range(1, 5):
            D.dynamics_iteration(a, it, w.deltat, w.n_imp)
        K.snapshot(a, p, w.n4, iteration=4, time_ps=4 * w.deltatps)
        psi_a, rimp_a, vimp_a = a.download("psi"), a.download("rimp"), a.download("vimp")
        e_a = a.energy()
    with Context(w) as b:
        K.restore(b, p)
        b.potenimp()
        b.poten()
        assert np.array_equal(b.download("psi"), psi_a)
        assert np.array_equal(b.download("rimp"), rimp_a)
        assert np.array_equal(b.download("vimp"), vimp_a)
        e_b = b.energy()
    for k in ("etot4", "ekin4", "elj4", "ecor4", "eHeX"):
        assert abs(e_b[k] - e_a[k]) <= 1e-12 * max(abs(e_a[k]), 1.0), k


def test_mixed_observables_and_restart(tmp_path):
    """The mixed path (HE_PREC_MIXED): observables from the binary32 psi plane and den against the
    FP64 run of the same trajectory, and a snapshot restored into a fresh mixed context (psi
    travels as binary64 text and is split into the pair again)."""
    w, psi = moving_droplet()
    obs = {}
    p = tmp_path / "psi_mixed.restart"
    for prec in ("f64", "mixed"):
        with Context(w, precision=prec) as ctx:
            D.dynamics_setup(ctx, psi, w.n_imp)
            for it in range(1, 6):
                D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
            obs[prec] = ctx.observables(w.n4)
            if prec == "mixed":
                K.snapshot(ctx, p, w.n4, iteration=5, time_ps=5 * w.deltatps)
                psi_m, e_m = ctx.download("psi"), ctx.energy()
    for k, r in obs["f64"].items():
        assert abs(obs["mixed"][k] - r) <= 1e-5 * max(abs(r), 1.0), (k, obs["mixed"][k], r)
    with Context(w, precision="mixed") as b:
        K.restore(b, p)
        b.potenimp()
        b.poten()
        back = b.download("psi")
        assert np.max(np.abs(back - psi_m)) <= 2.0 ** -44 * np.max(np.abs(psi_m))
        assert abs(b.energy()["etot"] - e_m["etot"]) <= 1e-6 * abs(e_m["etot"])
