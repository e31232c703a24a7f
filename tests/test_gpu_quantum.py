"""Quantum-impurity path (Dynamics_quantum_impurities) on the device against the CPU oracle.

Covers FT_V_spline's momentum table (the device transform of the cubic pieces, k_ftv), the
uimp_k / uimp_k_k kernels, potenimp/poten with potx4 and upotx, the RK-Gill and Hamming steppers
for He and impurity wave functions together, energy() with ekinx / eHeX / eimpu_impu, and the
per-step impurity moments.  Tolerances: 1e-10 of the field's max per step (as the classical path);
the momentum table to 1e-11 of max |V(p)|.
"""
import numpy as np
import pytest

from oracle import oracle as O
from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200.context import Context, ft_v_spline_table

pytestmark = pytest.mark.gpu

RTOL_STEP = 1e-10
NSPLINE = 10001  # radial spline nodes for the grid tests (the oracle transform is O(N_p*N))


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


def small_q(n=32, n_imp=1, **kw):
    w = C.quantum_2000(n=n)
    w = C.replace(w, xmax=12.0, ymax=12.0, zmax=12.0, n4=300, n_spline=NSPLINE, deltatps=5e-4,
                  nq_imp=n_imp, mq_imp_u=(23.0, 40.0)[:n_imp],
                  psix_center=((0.0, 0.0, 0.0), (2.5, -1.0, 1.5))[:n_imp],
                  psix_kick_aps=((0.0, 1.0, 2.0), (-1.5, 0.0, 0.5))[:n_imp], **kw)
    return w


def both(w):
    """Oracle and device context with the same state after set-up (potenimp + poten)."""
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    psix = [C.psix_initial(w, k) for k in range(w.nq_imp)]
    o = O.QDynamics(w.as_dict())
    ctx = Context(w, mode="quantum")
    ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"))
    D.quantum_setup(o, psi, psix)
    D.quantum_setup(ctx, psi, psix)
    return o, ctx


MORSE = [1, 2.0, 6.5, 0.8, C.MORSE_RCUT, C.MORSE_UMAX]


@pytest.mark.parametrize("parabolic", [0, 1])
def test_ft_v_spline_table_matches_oracle(parabolic):
    pmax, hp = 100.0, 0.01
    dev = ft_v_spline_table(MORSE, pmax, hp, n_spline=NSPLINE, parabolic=parabolic)
    ref = O.ft_vpp_table(MORSE, pmax, hp, nspline=NSPLINE, parabolic=parabolic)
    assert dev.shape == ref.shape == (10001,)
    assert rel(dev, ref) < 1e-11


def test_ft_v_spline_full_size_points():
    """The reference's N_FT_V_spline = 100001 nodes: sampled momenta of the device table against
    the oracle's transform at those momenta (above small_q, where no redefinition applies)."""
    pmax, hp = 100.0, 0.01
    dev = ft_v_spline_table(MORSE, pmax, hp)
    idx = [2, 3, 5, 17, 60, 250, 999, 4000, 10000]
    ref = np.array([O.ft_vpp_point(MORSE, i * hp) for i in idx])
    assert np.max(np.abs(dev[idx] - ref)) < 1e-11 * np.max(np.abs(dev))


@pytest.mark.parametrize("n_imp", [1, 2])
def test_quantum_fields_match_oracle(n_imp):
    kw = dict(ii_kind=1, ii_D=1.0, ii_re=4.0, ii_a=1.0, ii_rcut=1.5,
              ii_umax=float(C.select_pot(1, 1.0, 4.0, 1.0, 0.0, 0.0, 1.5))) if n_imp == 2 else {}
    w = small_q(n_imp=n_imp, **kw)
    o, ctx = both(w)
    with ctx:
        uk = ctx.download("uimpk")
        for i in range(n_imp):
            assert rel(uk[..., i].ravel(order="F"), o.get(f"uimpk:{i}")) < 1e-11
        if n_imp == 2:
            ukk = ctx.download("uimpkk")
            assert rel(ukk[..., 0, 1].ravel(order="F"), o.get("uimpkk1:0")) < 1e-11
            assert np.all(ukk[..., 0, 0] == 0.0)
        for name in ("potx4", "pot4", "dencg", "delj4"):
            assert rel(ctx.download(name).ravel(order="F"), o.get(name)) < 1e-12, name
        up = ctx.download("upotx")
        for i in range(n_imp):
            assert rel(up[..., i].ravel(order="F"), o.get(f"upotx:{i}")) < 1e-12
        assert rel(ctx.download("fden").ravel(order="F"), o.get("fden")) < 1e-12


@pytest.mark.parametrize("n_imp", [1, 2])
def test_quantum_dynamics_matches_oracle(n_imp):
    kw = dict(ii_kind=1, ii_D=1.0, ii_re=4.0, ii_a=1.0, ii_rcut=1.5,
              ii_umax=float(C.select_pot(1, 1.0, 4.0, 1.0, 0.0, 0.0, 1.5))) if n_imp == 2 else {}
    w = small_q(n_imp=n_imp, **kw)
    o, ctx = both(w)
    with ctx:
        eo, ed = o.energy(), ctx.energy()
        for k in ("etot4", "ekin4", "elj4", "ecor4", "ekinx", "eHeX", "eimpu_impu", "etot"):
            assert abs(ed[k] - eo[k]) <= 1e-11 * max(abs(eo[k]), 1.0), (k, ed[k], eo[k])
        for it in range(1, 9):
            eo_ = D.quantum_iteration(o, it, w.deltat)
            ed_ = D.quantum_iteration(ctx, it, w.deltat, errors=True)
            if it > 3:
                assert abs(ed_[0] - eo_[0]) <= 1e-8 * abs(eo_[0]) + 1e-22
                assert abs(ed_[1] - eo_[1]) <= 1e-8 * abs(eo_[1]) + 1e-22
            assert rel(ctx.download("psi").ravel(order="F"), o.get("psi")) < RTOL_STEP, it
            px = ctx.download("psix")
            for i in range(n_imp):
                assert rel(px[..., i].ravel(order="F"), o.get(f"psix:{i}")) < RTOL_STEP, (it, i)
            assert rel(ctx.download("den").ravel(order="F"), o.get("den")) < RTOL_STEP
        eo, ed = o.energy(), ctx.energy()
        for k in ("etot4", "ekin4", "elj4", "ecor4", "esolid", "ekinx", "eHeX", "eimpu_impu",
                  "eimpu", "etot"):
            assert abs(ed[k] - eo[k]) <= RTOL_STEP * max(abs(eo[k]), 1.0), (k, ed[k], eo[k])
        mo, md = o.moments(), ctx.qimp_moments()
        assert np.max(np.abs(md - mo)) < 1e-11
        # the impurity rings: psixold / hpsixold slots and the ring indices
        assert ctx.download("ring")[:5].tolist() == o.ring()
        pxo = ctx.download("psixold")
        for i in range(n_imp):
            for s in range(3):
                assert rel(pxo[..., s, i].ravel(order="F"), o.get(f"psixold{s + 1}:{i}")) < RTOL_STEP
        hxo = ctx.download("hpsixold")
        for i in range(n_imp):
            for s in range(2):
                assert rel(hxo[..., s, i].ravel(order="F"), o.get(f"hpsixold{s + 1}:{i}")) < RTOL_STEP
        assert rel(ctx.download("pcx")[..., 0].ravel(order="F"), o.get("pcx:0")) < RTOL_STEP
        denx = ctx.download("denx")
        ref = sum(np.abs(o.get(f"psix:{i}")) ** 2 for i in range(n_imp))
        assert rel(denx.ravel(order="F"), ref) < RTOL_STEP


def test_quantum_host_kernels_and_mu4():
    """Host-supplied uimp_k (the shim's upload of potenimpini's table) and a non-zero mu4."""
    w = small_q(mu4=-7.15)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    psix = [C.psix_initial(w, 0)]
    o = O.QDynamics(w.as_dict())
    with Context(w, mode="quantum") as ctx:
        ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"))
        uk = o.get("uimpk:0").reshape((w.nx // 2 + 1, w.ny, w.nz), order="F")
        ctx.set_quantum_impurities(w, uimp_k=uk[..., None])
        D.quantum_setup(o, psi, psix)
        D.quantum_setup(ctx, psi, psix)
        for it in range(1, 6):
            D.quantum_iteration(o, it, w.deltat)
            D.quantum_iteration(ctx, it, w.deltat)
        assert rel(ctx.download("psi").ravel(order="F"), o.get("psi")) < RTOL_STEP
        assert rel(ctx.download("psix")[..., 0].ravel(order="F"), o.get("psix:0")) < RTOL_STEP
