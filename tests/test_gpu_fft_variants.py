"""The 64^3 convolutions of the field evaluation with the y and z passes fused over a thread-block
cluster (fft_yz.cuh) against the separate y / z passes, and against the CPU oracle.

The fused kernel's line transforms are those of the register y pass; the separate binary64 z
pass is the shared-memory Stockham transform, so the two agree to rounding (binary64: 1e-12 of
each field's max; binary32: the 2e-6 bar of the mixed chain)."""
import numpy as np
import pytest

from oracle import oracle as O
from he_dft_2024_b200 import config as C
from he_dft_2024_b200.context import Context
from he_dft_2024_b200 import driver as D

pytestmark = pytest.mark.gpu

FIELDS = ("pot4", "dencg", "delj4", "fden")


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_fused_yz_convolutions_match_separate_passes(precision):
    w = C.replace(C.tddft_1000(n=64), n_imp=0, m_imp_u=(), rimp0=(), vimp0_aps=(), noise=0.05)
    den = C.woods_saxon(w)
    out = {}
    for fused in (0, 1):
        with Context(w, precision=precision) as ctx:
            if precision == "mixed":
                ctx.set_fft_variant("xy", 0, 8)
            ctx.set_fft_variant("yz", fused, 8)
            ctx.upload("den", den)
            ctx.poten()
            out[fused] = {k: ctx.download(k) for k in FIELDS}
    tol = 1e-12 if precision == "f64" else 2e-6
    for k in FIELDS:
        assert rel(out[1][k], out[0][k]) < tol, (k, rel(out[1][k], out[0][k]))


def test_fused_yz_refused_off_64():
    w = C.replace(C.tddft_1000(n=32), n_imp=0, m_imp_u=(), rimp0=(), vimp0_aps=())
    with Context(w) as ctx:
        with pytest.raises(Exception):
            ctx.set_fft_variant("yz", 1, 8)


@pytest.mark.parametrize("mode", ["dynamics", "statics"])
def test_fused_yz_runs_match_oracle(mode):
    """64^3 with the fused convolutions forced on: 6 driver iterations (dynamics with one
    impurity, or statics) against the oracle at the FP64 bar per step."""
    if mode == "dynamics":
        w = C.replace(C.tddft_1000(n=64), xmax=40.0, ymax=40.0, zmax=40.0, n4=500,
                      rimp0=((0.5, -0.3, 12.0),), deltatps=5e-4)
        o = O.Dynamics(w.as_dict(), m_imp_u=w.m_imp_u)
    else:
        w = C.statics_500()
        o = O.Statics(w.as_dict())
    with Context(w, mode=mode) as ctx:
        ctx.set_fft_variant("yz", 1, 8)
        ctx.set_kernels(o.get("fvlj4"), o.get("wcgk"))
        if mode == "dynamics":
            psi0 = D.initial_wavefunction(w, C.woods_saxon(w), kick=(0.0, 0.0, 0.05))
            for s in (o, ctx):
                D.dynamics_setup(s, psi0, w.n_imp)
        else:
            mus = [D.statics_setup(s, C.woods_saxon(w), w.n4) for s in (o, ctx)]
        for it in range(1, 7):
            if mode == "dynamics":
                for s in (o, ctx):
                    D.dynamics_iteration(s, it, w.deltat, w.n_imp)
            else:
                mus = [D.statics_iteration(s, it, w.deltat_statics, m, w.n4)[0]
                       for s, m in zip((o, ctx), mus)]
                assert abs(mus[1] - mus[0]) <= 1e-10 * abs(mus[0]), it
            eo, eg = o.energy()["etot"], ctx.energy()["etot"]
            assert abs(eg - eo) <= 1e-10 * abs(eo), it
            lo, lg = np.linalg.norm(o.get("den")), np.linalg.norm(ctx.download("den"))
            assert abs(lg - lo) <= 1e-10 * lo, it


@pytest.mark.parametrize("n", [64, 128])
@pytest.mark.parametrize("tile", [8, 16])
def test_register_z_pass_matches_shared_memory_pass_f64(n, tile):
    """The binary64 convolution with the z lines transformed in registers (k_zconv_reg) against
    the shared-memory Stockham z pass (k_zconv), separate y / z passes both times."""
    w = C.replace(C.tddft_1000(n=n), n_imp=0, m_imp_u=(), rimp0=(), vimp0_aps=(), noise=0.05)
    den = C.woods_saxon(w)
    out = {}
    for zreg in (0, 1):
        with Context(w) as ctx:
            if n == 64:
                ctx.set_fft_variant("yz", 0, 8)
            ctx.set_fft_variant("z", zreg, tile)
            ctx.upload("den", den)
            ctx.poten()
            out[zreg] = {k: ctx.download(k) for k in FIELDS}
    for k in FIELDS:
        assert rel(out[1][k], out[0][k]) < 1e-12, (k, rel(out[1][k], out[0][k]))
