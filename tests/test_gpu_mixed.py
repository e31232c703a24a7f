"""The mixed-precision path (HE_PREC_MIXED) against the binary64 path on the same inputs: the
mean field's FFT chain, the stencils and H psi in binary32; psi and its history as compensated
binary32 pairs; reductions and the impurity's Newton integration in binary64.

Accuracy bar: the metric's |delta E/N| < 1e-5 K between the mixed and the FP64 runs of the
classical-impurity workload, checked here over 200 driver iterations at 64^3 (and fields after one
evaluation to binary32 accuracy)."""
import numpy as np
import pytest

from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200.context import Context

pytestmark = pytest.mark.gpu


def workload(n=64):
    w = C.tddft_1000(n=n)
    return C.replace(w, xmax=20.0 * n / 64, ymax=20.0 * n / 64, zmax=20.0 * n / 64, n4=300,
                     rimp0=((0.5, -0.3, 8.0),), deltatps=2e-4)


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


def test_mixed_field_matches_f64_to_binary32_accuracy():
    w = workload(32)
    den = C.woods_saxon(w)
    out = {}
    for prec in ("f64", "mixed"):
        with Context(w, precision=prec) as ctx:
            ctx.upload("den", den)
            ctx.poten()
            out[prec] = {k: ctx.download(k) for k in ("pot4", "dencg", "delj4", "fden")}
    # binary32 rounding (not binary64, and not wrong): the FFT outputs carry a few ulp of binary32
    # relative to their largest value.  dencg is packed with the ~1e3 larger delj4 in one
    # complex line of the C2R pass; without the power-of-two scale of the binary32 wcgk copy its
    # error would be ~1e-5 of its maximum
    bound = {"pot4": 2e-6, "dencg": 2e-6, "delj4": 2e-6, "fden": 2e-6}
    for k, b in bound.items():
        r = rel(out["mixed"][k], out["f64"][k])
        assert 1e-12 < r < b, (k, r)


def test_mixed_energy_per_atom_within_1e5_K_over_200_steps():
    w = workload(64)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    e = {}
    for prec in ("f64", "mixed"):
        with Context(w, precision=prec) as ctx:
            D.dynamics_setup(ctx, psi, w.n_imp)
            hist = []
            for it in range(1, 201):
                D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
                if it % 50 == 0:
                    hist.append(ctx.energy()["etot"] / w.n4)
            e[prec] = (np.array(hist), ctx.download("rimp"), np.sum(ctx.download("den") ** 2))
    de = np.max(np.abs(e["mixed"][0] - e["f64"][0]))
    assert de < 1e-5, de
    assert np.max(np.abs(e["mixed"][1] - e["f64"][1])) < 1e-6
    assert abs(e["mixed"][2] - e["f64"][2]) < 1e-6 * e["f64"][2]


def test_mixed_rejects_unsupported_modes():
    from he_dft_2024_b200._lib import HeError
    w = workload(32)
    with Context(w, precision="mixed") as ctx:
        with pytest.raises(HeError):
            ctx.derden()
    # core4 = 'OTC' is covered (test_gpu_mixed_otc.py)


def test_mixed_field_formats_round_trip():
    """psi is held as a compensated pair (about 48 bits), pc as binary32, den as binary32; the
    host side is binary64 either way."""
    w = workload(32)
    rng = np.random.default_rng(5)
    shape = (w.nx, w.ny, w.nz)
    z = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    r = rng.random(shape)
    with Context(w, precision="mixed") as ctx:
        for name in ("psi", "psiold2"):
            ctx.upload(name, z)
            back = ctx.download(name)
            err = np.max(np.abs(back - z)) / np.max(np.abs(z))
            assert 0 < err < 2.0 ** -45, (name, err)
        for name in ("pc", "hpsiold1"):
            ctx.upload(name, z)
            back = ctx.download(name)
            assert np.array_equal(back, z.astype(np.complex64).astype(np.complex128)), name
        for name in ("den", "pot4"):
            ctx.upload(name, r)
            back = ctx.download(name)
            assert np.array_equal(back, r.astype(np.float32).astype(np.float64)), name


# ---- quantum impurities (Dynamics_quantum_impurities) in the mixed path ------------------------

def quantum_workload(n=32, n_imp=2):
    w = C.quantum_2000(n=n)
    return C.replace(w, xmax=12.0, ymax=12.0, zmax=12.0, n4=300, n_spline=10001, deltatps=5e-4,
                     nq_imp=n_imp, mq_imp_u=(23.0, 40.0)[:n_imp],
                     psix_center=((0.0, 0.0, 0.0), (2.5, -1.0, 1.5))[:n_imp],
                     psix_kick_aps=((0.0, 1.0, 2.0), (-1.5, 0.0, 0.5))[:n_imp])


def test_mixed_quantum_trajectory_matches_f64():
    """Two impurity wave functions with their X-X kernel, 40 driver iterations: energy per He
    atom, the impurities' kinetic and interaction energies and their centres against the FP64
    run of the same state."""
    w = quantum_workload(32, 2)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    psix = [C.psix_initial(w, k) for k in range(w.nq_imp)]
    res = {}
    for prec in ("f64", "mixed"):
        with Context(w, mode="quantum", precision=prec) as ctx:
            D.quantum_setup(ctx, psi, psix)
            for it in range(1, 41):
                D.quantum_iteration(ctx, it, w.deltat)
            res[prec] = (ctx.energy(), ctx.qimp_moments(), np.sum(ctx.download("den") ** 2),
                         ctx.download("psix"))
    e64, em = res["f64"][0], res["mixed"][0]
    assert abs(em["etot"] - e64["etot"]) / w.n4 < 1e-5, (em["etot"], e64["etot"])
    for k in ("ekinx", "eHeX", "eimpu_impu"):
        assert abs(em[k] - e64[k]) <= 1e-5 * max(abs(e64[k]), 1.0), (k, em[k], e64[k])
    m64, mm = res["f64"][1], res["mixed"][1]
    assert np.max(np.abs(mm - m64)) < 1e-6, np.max(np.abs(mm - m64))
    assert abs(res["mixed"][2] - res["f64"][2]) < 1e-6 * res["f64"][2]
    px = res["mixed"][3] - res["f64"][3]
    assert 0 < np.max(np.abs(px)) < 1e-5 * np.max(np.abs(res["f64"][3]))


def test_mixed_quantum_field_formats_round_trip():
    w = quantum_workload(32, 2)
    rng = np.random.default_rng(9)
    shape = (w.nx, w.ny, w.nz, 2)
    z = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    r = rng.random(shape)
    with Context(w, mode="quantum", precision="mixed") as ctx:
        D.quantum_setup(ctx, D.initial_wavefunction(w, C.woods_saxon(w)),
                        [C.psix_initial(w, k) for k in range(2)])
        ctx.upload("psix", z)
        back = ctx.download("psix")
        assert 0 < np.max(np.abs(back - z)) / np.max(np.abs(z)) < 2.0 ** -45
        ctx.upload("pcx", z)
        assert np.array_equal(ctx.download("pcx"), z.astype(np.complex64).astype(np.complex128))
        ctx.upload("upotx", r)
        assert np.array_equal(ctx.download("upotx"), r.astype(np.float32).astype(np.float64))
        denx = ctx.download("denx")
        assert np.allclose(denx, np.sum(np.abs(z) ** 2, axis=-1), rtol=1e-6)


@pytest.mark.parametrize("n", [64, 96, 128])
def test_mixed_fused_xy_passes_match_f64(n):
    """The plane-fused field evaluation (fft_xy.cuh) against the FP64 fields, and a few steps of
    it against the separate passes."""
    w = workload(n)
    den = C.woods_saxon(w)
    out = {}
    for prec, fused in (("f64", None), ("mixed", 1), ("mixed", 0)):
        with Context(w, precision=prec) as ctx:
            if fused is not None:
                ctx.set_fft_variant("xy", fused, 8)
            ctx.upload("den", den)
            ctx.poten()
            out[(prec, fused)] = {k: ctx.download(k) for k in ("pot4", "dencg", "delj4", "fden")}
    for k, b in {"pot4": 2e-6, "dencg": 2e-6, "delj4": 2e-6, "fden": 2e-6}.items():
        r = rel(out[("mixed", 1)][k], out[("f64", None)][k])
        assert 1e-12 < r < b, (k, r)
        r2 = rel(out[("mixed", 1)][k], out[("mixed", 0)][k])
        assert r2 < b, (k, r2)


@pytest.mark.parametrize("zvar,tile", [(0, 8), (1, 8), (1, 16)])
def test_mixed_fft_variants_agree(zvar, tile):
    """Each z-pass variant of the binary32 chain (shared-memory Stockham, register transform)
    and the pipelined x pass give the FP64 fields to binary32 accuracy."""
    w = workload(64)
    den = C.woods_saxon(w)
    out = {}
    for prec in ("f64", "mixed"):
        with Context(w, precision=prec) as ctx:
            if prec == "mixed":
                ctx.set_fft_variant("z", zvar, tile)
                ctx.set_fft_variant("x", zvar, tile)
            ctx.upload("den", den)
            ctx.poten()
            out[prec] = {k: ctx.download(k) for k in ("pot4", "dencg", "delj4", "fden")}
    for k, b in {"pot4": 2e-6, "dencg": 2e-6, "delj4": 2e-6, "fden": 2e-6}.items():
        r = rel(out["mixed"][k], out["f64"][k])
        assert 1e-12 < r < b, (k, r)


@pytest.mark.parametrize("icon", [8, 18, 24])
def test_mixed_boundaries_match_f64(icon):
    """Periodic (8), antiperiodic (18) and reflecting (24) boundaries in the binary32 stencils:
    a few driver iterations against the FP64 run."""
    w = C.replace(workload(32), icon=icon, noise=0.05)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    res = {}
    for prec in ("f64", "mixed"):
        with Context(w, precision=prec) as ctx:
            D.dynamics_setup(ctx, psi, w.n_imp)
            for it in range(1, 9):
                D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
            res[prec] = (ctx.download("psi"), ctx.energy()["etot"] / w.n4)
    r = rel(res["mixed"][0], res["f64"][0])
    assert 1e-12 < r < 1e-5, r
    assert abs(res["mixed"][1] - res["f64"][1]) < 1e-5



def test_mixed_statics_matches_f64():
    """Imaginary time (He_statics) in the mixed path: psi, psiold and pc as compensated pairs,
    H psi and the FFT chain in binary32, norm / mu / energy sums in binary64; 30 iterations of a
    40^3 droplet against the FP64 run."""
    w = C.replace(C.statics_500(), nx=40, ny=40, nz=40, xmax=14.0, ymax=14.0, zmax=14.0)
    den0 = C.woods_saxon(w)
    res = {}
    for prec in ("f64", "mixed"):
        with Context(w, mode="statics", precision=prec) as ctx:
            mu = D.statics_setup(ctx, den0, w.n4)
            for it in range(1, 31):
                mu, err = D.statics_iteration(ctx, it, w.deltat_statics, mu, w.n4)
            den = ctx.download("den")
            res[prec] = (mu, ctx.energy()["etot"] / w.n4, np.sqrt(np.sum(den * den)),
                         ctx.varmu(w.n4, mu), ctx.download("psi"))
    m, f = res["mixed"], res["f64"]
    assert abs(m[0] - f[0]) < 1e-5 * abs(f[0]), (m[0], f[0])       # mu
    assert abs(m[1] - f[1]) < 1e-5, (m[1], f[1])                  # E/N, K
    assert abs(m[2] - f[2]) < 1e-6 * f[2]                         # rho L2
    assert 1e-12 < rel(m[4], f[4]) < 1e-5
