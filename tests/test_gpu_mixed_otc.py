"""core4 = 'OTC' in the mixed-precision path (classical and quantum-impurity dynamics, statics): the alpha_s
term (term_alfa.f90) runs in binary64 on a binary64 copy of the binary32 density, and its field
enters the binary32 pot4 epilogue.  Compared with the FP64 run of the same state (itself pinned to
the oracle in test_gpu_alphas.py), at the mixed path's bars: fields to 2e-6 of their max, energy
per atom to 1e-5 K over the run."""
import numpy as np
import pytest

from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200.context import Context

pytestmark = pytest.mark.gpu

ALPHA_FIELDS = ("denalf", "falfs", "intxalf", "intyalf", "intzalf", "ualphas")


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("n", [32, 64])
def test_mixed_otc_classical_dynamics_matches_f64(n):
    w = C.tddft_1000(n=n)
    w = C.replace(w, xmax=20.0 * n / 32, ymax=20.0 * n / 32, zmax=20.0 * n / 32, n4=300,
                  core="OTC", lsolid=0, rimp0=((0.5, -0.3, 8.0),), deltatps=5e-4, noise=0.02)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    out = {}
    for prec in ("f64", "mixed"):
        with Context(w, precision=prec) as ctx:
            D.dynamics_setup(ctx, psi, w.n_imp)
            fields = {k: ctx.download(k) for k in ALPHA_FIELDS + ("pot4",)}
            for it in range(1, 41):
                D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
            out[prec] = (fields, ctx.energy(), ctx.download("den"), ctx.download("rimp"))
    f64, mx = out["f64"], out["mixed"]
    for k in ALPHA_FIELDS + ("pot4",):
        assert rel(mx[0][k], f64[0][k]) < 2e-6, (k, rel(mx[0][k], f64[0][k]))
    assert mx[1]["ealphas"] != 0.0
    assert abs(mx[1]["etot"] - f64[1]["etot"]) / w.n4 < 1e-5
    assert abs(mx[1]["ealphas"] - f64[1]["ealphas"]) <= 1e-5 * abs(f64[1]["ealphas"])
    assert abs(np.linalg.norm(mx[2]) - np.linalg.norm(f64[2])) < 1e-6 * np.linalg.norm(f64[2])
    assert np.max(np.abs(mx[3] - f64[3])) < 1e-6


def test_mixed_otc_quantum_dynamics_matches_f64():
    w = C.quantum_2000(n=32)
    w = C.replace(w, xmax=12.0, ymax=12.0, zmax=12.0, n4=300, n_spline=4001, deltatps=5e-4,
                  core="OTC", lsolid=0)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    psix = [C.psix_initial(w, 0)]
    out = {}
    for prec in ("f64", "mixed"):
        with Context(w, mode="quantum", precision=prec) as ctx:
            D.quantum_setup(ctx, psi, psix)
            ua = ctx.download("ualphas")
            for it in range(1, 21):
                D.quantum_iteration(ctx, it, w.deltat)
            out[prec] = (ua, ctx.energy(), ctx.qimp_moments())
    f64, mx = out["f64"], out["mixed"]
    assert rel(mx[0], f64[0]) < 2e-6
    assert abs(mx[1]["etot"] - f64[1]["etot"]) / w.n4 < 1e-5
    assert abs(mx[1]["ealphas"] - f64[1]["ealphas"]) <= 1e-5 * abs(f64[1]["ealphas"])
    assert np.max(np.abs(mx[2] - f64[2])) < 1e-6


def test_mixed_otc_statics_matches_f64():
    """4He_500 statics with OTC on 32^3: set-up and 30 imaginary-time iterations, mu and E/N."""
    w = C.replace(C.statics_500(), nx=32, ny=32, nz=32, xmax=11.2, ymax=11.2, zmax=11.2,
                  core="OTC", lsolid=0)
    den = C.woods_saxon(w)
    out = {}
    for prec in ("f64", "mixed"):
        with Context(w, mode="statics", precision=prec) as ctx:
            mu = D.statics_setup(ctx, den, w.n4)
            ua = ctx.download("ualphas")
            for it in range(1, 31):
                mu = D.statics_iteration(ctx, it, w.deltat_statics, mu, w.n4)[0]
            out[prec] = (mu, ctx.energy(), ua)
    f64, mx = out["f64"], out["mixed"]
    assert rel(mx[2], f64[2]) < 2e-6
    assert abs(mx[0] - f64[0]) <= 1e-5 * abs(f64[0])
    assert abs(mx[1]["etot"] - f64[1]["etot"]) / w.n4 < 1e-5
    assert mx[1]["ealphas"] != 0.0
    assert abs(mx[1]["ealphas"] - f64[1]["ealphas"]) <= 1e-5 * abs(f64[1]["ealphas"])
