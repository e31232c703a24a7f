"""The benchmark's own sizes, not only the small grids of the other parity tests: 4He_1000 on
128^3 (the default bench line) against the CPU oracle from the identical device state, and the
mixed-precision path against binary64 at 128^3 and on 4He_5000 at 256^3 (h = 0.5 A)."""
import os
import sys

import numpy as np
import pytest

from oracle import oracle as O
from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200.context import Context

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402  (the field lists of its full-size spot check)

pytestmark = pytest.mark.gpu


def start(ctx, w, pmc=2):
    den0 = C.woods_saxon(w)
    D.dynamics_setup(ctx, D.initial_wavefunction(w, den0), w.n_imp)
    for it in range(1, 4 + pmc):
        D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
    return 4 + pmc


def test_128_device_matches_oracle_from_the_same_state():
    w = C.tddft_1000()
    assert (w.nx, w.ny, w.nz) == (128, 128, 128)
    with Context(w) as ctx:
        it = start(ctx, w)
        o = bench.copy_state_to_oracle(ctx, w, os.cpu_count() or 1)
        for k in range(4):
            D.dynamics_iteration(o, it + k, w.deltat, w.n_imp)
            D.dynamics_iteration(ctx, it + k, w.deltat, w.n_imp)
        for name in ("psi", "den", "pot4"):
            g = ctx.download(name).ravel(order="F")
            r = np.asarray(o.get(name)).ravel()
            assert np.max(np.abs(g - r)) <= 1e-12 * np.max(np.abs(r)), name
        assert np.max(np.abs(ctx.download("rimp").ravel(order="F") - np.asarray(o.get("rimp")).ravel())) < 1e-12


@pytest.mark.parametrize("n,steps", [(128, 200), (256, 60)])
def test_mixed_matches_f64_at_full_size(n, steps):
    w = C.tddft_5000_256() if n == 256 else C.tddft_1000(n=128)
    res = {}
    for prec in ("f64", "mixed"):
        with Context(w, precision=prec) as ctx:
            it = start(ctx, w, pmc=0)
            for k in range(steps):
                D.dynamics_iteration(ctx, it + k, w.deltat, w.n_imp)
            den = ctx.download("den")
            res[prec] = (ctx.energy()["etot"] / w.n4, np.sqrt(np.sum(den * den)), ctx.download("rimp")[0, 2])
    e64, em = res["f64"], res["mixed"]
    assert abs(em[0] - e64[0]) < 1e-5, (em[0], e64[0])          # K per atom
    assert abs(em[1] - e64[1]) < 1e-6 * e64[1]
    assert abs(em[2] - e64[2]) < 1e-6                            # A
