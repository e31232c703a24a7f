"""Served trajectories on the device (he_dft_2024_b200/serving.py): a trajectory advanced by the
continuous-batching scheduler, on a context that served other trajectories before it, ends in
the same state as the same request run alone in a fresh context, in binary64 and in the mixed
precision path."""
import numpy as np
import pytest

from he_dft_2024_b200 import driver as D
from he_dft_2024_b200 import serving as S
from he_dft_2024_b200.context import Context

pytestmark = pytest.mark.gpu


def small_requests():
    out = []
    for i, (n4, speed) in enumerate(((60, 200.0), (80, 450.0), (70, 120.0))):
        r = S.Request(rid=i, arrival_s=0.01 * i, n4=n4, speed_ms=speed, steps=7)
        r.n, r.h = 32, 0.7
        out.append(r)
    return out


def make_context(w, precision):
    """A context with the FFT pass variants pinned: each context's autotuner picks its own
    variants, and in binary32 different variants round differently, so the served and the
    standalone run are compared on the same kernels."""
    ctx = Context(w, precision=precision)
    ctx.set_fft_variant("x", 0, 8)
    ctx.set_fft_variant("y", 1, 8)
    ctx.set_fft_variant("z", 0, 8)
    return ctx


def alone(r, precision="f64"):
    w = r.workload()
    with make_context(w, precision) as ctx:
        S.start_trajectory(ctx, w)
        for it in range(1, r.steps + 1):
            D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
        return ctx.download("rimp"), ctx.energy()


@pytest.mark.parametrize("precision", ["f64", "mixed"])
@pytest.mark.parametrize("budget_gb", [100.0, 1e-3])
def test_served_trajectories_match_standalone_runs(budget_gb, precision):
    reqs = small_requests()
    srv = S.Server(lambda w: make_context(w, precision), hbm_budget_gb=budget_gb)
    rep = srv.run(reqs)
    assert rep["requests"] == 3 and rep["grid_pt_steps_per_s"] > 0
    if budget_gb < 1:
        assert srv.peak_active == 1  # one context served all three, one after the other
    for r in reqs:
        rimp, e = alone(r, precision)
        np.testing.assert_allclose(r.final["rimp"], rimp, rtol=1e-12, atol=1e-14)
        for k in ("etot", "etot4", "ekin4", "eHeX", "ekinx"):
            assert abs(r.final["energy"][k] - e[k]) <= 1e-12 * max(abs(e[k]), 1.0), (k, r.rid)
