"""The quantum batch step replayed from CUDA graphs (bench.py --workload quantum): a cycle of
captured steps, replayed, leaves exactly the state that the same steps launched one by one
leave.  The cycle is found with he_state_fingerprint (the ring buffers' relabelling repeats)."""
import numpy as np
import pytest
import torch

from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200.context import Context

pytestmark = pytest.mark.gpu


def small_quantum():
    w = C.quantum_2000(n=32)
    return C.replace(w, xmax=12.0, ymax=12.0, zmax=12.0, n4=300, n_spline=10001,
                     deltatps=5e-4, nq_imp=1, mq_imp_u=(23.0,), psix_center=((0.0, 0.0, 0.0),),
                     psix_kick_aps=((0.0, 1.0, 2.0),))


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_graph_cycle_replays_eager_steps(precision):
    w = small_quantum()
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    psix = [C.psix_initial(w, 0)]
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctxs = []
    for _ in range(2):
        c = Context(w, mode="quantum", precision=precision)
        # the same FFT variants in both contexts (each autotunes on its own timings otherwise)
        c.set_fft_variant("x", 0, 8)
        c.set_fft_variant("y", 1, 8)
        c.set_fft_variant("z", 0, 8)
        c.set_stream(stream.cuda_stream)
        D.quantum_setup(c, psi, psix)
        for it in range(1, 6):
            D.quantum_iteration(c, it, w.deltat)
        ctxs.append(c)
    eager, graphed = ctxs
    start = graphed.state_fingerprint()  # (of this context's own buffers)
    graphs = []
    for _ in range(64):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
            D.quantum_iteration(graphed, 6, w.deltat)
        graphs.append(g)
        if graphed.state_fingerprint() == start:
            break
    assert graphed.state_fingerprint() == start, "no cycle within 64 steps"
    for rep in range(2):
        for g in graphs:
            g.replay()
    for k in range(2 * len(graphs)):
        D.quantum_iteration(eager, 6 + k, w.deltat)
    torch.cuda.synchronize()
    for name in ("psi", "psix", "den", "pot4"):
        assert np.array_equal(graphed.download(name), eager.download(name)), name
    assert graphed.energy()["etot"] == eager.energy()["etot"]
    del graphs
    for c in ctxs:
        c.close()
    torch.cuda.set_stream(torch.cuda.default_stream())


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_graph_cycle_replays_eager_classical_steps(precision):
    """The classical step (impurity work forked onto the side stream and joined with he_join at
    the end of each recorded step) replayed from a captured cycle equals the eager steps."""
    w = C.tddft_1000(n=32)
    w = C.replace(w, xmax=10.0, ymax=10.0, zmax=10.0, n4=300, rimp0=((0.5, -0.3, 8.0),),
                  deltatps=2e-4)
    den = C.woods_saxon(w)
    psi = D.initial_wavefunction(w, den)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctxs = []
    for _ in range(2):
        c = Context(w, precision=precision)
        c.set_stream(stream.cuda_stream)
        D.dynamics_setup(c, psi, w.n_imp)
        for it in range(1, 6):
            D.dynamics_iteration(c, it, w.deltat, w.n_imp)
        ctxs.append(c)
    eager, graphed = ctxs
    graphed.join()  # pending side-stream work of the eager steps, outside the recording
    start = graphed.state_fingerprint()
    graphs = []
    for _ in range(64):
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream, capture_error_mode="relaxed"):
            D.dynamics_iteration(graphed, 6, w.deltat, w.n_imp)
            graphed.join()
        graphs.append(g)
        if graphed.state_fingerprint() == start:
            break
    assert graphed.state_fingerprint() == start, "no cycle within 64 steps"
    for rep in range(2):
        for g in graphs:
            g.replay()
    for k in range(2 * len(graphs)):
        D.dynamics_iteration(eager, 6 + k, w.deltat, w.n_imp)
    torch.cuda.synchronize()
    for name in ("psi", "den", "pot4", "rimp", "vimp"):
        assert np.array_equal(graphed.download(name), eager.download(name)), name
    assert graphed.energy()["etot"] == eager.energy()["etot"]
    del graphs
    for c in ctxs:
        c.close()
    torch.cuda.set_stream(torch.cuda.default_stream())


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_statics_iterations_match_per_iteration_calls(precision):
    """he_statics_iterations (passes replayed from per-relabelling graphs, one host read at the
    end) against the driver's own per-iteration steppcr + refresh + poten calls: identical
    mu, mu4err, errpc and fields after 46 passes, i.e. past one 30-pass relabelling cycle."""
    w = C.statics_500()  # 64^3
    den0 = C.woods_saxon(w)
    dt = w.deltat_statics
    out = []
    for batched in (False, True):
        with Context(w, mode="statics", precision=precision) as ctx:
            ctx.set_fft_variant("x", 0, 8)  # both contexts on the same kernels
            ctx.set_fft_variant("y", 1, 8)
            ctx.set_fft_variant("z", 0, 8)
            mu = D.statics_setup(ctx, den0, w.n4)
            it = 1
            for _ in range(5):  # the 4 RK iterations and the first predictor-corrector one
                mu, _ = D.statics_iteration(ctx, it, dt, mu, w.n4)
                it += 1
            l0 = ctx.launches
            if batched:
                mu, err = ctx.statics_iterations(1, dt, mu, w.n4)    # the eager first pass
                mid = ctx.statics_iterations(44, dt, mu, w.n4)       # captures the cycle, replays
                mu, err = ctx.statics_iterations(1, dt, mid[0], w.n4)
            else:
                for k in range(46):
                    mu, err = D.statics_iteration(ctx, it, dt, mu, w.n4)
                    it += 1
                    if k == 44:
                        mid = (mu, err)
            out.append((mu, err, ctx.errpc, ctx.download("psi"), ctx.download("den"),
                        ctx.download("pot4"), ctx.launches - l0, mid))
    (mu_e, err_e, pc_e, psi_e, den_e, pot_e, l_e, mid_e) = out[0]
    (mu_b, err_b, pc_b, psi_b, den_b, pot_b, l_b, mid_b) = out[1]
    assert mid_b == mid_e  # mu4err of a batch from the pass before its last, kept on the device
    assert mu_b == mu_e and err_b == err_e and pc_b == pc_e
    assert np.array_equal(psi_b, psi_e)
    assert np.array_equal(den_b, den_e)
    assert np.array_equal(pot_b, pot_e)
    assert l_b == l_e + 46  # plus the one slot copy per pass
