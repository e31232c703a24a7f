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
