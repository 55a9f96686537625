"""Learned warm start: the hand-written MPNN kernels against the CPU oracle
(forward and gradients), the solver's SDPAB_INIT_DUAL start, and what a
trained network gains over the standard start."""
import numpy as np
import pytest

from golden_util import rel

pytestmark = pytest.mark.gpu


def _graphs(seeds, nmin=12, nmax=24):
    from sdpa_b200 import warmstart as W
    return [W.batch_graph(s, nmin, nmax) for s in seeds]


def test_mpnn_forward_and_gradients_match_oracle():
    from oracle import mpnn_ref as R
    from sdpa_b200 import warmstart as W
    graphs = _graphs(range(5))
    gb = W.make_graph_batch(graphs)
    rng = np.random.default_rng(3)
    target = rng.uniform(1.0, 2.0, gb.num_nodes).astype(np.float32)
    mask = (rng.random(gb.num_nodes) < 0.9).astype(np.float32)
    model = W.MPNN(seed=5)
    dg = W.DeviceGraphs(gb, mask, target)
    r = model.forward(dg).cpu().numpy()
    w = model.state()
    A = R.adjacency(gb.num_nodes, gb.rowptr, gb.col, gb.aval)
    r_ref, _ = R.forward(w, gb.feat, A)
    assert np.max(np.abs(r - r_ref)) <= 1e-4 * max(1.0, np.max(np.abs(r_ref)))
    loss = float(model.loss_grad(dg).item())
    g = model.grads.cpu().numpy()
    loss_ref, g_ref = R.loss_grad(w, gb.feat, A, target.astype(np.float64), mask.astype(np.float64))
    assert abs(loss - loss_ref) <= 1e-4 * max(1.0, loss_ref)
    # FP32 accumulation vs float64: relative to the largest gradient entry
    assert np.max(np.abs(g - g_ref)) <= 1e-3 * np.max(np.abs(g_ref))


def test_dual_start_from_exact_solution_saves_iterations():
    from sdpa_b200 import warmstart as W
    graphs = _graphs(range(100, 116), 40, 90)
    P, cold = W.solve_graphs(graphs)
    xs = [cold.x_of(P, q).copy() for q in range(P.count)]
    P2, warm = W.solve_graphs(graphs, init_x=xs)
    assert np.all(warm.phase == 7) and np.all(warm.status == 0)
    for q in range(P.count):
        assert rel(warm.primal_obj[q], cold.primal_obj[q]) < 1e-6
        assert np.max(np.abs(warm.x_of(P2, q) - cold.x_of(P, q))) < 1e-5
    assert warm.iterations.mean() < cold.iterations.mean() - 3


def test_dual_start_outside_its_class_falls_back():
    from sdpa_b200 import batch, instances
    insts = [instances.lovasz_theta(20, 0.5, 1)]
    P = batch.pack(insts)
    cold = batch.solve_host(P)
    warm = batch.solve_host(P, init=(np.array([2], np.int32), np.ones(P.nvec), None, None))
    assert warm.status[0] == 1 and warm.phase[0] == 7
    assert warm.iterations[0] == cold.iterations[0]
    assert rel(warm.primal_obj[0], cold.primal_obj[0]) < 1e-12


def test_trained_network_reduces_iterations():
    """Train on solver-generated solutions, then compare held-out solves from
    the network's proposal against the standard start (same tolerance)."""
    from sdpa_b200 import warmstart as W
    train_g = [W.batch_graph(s, 40, 100) for s in range(1000, 1600)]
    P, sol = W.solve_graphs(train_g)
    t, m = W.targets_from_solution(train_g, P, sol)
    model = W.MPNN(seed=0)
    hist = W.train(model, train_g, t, m, epochs=12, batch_graphs=64, lr=3e-3)
    assert hist[-1] < 0.25 * hist[0]
    test_g = [W.batch_graph(s, 40, 100) for s in range(50000, 50064)]
    Pc, cold = W.solve_graphs(test_g)
    Pw, warm = W.solve_graphs(test_g, init_x=W.propose_x(model, test_g))
    assert np.all(warm.phase == 7)
    for q in range(Pc.count):
        assert rel(warm.primal_obj[q], cold.primal_obj[q]) < 1e-6
    assert warm.iterations.mean() < cold.iterations.mean() - 1.0


@pytest.mark.parametrize("precision", [0, 1])
def test_shipped_network_warm_start_parity_heldout(precision):
    """The shipped network (sdpa_b200/data) through the device pipeline
    (network -> proposal kernel -> batched solver) on the held-out seeds:
    pdOPT everywhere, objectives within 1e-6 of the reference, x at least as
    close to the reference's tight optimum as the reference's own x, and
    fewer iterations than the reference needed."""
    import torch
    from sdpa_b200 import batch as B
    from sdpa_b200 import warmstart as W
    from golden_util import tight, x_within_reference_accuracy
    meta, tz = tight()
    names = sorted(meta["heldout_default"], key=lambda k: int(k[2:]))
    graphs = [W.batch_graph(int(nm[2:]), 50, 200) for nm in names]
    P = B.pack([g.instance() for g in graphs])
    db = B.DeviceBatch(P)
    pipe = W.WarmPipeline(W.default_model(), graphs, db)
    pipe.run(precision=precision)
    torch.cuda.synchronize()
    r = db.result()
    iters_ref = []
    for q, nm in enumerate(names):
        g = meta["heldout_default"][nm]
        iters_ref.append(g["iterations"])
        assert r.phase[q] == 7, nm
        assert rel(r.primal_obj[q], g["primal_obj"]) < 1e-6, nm
        assert rel(r.dual_obj[q], g["dual_obj"]) < 1e-6, nm
        assert x_within_reference_accuracy(r.x_of(P, q), tz[nm + ".xvec"], tz[nm + ".tight"]), nm
    assert r.iterations.mean() < np.mean(iters_ref) - 2.0
