"""The CPU oracle of the warm-start network checks itself: analytic
gradients against central finite differences (float64), and the parameter
layout against the C ABI's parameter count."""
import numpy as np

from oracle import mpnn_ref as R


def _small_graph(seed=0, n=9):
    rng = np.random.default_rng(seed)
    A = np.zeros((n, n))
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.size) < 0.5
    w = rng.uniform(0.1, 1.0, keep.sum())
    W = np.zeros((n, n))
    W[iu[keep], ju[keep]] = w
    W = W + W.T
    d = W.sum(1)
    A = W / (d[:, None] + 1.0)
    feat = rng.standard_normal((n, R.F0))
    return A, feat


def test_oracle_gradient_matches_finite_differences():
    _, _, npar = R.offsets()
    rng = np.random.default_rng(1)
    # weights exactly representable in BF16 so the rounding is the identity
    w = R.bf16_round(rng.standard_normal(npar).astype(np.float32) * 0.2)
    A, feat = _small_graph()
    t = rng.standard_normal(A.shape[0])
    mask = (rng.random(A.shape[0]) < 0.8).astype(float)
    loss, g = R.loss_grad(w, feat, A, t, mask)
    idx = rng.choice(npar, 40, replace=False)
    for k in idx:
        # central difference on the float64 network (no BF16 rounding of the step)
        h = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[k] += h
        wm[k] -= h
        lp = _loss64(wp, feat, A, t, mask)
        lm = _loss64(wm, feat, A, t, mask)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(1.0, abs(g[k])), (k, fd, g[k])


def _loss64(w, feat, A, t, mask):
    offs, oo, _ = R.offsets()
    h = feat
    for l, (ws, wn, b) in enumerate(offs):
        Ws = w[ws:wn].reshape(R.H, R.fin(l))
        Wn = w[wn:b].reshape(R.H, R.fin(l))
        h = np.maximum(h @ Ws.T + (A @ h) @ Wn.T + w[b:b + R.H], 0.0)
    r = h @ w[oo:oo + R.H] + w[oo + R.H]
    d = (r - t) * mask
    return float(np.sum(d * d) / mask.sum())


def test_parameter_count_matches_abi():
    from sdpa_b200 import _native as N
    _, _, npar = R.offsets()
    assert N.lib().sdpab_mpnn_num_params() == npar
