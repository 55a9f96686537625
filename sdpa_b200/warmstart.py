"""Learned warm start for batched MaxCut SDPs.

A 3-layer message-passing network (sdpa_b200/csrc/mpnn.cu: BF16 weights,
FP32 accumulation, hand-written forward/backward/Adam kernels driven through
the C ABI) predicts per node r_i = 4 x_i / d_i, where x is SDPA's x vector of
the MaxCut SDP and d the weighted degree.  The proposed x goes to the batched
solver with flag SDPAB_INIT_DUAL, which shifts it until X = diag(x) - L/4 is
strictly positive definite, sets Y = D X^-1 D with unit diagonal, and falls
back to the standard start otherwise; the interior-point method always runs
to its own tolerance.  Training targets are solutions the solver itself
produces.  torch tensors are used only as device allocations.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from . import batch as B
from . import instances as I

H = 64
F0 = 8
INIT_DUAL = 2


@dataclass
class Graph:
    n: int
    ei: np.ndarray
    ej: np.ndarray
    w: np.ndarray

    @property
    def degree(self) -> np.ndarray:
        d = np.zeros(self.n)
        np.add.at(d, self.ei, self.w)
        np.add.at(d, self.ej, self.w)
        return d

    def instance(self) -> I.Instance:
        return I.maxcut_from_graph(self.n, self.ei, self.ej, self.w)


def batch_graph(seed: int, nmin: int = 50, nmax: int = 200) -> Graph:
    return Graph(*I.batch_maxcut_graph(seed, nmin, nmax))


def node_features(g: Graph) -> np.ndarray:
    """Eight per-node features: weighted degree and edge count (relative to the
    graph means), graph size and density, a standardised degree, sqrt degree,
    and a constant."""
    n = g.n
    d = g.degree
    k = np.zeros(n)
    np.add.at(k, g.ei, 1.0)
    np.add.at(k, g.ej, 1.0)
    md, mk = max(d.mean(), 1e-9), max(k.mean(), 1e-9)
    f = np.empty((n, F0), np.float32)
    f[:, 0] = d / md
    f[:, 1] = k / mk
    f[:, 2] = np.log(n) / 5.0
    f[:, 3] = md / n * 4.0
    f[:, 4] = mk / n * 4.0
    f[:, 5] = (d - md) / (d.std() + 1e-9)
    f[:, 6] = np.sqrt(d / md)
    f[:, 7] = 1.0
    return f


@dataclass
class GraphBatch:
    """Host arrays of a batch of graphs in the layout of sdpab_graph_batch."""
    num_nodes: int
    rowptr: np.ndarray
    col: np.ndarray
    aval: np.ndarray
    aval_t: np.ndarray
    feat: np.ndarray
    offsets: np.ndarray   # node offset of every graph
    degree: np.ndarray    # weighted degree per node


def make_graph_batch(graphs: list[Graph]) -> GraphBatch:
    rows, cols, av, avt, feats, degs, offs = [], [], [], [], [], [], []
    off = 0
    for g in graphs:
        d = g.degree
        src = np.concatenate([g.ei, g.ej])
        dst = np.concatenate([g.ej, g.ei])
        w = np.concatenate([g.w, g.w])
        rows.append(dst + off)
        cols.append(src + off)
        av.append(w / (d[dst] + 1.0))
        avt.append(w / (d[src] + 1.0))
        feats.append(node_features(g))
        degs.append(d)
        offs.append(off)
        off += g.n
    dst = np.concatenate(rows)
    order = np.argsort(dst, kind="stable")
    dst = dst[order]
    col = np.concatenate(cols)[order].astype(np.int32)
    aval = np.concatenate(av)[order].astype(np.float32)
    aval_t = np.concatenate(avt)[order].astype(np.float32)
    rowptr = np.zeros(off + 1, np.int64)
    np.add.at(rowptr, dst + 1, 1)
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return GraphBatch(off, rowptr, col, aval, aval_t, np.concatenate(feats).astype(np.float32),
                      np.array(offs, np.int64), np.concatenate(degs))


class DeviceGraphs:
    """A GraphBatch resident on the GPU plus the sdpab_graph_batch view."""

    def __init__(self, gb: GraphBatch, mask: np.ndarray | None = None, target: np.ndarray | None = None):
        import torch
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        self.gb = gb
        self.rowptr, self.col = t(gb.rowptr), t(gb.col)
        self.aval, self.aval_t, self.feat = t(gb.aval), t(gb.aval_t), t(gb.feat)
        self.mask = t(mask.astype(np.float32)) if mask is not None else None
        self.target = t(target.astype(np.float32)) if target is not None else None
        mc = int(mask.sum()) if mask is not None else 0
        self.c = N.GraphBatch(gb.num_nodes, int(gb.col.size), self.rowptr.data_ptr(), self.col.data_ptr(),
                              self.aval.data_ptr(), self.aval_t.data_ptr(), self.feat.data_ptr(), mc)


class MPNN:
    """Parameters (FP32 master + BF16 working copy) and the C ABI calls."""

    def __init__(self, seed: int = 0):
        import torch
        self.L = N.lib()
        self.P = int(self.L.sdpab_mpnn_num_params())
        rng = np.random.default_rng(seed)
        w = np.zeros(self.P, np.float32)
        off = 0
        for l in range(3):
            fin = F0 if l == 0 else H
            for _ in range(2):
                w[off:off + H * fin] = rng.standard_normal(H * fin) * np.sqrt(1.0 / (2 * fin))
                off += H * fin
            off += H  # bias 0
        w[off:off + H] = rng.standard_normal(H) * np.sqrt(1.0 / H)
        w[off + H] = 1.3  # typical ratio
        self.master = torch.from_numpy(w).cuda()
        self.wb = torch.zeros(self.P, dtype=torch.int16, device="cuda")
        self.m1 = torch.zeros_like(self.master)
        self.m2 = torch.zeros_like(self.master)
        self.grads = torch.zeros_like(self.master)
        self.step = 0
        self._sync_bf16()

    def _sync_bf16(self):
        N.check(self.L.sdpab_mpnn_to_bf16(self.master.data_ptr(), self.wb.data_ptr(), None), "mpnn_to_bf16")

    def forward(self, dg: DeviceGraphs, act=None, out=None, stream=None):
        import torch
        n = dg.gb.num_nodes
        if act is None:
            act = torch.empty(int(self.L.sdpab_mpnn_act_floats(n)), dtype=torch.float32, device="cuda")
        if out is None:
            out = torch.empty(n, dtype=torch.float32, device="cuda")
        N.check(self.L.sdpab_mpnn_forward(ctypes.byref(dg.c), self.wb.data_ptr(), act.data_ptr(),
                                          out.data_ptr(), stream), "mpnn_forward")
        return out

    def loss_grad(self, dg: DeviceGraphs):
        import torch
        n = dg.gb.num_nodes
        act = torch.empty(int(self.L.sdpab_mpnn_act_floats(n)), dtype=torch.float32, device="cuda")
        scr = torch.empty(int(self.L.sdpab_mpnn_scratch_floats(n)), dtype=torch.float32, device="cuda")
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        N.check(self.L.sdpab_mpnn_loss_grad(ctypes.byref(dg.c), self.wb.data_ptr(), act.data_ptr(),
                                            scr.data_ptr(), dg.target.data_ptr(),
                                            dg.mask.data_ptr() if dg.mask is not None else None,
                                            self.grads.data_ptr(), loss.data_ptr(), None), "mpnn_loss_grad")
        return loss

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
        self.step += 1
        N.check(self.L.sdpab_mpnn_adam(self.master.data_ptr(), self.wb.data_ptr(), self.grads.data_ptr(),
                                       self.m1.data_ptr(), self.m2.data_ptr(), self.step, lr, b1, b2, eps, wd,
                                       None), "mpnn_adam")

    def state(self) -> np.ndarray:
        return self.master.cpu().numpy().copy()

    def load(self, w: np.ndarray):
        import torch
        self.master.copy_(torch.from_numpy(np.asarray(w, np.float32)))
        self._sync_bf16()


class WarmPipeline:
    """Device-resident warm-started batched solve: network forward, proposal
    kernel and the persistent solver, all on one stream (capturable in a CUDA
    graph).  The graphs must be in the order of the packed batch."""

    def __init__(self, model: MPNN, graphs: list[Graph], db: "B.DeviceBatch", margin: float = 0.0):
        import torch
        self.model, self.db = model, db
        gb = make_graph_batch(graphs)
        self.dg = DeviceGraphs(gb)
        n = gb.num_nodes
        assert n == db.P.nvec, "graph nodes must match the packed constraints"
        fb = np.empty(n)
        for q, g in enumerate(graphs):
            o = gb.offsets[q]
            d = gb.degree[o:o + g.n]
            fb[o:o + g.n] = 0.01 * max(d.mean() / 4.0, 1e-3)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        self.degree, self.fallback = t(gb.degree.astype(np.float64)), t(fb)
        self.act = torch.empty(int(N.lib().sdpab_mpnn_act_floats(n)), dtype=torch.float32, device="cuda")
        self.r = torch.empty(n, dtype=torch.float32, device="cuda")
        self.xprop = torch.zeros(n, dtype=torch.float64, device="cuda")
        self.flag = torch.full((db.P.count,), INIT_DUAL, dtype=torch.int32, device="cuda")
        db.init = N.BatchInit(self.flag.data_ptr(), self.xprop.data_ptr(), None, None, margin)
        self.n = n

    def run(self, precision=N.PREC_FP64, stream=None, **shape):
        """shape: launch shape and mixed-mode options of DeviceBatch.solve."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        self.model.forward(self.dg, self.act, self.r, s.cuda_stream)
        N.check(N.lib().sdpab_mpnn_propose_x(self.n, self.r.data_ptr(), self.degree.data_ptr(),
                                             self.fallback.data_ptr(), self.xprop.data_ptr(), s.cuda_stream),
                "mpnn_propose_x")
        self.db.solve(precision=precision, stream=s, **shape)


def default_model() -> MPNN:
    """The network trained by sdpa_b200.train_warmstart (weights in sdpa_b200/data)."""
    import os
    m = MPNN(seed=0)
    m.load(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "mpnn_maxcut.npy")))
    return m


def solve_graphs(graphs: list[Graph], precision=N.PREC_FP64, init_x: list | None = None, margin: float = 0.0):
    """Batched solve (host-pointer C ABI) of the MaxCut SDPs of `graphs`;
    init_x: proposed x per graph (SDPAB_INIT_DUAL)."""
    P = B.pack([g.instance() for g in graphs])
    init = None
    if init_x is not None:
        flag = np.full(P.count, INIT_DUAL, np.int32)
        xv = np.zeros(P.nvec)
        for q, x in enumerate(init_x):
            xv[P.vec_off[q]:P.vec_off[q] + P.m[q]] = x
        init = (flag, xv, None, None, margin)
    return P, B.solve_host(P, precision=precision, init=init)


def targets_from_solution(graphs: list[Graph], P, res) -> tuple[np.ndarray, np.ndarray]:
    """r_i = 4 x_i / d_i with a mask of the nodes that have edges."""
    ts, ms = [], []
    for q, g in enumerate(graphs):
        x = res.x_of(P, q)
        d = g.degree
        m = d > 1e-9
        t = np.where(m, 4.0 * x / np.maximum(d, 1e-9), 0.0)
        ts.append(t)
        ms.append(m.astype(np.float32))
    return np.concatenate(ts).astype(np.float32), np.concatenate(ms)


def propose_x(model: MPNN, graphs: list[Graph]) -> list[np.ndarray]:
    """Network proposal of x for every graph (x_i = r_i d_i / 4; isolated
    nodes get a small positive value)."""
    gb = make_graph_batch(graphs)
    dg = DeviceGraphs(gb)
    r = model.forward(dg).cpu().numpy().astype(np.float64)
    out = []
    for q, g in enumerate(graphs):
        o = gb.offsets[q]
        d = gb.degree[o:o + g.n]
        scale = max(d.mean() / 4.0, 1e-3)
        out.append(np.where(d > 1e-9, r[o:o + g.n] * d / 4.0, 0.01 * scale))
    return out


def train(model: MPNN, graphs: list[Graph], targets: np.ndarray, masks: np.ndarray, epochs: int = 30,
          batch_graphs: int = 256, lr: float = 2e-3, seed: int = 0, log=None):
    """Minibatch Adam over graphs (cosine learning-rate decay).  The graphs
    are grouped into fixed batches once, kept on the device, and the batch
    order is shuffled every epoch.  Returns the per-epoch mean loss."""
    rng = np.random.default_rng(seed)
    offs = np.concatenate([[0], np.cumsum([g.n for g in graphs])])
    idx = np.arange(len(graphs))
    rng.shuffle(idx)
    dev_batches = []
    for b0 in range(0, len(idx), batch_graphs):
        sel = idx[b0:b0 + batch_graphs]
        gb = make_graph_batch([graphs[s] for s in sel])
        t = np.concatenate([targets[offs[s]:offs[s + 1]] for s in sel])
        m = np.concatenate([masks[offs[s]:offs[s + 1]] for s in sel])
        dev_batches.append(DeviceGraphs(gb, m, t))
    hist = []
    order = np.arange(len(dev_batches))
    for ep in range(epochs):
        rng.shuffle(order)
        cur_lr = lr * (0.5 * (1 + np.cos(np.pi * ep / max(epochs, 1))))
        losses = []
        for b in order:
            losses.append(model.loss_grad(dev_batches[b]))
            model.adam(lr=float(cur_lr))
        hist.append(float(sum(float(x.item()) for x in losses) / max(len(losses), 1)))
        if log:
            log(f"epoch {ep} loss {hist[-1]:.5f}")
    return hist
