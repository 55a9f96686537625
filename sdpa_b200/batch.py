"""Batched solve of many small SDPs through the C ABI
(sdpab_batch_solve / sdpab_batch_solve_host).

`pack(instances)` turns `Instance`s into the flat arrays of `sdpab_batch`.
An instance with several blocks (SDP blocks and an LP block, as in a .dat-s
bLOCKsTRUCT) has its blocks laid along the diagonal of one n x n matrix,
n = sum |size|, and carries the block orders.  A batch carries a block
structure (which selects the solver with block support and F1 Schur
columns) when an instance has several blocks, or one block of order above
200, or a constraint with more than 2n effective entries (the cases where
the reference's formula choice can pick F1); a batch of MaxCut-like
instances passes none and runs the F3-only solver.  `solve_host` runs the host-pointer
entry point (copies
inside the call); `DeviceBatch` keeps a packed batch resident in device
memory (torch tensors as allocation plumbing only) and solves it with the
device-pointer entry point on a given stream.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native as N
from .instances import Instance


@dataclass
class Packed:
    count: int
    nmax: int
    mmax: int
    n: np.ndarray          # int32
    m: np.ndarray          # int32
    vec_off: np.ndarray    # int64
    b: np.ndarray          # float64
    mat_off: np.ndarray    # int64
    mat_ptr: np.ndarray    # int64
    row: np.ndarray        # int32 (0-based)
    col: np.ndarray        # int32
    val: np.ndarray        # float64
    dense_off: np.ndarray  # int64
    nvec: int
    nden: int
    nblock: np.ndarray | None = None    # int32 [count] (None: every instance is one SDP block)
    blk_off: np.ndarray | None = None   # int32 [count] offset into blk_size
    blk_size: np.ndarray | None = None  # int32 signed block orders (negative = LP)

    def arrays(self):
        """The sdpab_batch arrays in field order (None where absent)."""
        return [getattr(self, k) for k in _ARRAYS]

    def h2d_bytes(self) -> int:
        return sum(a.nbytes for a in self.arrays() if a is not None) + 4 * self.count

    def blocks_of(self, q: int) -> list[int]:
        if self.nblock is None:
            return [int(self.n[q])]
        o = int(self.blk_off[q])
        return [int(x) for x in self.blk_size[o:o + int(self.nblock[q])]]


_ARRAYS = ("n", "m", "vec_off", "b", "mat_off", "mat_ptr", "row", "col", "val", "dense_off", "nblock", "blk_off",
           "blk_size")


def _needs_general(it: Instance) -> bool:
    """Several blocks, a block of order > 200, or a constraint whose
    NonZeroEffect (diagonal 1, off-diagonal 2) exceeds 2n."""
    if len(it.blocks) != 1 or int(it.blocks[0]) < 2:
        return True
    n = int(it.blocks[0])
    if n > 200:
        return True
    sel = it.k > 0
    eff = np.bincount(it.k[sel], weights=np.where(it.i[sel] == it.j[sel], 1.0, 2.0), minlength=it.m + 1)
    return bool(eff.max(initial=0.0) > 2 * n)


def pack(instances: list[Instance]) -> Packed:
    cnt = len(instances)
    n = np.zeros(cnt, np.int32)
    m = np.zeros(cnt, np.int32)
    vec_off = np.zeros(cnt, np.int64)
    mat_off = np.zeros(cnt, np.int64)
    dense_off = np.zeros(cnt, np.int64)
    bs, ptrs, rows, cols, vals = [], [], [], [], []
    structured = any(_needs_general(it) for it in instances)
    nblock = np.zeros(cnt, np.int32)
    blk_off = np.zeros(cnt, np.int32)
    sizes = []
    nv = npn = ne = nd = 0
    for q, it in enumerate(instances):
        blocks = [int(x) for x in it.blocks]
        if not blocks or any(x == 0 for x in blocks) or len(blocks) > N.BATCH_MAX_BLOCKS:
            raise ValueError(f"instance {q}: 1..{N.BATCH_MAX_BLOCKS} blocks of non-zero order are supported")
        offs = np.concatenate([[0], np.cumsum(np.abs(blocks))]).astype(np.int64)
        nb = int(offs[-1])
        n[q], m[q] = nb, it.m
        nblock[q], blk_off[q] = len(blocks), len(sizes)
        sizes.extend(blocks)
        vec_off[q], mat_off[q], dense_off[q] = nv, npn, nd
        order = np.lexsort((it.j, it.i, it.l, it.k))
        k = it.k[order]
        base = offs[it.l[order] - 1]
        r = base + it.i[order] - 1
        c = base + it.j[order] - 1
        v = it.v[order]
        # entries are stored upper-triangular
        sw = r > c
        r2 = np.where(sw, c, r)
        c2 = np.where(sw, r, c)
        counts = np.bincount(k, minlength=it.m + 1)
        ptr = ne + np.concatenate([[0], np.cumsum(counts)])
        bs.append(np.asarray(it.c, np.float64))
        ptrs.append(ptr.astype(np.int64))
        rows.append(r2.astype(np.int32))
        cols.append(c2.astype(np.int32))
        vals.append(v.astype(np.float64))
        nv += it.m
        npn += it.m + 2
        ne += k.size
        nd += nb * nb
    P = Packed(cnt, int(n.max()), int(m.max()), n, m, vec_off, np.concatenate(bs), mat_off,
               np.concatenate(ptrs), np.concatenate(rows), np.concatenate(cols),
               np.concatenate(vals), dense_off, nv, nd)
    if structured:
        P.nblock, P.blk_off, P.blk_size = nblock, blk_off, np.asarray(sizes, np.int32)
    return P


@dataclass
class BatchResult:
    primal_obj: np.ndarray
    dual_obj: np.ndarray
    mu: np.ndarray
    primal_error: np.ndarray
    dual_error: np.ndarray
    iterations: np.ndarray
    phase: np.ndarray
    status: np.ndarray
    xvec: np.ndarray | None = None
    X: np.ndarray | None = None
    Y: np.ndarray | None = None

    def x_of(self, P: Packed, q: int) -> np.ndarray:
        return self.xvec[P.vec_off[q]:P.vec_off[q] + P.m[q]]

    def mat_of(self, which: np.ndarray, P: Packed, q: int) -> np.ndarray:
        nb = int(P.n[q])
        return which[P.dense_off[q]:P.dense_off[q] + nb * nb].reshape(nb, nb, order="F")

    def block_of(self, which: np.ndarray, P: Packed, q: int, l: int) -> np.ndarray:
        """Block l (0-based) of instance q's X or Y, as getResultXMat(l+1) /
        getResultYMat(l+1): the dense SDP block, or an LP block's vector."""
        M = self.mat_of(which, P, q)
        blocks = P.blocks_of(q)
        o = int(np.sum(np.abs(blocks[:l])))
        k = abs(blocks[l])
        if blocks[l] < 0:
            return np.diag(M)[o:o + k].copy()
        return M[o:o + k, o:o + k].copy()


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p).value


def _params(params):
    if params is None:
        return N.default_params(0)
    if isinstance(params, N.Params):
        return params
    p = N.default_params(0)
    for k, v in params.items():
        setattr(p, k, v)
    return p


def _config(precision=N.PREC_FP64, ctas_per_sm=0, mixed_switch_gap=0.0, staging=0, mixed_products=0,
            block_threads=0, refine_tol=0.0, factor_smem=0):
    return N.BatchConfig(precision, ctas_per_sm, mixed_switch_gap, staging, mixed_products, block_threads,
                         refine_tol, factor_smem)


def solve_host(P: Packed, params=None, precision=N.PREC_FP64, want_x=True, want_mats=False,
               init=None, ctas_per_sm=0, staging=0, block_threads=0, mixed_products=0,
               mixed_switch_gap=0.0, refine_tol=0.0, factor_smem=0) -> BatchResult:
    """sdpab_batch_solve_host on host arrays.  init = (flag, xvec, X, Y
    [, margin [, V, rank [, init_mu]]]) in the packed layouts (user X / Y as in
    SDPA::inputInitXMat / inputInitYMat; V: the SDPAB_INIT_FACTOR factors,
    instance q's n x rank rows at vec_off[q] * rank).
    The launch shape (block_threads, ctas_per_sm, staging) and the mixed
    mode's options are those of sdpab_batch_config (0 = defaults)."""
    L = N.lib()
    cnt = P.count
    arrs = [None if a is None else np.ascontiguousarray(a) for a in P.arrays()]
    bt = N.Batch(cnt, P.nmax, P.mmax, *[_ptr(a) for a in arrs])
    res = BatchResult(*[np.zeros(cnt) for _ in range(5)], *[np.zeros(cnt, np.int32) for _ in range(3)])
    res.xvec = np.zeros(P.nvec) if want_x else None
    res.X = np.zeros(P.nden) if want_mats else None
    res.Y = np.zeros(P.nden) if want_mats else None
    br = N.BatchResult(_ptr(res.xvec), _ptr(res.X), _ptr(res.Y), _ptr(res.primal_obj), _ptr(res.dual_obj),
                       _ptr(res.mu), _ptr(res.primal_error), _ptr(res.dual_error), _ptr(res.iterations),
                       _ptr(res.phase), _ptr(res.status))
    bi = None
    keep = []
    if init is not None:
        conv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        flag, xv, Xu, Yu = np.ascontiguousarray(init[0], np.int32), conv(init[1]), conv(init[2]), conv(init[3])
        margin = float(init[4]) if len(init) > 4 else 0.0
        Vf = conv(init[5]) if len(init) > 5 else None
        rank = int(init[6]) if len(init) > 6 else 0
        init_mu = float(init[7]) if len(init) > 7 else 0.0
        keep = [flag, xv, Xu, Yu, Vf]
        bi = ctypes.byref(N.BatchInit(_ptr(flag), _ptr(xv), _ptr(Xu), _ptr(Yu), margin, _ptr(Vf), rank, init_mu))
    prm = _params(params)
    cfg = _config(precision, ctas_per_sm, mixed_switch_gap, staging, mixed_products, block_threads, refine_tol,
                  factor_smem)
    N.check(L.sdpab_batch_solve_host(ctypes.byref(bt), bi, ctypes.byref(prm), ctypes.byref(cfg),
                                     ctypes.byref(br)), "sdpab_batch_solve_host")
    del keep
    return res


class DeviceBatch:
    """A packed batch resident in device memory (torch tensors hold the
    allocations), solved by sdpab_batch_solve on a CUDA stream."""

    def __init__(self, P: Packed, device="cuda", want_mats=False):
        import torch
        self.P = P
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.d = {k: t(a) for k, a in zip(_ARRAYS, P.arrays()) if a is not None}
        order = np.argsort(-(P.n.astype(np.int64) ** 2 + P.m), kind="stable").astype(np.int32)
        self.order = t(order)
        cnt = P.count
        f64 = dict(dtype=torch.float64, device=device)
        i32 = dict(dtype=torch.int32, device=device)
        self.sc = torch.zeros(5, cnt, **f64)
        self.ic = torch.zeros(3, cnt, **i32)
        self.xvec = torch.zeros(P.nvec, **f64)
        self.X = torch.zeros(P.nden, **f64) if want_mats else None
        self.Y = torch.zeros(P.nden, **f64) if want_mats else None
        self.init = None
        dp = lambda x: x.data_ptr()
        self._bt = N.Batch(cnt, P.nmax, P.mmax, *[dp(self.d[k]) if k in self.d else None for k in _ARRAYS])
        self._br = N.BatchResult(dp(self.xvec), dp(self.X) if want_mats else None,
                                 dp(self.Y) if want_mats else None,
                                 *[dp(self.sc[q]) for q in range(5)], *[dp(self.ic[q]) for q in range(3)])

    def set_init(self, flag, xvec, X=None, Y=None, margin: float = 0.0):
        """Device copies of an initial point (X, Y may be None for SDPAB_INIT_DUAL)."""
        import torch
        dev = self.xvec.device
        conv = lambda a, t: None if a is None else torch.as_tensor(np.ascontiguousarray(a, t), device=dev)
        self._init_t = [conv(flag, np.int32), conv(xvec, np.float64), conv(X, np.float64), conv(Y, np.float64)]
        self.init = N.BatchInit(*[None if x is None else x.data_ptr() for x in self._init_t], margin)

    def subset(self, order_tensor) -> "N.Batch":
        """The batch struct restricted to the instances listed (device int32
        tensor, in the order the solver takes them); pass it with that
        tensor as `order` to solve only those."""
        b = N.Batch.from_buffer_copy(self._bt)
        b.count = int(order_tensor.numel())
        return b

    def solve(self, params=None, precision=N.PREC_FP64, stream=None, ctas_per_sm=0, staging=0, block_threads=0,
              mixed_products=0, mixed_switch_gap=0.0, refine_tol=0.0, factor_smem=0, order=None):
        """block_threads / ctas_per_sm / staging: launch shape (0 = defaults;
        see sdpa_b200.autotune); mixed_products / mixed_switch_gap: options of
        the mixed mode (sdpab_batch_config); order: a device int32 tensor of
        instance indices to solve only those, in that order (default: all,
        largest first)."""
        import torch
        prm = _params(params)
        cfg = _config(precision, ctas_per_sm, mixed_switch_gap, staging, mixed_products, block_threads, refine_tol,
                      factor_smem)
        s = stream if stream is not None else torch.cuda.current_stream()
        bt = self._bt if order is None else self.subset(order)
        od = self.order if order is None else order
        N.check(N.lib().sdpab_batch_solve(ctypes.byref(bt),
                                          ctypes.byref(self.init) if self.init is not None else None,
                                          ctypes.byref(prm), ctypes.byref(cfg), ctypes.byref(self._br),
                                          od.data_ptr(), s.cuda_stream), "sdpab_batch_solve")

    def result(self) -> BatchResult:
        sc = self.sc.cpu().numpy()
        ic = self.ic.cpu().numpy()
        r = BatchResult(*sc, *ic)
        r.xvec = self.xvec.cpu().numpy()
        if self.X is not None:
            r.X = self.X.cpu().numpy()
            r.Y = self.Y.cpu().numpy()
        return r
