"""Low-rank warm start of MaxCut-type batches (SDPAB_INIT_FACTOR).

For instances whose constraints are X_ii = b_i (one SDP block, m = n), the
dual problem max <F0, Y> s.t. Y_ii = b_i, Y >= 0 is solved approximately in
the factored form Y = V V^T by the mixing method (sdpab_lowrank_factor, one
warp per instance), and the interior-point method starts near its central
path from V (the SDPAB_INIT_FACTOR start of sdpab_batch_solve): the start
is centred and within 3e-6 to about 1e-4 (relative, set by the factor's
accuracy) of optimal, so the solve to a relative gap of 1e-7 takes about
three iterations instead of about fourteen from lambda* I.  The
interior-point method still runs to its own tolerance; the factor only moves
its starting point.  Nothing of this is in the reference, which starts from
lambda* I or from a given point.

`FactorPipeline` issues the factor and the solve on one stream, so the pair
can be captured in one CUDA graph.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N

INIT_FACTOR = 3
DEFAULT_SWEEPS = 220
DEFAULT_TOL = 1e-10
DEFAULT_MU = 3e-6


class FactorPipeline:
    """Mixing-method factor + persistent solver from the factor start, for a
    resident DeviceBatch.  Instances not of the form X_ii = b_i report
    sweeps -1 and take the standard start (status 1)."""

    def __init__(self, db, rank: int = 0, max_sweeps: int = DEFAULT_SWEEPS, tol: float = DEFAULT_TOL,
                 init_mu: float = DEFAULT_MU, seed: int = 1, work_quantile: float = 0.0):
        """work_quantile q in (0, 1]: the instances with more work per sweep
        (rows plus neighbour records) than the q-quantile of the batch get
        proportionally fewer sweeps, so that none takes longer than
        max_sweeps sweeps of that quantile (0: no such cap)."""
        import torch
        self.db = db
        P = db.P
        L = N.lib()
        self.rank = int(rank) if rank > 0 else int(L.sdpab_lowrank_default_rank(P.nmax))
        self.max_sweeps, self.tol, self.seed = int(max_sweeps), float(tol), int(seed)
        dev = db.xvec.device
        self.V = torch.zeros(max(1, P.nvec) * self.rank, dtype=torch.float64, device=dev)
        self.sweeps = torch.zeros(P.count, dtype=torch.int32, device=dev)
        self.flag = torch.full((P.count,), INIT_FACTOR, dtype=torch.int32, device=dev)
        self.num_entries = int(db.d["val"].numel())
        # the mixing kernel's queue order: most work per sweep first (rows
        # plus neighbour records), so the longest instances start first
        f0 = P.mat_ptr[P.mat_off + 1] - P.mat_ptr[P.mat_off]
        cost = P.n.astype(np.int64) + 2 * f0.astype(np.int64)
        order = np.argsort(-cost, kind="stable").astype(np.int32)
        self.order = torch.from_numpy(order).to(dev)
        # the kernel's n + L: rows plus off-diagonal records (both triangles)
        work = 2 * f0.astype(np.int64) - P.n.astype(np.int64)
        self.sweep_work = (int(self.max_sweeps * np.quantile(work, work_quantile))
                           if 0.0 < work_quantile <= 1.0 and P.count > 0 else 0)
        db.init = N.BatchInit(self.flag.data_ptr(), None, None, None, 0.0, self.V.data_ptr(), self.rank,
                              float(init_mu))

    def factor(self, stream=None, order=None):
        """The factor of every instance (or of those in `order`)."""
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        od = self.order if order is None else order
        bt = self.db._bt if order is None else self.db.subset(order)
        N.check(N.lib().sdpab_lowrank_factor(ctypes.byref(bt), self.num_entries, self.rank,
                                             self.max_sweeps, self.tol, self.sweep_work, self.seed,
                                             self.V.data_ptr(),
                                             self.sweeps.data_ptr(), od.data_ptr(), s.cuda_stream),
                "sdpab_lowrank_factor")

    def run(self, precision=N.PREC_FP64, stream=None, **shape):
        """shape: launch shape and mixed-mode options of DeviceBatch.solve.
        (Factoring the longest instances on a side stream while the rest
        are solved was measured slower: those instances then finish the
        solve alone.)"""
        self.factor(stream)
        self.db.solve(precision=precision, stream=stream, **shape)
