"""sdpab_batch_solve_noalloc: the batched solve on the library's fixed scratch
region, for callers that cannot call cudaMalloc while they run (for example a
process whose own pool already holds the device's memory, or a service that
must not allocate after start-up).  Its results must agree with the
allocating entry point sdpab_batch_solve on the same device-resident batch,
on two calls in a row (the region is reused and keeps the previous call's
contents).  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OBJ_TOL = 1e-6   # relative, as the other parity tests
X_TOL = 1e-5     # absolute on x


def test_noalloc_matches_allocating_entry_point():
    import torch
    from sdpa_b200 import _native as N
    from sdpa_b200 import batch, instances

    insts = [instances.batch_maxcut(s) for s in range(40)]
    P = batch.pack(insts)
    db = batch.DeviceBatch(P)
    db.solve()                      # allocating entry point
    torch.cuda.synchronize()
    ref = db.result()
    assert np.all(ref.phase == 7)

    # drop the allocating path's workspace: the calls below must not grow it
    # again, nor take any other device memory
    N.check(N.lib().sdpab_release_workspace(), "sdpab_release_workspace")
    torch.cuda.synchronize()
    assert N.lib().sdpab_workspace_bytes() == 0
    free_before = torch.cuda.mem_get_info()[0]
    prm = N.default_params(0)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        db.sc.fill_(float("nan"))
        db.ic.fill_(-99)
        db.xvec.fill_(float("nan"))
        rc = N.lib().sdpab_batch_solve_noalloc(ctypes.byref(db._bt), None, ctypes.byref(prm),
                                               ctypes.byref(db._br), db.order.data_ptr(), stream)
        N.check(rc, "sdpab_batch_solve_noalloc")
        torch.cuda.synchronize()
        got = db.result()
        assert np.all(got.status == 0), call
        assert np.all(got.phase == ref.phase), call
        assert np.array_equal(got.iterations, ref.iterations), call
        rp = np.abs(got.primal_obj - ref.primal_obj) / np.maximum(1.0, np.abs(ref.primal_obj))
        rd = np.abs(got.dual_obj - ref.dual_obj) / np.maximum(1.0, np.abs(ref.dual_obj))
        assert rp.max() < OBJ_TOL and rd.max() < OBJ_TOL, call
        assert np.max(np.abs(got.xvec - ref.xvec)) < X_TOL, call
    assert N.lib().sdpab_workspace_bytes() == 0
    assert torch.cuda.mem_get_info()[0] >= free_before


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from sdpa_b200 import _native as N
    from sdpa_b200 import batch, instances
    P = batch.pack([instances.batch_maxcut(1)])
    db = batch.DeviceBatch(P)
    db._bt.nmax = 600   # one block would need 14*600^2 + m^2 doubles > 32 MiB
    prm = N.default_params(0)
    rc = N.lib().sdpab_batch_solve_noalloc(ctypes.byref(db._bt), None, ctypes.byref(prm),
                                           ctypes.byref(db._br), None, None)
    assert rc == N.ESIZE
    assert b"scratch" in N.lib().sdpab_last_error()
