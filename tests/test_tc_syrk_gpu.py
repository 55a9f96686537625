"""The tensor-core (tcgen05, split TF32) kernels against FP64 numpy
references: the lower update C -= P P^T of the mixed-precision Schur
factorisation (partial tiles, K not a multiple of the staging width, the
upper triangle untouched) and the batched F1 product C_q = A_q B^T, both
with FP32-level error."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,K", [(128, 32), (200, 128), (300, 70), (517, 128)])
def test_tc_syrk_matches_fp64(M, K):
    import torch
    from sdpa_b200 import _native as N
    rng = np.random.default_rng(M * 1000 + K)
    P = rng.standard_normal((M, K)).astype(np.float32)
    C0 = rng.standard_normal((M, M)).astype(np.float32)
    ld = M + 3  # leading dimensions larger than M
    Pd = torch.zeros((K, ld), dtype=torch.float32, device="cuda")   # column-major M x K: [k, r]
    Cd = torch.zeros((M, ld), dtype=torch.float32, device="cuda")   # column-major M x M: [c, r]
    Pd[:, :M] = torch.from_numpy(P.T.copy()).cuda()
    Cd[:, :M] = torch.from_numpy(C0.T.copy()).cuda()
    work = torch.empty(int(N.lib().sdpab_tc_syrk_work_bytes(M, K)) // 4 + 4, dtype=torch.float32, device="cuda")
    N.check(N.lib().sdpab_tc_syrk(M, K, Pd.data_ptr(), ld, Cd.data_ptr(), ld, work.data_ptr(), -1, None), "tc_syrk")
    C = Cd[:, :M].cpu().numpy().T  # back to row-major M x M
    ref = C0.astype(np.float64) - P.astype(np.float64) @ P.astype(np.float64).T
    low = np.tril(np.ones((M, M), bool))
    err = np.max(np.abs(C[low] - ref[low]))
    scale = np.max(np.abs(P.astype(np.float64) @ P.astype(np.float64).T))
    assert err <= 2e-6 * scale, (err, scale)
    np.testing.assert_array_equal(C[~low], C0[~low])  # strictly upper triangle untouched
    assert np.all(Cd[:, M:].cpu().numpy() == 0)  # nothing written outside M x M


@pytest.mark.parametrize("M,N,K,batch", [(128, 128, 16, 1), (200, 300, 70, 3), (500, 500, 500, 2), (37, 129, 131, 4)])
def test_tc_gemm_matches_fp64(M, N, K, batch):
    """The split-TF32 product of the mixed-precision F1 assembly,
    C_q = A_q B^T with FP64 operands: partial tiles, K not a multiple of the
    staging width, a batch with strides, FP32-level error against FP64."""
    import torch
    from sdpa_b200 import _native as N_
    rng = np.random.default_rng(M * 7 + N * 5 + K * 3 + batch)
    A = rng.standard_normal((batch, M, K))
    B = rng.standard_normal((N, K))
    lda, ldb, ldc = M + 2, N + 1, M + 5
    sA, sC = lda * K + 7, ldc * N + 3
    Ad = torch.zeros(batch * sA, dtype=torch.float64, device="cuda")
    Bd = torch.zeros(ldb * K, dtype=torch.float64, device="cuda")
    Cd = torch.zeros(batch * sC, dtype=torch.float64, device="cuda")
    for q in range(batch):
        blk = np.zeros((K, lda))
        blk[:, :M] = A[q].T
        Ad[q * sA:q * sA + lda * K] = torch.from_numpy(blk.ravel()).cuda()
    bb = np.zeros((K, ldb))
    bb[:, :N] = B.T
    Bd[:] = torch.from_numpy(bb.ravel()).cuda()
    work = torch.empty(int(N_.lib().sdpab_tc_gemm_work_bytes(M, N, K, batch)) // 8 + 4, dtype=torch.float64,
                       device="cuda")
    N_.check(N_.lib().sdpab_tc_gemm(M, N, K, batch, Ad.data_ptr(), lda, sA, Bd.data_ptr(), ldb, Cd.data_ptr(), ldc,
                                    sC, work.data_ptr(), -1, None), "tc_gemm")
    Ch = Cd.cpu().numpy()
    for q in range(batch):
        C = Ch[q * sC:q * sC + ldc * N].reshape(N, ldc)[:, :M].T
        ref = A[q] @ B.T
        bound = np.abs(A[q]) @ np.abs(B).T
        assert np.all(np.abs(C - ref) <= 5e-6 * bound + 1e-300), np.max(np.abs(C - ref) / bound)
        pad = Ch[q * sC:q * sC + ldc * N].reshape(N, ldc)[:, M:]
        assert np.all(pad == 0)  # nothing written outside M x N


def test_tc_syrk_gives_up_with_its_status_and_recovers():
    """A wait bound of zero polls: every block gives up at its first wait,
    before any MMA is issued, drains its copies and frees its tensor memory;
    the call returns SDPAB_ECUDA with the time-out message and leaves C as it
    was.  The next call with the default bound is correct (the context is
    intact)."""
    import torch
    from sdpa_b200 import _native as N
    M, K = 200, 64
    rng = np.random.default_rng(7)
    P = torch.from_numpy(rng.standard_normal((K, M)).astype(np.float32)).cuda()  # column-major M x K
    C0 = rng.standard_normal((M, M)).astype(np.float32)
    Cd = torch.from_numpy(C0.T.copy()).cuda()
    work = torch.empty(int(N.lib().sdpab_tc_syrk_work_bytes(M, K)) // 4 + 4, dtype=torch.float32, device="cuda")
    rc = N.lib().sdpab_tc_syrk(M, K, P.data_ptr(), M, Cd.data_ptr(), M, work.data_ptr(), 0, None)
    assert rc == N.ECUDA
    assert b"timed out" in N.lib().sdpab_last_error()
    np.testing.assert_array_equal(Cd.cpu().numpy(), C0.T)
    N.check(N.lib().sdpab_tc_syrk(M, K, P.data_ptr(), M, Cd.data_ptr(), M, work.data_ptr(), -1, None), "tc_syrk")
    Pn = P.cpu().numpy().T.astype(np.float64)
    ref = C0.astype(np.float64) - Pn @ Pn.T
    low = np.tril(np.ones((M, M), bool))
    assert np.max(np.abs(Cd.cpu().numpy().T[low] - ref[low])) <= 2e-6 * np.max(np.abs(Pn @ Pn.T))


def test_tc_gemm_gives_up_with_its_status_and_recovers():
    import torch
    from sdpa_b200 import _native as N_
    M, N, K, batch = 150, 150, 150, 2
    rng = np.random.default_rng(8)
    A = torch.from_numpy(rng.standard_normal(batch * M * K)).cuda()
    B = torch.from_numpy(rng.standard_normal(N * K)).cuda()
    C = torch.full((batch * M * N,), 3.0, dtype=torch.float64, device="cuda")
    work = torch.empty(int(N_.lib().sdpab_tc_gemm_work_bytes(M, N, K, batch)) // 8 + 4, dtype=torch.float64,
                       device="cuda")
    args = (M, N, K, batch, A.data_ptr(), M, M * K, B.data_ptr(), N, C.data_ptr(), M, M * N, work.data_ptr())
    rc = N_.lib().sdpab_tc_gemm(*args, 0, None)
    assert rc == N_.ECUDA and b"timed out" in N_.lib().sdpab_last_error()
    assert torch.all(C == 3.0)
    N_.check(N_.lib().sdpab_tc_gemm(*args, -1, None), "tc_gemm")
    An = A.cpu().numpy().reshape(batch, K, M).transpose(0, 2, 1)
    Bn = B.cpu().numpy().reshape(K, N).T
    Cn = C.cpu().numpy().reshape(batch, N, M).transpose(0, 2, 1)
    for q in range(batch):
        ref = An[q] @ Bn.T
        assert np.max(np.abs(Cn[q] - ref)) <= 2e-6 * np.max(np.abs(ref))


@pytest.mark.parametrize("polls", [0, 1])
def test_mixed_solve_falls_back_when_tensor_cores_give_up(polls):
    """The mixed-precision solve of a random SDP with m = 300 (tensor-core
    trailing updates of the FP32 Schur factor) and an order-80 block (tensor-
    core F1 products), with the tensor-core waits bounded to `polls` polls:
    the pipelines give up, the solver counts it and uses the FP64 factor /
    SIMT products for those iterations, and the solve still matches the
    reference (objectives within 1e-6, x within the reference's accuracy).
    The same solve with the default bound has no time-outs."""
    import json
    import os
    from golden_util import GOLDEN, rel, x_within_reference_accuracy
    from sdpa_b200 import instances
    from sdpa_b200.sdpa import SDPA
    meta = json.load(open(os.path.join(GOLDEN, "tcfb.json")))["rnd300"]
    arr = np.load(os.path.join(GOLDEN, "tcfb.npz"))
    inst = instances.random_sdp(m=300, n=80, nlp=6, density=0.1, seed=11)
    for limit in (polls, -1):
        s = SDPA()
        s.inputProblem(inst)
        s.setPrecision(1)
        s.setTensorCoreWaitLimit(limit)
        s.solve()
        t = s.tensorCoreTimeouts()
        assert (t > 0) if limit >= 0 else (t == 0), (limit, t)
        assert s.getPhaseString() == "pdOPT"
        assert rel(s.getPrimalObj(), meta["primal_obj"]) < 1e-6
        assert rel(s.getDualObj(), meta["dual_obj"]) < 1e-6
        assert x_within_reference_accuracy(s.getResultXVec(), arr["rnd300.xvec"], arr["rnd300.tight"])
