"""The tensor-core (tcgen05, split TF32) lower update C -= P P^T of the
mixed-precision Schur factorisation against an FP64 numpy reference:
partial tiles, K not a multiple of the staging width, the upper triangle
untouched, FP32-level error."""
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
    N.check(N.lib().sdpab_tc_syrk(M, K, Pd.data_ptr(), ld, Cd.data_ptr(), ld, work.data_ptr(), None), "tc_syrk")
    C = Cd[:, :M].cpu().numpy().T  # back to row-major M x M
    ref = C0.astype(np.float64) - P.astype(np.float64) @ P.astype(np.float64).T
    low = np.tril(np.ones((M, M), bool))
    err = np.max(np.abs(C[low] - ref[low]))
    scale = np.max(np.abs(P.astype(np.float64) @ P.astype(np.float64).T))
    assert err <= 2e-6 * scale, (err, scale)
    np.testing.assert_array_equal(C[~low], C0[~low])  # strictly upper triangle untouched
    assert np.all(Cd[:, M:].cpu().numpy() == 0)  # nothing written outside M x M
