// Minimum eigenvalue of L D L^T for the step length (Jal::getMinEigen,
// sdpa_jordan.cpp:58-109): Lanczos for n > 20 (Lal::getMinEigen,
// sdpa_linear.cpp:29-143), all eigenvalues for n <= 20 (dsyev branch,
// sdpa_linear.cpp:145-182).  Executed by one block of BT threads (256, the
// default NT, or 128); shared by the batched persistent solver and the
// host-driven solver.
#pragma once
#include "cta_linalg.cuh"

namespace sdpab {

constexpr int NT = 256;
constexpr int TRI_MAX = 64;  // Lanczos tridiagonal order bound (sqrt(n)+11 for n < 2800)
// Largest Lanczos matrix kept in shared memory (n <= 110 in FP64); larger
// blocks run the Lanczos matvecs from global memory.
constexpr int LANCZOS_SMEM_DOUBLES = 12288;

// One Lanczos process: vectors (n), tridiagonal (d, e), work (6 TRI_MAX;
// the dense n <= 20 path keeps its Householder vectors there) and the slots
// warp j publishes its Ritz results in.
struct LanczosVec {
  double *q, *qold, *r, *w;
  double *d, *e, *work;
  double* val;  // [0] Ritz minimum, [1] last eigenvector component, [2] fresh flag
};

struct EigScratch {
  LanczosVec v[2];  // up to two processes run in lockstep (X and Z)
  double* M;        // dense n <= 20 matrix (400)
  cta::Reducer* R;
};

// Shared-memory doubles of an EigScratch for blocks of order <= nmax;
// `sets` = number of Lanczos processes that may run together (1 or 2).
__host__ __device__ inline long long eig_scratch_doubles(int nmax, int sets = 2)
{
  return (long long)sets * (4LL * nmax + 8 * TRI_MAX + 4) + 400;
}

static __device__ inline void eig_scratch_carve(EigScratch& s, double* p, int nmax, cta::Reducer* R,
                                                int sets = 2)
{
  s.v[1] = LanczosVec{};
  for (int j = 0; j < sets; ++j) {
    LanczosVec& v = s.v[j];
    v.q = p; p += nmax;
    v.qold = p; p += nmax;
    v.r = p; p += nmax;
    v.w = p; p += nmax;
    v.d = p; p += TRI_MAX;
    v.e = p; p += TRI_MAX;
    v.work = p; p += 6 * TRI_MAX;
    v.val = p; p += 4;
  }
  s.M = p;
  s.R = R;
}

// Lal::getMinEigen (sdpa_linear.cpp:29-143) for NM independent matrices in
// lockstep: Lanczos on each M_j = L D L^T with the reference's start vector
// (all ones), stopping rule and error correction, each process advancing
// only while its own stopping test says so.  M_j is formed beforehand by two
// GEMMs (the reference applies L^T, D, L to each Lanczos vector; the
// products agree to rounding), so each step is one coalesced matvec.  The
// tridiagonal eigen-solve (dsteqr in the reference) is a warp multisection +
// Newton for the smallest Ritz value, which also yields the last component
// of its eigenvector.
//
// Schedule.  Running X and Z together shares every block barrier between
// them.  The tridiagonal solve that step k calls for only decides whether
// step k+1 happens, so it runs (warp j for process j) while the other warps
// already compute step k+1's matvec; if the stopping test then ends the
// process, that matvec is discarded.  The values computed and the decisions
// taken are those of the plain sequence: per step, alpha = q.Mq, the
// residual, beta, and at the steps the reference chooses (kk >= sqrt(k),
// k = n-1 or k > sqrt(n+9)) the Ritz value and error of the tridiagonal.
template <int NM, int BT = NT>
static __device__ void lanczos_min_eig_multi(int n, const double* const* Ms, EigScratch& s, double* out)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int NW = BT / 32;
  double beta[NM], mn[NM], mn_old[NM], err[NM];
  int k[NM], kk[NM];
  bool act[NM], pend[NM];
  const double sqn = sqrt((double)n);
#pragma unroll
  for (int j = 0; j < NM; ++j) {
    LanczosVec& v = s.v[j];
    for (int i = tid; i < n; i += BT) { v.qold[i] = 0.0; v.r[i] = 1.0; }
    for (int i = tid; i < TRI_MAX; i += BT) { v.d[i] = 1.0e50; v.e[i] = 0.0; }
    beta[j] = sqn;
    mn[j] = 1.0e51;
    mn_old[j] = 1.0e52;
    err[j] = 1.0e10;
    k[j] = kk[j] = 0;
    act[j] = true;
    pend[j] = false;
  }
  __syncthreads();
  for (;;) {
    // (a) the next step of every running process works on q = r / beta,
    // formed where it is read (r is published by the previous step's last
    // barrier), so the step has two barriers
    double ib[NM];
#pragma unroll
    for (int j = 0; j < NM; ++j) ib[j] = 1.0 / beta[j];
    // (b) warps 0 / 1 solve the pending tridiagonals while the remaining
    // warps multiply; CW columns of every running matrix per warp and pass,
    // all loads of a pass issued before its FMAs
    bool any_pend = false;
#pragma unroll
    for (int j = 0; j < NM; ++j) any_pend |= pend[j];
    const int w0 = any_pend ? NM : 0;
#pragma unroll
    for (int j = 0; j < NM; ++j) {
      if (wid != j || !pend[j]) continue;
      LanczosVec& v = s.v[j];
      __syncwarp();  // e[k] was written by this warp's lane 0
      double ul;
      const double lam = cta::tridiag_min_eig_warp(k[j], v.d, v.e, mn[j], &ul, v.work);
      if (lane == 0) {
        v.val[0] = lam;
        v.val[1] = ul;
      }
    }
    constexpr int CW = (NM == 2) ? 2 : 4;
    double part[NM];
#pragma unroll
    for (int j = 0; j < NM; ++j) part[j] = 0.0;
    if (wid >= w0) {
      const int nwk = NW - w0;
      for (int i0 = (wid - w0) * CW; i0 < n; i0 += CW * nwk) {
        double acc[NM][CW];
#pragma unroll
        for (int j = 0; j < NM; ++j)
#pragma unroll
          for (int c = 0; c < CW; ++c) acc[j][c] = 0.0;
        for (int kx0 = 0; kx0 < n; kx0 += 128) {
          double qv[NM][4], mv[NM][CW][4];
#pragma unroll
          for (int j = 0; j < NM; ++j) {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int kx = kx0 + lane + 32 * u;
              qv[j][u] = (act[j] && kx < n) ? s.v[j].r[kx] * ib[j] : 0.0;
#pragma unroll
              for (int c = 0; c < CW; ++c)
                mv[j][c][u] = (act[j] && kx < n && i0 + c < n) ? Ms[j][kx + (size_t)n * (i0 + c)] : 0.0;
            }
          }
#pragma unroll
          for (int j = 0; j < NM; ++j)
#pragma unroll
            for (int c = 0; c < CW; ++c)
#pragma unroll
              for (int u = 0; u < 4; ++u) acc[j][c] += mv[j][c][u] * qv[j][u];
        }
#pragma unroll
        for (int j = 0; j < NM; ++j) {
          double wv = 0.0;
#pragma unroll
          for (int c = 0; c < CW; ++c) {
            for (int o = 16; o > 0; o >>= 1) acc[j][c] += __shfl_xor_sync(0xffffffffu, acc[j][c], o);
            if (lane == c) wv = acc[j][c];
          }
          if (act[j] && lane < CW && i0 + lane < n) {
            s.v[j].w[i0 + lane] = wv;
            part[j] += (s.v[j].r[i0 + lane] * ib[j]) * wv;
          }
        }
      }
    }
    double alpha[NM];
    cta::block_sum_n<BT, NM>(part, alpha, *s.R);  // publishes w and the tridiagonal results
    // (c) take in the Ritz values, then the reference's test for this step
    bool any = false;
#pragma unroll
    for (int j = 0; j < NM; ++j) {
      if (pend[j]) {
        mn_old[j] = mn[j];
        mn[j] = s.v[j].val[0];
        err[j] = s.v[j].val[1];
        pend[j] = false;
      }
      if (act[j])
        act[j] = k[j] < n && k[j] < sqn + 10 && k[j] < TRI_MAX - 1 && beta[j] > 1.0e-16 &&
                 (fabs(mn[j] - mn_old[j]) > 1.0e-5 * fabs(mn[j]) + 1.0e-8 ||
                  fabs(err[j] * beta[j]) > 1.0e-2 * fabs(mn[j]) + 1.0e-4);
      any |= act[j];
    }
    if (!any) break;
    // (d) finish the step: residual, its norm, and whether this step's
    // tridiagonal (order k+1) is to be solved
    double rpart[NM];
#pragma unroll
    for (int j = 0; j < NM; ++j) {
      rpart[j] = 0.0;
      if (!act[j]) continue;
      LanczosVec& v = s.v[j];
      for (int i = tid; i < n; i += BT) {
        const double qi = v.r[i] * ib[j];
        const double rv = (v.w[i] - alpha[j] * qi) - beta[j] * v.qold[i];
        v.qold[i] = qi;
        v.r[i] = rv;
        rpart[j] += rv * rv;
      }
      const int kj = k[j];
      if (tid == 0) v.d[kj] = alpha[j];
      if (kk[j] >= sqrt((double)kj) || kj == n - 1 || kj > sqrt((double)n + 9)) {
        pend[j] = true;
        kk[j] = 0;
      }
    }
    double rr[NM];
    cta::block_sum_n<BT, NM>(rpart, rr, *s.R);
#pragma unroll
    for (int j = 0; j < NM; ++j) {
      if (!act[j]) continue;
      beta[j] = sqrt(rr[j]);
      // written by the lane that later solves this process's tridiagonal
      if (wid == j && lane == 0) s.v[j].e[k[j]] = beta[j];
      ++k[j];
      ++kk[j];
    }
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < NM; ++j) out[j] = mn[j] - fabs(err[j] * beta[j]);
}

template <int BT = NT>
static __device__ double lanczos_min_eig(int n, const double* M, EigScratch& s)
{
  const double* Ms[1] = {M};
  double out[1];
  lanczos_min_eig_multi<1, BT>(n, Ms, s, out);
  return out[0];
}

// n <= 20: minimum eigenvalue of the lower triangle of M = L D L^T
// (Jal::getMinEigen QR branch + dsyev, sdpa_jordan.cpp:81-89,
// sdpa_linear.cpp:145-182) via Householder tridiagonalisation (warp 0) and
// multisection.
template <int BT = NT>
static __device__ double dense_min_eig(int n, const double* W2, EigScratch& s)
{
  const int tid = threadIdx.x, lane = tid & 31;
  LanczosVec& lv = s.v[0];
  double* M = s.M;  // n x n symmetric copy of the lower triangle
  for (int t = tid; t < n * n; t += BT) {
    const int i = t % n, j = t / n;
    M[i + n * j] = (i >= j) ? W2[i + (size_t)n * j] : W2[j + (size_t)n * i];
  }
  __syncthreads();
  if (tid < 32) {
    double* v = lv.work;        // n
    double* p = lv.work + 32;   // n
    for (int k = 0; k + 2 < n; ++k) {
      const int len = n - k - 1;
      const double x = (lane < len) ? M[(k + 1 + lane) + n * k] : 0.0;
      double nrm2 = x * x;
      for (int o = 16; o > 0; o >>= 1) nrm2 += __shfl_xor_sync(0xffffffffu, nrm2, o);
      const double x0 = __shfl_sync(0xffffffffu, x, 0);
      const double alpha = (x0 >= 0.0) ? -sqrt(nrm2) : sqrt(nrm2);
      const double vi = (lane == 0) ? x - alpha : x;
      const double vn2 = nrm2 - x0 * x0 + (x0 - alpha) * (x0 - alpha);
      if (lane == 0) lv.e[k] = (nrm2 > 0.0) ? alpha : 0.0;
      if (!(vn2 > 0.0)) { __syncwarp(); continue; }
      if (lane < len) v[lane] = vi;
      __syncwarp();
      // p = (2 / vn2) S v on the trailing block; K = v^T p / v^T v; w = p - K v
      double pi = 0.0;
      if (lane < len) {
        for (int c = 0; c < len; ++c) pi += M[(k + 1 + lane) + n * (k + 1 + c)] * v[c];
        pi *= 2.0 / vn2;
      }
      double kv = (lane < len) ? pi * v[lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) kv += __shfl_xor_sync(0xffffffffu, kv, o);
      kv /= vn2;
      const double wi = pi - kv * vi;
      if (lane < len) p[lane] = wi;
      __syncwarp();
      if (lane < len) {
        for (int c = 0; c < len; ++c)
          M[(k + 1 + lane) + n * (k + 1 + c)] -= v[lane] * p[c] + p[lane] * v[c];
      }
      __syncwarp();
    }
    if (lane < n) lv.d[lane] = M[lane + n * lane];
    if (n >= 2 && lane == 0) lv.e[n - 2] = M[(n - 1) + n * (n - 2)];
    __syncwarp();
    double ul;
    const double lam = cta::tridiag_min_eig_warp(n, lv.d, lv.e, 1.0e300, &ul, lv.work + 128);
    if (lane == 0) lv.val[0] = lam;
  }
  __syncthreads();
  const double r = lv.val[0];
  __syncthreads();
  return r;
}

// Minimum eigenvalues of L D L^T for the step length (Jal::getMinEigen,
// sdpa_jordan.cpp:58-109: Lanczos for n > 20, all eigenvalues for n <= 20),
// for both of an iteration, lambda_min(Lx Dx Lx^T) and lambda_min(Lz Dz Lz^T),
// with the two Lanczos processes in lockstep.
// Wx1, Wx2, Wz1, Wz2: n x n scratch (Wx2 and Wz2 receive the formed
// matrices).  The matrices are staged in shared memory while they fit.
// z_diag: Dz is diagonal and given as the vector of its diagonal (n values),
// so Dz Lz^T is a row scaling of Lz^T (no GEMM).
// Wx2 = Lx Dx Lx^T and Wz2 = Lz Dz Lz^T (Wx1, Wz1 scratch).
template <int BT = NT>
static __device__ void form_ldlt_pair(int n, const double* Lx, const double* Dx, const double* Lz,
                                      const double* Dz, double* Wx1, double* Wx2, double* Wz1, double* Wz2,
                                      double* gsm, bool z_diag)
{
  cta::gemm<BT>(n, false, Dx, n, true, Lx, n, Wx1, n, 1.0, 0.0, gsm);
  cta::gemm<BT>(n, false, Lx, n, false, Wx1, n, Wx2, n, 1.0, 0.0, gsm);
  if (z_diag) {
    for (int t = threadIdx.x; t < n * n; t += BT) {
      const int i = t % n, j = t / n;
      Wz1[t] = Dz[i] * Lz[j + (size_t)n * i];
    }
    __syncthreads();
  } else {
    cta::gemm<BT>(n, false, Dz, n, true, Lz, n, Wz1, n, 1.0, 0.0, gsm);
  }
  cta::gemm<BT>(n, false, Lz, n, false, Wz1, n, Wz2, n, 1.0, 0.0, gsm);
}

template <int BT = NT>
static __device__ void min_eig_pair(int n, const double* Lx, const double* Dx, const double* Lz,
                                    const double* Dz, double* Wx1, double* Wx2, double* Wz1, double* Wz2,
                                    double* gsm, int gsm_doubles, EigScratch& s, double* out, bool z_diag = false)
{
  form_ldlt_pair<BT>(n, Lx, Dx, Lz, Dz, Wx1, Wx2, Wz1, Wz2, gsm, z_diag);
  if (n <= 20) {
    out[0] = dense_min_eig<BT>(n, Wx2, s);
    out[1] = dense_min_eig<BT>(n, Wz2, s);
    return;
  }
  const double* Ms[2] = {Wx2, Wz2};
  const int nn = n * n;
  if (2 * nn <= gsm_doubles) {
    for (int t = threadIdx.x; t < nn; t += BT) { gsm[t] = Wx2[t]; gsm[nn + t] = Wz2[t]; }
    __syncthreads();
    Ms[0] = gsm;
    Ms[1] = gsm + nn;
  } else if (nn <= gsm_doubles) {
    for (int t = threadIdx.x; t < nn; t += BT) gsm[t] = Wx2[t];
    __syncthreads();
    Ms[0] = gsm;
  }
  lanczos_min_eig_multi<2, BT>(n, Ms, s, out);
}

// The same for block-diagonal X and Z: nb blocks of signed orders bsz at
// offsets boff along the diagonal of the n x n matrices (order >= 2: SDP
// block; otherwise LP entries, one per diagonal position).  As in
// Jal::getMinEigen (sdpa_jordan.cpp:58-109) every SDP block gets its own
// minimum eigenvalue (Lanczos for order > 20, all eigenvalues otherwise, on
// a compact copy of the block), every LP entry contributes x_t l_t^2 (the
// diagonal of L D L^T there), and the smallest value is the result.  Not
// inlined: only block-structured instances take this path, and a second
// inlined Lanczos would raise the register pressure of the whole solver.
template <int BT = NT>
static __device__ __noinline__ void min_eig_pair_blocks(int n, int nb, const int* boff, const int* bsz,
                                                        const double* Lx, const double* Dx, const double* Lz,
                                                        const double* Dz, double* Wx1, double* Wx2, double* Wz1,
                                                        double* Wz2, double* gsm, int gsm_doubles, EigScratch& s,
                                                        double* out, bool z_diag)
{
  form_ldlt_pair<BT>(n, Lx, Dx, Lz, Dz, Wx1, Wx2, Wz1, Wz2, gsm, z_diag);
  double mx = 1.0e50, mz = 1.0e50;
  for (int l = 0; l < nb; ++l) {
    if (bsz[l] >= 2) continue;
    const int o = boff[l], cnt = bsz[l] < 0 ? -bsz[l] : bsz[l];
    for (int t = threadIdx.x; t < cnt; t += BT) {
      const size_t d = (size_t)(o + t) * (n + 1);
      mx = fmin(mx, Wx2[d]);
      mz = fmin(mz, Wz2[d]);
    }
  }
  mx = -cta::block_max<BT>(-mx, *s.R);
  mz = -cta::block_max<BT>(-mz, *s.R);
  for (int l = 0; l < nb; ++l) {
    const int k = bsz[l];
    if (k < 2) continue;
    const int o = boff[l];
    const int kk = k * k;
    double* Mx = (2 * kk <= gsm_doubles) ? gsm : Wx1;
    double* Mz = (2 * kk <= gsm_doubles) ? gsm + kk : Wz1;
    for (int t = threadIdx.x; t < kk; t += BT) {
      const size_t g = (size_t)(o + t % k) + (size_t)n * (o + t / k);
      Mx[t] = Wx2[g];
      Mz[t] = Wz2[g];
    }
    __syncthreads();
    double r[2];
    if (k <= 20) {
      r[0] = dense_min_eig<BT>(k, Mx, s);
      r[1] = dense_min_eig<BT>(k, Mz, s);
    } else {
      const double* Ms[2] = {Mx, Mz};
      lanczos_min_eig_multi<2, BT>(k, Ms, s, r);
    }
    mx = fmin(mx, r[0]);
    mz = fmin(mz, r[1]);
    __syncthreads();
  }
  out[0] = mx;
  out[1] = mz;
}

}  // namespace sdpab
