// Minimum eigenvalue of L D L^T for the step length (Jal::getMinEigen,
// sdpa_jordan.cpp:58-109): Lanczos for n > 20 (Lal::getMinEigen,
// sdpa_linear.cpp:29-143), all eigenvalues for n <= 20 (dsyev branch,
// sdpa_linear.cpp:145-182).  Executed by one 256-thread block; shared by the
// batched persistent solver and the host-driven solver.
#pragma once
#include "cta_linalg.cuh"

namespace sdpab {

constexpr int NT = 256;
constexpr int TRI_MAX = 64;  // Lanczos tridiagonal order bound (sqrt(n)+11 for n < 2800)
// Largest Lanczos matrix kept in shared memory (n <= 110 in FP64); larger
// blocks run the Lanczos matvecs from global memory.
constexpr int LANCZOS_SMEM_DOUBLES = 12288;

struct EigScratch {
  double *q, *qold, *r, *w, *t;   // Lanczos vectors (n)
  double *d, *e, *work;           // tridiagonal (TRI_MAX), work 6*TRI_MAX
  double* M;                      // dense n <= 20 matrix (400)
  cta::Reducer* R;
  double* s_val;                  // broadcast slot
};

// Lal::getMinEigen (sdpa_linear.cpp:29-143): Lanczos on M = L D L^T with
// the reference's start vector (all ones), stopping rule and error
// correction.  M is formed once by two GEMMs (the reference applies L^T, D, L
// to each Lanczos vector; the products agree to rounding), so each step is a
// single coalesced matvec.  The tridiagonal eigen-solve (dsteqr in the
// reference) is a warp multisection for the smallest Ritz value plus inverse
// iteration for the last component of its eigenvector.
static __device__ double lanczos_min_eig(int n, const double* M, EigScratch& s)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  // every thread owns the vector entries i = tid, tid + NT, ...
  for (int i = tid; i < n; i += NT) { s.q[i] = 0.0; s.r[i] = 1.0; }
  if (wid == 0) {
    for (int i = lane; i < TRI_MAX; i += 32) { s.d[i] = 1.0e50; s.e[i] = 0.0; }
  }
  double beta = sqrt((double)n);
  double mn = 1.0e51, mn_old = 1.0e52, err = 1.0e10;
  int k = 0, kk = 0;
  const double sqn = sqrt((double)n);
  while (k < n && k < sqn + 10 && k < TRI_MAX - 1 && beta > 1.0e-16 &&
         (fabs(mn - mn_old) > 1.0e-5 * fabs(mn) + 1.0e-8 ||
          fabs(err * beta) > 1.0e-2 * fabs(mn) + 1.0e-4)) {
    const double ib = 1.0 / beta;
    for (int i = tid; i < n; i += NT) { s.qold[i] = s.q[i]; s.q[i] = s.r[i] * ib; }
    __syncthreads();
    // w = M q: each warp takes 4 columns at a time (M column i dotted with q)
    double part = 0.0;
    for (int i0 = wid * 4; i0 < n; i0 += NT / 8) {
      double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      const double* c0 = M + (size_t)n * i0;
      for (int kx = lane; kx < n; kx += 32) {
        const double qk = s.q[kx];
        a0 += c0[kx] * qk;
        if (i0 + 1 < n) a1 += c0[kx + n] * qk;
        if (i0 + 2 < n) a2 += c0[kx + 2 * n] * qk;
        if (i0 + 3 < n) a3 += c0[kx + 3 * n] * qk;
      }
      for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        a3 += __shfl_xor_sync(0xffffffffu, a3, o);
      }
      if (lane < 4 && i0 + lane < n) {
        const double wv = (lane == 0) ? a0 : (lane == 1) ? a1 : (lane == 2) ? a2 : a3;
        s.w[i0 + lane] = wv;
        part += s.q[i0 + lane] * wv;
      }
    }
    const double alpha = cta::block_sum<NT>(part, *s.R);  // barrier also publishes w
    double rpart = 0.0;
    for (int i = tid; i < n; i += NT) {
      const double rv = (s.w[i] - alpha * s.q[i]) - beta * s.qold[i];
      s.r[i] = rv;
      rpart += rv * rv;
    }
    if (wid == 0) {
      if (lane == 0) s.d[k] = alpha;
      __syncwarp();
      if (kk >= sqrt((double)k) || k == n - 1 || k > sqrt((double)n + 9)) {
        const double lam = cta::tridiag_min_eig_warp(k + 1, s.d, s.e);
        if (lane == 0) {
          s.s_val[0] = lam;
          s.s_val[1] = cta::tridiag_evec_last(k + 1, s.d, s.e, lam, s.work);
          s.s_val[2] = 1.0;
        }
      } else if (lane == 0) {
        s.s_val[2] = 0.0;
      }
    }
    // the barrier of this reduction also publishes warp 0's eigen result
    const double rr = cta::block_sum<NT>(rpart, *s.R);
    if (s.s_val[2] != 0.0) {
      kk = 0;
      mn_old = mn;
      mn = s.s_val[0];
      err = s.s_val[1];
    }
    beta = sqrt(rr);
    if (tid == 0) s.e[k] = beta;
    ++k;
    ++kk;
  }
  __syncthreads();
  return mn - fabs(err * beta);
}

// n <= 20: minimum eigenvalue of the lower triangle of M = L D L^T
// (Jal::getMinEigen QR branch + dsyev, sdpa_jordan.cpp:81-89,
// sdpa_linear.cpp:145-182) via Householder tridiagonalisation (warp 0) and
// multisection.
static __device__ double dense_min_eig(int n, const double* W2, EigScratch& s)
{
  const int tid = threadIdx.x, lane = tid & 31;
  double* M = s.M;  // n x n symmetric copy of the lower triangle
  for (int t = tid; t < n * n; t += NT) {
    const int i = t % n, j = t / n;
    M[i + n * j] = (i >= j) ? W2[i + (size_t)n * j] : W2[j + (size_t)n * i];
  }
  __syncthreads();
  if (tid < 32) {
    double* v = s.work;        // n
    double* p = s.work + 32;   // n
    for (int k = 0; k + 2 < n; ++k) {
      const int len = n - k - 1;
      const double x = (lane < len) ? M[(k + 1 + lane) + n * k] : 0.0;
      double nrm2 = x * x;
      for (int o = 16; o > 0; o >>= 1) nrm2 += __shfl_xor_sync(0xffffffffu, nrm2, o);
      const double x0 = __shfl_sync(0xffffffffu, x, 0);
      const double alpha = (x0 >= 0.0) ? -sqrt(nrm2) : sqrt(nrm2);
      const double vi = (lane == 0) ? x - alpha : x;
      const double vn2 = nrm2 - x0 * x0 + (x0 - alpha) * (x0 - alpha);
      if (lane == 0) s.e[k] = (nrm2 > 0.0) ? alpha : 0.0;
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
    if (lane < n) s.d[lane] = M[lane + n * lane];
    if (n >= 2 && lane == 0) s.e[n - 2] = M[(n - 1) + n * (n - 2)];
    __syncwarp();
    const double lam = cta::tridiag_min_eig_warp(n, s.d, s.e);
    if (lane == 0) s.s_val[0] = lam;
  }
  __syncthreads();
  const double r = s.s_val[0];
  __syncthreads();
  return r;
}

// Minimum eigenvalue of L D L^T (Jal::getMinEigen, sdpa_jordan.cpp:58-109):
// Lanczos for n > 20, dense for n <= 20.  W1, W2: n x n scratch.
static __device__ double min_eig(int n, const double* L, const double* D, double* W1, double* W2,
                          double* gsm, int gsm_doubles, EigScratch& s)
{
  cta::gemm<NT>(n, false, D, n, true, L, n, W1, n, 1.0, 0.0, gsm);   // D L^T
  cta::gemm<NT>(n, false, L, n, false, W1, n, W2, n, 1.0, 0.0, gsm); // L (D L^T)
  if (n <= 20) return dense_min_eig(n, W2, s);
  const double* M = W2;
  if (n * n <= gsm_doubles) {  // stage M in shared memory for the Lanczos steps
    for (int t = threadIdx.x; t < n * n; t += NT) gsm[t] = W2[t];
    __syncthreads();
    M = gsm;
  }
  return lanczos_min_eig(n, M, s);
}


}  // namespace sdpab
