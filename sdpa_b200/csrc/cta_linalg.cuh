// CTA-cooperative dense linear algebra for one small SDP block (order n up to
// a few hundred), the building blocks of the batched persistent solver.
// Every routine is called by ALL threads of the block with identical
// arguments and ends with a __syncthreads(); matrices are column-major FP64
// in global memory (L2-resident working set), tiles are staged through shared
// memory.  Nothing here waits on another block.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace sdpab {
namespace cta {

// ------------------------------------------------------------ reductions
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

template <int NT>
__device__ __forceinline__ double block_max(double v, double* red)
{
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = red[0];
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) s = fmax(s, red[w]);
  __syncthreads();
  return s;
}

// Full Frobenius inner product of two n x n column-major matrices.
template <int NT>
__device__ double dot_mat(int n, const double* A, int lda, const double* B, int ldb, double* red)
{
  double s = 0.0;
  const int tot = n * n;
  for (int t = threadIdx.x; t < tot; t += NT) {
    int i = t % n, j = t / n;
    s += A[i + (size_t)lda * j] * B[i + (size_t)ldb * j];
  }
  return block_sum<NT>(s, red);
}

template <int NT>
__device__ double trace(int n, const double* A, int lda, double* red)
{
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) s += A[i + (size_t)lda * i];
  return block_sum<NT>(s, red);
}

template <int NT>
__device__ double dot_vec(int n, const double* a, const double* b, double* red)
{
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) s += a[i] * b[i];
  return block_sum<NT>(s, red);
}

// ------------------------------------------------------------ GEMM
// C = alpha * op(A) * op(B) + beta * C for square n x n operands.
// 64 x 64 output tiles, 256 threads as a 16 x 16 grid with 4 x 4 outputs each
// (rows ty + 16 i, columns tx + 16 j), K staged in chunks of 32.
// smem: 2 * 32 * 64 doubles.
constexpr int GT = 64, GK = 32;
template <int NT>
__device__ void gemm(int n, bool tA, const double* A, int lda, bool tB, const double* B, int ldb,
                     double* C, int ldc, double alpha, double beta, double* smem)
{
  static_assert(NT == 256, "gemm tile mapping assumes 256 threads");
  double* As = smem;             // [GK][GT]  As[k*GT + r]
  double* Bs = smem + GK * GT;   // [GK][GT]  Bs[k*GT + c]
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int tiles = (n + GT - 1) / GT;
  for (int tile = 0; tile < tiles * tiles; ++tile) {
    const int r0 = (tile % tiles) * GT, c0 = (tile / tiles) * GT;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    for (int k0 = 0; k0 < n; k0 += GK) {
      // stage op(A)[r0:r0+64, k0:k0+32] and op(B)[k0:k0+32, c0:c0+64]
      for (int t = threadIdx.x; t < GK * GT; t += NT) {
        int r, k;
        if (!tA) { r = t % GT; k = t / GT; } else { k = t % GK; r = t / GK; }
        int gr = r0 + r, gk = k0 + k;
        double v = 0.0;
        if (gr < n && gk < n) v = tA ? A[gk + (size_t)lda * gr] : A[gr + (size_t)lda * gk];
        As[k * GT + r] = v;
      }
      for (int t = threadIdx.x; t < GK * GT; t += NT) {
        int c, k;
        if (!tB) { k = t % GK; c = t / GK; } else { c = t % GT; k = t / GT; }
        int gc = c0 + c, gk = k0 + k;
        double v = 0.0;
        if (gc < n && gk < n) v = tB ? B[gc + (size_t)ldb * gk] : B[gk + (size_t)ldb * gc];
        Bs[k * GT + c] = v;
      }
      __syncthreads();
      const int kmax = min(GK, n - k0);
      for (int k = 0; k < kmax; ++k) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[k * GT + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[k * GT + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      int gr = r0 + ty + 16 * i;
      if (gr >= n) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int gc = c0 + tx + 16 * j;
        if (gc >= n) continue;
        double* cp = C + gr + (size_t)ldc * gc;
        *cp = (beta == 0.0) ? alpha * acc[i][j] : alpha * acc[i][j] + beta * (*cp);
      }
    }
  }
  __syncthreads();
}

// ------------------------------------------------------------ Cholesky
// In-place lower Cholesky (right-looking).  adjust = true applies the
// reference's Schur-complement rule (rATL_dpotrfL, sdpa_dpotrf.cpp:31-33):
// pivot < -1e-6 fails, pivot < 1e-14 becomes 1e100.  adjust = false is
// LAPACK dpotrf's rule (pivot <= 0 or NaN fails).  Returns 0 on success, else
// the failing column + 1.  The strict upper triangle is zeroed.
template <int NT>
__device__ int cholesky(int n, double* A, int lda, bool adjust, int* s_flag)
{
  for (int j = 0; j < n; ++j) {
    if (threadIdx.x == 0) {
      double d = A[j + (size_t)lda * j];
      int fail = 0;
      if (adjust) {
        if (d < -1.0e-6 || d != d) fail = 1;
        else if (d < 1.0e-14) d = 1.0e100;
      } else if (!(d > 0.0)) {
        fail = 1;
      }
      if (!fail) A[j + (size_t)lda * j] = sqrt(d);
      *s_flag = fail ? j + 1 : 0;
    }
    __syncthreads();
    if (*s_flag) { int f = *s_flag; __syncthreads(); return f; }
    const double inv = 1.0 / A[j + (size_t)lda * j];
    for (int i = j + 1 + threadIdx.x; i < n; i += NT) A[i + (size_t)lda * j] *= inv;
    __syncthreads();
    const int rem = n - j - 1;
    for (int t = threadIdx.x; t < rem * rem; t += NT) {
      int i = j + 1 + t % rem, k = j + 1 + t / rem;
      if (i >= k) A[i + (size_t)lda * k] -= A[i + (size_t)lda * j] * A[k + (size_t)lda * j];
    }
    __syncthreads();
  }
  for (int t = threadIdx.x; t < n * n; t += NT) {
    int i = t % n, k = t / n;
    if (i < k) A[i + (size_t)lda * k] = 0.0;
  }
  __syncthreads();
  return 0;
}

// Linv = L^{-1} for lower-triangular L (right-looking forward substitution on
// all columns at once).  Linv must not alias L.
template <int NT>
__device__ void tri_inverse(int n, const double* L, int ldl, double* Li, int ldi)
{
  for (int t = threadIdx.x; t < n * n; t += NT) {
    int i = t % n, j = t / n;
    Li[i + (size_t)ldi * j] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    const double inv = 1.0 / L[k + (size_t)ldl * k];
    for (int j = threadIdx.x; j <= k; j += NT) Li[k + (size_t)ldi * j] *= inv;
    __syncthreads();
    const int rows = n - k - 1, cols = k + 1;
    for (int t = threadIdx.x; t < rows * cols; t += NT) {
      int i = k + 1 + t % rows, j = t / rows;
      Li[i + (size_t)ldi * j] -= L[i + (size_t)ldl * k] * Li[k + (size_t)ldi * j];
    }
    __syncthreads();
  }
}

// x = L^{-T} L^{-1} x for a Cholesky factor L (lower), vector in shared memory.
// Row-oriented substitution: each step is a block-wide dot product.
template <int NT>
__device__ void chol_solve(int n, const double* L, int ldl, double* x, double* red)
{
  // forward: L z = x
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int k = threadIdx.x; k < i; k += NT) s += L[i + (size_t)ldl * k] * x[k];
    s = block_sum<NT>(s, red);
    if (threadIdx.x == 0) x[i] = (x[i] - s) / L[i + (size_t)ldl * i];
    __syncthreads();
  }
  // backward: L^T x = z
  for (int i = n - 1; i >= 0; --i) {
    double s = 0.0;
    for (int k = i + 1 + threadIdx.x; k < n; k += NT) s += L[k + (size_t)ldl * i] * x[k];
    s = block_sum<NT>(s, red);
    if (threadIdx.x == 0) x[i] = (x[i] - s) / L[i + (size_t)ldl * i];
    __syncthreads();
  }
}

// ------------------------------------------------------------ eigenvalues
// Number of eigenvalues < x of the symmetric tridiagonal (d, e) of order k
// (Sturm sequence count).
__device__ __forceinline__ int sturm_count(int k, const double* d, const double* e, double x)
{
  int cnt = 0;
  double q = 1.0;
  for (int i = 0; i < k; ++i) {
    double off = (i > 0) ? e[i - 1] * e[i - 1] : 0.0;
    q = d[i] - x - ((i > 0) ? off / q : 0.0);
    if (q == 0.0) q = -1.0e-300;
    if (q < 0.0) ++cnt;
  }
  return cnt;
}

// Smallest eigenvalue of a symmetric tridiagonal (d, e) of order k by warp
// multisection of the Gershgorin interval (each round splits the bracket into
// 33 parts).  Called by one full warp; every lane returns the value.
__device__ double tridiag_min_eig_warp(int k, const double* d, const double* e)
{
  const int lane = threadIdx.x & 31;
  double lo = 1.0e300, hi = -1.0e300;
  for (int i = 0; i < k; ++i) {
    double r = ((i > 0) ? fabs(e[i - 1]) : 0.0) + ((i < k - 1) ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
  }
  double span = fmax(fabs(lo), fabs(hi));
  lo -= 1.0e-15 * span + 1.0e-300;
  hi += 1.0e-15 * span + 1.0e-300;
  for (int round = 0; round < 24; ++round) {
    double w = (hi - lo) / 33.0;
    double x = lo + w * (lane + 1);
    int c = sturm_count(k, d, e, x);
    unsigned ball = __ballot_sync(0xffffffffu, c >= 1);
    // first lane whose point has at least one eigenvalue below it
    int f = ball ? (__ffs(ball) - 1) : 32;
    double nlo = lo + w * f;
    double nhi = (f < 32) ? lo + w * (f + 1) : hi;
    lo = nlo;
    hi = nhi;
    if (hi - lo <= 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1.0e-300) break;
  }
  return 0.5 * (lo + hi);
}

// Last component (index k-1) of the unit eigenvector of the tridiagonal (d, e)
// for eigenvalue lam, by two steps of inverse iteration with partial
// pivoting.  Called by one thread; work needs 5*k doubles.
__device__ double tridiag_evec_last(int k, const double* d, const double* e, double lam,
                                    double* work)
{
  if (k == 1) return 1.0;
  double* a = work;          // sub
  double* b = work + k;      // diag
  double* c = work + 2 * k;  // super
  double* c2 = work + 3 * k; // second super (fill-in from pivoting)
  double* v = work + 4 * k;
  double span = 0.0;
  for (int i = 0; i < k; ++i) span = fmax(span, fabs(d[i]) + ((i < k - 1) ? fabs(e[i]) : 0.0));
  double shift = lam - 1.0e-13 * (span + 1.0e-300);
  for (int i = 0; i < k; ++i) v[i] = 1.0;
  // LU with partial pivoting of the tridiagonal T - shift I.
  double* piv_l = work + 5 * k;  // multipliers, k doubles
  int pivrow[64];
  for (int i = 0; i < k; ++i) { a[i] = (i > 0) ? e[i - 1] : 0.0; b[i] = d[i] - shift; c[i] = (i < k - 1) ? e[i] : 0.0; c2[i] = 0.0; }
  for (int i = 0; i < k - 1; ++i) {
    // rows i and i+1; a[i+1] is the entry below the pivot
    if (fabs(a[i + 1]) > fabs(b[i])) {
      // swap rows i and i+1
      double t;
      t = b[i]; b[i] = a[i + 1]; a[i + 1] = t;
      t = c[i]; c[i] = b[i + 1]; b[i + 1] = t;
      t = c2[i]; c2[i] = c[i + 1]; c[i + 1] = t;
      pivrow[i] = 1;
    } else {
      pivrow[i] = 0;
    }
    double piv = (b[i] != 0.0) ? b[i] : 1.0e-300;
    double l = a[i + 1] / piv;
    piv_l[i] = l;
    b[i + 1] -= l * c[i];
    c[i + 1] -= l * c2[i];
  }
  if (b[k - 1] == 0.0) b[k - 1] = 1.0e-300;
  for (int itn = 0; itn < 2; ++itn) {
    // apply row swaps and L^{-1}
    for (int i = 0; i < k - 1; ++i) {
      if (pivrow[i]) { double t = v[i]; v[i] = v[i + 1]; v[i + 1] = t; }
      v[i + 1] -= piv_l[i] * v[i];
    }
    // back substitution with U (diag b, super c, super2 c2)
    for (int i = k - 1; i >= 0; --i) {
      double s = v[i];
      if (i + 1 < k) s -= c[i] * v[i + 1];
      if (i + 2 < k) s -= c2[i] * v[i + 2];
      double piv = (b[i] != 0.0) ? b[i] : 1.0e-300;
      v[i] = s / piv;
    }
    double nrm = 0.0;
    for (int i = 0; i < k; ++i) nrm = fmax(nrm, fabs(v[i]));
    for (int i = 0; i < k; ++i) v[i] /= nrm;
  }
  double s2 = 0.0;
  for (int i = 0; i < k; ++i) s2 += v[i] * v[i];
  return v[k - 1] / sqrt(s2);
}

}  // namespace cta
}  // namespace sdpab
