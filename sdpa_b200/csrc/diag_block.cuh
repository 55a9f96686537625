// Diagonal block of the grid-level Cholesky: factor a block of order <= 128
// and form the inverse of its factor in ONE launch of one block of threads,
// with the block resident in shared memory.  The grid factorisation's
// critical path is a chain of these (one per 128 columns), so latency, not
// arithmetic, is what matters:
//  * the 32 x 32 diagonal factorisations run in one warp with each row in a
//    lane's registers and the columns broadcast by shuffles; there are no
//    divergent branches: entries above the diagonal are updated too and
//    never read;
//  * the panel solve below each diagonal block is one thread per row, and
//    the trailing update one warp per 32 x 32 tile (4 x 8 entries per lane,
//    paired shared-memory loads);
//  * the inverse is formed in place, blocked by 32: the diagonal blocks are
//    inverted concurrently, one warp each, then the block columns from the
//    right, Li[R, j] = -Li[R, R] L[R, j] Li[j, j].
// Pivot rules as the CTA Cholesky (adjust = the reference's Schur rule,
// rATL_dpotrfL, sdpa_dpotrf.cpp:31-33).
#pragma once
#include "cta_linalg.cuh"

namespace sdpab {

constexpr int DB_MAX = 128;             // largest block
constexpr int DB_LDS = DB_MAX + 4;      // leading dimension of the resident block (even: paired loads)
constexpr int DB_WLD = DB_MAX - 32 + 4; // leading dimension of the inverse's work panel
constexpr int DB_NT = 256;

template <typename T>
constexpr size_t diag_block_smem()
{
  return ((size_t)DB_MAX * DB_LDS + (size_t)DB_WLD * 32 + DB_MAX) * sizeof(T);
}

static_assert(diag_block_smem<double>() <= 227 * 1024, "the resident block must fit one block's shared memory");

template <typename T>
struct DbPair;
template <>
struct DbPair<double> {
  using type = double2;
};
template <>
struct DbPair<float> {
  using type = float2;
};

// pivot of column j: sets ljj and inv = 1 / ljj, or returns j + 1
template <typename T>
__device__ __forceinline__ int db_pivot(T d, bool adjust, int j, T& ljj, T& inv)
{
  if (adjust) {
    if (d < (T)-1.0e-6 || d != d) return j + 1;
    if (d < (T)1.0e-14) d = cta::adjust_huge<T>();
  } else if (!(d > (T)0)) {
    return j + 1;
  }
  ljj = sqrt(d);
  inv = (T)1 / ljj;
  return 0;
}

// one warp: factor S[kb:kb+bs, kb:kb+bs] (bs <= 32) in place; dinv[kb + j] =
// 1 / L_jj.  Returns 0 or the failing column (relative to S) + 1.
template <typename T>
__device__ __forceinline__ int db_potrf32(T* S, int kb, int bs, bool adjust, T* dinv)
{
  const int lane = threadIdx.x & 31;
  T a[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) a[c] = (c <= lane && lane < bs) ? S[kb + lane + DB_LDS * (kb + c)] : (T)0;
  int fail = 0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j >= bs) break;  // warp-uniform
    T ljj = 0, inv = 0;
    fail = db_pivot<T>(__shfl_sync(0xffffffffu, a[j], j), adjust, kb + j, ljj, inv);
    if (fail) break;     // warp-uniform
    if (lane == j) dinv[kb + j] = inv;
    a[j] = (lane == j) ? ljj : a[j] * inv;
    const T lrj = a[j];
#pragma unroll
    for (int c = j + 1; c < 32; ++c) a[c] = fma(-lrj, __shfl_sync(0xffffffffu, lrj, c), a[c]);
  }
  if (!fail && lane < bs) {
#pragma unroll
    for (int c = 0; c < 32; ++c)
      if (c <= lane) S[kb + lane + DB_LDS * (kb + c)] = a[c];
  }
  return fail;
}

// Factor the n x n block A (lda; n <= 128) in place: lower triangle = L,
// strict upper = 0.  If Li is given, also Li = L^-1 (ldi; upper = 0).  A
// failure writes col0 + failing column + 1 to *flag (if still 0); a set
// *flag on entry skips the launch's work.
template <typename T>
__global__ void __launch_bounds__(DB_NT) k_chol_inv_diag(int n, T* A, int lda, int adjust, int col0, int* flag,
                                                         T* Li, int ldi)
{
  using P2 = typename DbPair<T>::type;
  extern __shared__ __align__(16) unsigned char db_raw[];
  T* S = (T*)db_raw;
  T* W = S + (size_t)DB_MAX * DB_LDS;
  T* dinv = W + (size_t)DB_WLD * 32;
  __shared__ int s_fail;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = DB_NT / 32;
  if (*flag) return;
  // lower triangle of A into S, zeros elsewhere (one warp per column)
  for (int c = warp; c < DB_MAX; c += NW)
    for (int r = lane; r < DB_MAX; r += 32) S[r + DB_LDS * c] = (r < n && c <= r) ? A[r + (size_t)lda * c] : (T)0;
  __syncthreads();
  // ---- factorisation, right-looking by 32
  for (int kb = 0; kb < n; kb += 32) {
    const int bs = min(32, n - kb);
    if (warp == 0) {
      const int f = db_potrf32<T>(S, kb, bs, adjust != 0, dinv);
      if (lane == 0) s_fail = f;
    }
    __syncthreads();
    if (s_fail) {
      if (tid == 0) atomicCAS(flag, 0, col0 + s_fail);
      return;
    }
    const int r0 = kb + 32, rem = n - r0;  // rem > 0 implies bs == 32
    if (rem <= 0) break;
    // panel: rows r0.. of columns kb..kb+31 times L_kk^-T, one thread per row
    for (int r = r0 + tid; r < n; r += DB_NT) {
      T x[32];
#pragma unroll
      for (int p = 0; p < 32; ++p) x[p] = S[r + DB_LDS * (kb + p)];
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        x[c] *= dinv[kb + c];
#pragma unroll
        for (int q = c + 1; q < 32; ++q) x[q] = fma(-x[c], S[kb + q + DB_LDS * (kb + c)], x[q]);
      }
#pragma unroll
      for (int p = 0; p < 32; ++p) S[r + DB_LDS * (kb + p)] = x[p];
    }
    __syncthreads();
    // trailing lower triangle: one warp per 32 x 32 tile (tr >= tc); lane
    // (rg, cg) owns rows 4 rg .. 4 rg + 3 and columns 8 cg .. 8 cg + 7
    const int nt = (rem + 31) / 32;
    if (warp < nt * (nt + 1) / 2) {
      int tr = 0;
      while ((tr + 1) * (tr + 2) / 2 <= warp) ++tr;
      const int tc = warp - tr * (tr + 1) / 2;
      const int rg = lane & 7, cg = lane >> 3;
      const int rb = r0 + 32 * tr + 4 * rg, cb = r0 + 32 * tc + 8 * cg;
      T acc[4][8];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int u = 0; u < 8; ++u) acc[i][u] = 0;
#pragma unroll 4
      for (int p = 0; p < 32; ++p) {
        const T* colp = S + DB_LDS * (kb + p);
        const P2 ra = *(const P2*)(colp + rb), rb2 = *(const P2*)(colp + rb + 2);
        const T xr[4] = {ra.x, ra.y, rb2.x, rb2.y};
        T xc[8];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const P2 q = *(const P2*)(colp + cb + 2 * v);
          xc[2 * v] = q.x;
          xc[2 * v + 1] = q.y;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int u = 0; u < 8; ++u) acc[i][u] = fma(xr[i], xc[u], acc[i][u]);
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (rb + i < n && cb + u <= rb + i) S[rb + i + DB_LDS * (cb + u)] -= acc[i][u];
    }
    __syncthreads();
  }
  for (int c = warp; c < n; c += NW)
    for (int r = lane; r < n; r += 32) A[r + (size_t)lda * c] = (c <= r) ? S[r + DB_LDS * c] : (T)0;
  if (!Li) return;
  __syncthreads();  // L is read out above before the inverse overwrites it
  // ---- inverse in place: diagonal blocks, one warp each (lane = column)
  const int nbk = (n + 31) / 32;
  if (warp < nbk) {
    const int kb = 32 * warp, bs = min(32, n - kb);
    T x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      T s = (lane == i) ? (T)1 : (T)0;
#pragma unroll
      for (int k = 0; k < i; ++k) s = fma(-S[kb + i + DB_LDS * (kb + k)], x[k], s);
      x[i] = (i < bs) ? s * dinv[kb + i] : (T)0;
    }
    __syncwarp();
    if (lane < bs) {
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (i >= lane && i < bs) S[kb + i + DB_LDS * (kb + lane)] = x[i];
    }
  }
  __syncthreads();
  // block columns from the right: Li[R, jb] = -Li[R, R] L[R, jb] Li[jb, jb]
  for (int jb = nbk - 2; jb >= 0; --jb) {
    const int c0 = 32 * jb, R0 = c0 + 32;
    const int cq = 4 * warp;  // this warp's 4 columns of the block column
    {
      T y[3][4];
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int u = 0; u < 4; ++u) y[t][u] = 0;
      for (int k = R0; k < n; ++k) {
        T xk[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) xk[u] = S[k + DB_LDS * (c0 + cq + u)];
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          const int i = R0 + 32 * t + lane;
          const T lik = (i < n) ? S[i + DB_LDS * k] : (T)0;  // zero above the diagonal
#pragma unroll
          for (int u = 0; u < 4; ++u) y[t][u] = fma(-lik, xk[u], y[t][u]);
        }
      }
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int u = 0; u < 4; ++u) W[32 * t + lane + DB_WLD * (cq + u)] = y[t][u];
    }
    __syncthreads();
    {
      T z[3][4];
#pragma unroll
      for (int t = 0; t < 3; ++t)
#pragma unroll
        for (int u = 0; u < 4; ++u) z[t][u] = 0;
#pragma unroll 4
      for (int k = 0; k < 32; ++k) {
        T dk[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) dk[u] = S[c0 + k + DB_LDS * (c0 + cq + u)];  // Li[jb, jb], zero above
#pragma unroll
        for (int t = 0; t < 3; ++t) {
          const T yk = W[32 * t + lane + DB_WLD * k];
#pragma unroll
          for (int u = 0; u < 4; ++u) z[t][u] = fma(yk, dk[u], z[t][u]);
        }
      }
#pragma unroll
      for (int t = 0; t < 3; ++t) {
        const int i = R0 + 32 * t + lane;
        if (i < n) {
#pragma unroll
          for (int u = 0; u < 4; ++u) S[i + DB_LDS * (c0 + cq + u)] = z[t][u];
        }
      }
    }
    __syncthreads();
  }
  for (int c = warp; c < n; c += NW)
    for (int r = lane; r < n; r += 32) Li[r + (size_t)ldi * c] = (c <= r) ? S[r + DB_LDS * c] : (T)0;
}

}  // namespace sdpab
