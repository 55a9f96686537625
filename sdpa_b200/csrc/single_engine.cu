// Device kernels and host orchestration of the host-driven solver
// (solver.h).  The operation sequence is the reference's (SDPA::solve,
// sdpa_solve.cpp:59-233; Newton::Mehrotra, sdpa_newton.cpp:2755-2809); the
// scalar rules are ipm_control.h.  Dense n x n blocks and the m x m Schur
// matrix stay resident in HBM; block-level pieces (diagonal-block Cholesky,
// Lanczos, Schur solve) run as single thread-block kernels built from
// cta_linalg.cuh / eig.cuh, everything else as grid kernels.
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <map>
#include <numeric>
#include <queue>
#include <string>
#include <vector>

#include "cta_linalg.cuh"
#include "diag_block.cuh"
#include "eig.cuh"
#include "ipm_control.h"
#include "sdpa_b200.h"
#include "sdpab_internal.h"
#include "solver.h"

namespace sdpab {

enum Formula { F1 = 1, F2 = 2, F3 = 3 };

// ------------------------------------------------------------------ kernels

__global__ void k_set_identity(int n, double* A, double v)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < (long long)n * n) A[t] = ((t % n) == (t / n)) ? v : 0.0;
}

// out = a * x + b * y (element-wise, len entries)
__global__ void k_axpby(long long len, double* out, double a, const double* x, double b, const double* y)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < len) out[t] = a * x[t] + (y ? b * y[t] : 0.0);
}

// out = a * x + b * y - z  (rMat of the corrector: beta mu Z^-1 - X - dX dZ Z^-1)
__global__ void k_axpby_sub(long long len, double* out, double a, const double* x, double b,
                            const double* y, const double* z)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < len) out[t] = (a * x[t] + b * y[t]) - z[t];
}

// dX = sym(R - W): lower = (lower + upper) / 2 mirrored (Lal::getSymmetrize,
// sdpa_linear.cpp:591-618, applied to R - X dZ Z^-1)
__global__ void k_sym_diff(int n, double* dX, const double* R, const double* W)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int i = t % n, j = t / n;
  if (i < j) return;
  const double lo = R[i + (size_t)n * j] - W[i + (size_t)n * j];
  const double up = R[j + (size_t)n * i] - W[j + (size_t)n * i];
  const double s = 0.5 * (lo + up);
  dX[i + (size_t)n * j] = s;
  dX[j + (size_t)n * i] = s;
}

// rows x cols copy between leading dimensions
template <typename T>
__global__ void k_copy2d_t(int rows, int cols, const T* src, int lds, T* dst, int ldd)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)rows * cols) return;
  const int i = t % rows, j = t / rows;
  dst[i + (size_t)ldd * j] = src[i + (size_t)lds * j];
}

// W += scale * sum_q coef[cons[q]] A_q (InputData::multi_plusToA,
// sdpa_dataset.cpp:427-433).  One warp per constraint, atomics for shared
// positions.
__global__ void k_sp_scatter(int nc, const int* cons, const long long* ptr, const int* row,
                             const int* col, const double* val, const double* coef, double scale,
                             double* W, int n)
{
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nc) return;
  const double s = scale * (coef ? coef[cons[warp]] : 1.0);
  for (long long e = ptr[warp] + lane; e < ptr[warp + 1]; e += 32) {
    const int r = row[e], c = col[e];
    const double v = s * val[e];
    atomicAdd(&W[r + (size_t)n * c], v);
    if (r != c) atomicAdd(&W[c + (size_t)n * r], v);
  }
}

// Schur complement by formula F3 for every pair whose dominant constraint
// uses F3 (compute_bMat_dense_SDP3 + calF3_thread_2, sdpa_newton.cpp:2019-2125,
// :1319-1403).  One thread per ordered (i, j) pair of the block's constraints.
__device__ __forceinline__ void f3_pair(long long t, int nc, const int* cons, const long long* ptr, const int* row,
                                        const int* col, const double* val, const int* nnz, const int* formula,
                                        const double* X, const double* Zi, int n, double* B, int m)
{
  const int il = (int)(t % nc), jl = (int)(t / nc);
  if (formula[jl] != F3) return;
  const int gi = cons[il], gj = cons[jl];
  const int inz = nnz[il], jnz = nnz[jl];
  if (jnz < inz || (inz == jnz && gi < gj)) return;
  double ret = 0.0;
  for (long long e1 = ptr[jl]; e1 < ptr[jl + 1]; ++e1) {
    const int al = row[e1], be = col[e1];
    const double* Xa = X + (size_t)n * al;
    const double* Xb = X + (size_t)n * be;
    const double* Za = Zi + (size_t)n * al;
    const double* Zb = Zi + (size_t)n * be;
    double sum = 0.0;
    for (long long e2 = ptr[il]; e2 < ptr[il + 1]; ++e2) {
      const int ga = row[e2], de = col[e2];
      double plu;
      if (al != be) {
        plu = (ga != de) ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] + Za[de] * Xb[ga] + Za[ga] * Xb[de]
                         : Zb[de] * Xa[ga] + Za[de] * Xb[ga];
      } else {
        plu = (ga != de) ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] : Zb[de] * Xa[ga];
      }
      sum += val[e2] * plu;
    }
    ret += val[e1] * sum;
  }
  atomicAdd(&B[gi + (size_t)m * gj], ret);
  if (gi != gj) atomicAdd(&B[gj + (size_t)m * gi], ret);
}

// Tr(A_i X A_j Z^-1) of one constraint pair by formula F3 (calF3_thread_2,
// sdpa_newton.cpp:1319-1403), the constraint with more entries as the outer
// loop (the value is symmetric in i and j).  The outer entries
// [e_beg, e_end) with stride e_step (a slice of the outer constraint's
// entries when several threads share one pair).
constexpr long long F3_HEAVY = 1024;  // entry pairs above which one pair gets a block of threads
__device__ __forceinline__ double f3_value_slice(int o, int in, long long e_beg, long long e_step,
                                                 const long long* ptr, const int* row, const int* col,
                                                 const double* val, const double* X, const double* Zi, int n)
{
  double ret = 0.0;
  for (long long e1 = ptr[o] + e_beg; e1 < ptr[o + 1]; e1 += e_step) {
    const int al = row[e1], be = col[e1];
    const double* Xa = X + (size_t)n * al;
    const double* Xb = X + (size_t)n * be;
    const double* Za = Zi + (size_t)n * al;
    const double* Zb = Zi + (size_t)n * be;
    double sum = 0.0;
    for (long long e2 = ptr[in]; e2 < ptr[in + 1]; ++e2) {
      const int ga = row[e2], de = col[e2];
      double plu;
      if (al != be) {
        plu = (ga != de) ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] + Za[de] * Xb[ga] + Za[ga] * Xb[de]
                         : Zb[de] * Xa[ga] + Za[de] * Xb[ga];
      } else {
        plu = (ga != de) ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] : Zb[de] * Xa[ga];
      }
      sum += val[e2] * plu;
    }
    ret += val[e1] * sum;
  }
  return ret;
}

// The whole Schur matrix by F3 when it has one source: one SDP block that
// every constraint touches, every constraint F3, no LP block (Lovasz theta,
// MaxCut).  Each entry is then written once, so B needs no zero fill and no
// atomics.  One block of threads per 32 x 32 tile on or below the diagonal
// (tile rows i, columns j of the constraint index); the tile's values go
// through shared memory, and both the tile and its mirror above the
// diagonal are stored with consecutive threads on consecutive rows
// (coalesced).  Threads as 32 x 8, four pairs each.
constexpr int F3T = 32;
// F3 value of a pair of single-entry constraints (r1, c1, v1), (r2, c2, v2)
// (the one-entry case of f3_value_slice; the first as the outer loop).
__device__ __forceinline__ double f3_value_11(int al, int be, double v1, int ga, int de, double v2, const double* X,
                                              const double* Zi, int n)
{
  const double* Xa = X + (size_t)n * al;
  const double* Xb = X + (size_t)n * be;
  const double* Za = Zi + (size_t)n * al;
  const double* Zb = Zi + (size_t)n * be;
  double plu;
  if (al != be) {
    plu = (ga != de) ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] + Za[de] * Xb[ga] + Za[ga] * Xb[de]
                     : Zb[de] * Xa[ga] + Za[de] * Xb[ga];
  } else {
    plu = (ga != de) ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] : Zb[de] * Xa[ga];
  }
  return v1 * (v2 * plu);
}

__global__ void __launch_bounds__(256) k_f3_tiles(int m, const long long* ptr, const int* row, const int* col,
                                                  const double* val, const int* nnz, const double* X,
                                                  const double* Zi, int n, double* B)
{
  __shared__ double tile[F3T][F3T + 1];
  // the tile's row and column constraints: entry count, NonZeroEffect and
  // (for single-entry constraints) the entry itself, loaded once per tile
  __shared__ long long s_cnt[2][F3T];
  __shared__ int s_nnz[2][F3T], s_r[2][F3T], s_c[2][F3T];
  __shared__ double s_v[2][F3T];
  const long long t = blockIdx.x;
  int ti = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((long long)(ti + 1) * (ti + 2) / 2 <= t) ++ti;
  while ((long long)ti * (ti + 1) / 2 > t) --ti;
  const int tj = (int)(t - (long long)ti * (ti + 1) / 2);
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  if (ty < 2) {
    const int q = (ty == 0 ? ti : tj) * F3T + tx;
    if (q < m) {
      const long long b0 = ptr[q], c = ptr[q + 1] - b0;
      s_cnt[ty][tx] = c;
      s_nnz[ty][tx] = nnz[q];
      s_r[ty][tx] = (c > 0) ? row[b0] : 0;
      s_c[ty][tx] = (c > 0) ? col[b0] : 0;
      s_v[ty][tx] = (c > 0) ? val[b0] : 0.0;
    }
  }
  __syncthreads();
  const int i = ti * F3T + tx;
#pragma unroll
  for (int k = 0; k < F3T / 8; ++k) {
    const int jl = ty + 8 * k, j = tj * F3T + jl;
    double v = 0.0;
    if (i < m && j < m && (ti > tj || tx >= jl)) {
      const long long ci = s_cnt[0][tx], cj = s_cnt[1][jl];
      if (ci == 1 && cj == 1) {
        // j outer when it dominates (equal NonZeroEffect: either order)
        if (s_nnz[1][jl] >= s_nnz[0][tx])
          v = f3_value_11(s_r[1][jl], s_c[1][jl], s_v[1][jl], s_r[0][tx], s_c[0][tx], s_v[0][tx], X, Zi, n);
        else
          v = f3_value_11(s_r[0][tx], s_c[0][tx], s_v[0][tx], s_r[1][jl], s_c[1][jl], s_v[1][jl], X, Zi, n);
      } else if (ci * cj <= F3_HEAVY) {
        // heavy pairs are left to k_f3_heavy (stored as 0 here, overwritten there)
        const int o = (s_nnz[1][jl] >= s_nnz[0][tx]) ? j : i, in = (o == j) ? i : j;
        v = f3_value_slice(o, in, 0, 1, ptr, row, col, val, X, Zi, n);
      }
    }
    tile[tx][jl] = v;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < F3T / 8; ++k) {
    const int jl = ty + 8 * k, j = tj * F3T + jl;
    if (i < m && j < m && (ti > tj || tx >= jl)) B[i + (size_t)m * j] = tile[tx][jl];
  }
#pragma unroll
  for (int k = 0; k < F3T / 8; ++k) {
    const int il = ty + 8 * k, i2 = ti * F3T + il, j2 = tj * F3T + tx;
    if (i2 < m && j2 < m && (ti > tj || il >= tx)) B[j2 + (size_t)m * i2] = tile[il][tx];
  }
}

// The heavy pairs of the one-source F3 assembly (entry pairs above
// F3_HEAVY, e.g. the trace constraint of Lovasz theta with itself): one
// block of 1024 threads per pair, the (outer, inner) entry pairs dealt over
// the threads, a fixed-order block reduction; runs after k_f3_tiles.
__global__ void __launch_bounds__(1024) k_f3_heavy(int m, const int* pairs, const long long* ptr, const int* row,
                                                   const int* col, const double* val, const int* nnz,
                                                   const double* X, const double* Zi, int n, double* B)
{
  __shared__ double red[32];
  const int i = pairs[2 * blockIdx.x], j = pairs[2 * blockIdx.x + 1];
  const int o = (nnz[j] >= nnz[i]) ? j : i, in = (o == j) ? i : j;
  // the (outer, inner) entry pairs dealt over the threads
  const long long ob = ptr[o], ib = ptr[in], ci = ptr[in + 1] - ib;
  const long long tot = (ptr[o + 1] - ob) * ci;
  double v = 0.0;
  for (long long f = threadIdx.x; f < tot; f += 1024) {
    const long long e1 = ob + f / ci, e2 = ib + f % ci;
    v += f3_value_11(row[e1], col[e1], val[e1], row[e2], col[e2], val[e2], X, Zi, n);
  }
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 32; ++w) s += red[w];
    B[i + (size_t)m * j] = s;
    B[j + (size_t)m * i] = s;
  }
}

// The F3 pairs of every SDP block in one launch: block b owns the flat pair
// indices [off[b], off[b + 1]) (nc_b^2 of them), found by binary search.
struct F3Desc {
  const int* cons;
  const long long* ptr;
  const int *row, *col;
  const double* val;
  const int *nnz, *form;
  const double *X, *Zi;
  int nc, n;
};

__global__ void k_f3_all(const F3Desc* d, const long long* off, int nb, double* B, int m)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= off[nb]) return;
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (off[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const F3Desc& q = d[lo];
  f3_pair(t - off[lo], q.nc, q.cons, q.ptr, q.row, q.col, q.val, q.nnz, q.form, q.X, q.Zi, q.n, B, m);
}

// F1 step 1 (Lal::let(work1,'=',xMat,'*',Aj), sdpa_newton.cpp:1859-1863):
// T_q = X A_j for a chunk of F1/F2 constraints, A_j given column-wise with
// both triangles (csc).  One block per (q, column c).
__global__ void k_f1_left(int n, int q0, const int* f1list, const long long* cptr_base,
                          const long long* csc_ptr, const int* csc_row, const double* csc_val,
                          const double* X, double* T)
{
  const int q = blockIdx.y, c = blockIdx.x;
  const int f = f1list[q0 + q];
  const long long* cp = cptr_base + (size_t)f * (n + 1);
  const long long beg = csc_ptr[f] + cp[c], end = csc_ptr[f] + cp[c + 1];
  double* Tc = T + (size_t)q * n * n + (size_t)n * c;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double s = 0.0;
    for (long long e = beg; e < end; ++e) s += X[i + (size_t)n * csc_row[e]] * csc_val[e];
    Tc[i] = s;
  }
}

// F1 step 3 (calF1, sdpa_newton.cpp:885-889, driver :1868-1907):
// B_ij += A_i . G_j for every i dominated by j, for the (up to 32) j of a
// chunk at once.  With A_i symmetric and stored as upper entries,
// A_i . G_j = sum over entries (r <= c) of v * H_j(r, c), where
// H_j(r, c) = G_j(r, c) + G_j(c, r) off the diagonal and G_j(r, r) on it.
// k_f1_pack forms H for the whole chunk as rows of 32 doubles, one row per
// upper position (packed index c (c + 1) / 2 + r, column q = chunk entry);
// k_f1_spmm then reads one 256-byte row per entry of A_i for all j of the
// chunk together (lane = q): each entry of A_i is read once per chunk, not
// once per j, and every G read is coalesced.
constexpr int F1_PACK_T = 16;                        // position tile (16 x 16)
constexpr int F1_PACK_LD = 33;                       // padded q stride of the staged tile
constexpr size_t F1_PACK_SMEM =
    ((size_t)F1_PACK_T * F1_PACK_T * F1_PACK_LD + F1_PACK_T * (F1_PACK_T + 1)) * sizeof(double);

__device__ __forceinline__ size_t f1_packed(int r, int c) { return (size_t)c * (c + 1) / 2 + r; }

// One block per 16 x 16 tile on or above the diagonal (blockIdx.x indexes
// those tiles row-major over the packed upper triangle of tiles).
__global__ void __launch_bounds__(256) k_f1_pack(int n, int cnt, const double* G, double* H)
{
  extern __shared__ double f1s[];
  double* St = f1s;                                       // [256][33]
  double* Tt = f1s + F1_PACK_T * F1_PACK_T * F1_PACK_LD;  // [16][17] transposed tile
  // tile (tr, tc) with tr <= tc from the linear index
  const long long k = blockIdx.x;
  int tc = (int)((sqrt(8.0 * (double)k + 1.0) - 1.0) * 0.5);
  while ((long long)tc * (tc + 1) / 2 > k) --tc;
  while ((long long)(tc + 1) * (tc + 2) / 2 <= k) ++tc;
  const int tr = (int)(k - (long long)tc * (tc + 1) / 2);
  const int r0 = tr * F1_PACK_T, c0 = tc * F1_PACK_T;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int r = r0 + tx, c = c0 + ty;
  const size_t nn = (size_t)n * n;
  for (int q = 0; q < cnt; ++q) {
    const double* Gq = G + q * nn;
    Tt[ty * (F1_PACK_T + 1) + tx] = (c0 + tx < n && r0 + ty < n) ? Gq[(c0 + tx) + (size_t)n * (r0 + ty)] : 0.0;
    const double a = (r < n && c < n) ? Gq[r + (size_t)n * c] : 0.0;
    __syncthreads();
    St[threadIdx.x * F1_PACK_LD + q] = (r == c) ? a : a + Tt[tx * (F1_PACK_T + 1) + ty];
    __syncthreads();
  }
  for (int t = threadIdx.x; t < F1_PACK_T * F1_PACK_T * cnt; t += blockDim.x) {
    const int lp = t / cnt, q = t - lp * cnt;
    const int rr = r0 + (lp & 15), cc = c0 + (lp >> 4);
    if (rr > cc || cc >= n) continue;
    H[f1_packed(rr, cc) * 32 + q] = St[lp * F1_PACK_LD + q];
  }
}

// Warp (constraint il, part blockIdx.y of its entries); lane q = chunk entry.
__global__ void __launch_bounds__(256) k_f1_spmm(int nc, int q0, int cnt, const int* f1list, const int* cons,
                                                 const long long* ptr, const int* pos, const double* val,
                                                 const int* nnz, const double* H, double* B, int m)
{
  const int lane = threadIdx.x & 31;
  const int il = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (il >= nc) return;
  const int gi = cons[il], inz = nnz[il];
  int gj = 0;
  bool dom = false;
  if (lane < cnt) {
    const int jl = f1list[q0 + lane];
    gj = cons[jl];
    const int jnz = nnz[jl];
    dom = !(jnz < inz || (inz == jnz && gi < gj));
  }
  if (!__any_sync(0xffffffffu, dom)) return;
  const long long beg = ptr[il], end = ptr[il + 1];
  const int parts = gridDim.y;
  double acc = 0.0;
  for (long long e0 = beg + 32LL * blockIdx.y; e0 < end; e0 += 32LL * parts) {
    const long long e = e0 + lane;
    const int p = (e < end) ? pos[e] : 0;
    const double v = (e < end) ? val[e] : 0.0;
    const int ne = (int)min(32LL, end - e0);
#pragma unroll 8
    for (int u = 0; u < 32; ++u) {
      if (u >= ne) break;
      const int pu = __shfl_sync(0xffffffffu, p, u);
      const double vu = __shfl_sync(0xffffffffu, v, u);
      acc += vu * H[(size_t)pu * 32 + lane];
    }
  }
  if (dom) {
    atomicAdd(&B[gi + (size_t)m * gj], acc);
    if (gi != gj) atomicAdd(&B[gj + (size_t)m * gi], acc);
  }
}

// F1/F2 columns of every SDP block of order <= SMALL_F1 in one launch (the
// same products as k_f1_left + gemm + k_f1_pack + k_f1_spmm, which a block
// of order 10 would otherwise pay four launches per chunk for).  One thread
// block per (SDP block, F1 constraint j), found by binary search over off:
// T = X A_j and G = T Z^-1 in shared memory, then one warp per constraint i
// of the block that j dominates: B_ij += A_i . G (upper entries of A_i,
// G(r, c) + G(c, r) off the diagonal).
constexpr int SMALL_F1 = 64;

struct F1Desc {
  const int* f1;
  const long long *cptr, *csc_ptr;
  const int* csc_row;
  const double* csc_val;
  const int* cons;
  const long long* ptr;
  const int *row, *col;
  const double* val;
  const int* nnz;
  const double *X, *Zi;
  int nc, n;
};

__global__ void __launch_bounds__(256) k_f1_small(const F1Desc* d, const long long* off, int nb, double* B, int m)
{
  extern __shared__ double f1sm[];
  const long long t = blockIdx.x;
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (off[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  const F1Desc& q = d[lo];
  const int n = q.n, nn = n * n;
  const int jl = q.f1[t - off[lo]];
  double* T = f1sm;
  double* G = f1sm + nn;
  const long long* cp = q.cptr + (size_t)jl * (n + 1);
  const long long base = q.csc_ptr[jl];
  for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
    const int i = idx % n, c = idx / n;
    double s = 0.0;
    for (long long e = base + cp[c]; e < base + cp[c + 1]; ++e) s += q.X[i + (size_t)n * q.csc_row[e]] * q.csc_val[e];
    T[idx] = s;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nn; idx += blockDim.x) {
    const int i = idx % n, c = idx / n;
    const double* zc = q.Zi + (size_t)n * c;
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += T[i + n * k] * __ldg(zc + k);
    G[idx] = s;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gj = q.cons[jl], jnz = q.nnz[jl];
  for (int il = warp; il < q.nc; il += blockDim.x >> 5) {
    const int gi = q.cons[il], inz = q.nnz[il];
    if (jnz < inz || (inz == jnz && gi < gj)) continue;
    double acc = 0.0;
    for (long long e = q.ptr[il] + lane; e < q.ptr[il + 1]; e += 32) {
      const int r = q.row[e], c = q.col[e];
      const double h = (r == c) ? G[r + n * c] : G[r + n * c] + G[c + n * r];
      acc += q.val[e] * h;
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      atomicAdd(&B[gi + (size_t)m * gj], acc);
      if (gi != gj) atomicAdd(&B[gj + (size_t)m * gi], acc);
    }
  }
}

// LP part of the Schur complement (compute_bMat_dense_LP,
// sdpa_newton.cpp:2562-2602): B_ij += x_t z_t^-1 a_it a_jt for each LP
// coordinate t and each pair of constraints touching it.  One block per t.
__global__ void k_lp_bmat(const long long* tptr, const int* tk, const double* tv, const double* x,
                          const double* zi, double* B, int m)
{
  const int t = blockIdx.x;
  const long long beg = tptr[t], cnt = tptr[t + 1] - beg;
  const double xz = x[t] * zi[t];
  for (long long p = threadIdx.x; p < cnt * cnt; p += blockDim.x) {
    const long long a1 = p % cnt, a2 = p / cnt;
    if (a2 < a1) continue;  // k2 >= k1 in list order
    const int j = tk[beg + a1], i = tk[beg + a2];
    const double v = xz * tv[beg + a2] * tv[beg + a1];
    atomicAdd(&B[i + (size_t)m * j], v);
    if (i != j) atomicAdd(&B[j + (size_t)m * i], v);
  }
}

// LP inner products per constraint: out[k] += sign * sum_t a_kt w_t
__global__ void k_lp_dot(int m, const long long* ptr, const int* idx, const double* val, const double* w,
                         double sign, double* out)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double s = 0.0;
  for (long long e = ptr[k]; e < ptr[k + 1]; ++e) s += val[e] * w[idx[e]];
  out[k] += sign * s;
}

// LP scatter: w_t += scale * sum_k coef_k a_kt (one thread per LP coordinate)
__global__ void k_lp_scatter(int nlp, const long long* tptr, const int* tk, const double* tv,
                             const double* coef, double scale, double* w)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nlp) return;
  double s = 0.0;
  for (long long e = tptr[t]; e < tptr[t + 1]; ++e) s += coef[tk[e]] * tv[e];
  w[t] += scale * s;
}

// Element-wise LP vectors
__global__ void k_lp_ops(int op, int nlp, double a, double b, double* o, const double* x, const double* y,
                         const double* z, const double* w)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nlp) return;
  switch (op) {
    case 0: o[t] = a * x[t] - y[t]; break;                         // R = a zi - x
    case 1: o[t] = (a * x[t] - y[t]) - z[t] * w[t] * x[t]; break;  // R = a zi - x - dx dz zi
    case 2: o[t] = x[t] * y[t] * z[t]; break;                      // x D zi
    case 3: o[t] = x[t] - y[t] * z[t] * w[t]; break;               // dx = R - x dz zi
    default: break;
  }
}

// 1/x, 1/sqrt(x) of the LP block (Jal::getInvChol / getInvCholAndInv LP part,
// sdpa_jordan.cpp:170-177, :201-203); flags x < 0.
__global__ void k_lp_inv(int nlp, const double* x, double* lx, double* xi, int* bad)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nlp) return;
  if (x[t] < 0.0) atomicOr(bad, 1);
  lx[t] = 1.0 / sqrt(x[t]);
  if (xi) xi[t] = 1.0 / x[t];
}

// Deterministic reductions (mode 0: dot product, mode 1: max |a|): per-block
// partials, then an in-order combination.
__global__ void k_dot_partial(long long len, const double* a, const double* b, double* part, int mode)
{
  double s = 0.0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < len;
       t += (long long)gridDim.x * blockDim.x) {
    if (mode == 0) s += a[t] * b[t];
    else s = fmax(s, fabs(a[t]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_xor_sync(0xffffffffu, s, o);
    s = (mode == 1) ? fmax(s, v) : s + v;
  }
  __shared__ double w[32];
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) r = (mode == 1) ? fmax(r, w[q]) : r + w[q];
    part[blockIdx.x] = r;
  }
}

__global__ void k_dot_final(int np, const double* part, double* out, int mode, int accumulate, double scale)
{
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double r = 0.0;
  for (int q = 0; q < np; ++q) r = (mode == 1) ? fmax(r, part[q]) : r + part[q];
  r *= scale;
  if (accumulate) *out = (mode == 1) ? fmax(*out, r) : *out + r;
  else *out = r;
}

// ---- all SDP blocks in one launch.  The n_q x n_q matrices of the blocks
// form one flat range (block q at [eoff[q], eoff[q + 1])); which matrix of a
// block is meant is a kind, looked up in tab[kind * nb + q].  A problem of
// 200 blocks of order 10 would otherwise pay one or two launches per block
// for every inner product, residual and update.
enum { MB_X, MB_Z, MB_DX, MB_DZ, MB_C, MB_X0, MB_Z0, MB_D, MB_R, MB_W1, MB_W2, MB_ZI, MB_KINDS };

// walks the part [c0, c1) of the flat range: f(q, local index, n_q, flat index)
template <typename F>
__device__ __forceinline__ void mb_walk(const long long* eoff, const int* nq, int nb, long long c0, long long c1,
                                        F f)
{
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (eoff[mid] <= c0) lo = mid;
    else hi = mid - 1;
  }
  for (int q = lo; q < nb && eoff[q] < c1; ++q) {
    const long long b = max(c0, eoff[q]), e = min(c1, eoff[q + 1]);
    for (long long t = b + threadIdx.x; t < e; t += blockDim.x) f(q, t - eoff[q], nq[q], t);
  }
}

// Deterministic reduction over every block (mode 0: sum of a .* b, mode 1:
// max |a|, mode 2: sum of the diagonals of a); block c of the grid takes the
// c-th chunk and writes part[c] (combined by k_dot_final).
__global__ void k_mb_reduce(const double* const* tab, int ka, int kb, const long long* eoff, const int* nq, int nb,
                            long long chunk, double* part, int mode)
{
  const double* const* A = tab + (size_t)ka * nb;
  const double* const* Bv = tab + (size_t)kb * nb;
  const long long c0 = blockIdx.x * chunk, c1 = min(eoff[nb], c0 + chunk);
  double s = 0.0;
  mb_walk(eoff, nq, nb, c0, c1, [&](int q, long long l, int n, long long) {
    const double a = A[q][l];
    if (mode == 0) s += a * Bv[q][l];
    else if (mode == 1) s = fmax(s, fabs(a));
    else if (l % (n + 1) == 0) s += a;
  });
  for (int o = 16; o > 0; o >>= 1) {
    const double v = __shfl_xor_sync(0xffffffffu, s, o);
    s = (mode == 1) ? fmax(s, v) : s + v;
  }
  __shared__ double w[32];
  if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) r = (mode == 1) ? fmax(r, w[q]) : r + w[q];
    part[blockIdx.x] = r;
  }
}

// out = a x + b y over every block (ky < 0: out = a x)
__global__ void k_mb_axpby(double* const* tab, int ko, double a, int kx, double b, int ky, const long long* eoff,
                           const int* nq, int nb, long long chunk)
{
  double* const* O = tab + (size_t)ko * nb;
  double* const* Xv = tab + (size_t)kx * nb;
  double* const* Yv = ky >= 0 ? tab + (size_t)ky * nb : nullptr;
  const long long c0 = blockIdx.x * chunk, c1 = min(eoff[nb], c0 + chunk);
  mb_walk(eoff, nq, nb, c0, c1, [&](int q, long long l, int, long long) {
    O[q][l] = a * Xv[q][l] + (Yv ? b * Yv[q][l] : 0.0);
  });
}

// The constraint entries of every block: block q's constraints are warps
// [coff[q], coff[q + 1]).
struct MbSparse {
  const int* cons;
  const long long* ptr;
  const int *row, *col;
  const double* val;
  int n, q;
};

__device__ __forceinline__ int mb_find(const long long* off, int nb, long long t)
{
  int lo = 0, hi = nb - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (off[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Per-constraint inner products out[cons] += sign * (A_k . W) over the
// entries each block holds (Lal::getInnerProduct(Sparse, Dense),
// sdpa_linear.cpp:318-460), W = tab[kw]; one warp per (block, constraint).
__global__ void k_mb_sp_dot(const MbSparse* d, const long long* coff, int ns, const double* const* tab, int kw,
                            int nb, double sign, double* out)
{
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= coff[ns]) return;
  const MbSparse& B = d[mb_find(coff, ns, warp)];
  const int k = (int)(warp - coff[&B - d]);
  const double* W = tab[(size_t)kw * nb + B.q];
  const int n = B.n;
  double s = 0.0;
  for (long long e = B.ptr[k] + lane; e < B.ptr[k + 1]; e += 32) {
    const int r = B.row[e], c = B.col[e];
    const double v = B.val[e];
    s += (r == c) ? v * W[r + (size_t)n * r] : v * (W[r + (size_t)n * c] + W[c + (size_t)n * r]);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) atomicAdd(&out[B.cons[k]], sign * s);
}

// k_sp_scatter over every block: W += scale * sum_k coef[cons] A_k, W = tab[kw]
__global__ void k_mb_sp_scatter(const MbSparse* d, const long long* coff, int ns, double* const* tab, int kw, int nb,
                                const double* coef, double scale)
{
  const long long warp = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= coff[ns]) return;
  const MbSparse& B = d[mb_find(coff, ns, warp)];
  const int k = (int)(warp - coff[&B - d]);
  double* W = tab[(size_t)kw * nb + B.q];
  const int n = B.n;
  const double s = scale * (coef ? coef[B.cons[k]] : 1.0);
  for (long long e = B.ptr[k] + lane; e < B.ptr[k + 1]; e += 32) {
    const int r = B.row[e], c = B.col[e];
    const double v = s * B.val[e];
    atomicAdd(&W[r + (size_t)n * c], v);
    if (r != c) atomicAdd(&W[c + (size_t)n * r], v);
  }
}

// C = alpha op(A) op(B) + beta C over 64 x 64 output tiles, one tile per
// block, z = batch (strided); lower skips tiles above the diagonal.
template <typename TM, typename TC>
__global__ void __launch_bounds__(NT) k_gemm(int M, int N, int K, int tA, const TM* A, int lda,
                                             long long sA, int tB, const TM* B, int ldb, long long sB,
                                             TM* C, int ldc, long long sC, double alpha, double beta,
                                             int lower)
{
  extern __shared__ double smem[];
  const int r0 = blockIdx.x * cta::GT, c0 = blockIdx.y * cta::GT;
  if (lower && r0 + cta::GT - 1 < c0) return;
  const int z = blockIdx.z;
  A += sA * z;
  B += sB * z;
  C += sC * z;
  const TM* Ap = tA ? A + (size_t)lda * r0 : A + r0;
  const TM* Bp = tB ? B + c0 : B + (size_t)ldb * c0;
  cta::gemm_rect<NT, TM, TC>(min(cta::GT, M - r0), min(cta::GT, N - c0), K, tA, Ap, lda, tB, Bp, ldb,
                             C + r0 + (size_t)ldc * c0, ldc, alpha, beta, smem, lower != 0, r0 - c0);
}

// FP64 GEMM, C = alpha op(A) op(B) + beta C, one 128 x 64 output tile per
// 256-thread block (z = batch, strided; lower skips tiles above the diagonal
// and entries with row < column), on the FP64 MMA (mma.sync m8n8k4): the 8
// warps as 4 x 2 over the tile's 16 x 8 blocks of 8 x 8, warp (wr, wc)
// owning blocks (wr + 4 i, wc + 2 j), i, j < 4: 16 MMAs per K step of 4 from
// 8 fragment loads.  K is staged in chunks of 32 by cp.async into two
// stages, [k][row] with strides of 132 / 68 doubles (= 4 mod 16, so each
// half-warp's fragment loads fall on distinct banks); 100 KB, two blocks
// per SM.
constexpr int DG_M = 128, DG_N = 64, DG_K = 32, DG_AS = DG_M + 4, DG_BS = DG_N + 4;
constexpr int DG_STAGE = DG_K * (DG_AS + DG_BS);
constexpr size_t DG_SMEM = 2 * (size_t)DG_STAGE * sizeof(double);

__global__ void __launch_bounds__(256, 2) k_dgemm(int M, int N, int K, int tA, const double* A, int lda,
                                                  long long sA, int tB, const double* B, int ldb, long long sB,
                                                  double* C, int ldc, long long sC, double alpha, double beta,
                                                  int lower)
{
  extern __shared__ __align__(16) double dsm[];
  const int r0 = blockIdx.x * DG_M, c0 = blockIdx.y * DG_N;
  if (lower && r0 + DG_M - 1 < c0) return;
  const int z = blockIdx.z;
  A += sA * z;
  B += sB * z;
  C += sC * z;
  const int tid = threadIdx.x;
  const int lane = tid & 31, w = tid >> 5, wr = w & 3, wc = w >> 2, q = lane & 3, p = lane >> 2;
  auto issue = [&](int k0, int st) {
    double* As = dsm + st * DG_STAGE;
    double* Bs = As + DG_K * DG_AS;
    for (int t = tid; t < DG_K * DG_M; t += 256) {
      int r, k;
      if (!tA) { r = t % DG_M; k = t / DG_M; } else { k = t % DG_K; r = t / DG_K; }
      const int gr = r0 + r, gk = k0 + k;
      const bool v = gr < M && gk < K;
      cta::cp_async_el<double>(&As[k * DG_AS + r],
                               v ? (tA ? A + gk + (size_t)lda * gr : A + gr + (size_t)lda * gk) : A, v);
    }
    for (int t = tid; t < DG_K * DG_N; t += 256) {
      int c, k;
      if (!tB) { k = t % DG_K; c = t / DG_K; } else { c = t % DG_N; k = t / DG_N; }
      const int gc = c0 + c, gk = k0 + k;
      const bool v = gc < N && gk < K;
      cta::cp_async_el<double>(&Bs[k * DG_BS + c],
                               v ? (tB ? B + gc + (size_t)ldb * gk : B + gk + (size_t)ldb * gc) : B, v);
    }
    cta::cp_async_commit();
  };
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nch = (K + DG_K - 1) / DG_K;
  if (nch > 0) issue(0, 0);
  for (int ch = 0; ch < nch; ++ch) {
    cta::cp_async_wait_all();
    __syncthreads();  // chunk ch visible; every thread is done with the other stage
    if (ch + 1 < nch) issue((ch + 1) * DG_K, (ch + 1) & 1);
    const double* As = dsm + (ch & 1) * DG_STAGE;
    const double* Bs = As + DG_K * DG_AS;
    // rows k >= K of the last chunk are zero-filled: whole steps of 4
    const int kmax = min(DG_K, K - ch * DG_K);
#pragma unroll 2
    for (int kk = 0; kk < kmax; kk += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[(kk + q) * DG_AS + (wr + 4 * i) * 8 + p];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[(kk + q) * DG_BS + (wc + 2 * j) * 8 + p];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) cta::dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gr = r0 + (wr + 4 * i) * 8 + p;
    if (gr >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gc = c0 + (wc + 2 * j) * 8 + 2 * q + h;
        if (gc >= N || (lower && gr < gc)) continue;
        double* cp = C + gr + (size_t)ldc * gc;
        *cp = (beta == 0.0) ? alpha * acc[i][j][h] : alpha * acc[i][j][h] + beta * (*cp);
      }
    }
  }
}

// Tile-sparse trailing update of the blocked Cholesky: one block per listed
// 128 x 128 tile pair (i, j) of the lower triangle, A_ij -= P_i P_j^T with
// P the scaled panel (columns kb .. kb + bs), lower-triangular on i == j.
// Tiles the symbolic factorisation leaves zero are not touched: they stay
// exactly zero, as in the dense factorisation.
template <typename T>
__global__ void __launch_bounds__(NT) k_syrk_pairs(const int* pairs, int n, int kb, int bs, T* A)
{
  extern __shared__ double smem[];
  const int i = pairs[2 * blockIdx.x], j = pairs[2 * blockIdx.x + 1];
  const int r0 = i * 128, c0 = j * 128;
  const int M = min(128, n - r0), N = min(128, n - c0);
  cta::gemm_rect<NT, T, T>(M, N, bs, false, A + r0 + (size_t)n * kb, n, true, A + c0 + (size_t)n * kb, n,
                           A + r0 + (size_t)n * c0, n, -1.0, 1.0, smem, i == j, 0);
}

// Li = L^{-1} of a bs x bs lower-triangular block (lda) into Li (ld bs)
template <typename T>
__global__ void __launch_bounds__(NT) k_tri_inv(int bs, const T* L, int lda, T* Li, int ldi, const int* flag)
{
  extern __shared__ double smem[];
  T* sD = (T*)(smem + cta::GEMM_RECT_SMEM);
  if (flag && *flag) return;
  cta::tri_inverse<NT, T>(bs, L, lda, Li, ldi, sD, smem);
}

// x = L^{-T} L^{-1} x (Lal::solveSystems, sdpa_linear.cpp:843-862)
template <typename T>
__global__ void __launch_bounds__(NT) k_chol_solve(int m, const T* L, T* x)
{
  extern __shared__ double smem[];
  cta::chol_solve<NT, T>(m, L, m, x, (T*)smem);
}

// element-wise conversion between precisions
template <typename TO, typename TI>
__global__ void k_convert(long long n, TO* out, const TI* in)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) out[t] = (TO)in[t];
}

// Blocked triangular solves with the stored diagonal-block inverses of the
// Cholesky factor (one block: x_b = Dinv_b x_b or Dinv_b^T x_b).
// 512 threads: row i = threadIdx.x % 128 (bs <= 128), column group
// g = threadIdx.x / 128 takes every fourth column; the four partial sums are
// reduced in shared memory.  Rows read Dinv coalesced (consecutive i) in
// the forward product; the transposed product reads row i's column
// segment, contiguous per thread.
template <typename T>
__global__ void __launch_bounds__(512) k_trsv_diag(int bs, const T* Dinv, T* x, int trans)
{
  __shared__ T xs[128];
  __shared__ T part[4][129];
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xs[i] = x[i];
  __syncthreads();
  const int i = threadIdx.x & 127, g = threadIdx.x >> 7;
  T s = (T)0;
  if (i < bs) {
    if (!trans)
      for (int p = g; p <= i; p += 4) s += Dinv[i + (size_t)bs * p] * xs[p];
    else
      for (int p = i + ((g - i) & 3); p < bs; p += 4) s += Dinv[p + (size_t)bs * i] * xs[p];
  }
  part[g][i] = s;
  __syncthreads();
  if (g == 0 && i < bs) x[i] = part[0][i] + part[1][i] + part[2][i] + part[3][i];
}

// forward update: x[r] -= sum_p L[r, kb+p] x[kb+p] for the rows below the
// block.  256-thread blocks of 32 rows x 8 column groups (each column read
// by 32 consecutive rows, 256 bytes in FP64), partial sums reduced in shared
// memory: eight times the threads of one thread per row, so a panel of
// ~10^4 rows spreads over a few hundred blocks.
template <typename T>
__global__ void __launch_bounds__(256) k_trsv_fwd_update(int rows, int bs, const T* Lp, int ld, const T* xb, T* xr)
{
  __shared__ T xs[256];
  __shared__ T part[8][33];
  for (int i = threadIdx.x; i < bs; i += blockDim.x) xs[i] = xb[i];
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int r = blockIdx.x * 32 + tx;
  T s = (T)0;
  if (r < rows)
    for (int p = ty; p < bs; p += 8) s += Lp[r + (size_t)ld * p] * xs[p];
  part[ty][tx] = s;
  __syncthreads();
  if (ty == 0 && r < rows) {
    T t = part[0][tx];
#pragma unroll
    for (int g = 1; g < 8; ++g) t += part[g][tx];
    xr[r] -= t;
  }
}

// backward update: x[i] -= sum_p L[kb+p, i] x[kb+p] for i < kb (one warp per i)
template <typename T>
__global__ void k_trsv_bwd_update(int kb, int bs, const T* Lrow, int ld, const T* xb, T* x)
{
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= kb) return;
  T s = (T)0;
  for (int p = lane; p < bs; p += 32) s += Lrow[p + (size_t)ld * warp] * xb[p];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) x[warp] -= s;
}

// x += (double) v
__global__ void k_add_f32(int m, double* x, const float* v)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < m) x[t] += (double)v[t];
}

// r = g - B x for the symmetric m x m FP64 Schur matrix (column i dotted with
// x, one warp per i): the FP64 residual of the iterative refinement.
__global__ void k_residual(int m, const double* B, const double* x, const double* g, double* r)
{
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= m) return;
  const double* col = B + (size_t)m * warp;
  double s = 0.0;
  for (int k = lane; k < m; k += 32) s += col[k] * x[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) r[warp] = g[warp] - s;
}

// minimum eigenvalue of a formed M = L D L^T (n x n, global) into *out
__global__ void __launch_bounds__(NT) k_min_eig(int n, const double* M, double* out)
{
  extern __shared__ double smem[];
  __shared__ double redbuf[4 * (NT / 32)];
  cta::Reducer RD{redbuf, 0};
  EigScratch es;
  eig_scratch_carve(es, smem, n, &RD, 1);
  const double v = (n > 20) ? lanczos_min_eig(n, M, es) : dense_min_eig(n, M, es);
  if (threadIdx.x == 0) *out = v;
}

// Many small SDP blocks: one 256-thread block per SDP block of order <= 96
// runs the per-block steps with the block-level routines of the batched
// engine, in one launch for all of them (instead of several launches and a
// host read-back per block).
constexpr int SMALL_BLOCK = 96;
constexpr int SB_GSM = 4 * 16 * 100;  // GEMM staging: the double-buffered n <= 96 MMA tile

struct BlockPtrs {
  double *X, *Z, *Zi, *LXi, *LZi, *W1, *W2, *R, *XDZ, *dX, *dZ, *D;
  // the constraints touching the block: global index, entry ranges, entries
  const int* cons;
  const long long* ptr;
  const int *row, *col;
  const double* val;
  int n, nc;
};

static size_t small_block_smem(int nmax)
{
  return (size_t)(SB_GSM + 2 * cta::SD_DOUBLES + eig_scratch_doubles(nmax, 2)) * sizeof(double);
}

// Solutions::update's inverses (sdpa_dataset.cpp:117-171) per block: the
// Cholesky factors of X and Z in lockstep (LAPACK's pivot rule), their
// inverses L_X^-1, L_Z^-1 and Z^-1 = L_Z^-T L_Z^-1; *flag = 1 if a factor fails.
__global__ void __launch_bounds__(NT) k_blocks_inverse(const BlockPtrs* bp, int* flag)
{
  extern __shared__ double smem[];
  __shared__ int s_flag2[2];
  double* gsm = smem;
  double* sD = gsm + SB_GSM;
  double* sD2 = sD + cta::SD_DOUBLES;
  const BlockPtrs b = bp[blockIdx.x];
  const int n = b.n, nn = n * n;
  for (int t = threadIdx.x; t < nn; t += NT) {
    b.W1[t] = b.X[t];
    b.W2[t] = b.Z[t];
  }
  __syncthreads();
  if (cta::cholesky_pair<NT, double>(n, b.W1, b.W2, n, sD, sD2, gsm, s_flag2)) {
    if (threadIdx.x == 0) atomicExch(flag, 1);
    return;
  }
  cta::tri_inverse_pair<NT, double>(n, b.W1, b.W2, n, b.LXi, b.LZi, n, sD, sD2, gsm);
  cta::gemm<NT>(n, true, b.LZi, n, false, b.LZi, n, b.Zi, n, 1.0, 0.0, gsm);
}

// Newton direction per block (compute_DzMat / compute_DxMat,
// sdpa_newton.cpp:2718-2752): dZ = D (dual infeasible) or 0, minus
// sum_k dy_k A_k; dX = sym(R - X dZ Z^-1) (Lal::getSymmetrize); the products
// in FP32 when lowp (mixed precision).
__global__ void __launch_bounds__(NT) k_blocks_direction(const BlockPtrs* bp, const double* dy, int dinf, int lowp)
{
  extern __shared__ double smem[];
  const BlockPtrs b = bp[blockIdx.x];
  const int n = b.n, nn = n * n;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < nn; t += NT) b.dZ[t] = dinf ? b.D[t] : 0.0;
  __syncthreads();
  for (int k = wid; k < b.nc; k += NT / 32) {
    const double sc = -dy[b.cons[k]];
    for (long long e = b.ptr[k] + lane; e < b.ptr[k + 1]; e += 32) {
      const int r = b.row[e], c = b.col[e];
      const double v = sc * b.val[e];
      atomicAdd(&b.dZ[r + (size_t)n * c], v);
      if (r != c) atomicAdd(&b.dZ[c + (size_t)n * r], v);
    }
  }
  __syncthreads();
  cta::gemm_prec<NT, double>(n, false, b.X, n, false, b.dZ, n, b.W1, n, 1.0, 0.0, smem, lowp != 0);
  cta::gemm_prec<NT, double>(n, false, b.W1, n, false, b.Zi, n, b.W2, n, 1.0, 0.0, smem, lowp != 0);
  for (int t = threadIdx.x; t < nn; t += NT) {
    const int i = t % n, j = t / n;
    if (i < j) continue;
    const double lo = b.R[i + (size_t)n * j] - b.W2[i + (size_t)n * j];
    const double up = b.R[j + (size_t)n * i] - b.W2[j + (size_t)n * i];
    const double v = 0.5 * (lo + up);
    b.dX[i + (size_t)n * j] = v;
    b.dX[j + (size_t)n * i] = v;
  }
}

// Corrector right-hand side per block (Newton::Mehrotra(CORRECTOR),
// sdpa_newton.cpp:2755-2809): R = (beta mu Z^-1 - X) - dX dZ Z^-1 and, when
// the point is dual infeasible, W1 = R - X D Z^-1.
__global__ void __launch_bounds__(NT) k_blocks_corrector(const BlockPtrs* bp, double bmu, int dinf, int lowp)
{
  extern __shared__ double smem[];
  const BlockPtrs b = bp[blockIdx.x];
  const int n = b.n, nn = n * n;
  cta::gemm_prec<NT, double>(n, false, b.dX, n, false, b.dZ, n, b.W1, n, 1.0, 0.0, smem, lowp != 0);
  cta::gemm_prec<NT, double>(n, false, b.W1, n, false, b.Zi, n, b.W2, n, 1.0, 0.0, smem, lowp != 0);
  for (int t = threadIdx.x; t < nn; t += NT) {
    const double r = (bmu * b.Zi[t] + -1.0 * b.X[t]) - b.W2[t];
    b.R[t] = r;
    if (dinf) b.W1[t] = 1.0 * r + -1.0 * b.XDZ[t];
  }
}

// Step length per block (Jal::getMinEigen, sdpa_jordan.cpp:58-109): the
// minimum eigenvalues of L_X^-1 dX L_X^-T and L_Z^-1 dZ L_Z^-T, with the
// two Lanczos processes in lockstep; out[2 b], out[2 b + 1].  R and XDZ are
// scratch here (rebuilt by the next predictor).
__global__ void __launch_bounds__(NT) k_blocks_step(const BlockPtrs* bp, int nmax, double* out)
{
  extern __shared__ double smem[];
  __shared__ double redbuf[4 * (NT / 32)];
  cta::Reducer RD{redbuf, 0};
  EigScratch es;
  eig_scratch_carve(es, smem + SB_GSM + 2 * cta::SD_DOUBLES, nmax, &RD, 2);
  const BlockPtrs b = bp[blockIdx.x];
  double mins[2];
  min_eig_pair(b.n, b.LXi, b.dX, b.LZi, b.dZ, b.W1, b.W2, b.R, b.XDZ, smem, SB_GSM, es, mins, false);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = mins[0];
    out[2 * blockIdx.x + 1] = mins[1];
  }
}

// ------------------------------------------------------------------ host side

static inline int nblk(long long n, int t = 256) { return (int)((n + t - 1) / t); }

struct SdpBlock {
  int n = 0;
  int fileBlock = 0;  // 1-based
  // device dense matrices (n x n)
  double *C = nullptr, *X = nullptr, *Z = nullptr, *Zi = nullptr, *LXi = nullptr, *LZi = nullptr;
  double *D = nullptr, *XDZ = nullptr, *R = nullptr, *dX = nullptr, *dZ = nullptr, *W1 = nullptr,
         *W2 = nullptr, *X0 = nullptr, *Z0 = nullptr, *Lt = nullptr;
  // constraints touching this block (host-built, device copies)
  int nc = 0;
  std::vector<int> hcons, hnnz, hform;
  std::vector<long long> hptr;
  std::vector<int> hrow, hcol;
  std::vector<double> hval;
  int *cons = nullptr, *nnz = nullptr, *form = nullptr, *row = nullptr, *col = nullptr;
  int* pos = nullptr;  // packed upper position c (c + 1) / 2 + r of each entry (F1 inner products)
  long long* ptr = nullptr;
  double* val = nullptr;
  // F1/F2 constraints (local indices) and their symmetric CSC
  std::vector<int> hf1;
  int* f1 = nullptr;
  long long *csc_cptr = nullptr, *csc_ptr = nullptr;
  int* csc_row = nullptr;
  double* csc_val = nullptr;
};

// A captured grid solve (chol_solve_graph).
struct SolveGraph {
  const void* L;
  const void* dinv;
  void* x;
  int m;
  cudaGraphExec_t exec;
};

struct DevState {
  int m = 0, nlp = 0, nDim = 0;
  std::vector<SolveGraph> solve_graphs;
  // look-ahead of the grid Cholesky: the next diagonal block is factored on
  // `side` (non-blocking) while the trailing update runs on the default stream
  cudaStream_t side = nullptr;
  cudaEvent_t ev_next = nullptr, ev_diag = nullptr;
  // tile-sparse Schur factorisation: for panel k, the trailing 128 x 128
  // tile pairs (i, j), i >= j >= k + 2, that the symbolic factorisation
  // marks nonzero, at pairs[2 pair_off[k] ..]
  // SDP blocks of order <= SMALL_BLOCK, handled by k_blocks_* (device
  // descriptors), the others one by one; per-block step-length minima
  std::vector<int> small_idx, large_idx;
  BlockPtrs* small_ptrs = nullptr;
  int small_nmax = 0;
  double* blk_mins = nullptr;
  // F3 assembly of all blocks in one launch (k_f3_all)
  F3Desc* f3_desc = nullptr;
  long long* f3_off = nullptr;
  long long f3_total = 0;
  int f3_nb = 0;
  // the Schur matrix has one source (k_f3_tiles): the SDP block of index
  // f3_direct_block, touched by every constraint, all F3, no LP block
  int f3_direct_block = -1;
  int* f3_heavy = nullptr;   // its heavy pairs (i, j), i >= j (k_f3_heavy)
  int f3_nheavy = 0;
  // F1 columns of the blocks of order <= SMALL_F1 in one launch (k_f1_small)
  F1Desc* f1_desc = nullptr;
  long long* f1_off = nullptr;
  long long f1_total = 0;
  int f1_nb = 0, f1_nmax = 0;
  // every SDP block as one flat range (k_mb_*): matrix table
  // [kind * nsdp + q], offsets and orders, constraint descriptors
  double** mb_tab = nullptr;
  long long* mb_eoff = nullptr;
  int* mb_nq = nullptr;
  long long mb_total = 0;
  MbSparse* mb_sp = nullptr;
  long long* mb_coff = nullptr;
  long long mb_ctotal = 0;
  int mb_ns = 0;
  bool sparse = false;
  std::vector<long long> pair_off;
  int* pairs = nullptr;
  long long dense_pairs = 0, sparse_pairs = 0;
  Params prm;
  std::vector<int> blockStruct, blockKind, blockIndex;  // kind 0 SDP, 2 LP; index = SDP idx or LP offset
  std::vector<SdpBlock> sdp;
  // LP
  double *lpC = nullptr, *lpx = nullptr, *lpz = nullptr, *lpzi = nullptr, *lplx = nullptr, *lplz = nullptr,
         *lpD = nullptr, *lpR = nullptr, *lpXDZ = nullptr, *lpdx = nullptr, *lpdz = nullptr, *lpW = nullptr,
         *lpx0 = nullptr, *lpz0 = nullptr, *lptmp = nullptr;
  long long *lp_ptr = nullptr, *lpT_ptr = nullptr;
  int *lp_idx = nullptr, *lpT_k = nullptr;
  double *lp_val = nullptr, *lpT_v = nullptr;
  // vectors
  double *b = nullptr, *y = nullptr, *dy = nullptr, *g = nullptr, *rp = nullptr, *ytmp = nullptr;
  double* B = nullptr;      // m x m
  double* Linv = nullptr;   // panel inverse scratch (NBG x NBG)
  double* T = nullptr;      // panel / F1 scratch
  size_t Tsize = 0;
  float *B32 = nullptr, *Linv32 = nullptr, *T32 = nullptr, *v32 = nullptr;  // mixed-precision Schur
  double* dinv = nullptr;   // diagonal-block inverses of the Schur factor (large m)
  float* dinv32 = nullptr;
  double* res = nullptr;    // refinement residual
  int mixed = 0;
  double mu_switch = 1.0e-2;
  double* part = nullptr;   // reduction partials
  double* sc = nullptr;     // scalar slots
  int* flag = nullptr;
  int* tc_err = nullptr;    // tensor-core update time-out flag (inside the flag allocation)
  bool tc = false;          // mixed mode: tensor-core trailing updates of the FP32 Schur factor
  void* tc_work = nullptr;  // their split operands (syrk_tf32x3_work_bytes(m, NBG))
  int* tc_f1_err = nullptr;   // time-out flag of the tensor-core F1 products
  void* tc_f1_work = nullptr; // split operands of the tensor-core F1 products (mixed mode)
  long long tc_wait = -1;     // polls per wait of the tensor-core pipelines (< 0: their default)
  std::vector<void*> allocs;
  double* alloc(size_t n)
  {
    void* p = nullptr;
    if (n == 0) n = 1;
    if (cudaMalloc(&p, n * sizeof(double)) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    return (double*)p;
  }
  template <class T>
  T* upload(const std::vector<T>& v)
  {
    void* p = nullptr;
    size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    allocs.push_back(p);
    if (!v.empty()) cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return (T*)p;
  }
  ~DevState()
  {
    for (SolveGraph& g : solve_graphs) cudaGraphExecDestroy(g.exec);
    if (ev_next) cudaEventDestroy(ev_next);
    if (ev_diag) cudaEventDestroy(ev_diag);
    if (side) cudaStreamDestroy(side);
    for (void* p : allocs) cudaFree(p);
  }
};

static const int NBG = 128;        // panel width of the grid-level Cholesky
static const int F1_CHUNK = 32;    // F1 constraints processed per batched GEMM (= warp lanes in k_f1_spmm)
static const int SMALL_SOLVE = 512;   // Schur orders up to this use the one-block solve

static size_t chol_smem() { return (cta::GEMM_RECT_SMEM + cta::SD_DOUBLES) * sizeof(double); }

template <typename TM, typename TC>
static void gemm_t(int M, int N, int K, bool tA, const TM* A, int lda, bool tB, const TM* B, int ldb, TM* C,
                   int ldc, double alpha, double beta, bool lower = false, int batch = 1, long long sA = 0,
                   long long sB = 0, long long sC = 0)
{
  if (M <= 0 || N <= 0) return;
  // The 128 x 64 tile pays off on the long-K products of the Schur build;
  // the Cholesky's panel and trailing updates (K <= 128) stay on 64 x 64.
  if constexpr (std::is_same<TM, double>::value && std::is_same<TC, double>::value) if (K > 128) {
    static std::atomic<unsigned long long> attr{0};
    smem_attr_per_device((const void*)k_dgemm, (int)DG_SMEM, attr);
    dim3 g((M + DG_M - 1) / DG_M, (N + DG_N - 1) / DG_N, batch);
    k_dgemm<<<g, 256, DG_SMEM>>>(M, N, K, tA, A, lda, sA, tB, B, ldb, sB, C, ldc, sC, alpha, beta, lower ? 1 : 0);
    return;
  }
  dim3 grid((M + cta::GT - 1) / cta::GT, (N + cta::GT - 1) / cta::GT, batch);
  k_gemm<TM, TC><<<grid, NT, cta::GEMM_RECT_SMEM * sizeof(double)>>>(M, N, K, tA, A, lda, sA, tB, B, ldb, sB,
                                                                       C, ldc, sC, alpha, beta, lower ? 1 : 0);
}

// FP64 matrices; lowp = FP32 products (mixed precision)
static void gemm(DevState& S, int M, int N, int K, bool tA, const double* A, int lda, bool tB,
                 const double* B, int ldb, double* C, int ldc, double alpha, double beta, bool lower = false,
                 int batch = 1, long long sA = 0, long long sB = 0, long long sC = 0, bool lowp = false)
{
  if (lowp)
    gemm_t<double, float>(M, N, K, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, lower, batch, sA, sB, sC);
  else
    gemm_t<double, double>(M, N, K, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, lower, batch, sA, sB, sC);
}

// Blocked right-looking Cholesky of an n x n matrix (lda = n) in place, in
// the matrix's own precision T (FP32 for the mixed-precision Schur factor).
// Linv: NBG x NBG scratch, Tb: n x NBG scratch.  Returns 0 or the failing
// column + 1.
//
// Look-ahead: the diagonal factor and inverse of block k+1 are single-block
// kernels on a chain that does not shrink with n.  After panel k is formed,
// only block column k+1 is updated first; block k+1 is then factored and
// inverted on the side stream while the trailing update of the remaining
// columns runs on the default stream (the side stream has the higher
// priority, so its blocks are scheduled first).  Events order the two streams; the
// shared Linv scratch is overwritten only after panel k's product has read
// it.
template <typename T>
static int cholesky_grid_t(DevState& S, T* A, int n, bool adjust, T* Linv, T* Tb, T* dinv_store = nullptr)
{
  cudaMemset(S.flag, 0, sizeof(int));
  if (!S.side) {
    // highest priority: its single-block kernels go ahead of the trailing
    // update's queued blocks instead of waiting for its last wave
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&S.side, cudaStreamNonBlocking, hi) != cudaSuccess) S.side = nullptr;
    if (S.side && (cudaEventCreateWithFlags(&S.ev_next, cudaEventDisableTiming) != cudaSuccess ||
                   cudaEventCreateWithFlags(&S.ev_diag, cudaEventDisableTiming) != cudaSuccess)) {
      cudaGetLastError();
      cudaStreamDestroy(S.side);
      S.side = nullptr;
    }
  }
  static_assert(NBG == DB_MAX, "diagonal blocks of the grid Cholesky are factored by k_chol_inv_diag");
  static std::atomic<unsigned long long> diag_attr{0};
  smem_attr_per_device((const void*)k_chol_inv_diag<T>, (int)diag_block_smem<T>(), diag_attr);
  auto Li_of = [&](int kb) { return dinv_store ? dinv_store + (size_t)(kb / NBG) * NBG * NBG : Linv; };
  // factor (and, if a panel or the stored inverses need it, invert) the
  // diagonal block at kb on stream st
  auto diag = [&](int kb, cudaStream_t st) {
    const int bs = std::min(NBG, n - kb);
    T* Ad = A + kb + (size_t)n * kb;
    T* Li = (n - kb - bs > 0 || dinv_store) ? Li_of(kb) : nullptr;
    k_chol_inv_diag<T><<<1, DB_NT, diag_block_smem<T>(), st>>>(bs, Ad, n, adjust ? 1 : 0, kb, S.flag, Li, bs);
  };
  diag(0, 0);
  for (int kb = 0; kb < n; kb += NBG) {
    const int bs = std::min(NBG, n - kb);
    const int rem = n - kb - bs;
    if (rem <= 0) break;
    if (kb > 0 && S.side) cudaStreamWaitEvent(0, S.ev_diag, 0);  // diagonal block kb (side stream)
    T* Li = Li_of(kb);
    T* P = A + (kb + bs) + (size_t)n * kb;
    // panel: P <- P L_bb^{-T}
    gemm_t<T, T>(rem, bs, bs, false, P, n, true, Li, bs, Tb, rem, 1.0, 0.0);
    k_copy2d_t<T><<<nblk((long long)rem * bs), 256>>>(rem, bs, Tb, rem, P, n);
    // block column kb+1 first, then its diagonal block on the side stream
    const int nb2 = std::min(NBG, rem);
    T* A22 = A + (kb + bs) + (size_t)n * (kb + bs);
    gemm_t<T, T>(rem, nb2, bs, false, P, n, true, P, n, A22, n, -1.0, 1.0, true);
    if (S.side) {
      cudaEventRecord(S.ev_next, 0);
      cudaStreamWaitEvent(S.side, S.ev_next, 0);
      diag(kb + bs, S.side);
      cudaEventRecord(S.ev_diag, S.side);
    } else {
      diag(kb + bs, 0);
    }
    // trailing: the columns after block kb+1 (FP32 with tensor cores in mixed
    // mode; only the nonzero tile pairs when the Schur pattern is sparse)
    const int rest = rem - nb2;
    if (rest <= 0) continue;
    if (S.sparse) {
      const int k = kb / NBG;
      const long long cnt = S.pair_off[k + 1] - S.pair_off[k];
      if (cnt > 0)
        k_syrk_pairs<T><<<(unsigned)cnt, NT, cta::GEMM_RECT_SMEM * sizeof(double)>>>(S.pairs + 2 * S.pair_off[k], n,
                                                                                     kb, bs, A);
      continue;
    }
    T* P2 = P + nb2;
    T* A33 = A22 + nb2 + (size_t)n * nb2;
    bool done = false;
    if constexpr (std::is_same<T, float>::value) {
      if (S.tc && S.tc_work) done = syrk_tf32x3(rest, bs, P2, n, A33, n, S.tc_work, S.tc_err, 0, S.tc_wait) == 0;
    }
    if (!done) gemm_t<T, T>(rest, rest, bs, false, P2, n, true, P2, n, A33, n, -1.0, 1.0, true);
  }
  if (S.side) cudaStreamWaitEvent(0, S.ev_diag, 0);  // the last diagonal block
  int f = 0;
  cudaMemcpy(&f, S.flag, sizeof(int), cudaMemcpyDeviceToHost);
  return f;
}

static int cholesky_grid(DevState& S, double* A, int n, bool adjust, double* dinv_store = nullptr)
{
  return cholesky_grid_t<double>(S, A, n, adjust, S.Linv, S.T, dinv_store);
}

// x = L^{-T} L^{-1} x with the factor of cholesky_grid_t and its stored
// diagonal-block inverses (grid-wide updates between the block solves).
template <typename T>
static void chol_solve_grid(int m, const T* L, const T* dinv, T* x, cudaStream_t st = 0)
{
  const int nb = (m + NBG - 1) / NBG;
  for (int b = 0; b < nb; ++b) {
    const int kb = b * NBG, bs = std::min(NBG, m - kb), rem = m - kb - bs;
    k_trsv_diag<T><<<1, 512, 0, st>>>(bs, dinv + (size_t)b * NBG * NBG, x + kb, 0);
    if (rem > 0)
      k_trsv_fwd_update<T><<<(rem + 31) / 32, 256, 0, st>>>(rem, bs, L + (kb + bs) + (size_t)m * kb, m, x + kb,
                                                            x + kb + bs);
  }
  for (int b = nb - 1; b >= 0; --b) {
    const int kb = b * NBG, bs = std::min(NBG, m - kb);
    k_trsv_diag<T><<<1, 512, 0, st>>>(bs, dinv + (size_t)b * NBG * NBG, x + kb, 1);
    if (kb > 0) k_trsv_bwd_update<T><<<nblk((long long)kb * 32), 256, 0, st>>>(kb, bs, L + kb, m, x + kb, x);
  }
}

// The grid solve is ~4 launches per 128-row block and direction (about 300
// for m = 10^4), each a few microseconds of work: captured once as a CUDA
// graph per (factor, diagonal inverses, right-hand side) and replayed on the
// default stream.  Capture failures fall back to direct launches.
template <typename T>
static void chol_solve_graph(DevState& S, int m, const T* L, const T* dinv, T* x)
{
  for (const SolveGraph& g : S.solve_graphs)
    if (g.L == (const void*)L && g.dinv == (const void*)dinv && g.x == (void*)x && g.m == m) {
      if (cudaGraphLaunch(g.exec, 0) == cudaSuccess) return;
      cudaGetLastError();
      chol_solve_grid<T>(m, L, dinv, x);
      return;
    }
  cudaStream_t cs = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
  if (ok) {
    chol_solve_grid<T>(m, L, dinv, x, cs);
    ok = cudaStreamEndCapture(cs, &graph) == cudaSuccess && graph != nullptr;
    if (ok) ok = cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  }
  if (graph) cudaGraphDestroy(graph);
  if (cs) cudaStreamDestroy(cs);
  if (!ok) {
    cudaGetLastError();
    chol_solve_grid<T>(m, L, dinv, x);
    return;
  }
  S.solve_graphs.push_back({(const void*)L, (const void*)dinv, (void*)x, m, exec});
  if (cudaGraphLaunch(exec, 0) != cudaSuccess) {
    cudaGetLastError();
    chol_solve_grid<T>(m, L, dinv, x);
  }
}

// Deterministic reduction of len elements into sc[slot]
static void dot(DevState& S, long long len, const double* a, const double* b, int slot, bool acc,
                int mode = 0, double scale = 1.0)
{
  const int g = (int)std::min<long long>(256, std::max<long long>(1, (len + 1023) / 1024));
  if (len > 0) k_dot_partial<<<g, 256>>>(len, a, b, S.part, mode);
  k_dot_final<<<1, 32>>>(len > 0 ? g : 0, S.part, S.sc + slot, mode, acc ? 1 : 0, scale);
}

static void read_scalars(DevState& S, double* h, int n)
{
  cudaMemcpy(h, S.sc, n * sizeof(double), cudaMemcpyDeviceToHost);
}

Solver::Solver() {}
Solver::~Solver() { release(); }

void Solver::release()
{
  delete d_;
  d_ = nullptr;
}

int Solver::dimacs(double* out)
{
  if (!d_) return set_error(SDPAB_ESTATE, "dimacs: no solve");
  DevState& S = *d_;
  std::vector<int> n;
  std::vector<const double*> X, Z, D;
  for (const SdpBlock& B : S.sdp) {
    n.push_back(B.n);
    X.push_back(B.X);
    Z.push_back(B.Z);
    D.push_back(B.D);
  }
  DimacsInput in{S.m, S.rp, (int)S.sdp.size(), n.data(), X.data(), Z.data(), D.data(),
                 S.nlp, S.lpx, S.lpz, S.lpD};
  return dimacs_device(in, out, 0);
}

int Solver::formula_count(int f) const
{
  if (!d_) return 0;
  int c = 0;
  for (const SdpBlock& b : d_->sdp)
    for (int x : b.hform) c += (x == f);
  return c;
}

// ------------------------------------------------------------ constraint order
// Groups of constraints (0-based) whose Schur entries couple: those with an
// entry in the same SDP block, or at the same LP coordinate (the aggregate
// sparsity pattern of B, Chordal's analysis, sdpa_chordal.cpp:365-524).
static std::vector<std::vector<int>> constraint_groups(const ProblemData& p)
{
  const int nb = (int)p.blockStruct.size();
  std::map<std::pair<int, int>, int> id;  // (block, LP coordinate or -1) -> group
  std::vector<std::vector<int>> g;
  for (const Entry& e : p.entries) {
    if (e.k < 1 || e.k > p.m || e.l < 1 || e.l > nb) continue;
    const int bs = p.blockStruct[e.l - 1];
    const std::pair<int, int> key(e.l, (bs > 1) ? -1 : std::min(e.i, e.j));
    auto it = id.find(key);
    int gi;
    if (it == id.end()) {
      gi = (int)g.size();
      id.emplace(key, gi);
      g.emplace_back();
    } else {
      gi = it->second;
    }
    g[gi].push_back(e.k - 1);
  }
  for (auto& v : g) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  return g;
}

// Trailing tile pairs of the symbolic 128 x 128 tile Cholesky of B with the
// constraints at positions pos[k] (the count the factorisation would visit).
static long long symbolic_tile_pairs(const std::vector<std::vector<int>>& groups, const std::vector<int>& pos, int m)
{
  const int nt = (m + NBG - 1) / NBG;
  std::vector<std::vector<char>> P(nt, std::vector<char>(nt, 0));
  std::vector<int> t;
  for (const auto& grp : groups) {
    t.clear();
    for (int k : grp) t.push_back(pos[k] / NBG);
    std::sort(t.begin(), t.end());
    t.erase(std::unique(t.begin(), t.end()), t.end());
    for (size_t a = 0; a < t.size(); ++a)
      for (size_t b = 0; b <= a; ++b) P[t[a]][t[b]] = 1;
  }
  long long pairs = 0;
  std::vector<int> R;
  for (int k = 0; k < nt; ++k) {
    R.clear();
    for (int i = k + 1; i < nt; ++i)
      if (P[i][k]) R.push_back(i);
    for (size_t a = 0; a < R.size(); ++a)
      for (size_t b = 0; b <= a; ++b) {
        P[R[a]][R[b]] = 1;
        if (R[b] >= k + 2) ++pairs;
      }
  }
  return pairs;
}

// Minimum-degree elimination order of the constraints on the group
// (clique) structure, by element absorption: eliminating a constraint merges
// the groups that hold it into one new group of their other members; a
// constraint's degree is taken as the sum of (size - 1) over its live
// groups, an upper bound of its true degree (as in approximate minimum
// degree orderings).  Ties go to the lower index, so the order is
// deterministic.  Returns position -> constraint.
static std::vector<int> min_degree_order(const std::vector<std::vector<int>>& groups, int m)
{
  std::vector<std::vector<int>> E = groups;
  std::vector<char> alive(E.size(), 1);
  std::vector<std::vector<int>> of(m);
  for (int e = 0; e < (int)E.size(); ++e)
    for (int k : E[e]) of[k].push_back(e);
  auto degree = [&](int k) {
    long long d = 0;
    for (int e : of[k])
      if (alive[e]) d += (long long)E[e].size() - 1;
    return d;
  };
  using Item = std::pair<long long, int>;
  std::priority_queue<Item, std::vector<Item>, std::greater<Item>> pq;
  std::vector<long long> deg(m);
  for (int k = 0; k < m; ++k) {
    deg[k] = degree(k);
    pq.push({deg[k], k});
  }
  std::vector<char> done(m, 0);
  std::vector<int> stamp(m, -1), order;
  order.reserve(m);
  while (!pq.empty()) {
    const Item it = pq.top();
    pq.pop();
    const int v = it.second;
    if (done[v] || it.first != deg[v]) continue;  // stale entry
    done[v] = 1;
    order.push_back(v);
    std::vector<int> U;
    for (int e : of[v]) {
      if (!alive[e]) continue;
      for (int u : E[e])
        if (!done[u] && stamp[u] != v) {
          stamp[u] = v;
          U.push_back(u);
        }
      alive[e] = 0;
      std::vector<int>().swap(E[e]);
    }
    if (U.empty()) continue;
    std::sort(U.begin(), U.end());
    const int ne = (int)E.size();
    E.push_back(U);
    alive.push_back(1);
    for (int u : U) {
      auto& L = of[u];
      L.erase(std::remove_if(L.begin(), L.end(), [&](int e) { return !alive[e]; }), L.end());
      L.push_back(ne);
      deg[u] = degree(u);
      pq.push({deg[u], u});
    }
  }
  return order;
}

// The constraints by the number of groups they touch, then by their first
// group, then by index: constraints local to one block come first, grouped
// by block, the coupling ones last (the arrowhead order, which keeps the
// couplings out of the diagonal tiles).
static std::vector<int> group_count_order(const std::vector<std::vector<int>>& groups, int m)
{
  std::vector<int> cnt(m, 0), first(m, 1 << 30);
  for (int g = 0; g < (int)groups.size(); ++g)
    for (int k : groups[g]) {
      ++cnt[k];
      first[k] = std::min(first[k], g);
    }
  std::vector<int> o(m);
  std::iota(o.begin(), o.end(), 0);
  std::stable_sort(o.begin(), o.end(), [&](int a, int b) {
    if (cnt[a] != cnt[b]) return cnt[a] < cnt[b];
    return first[a] < first[b];
  });
  return o;
}

// The order with the fewest symbolic tile pairs among the caller's, the
// minimum-degree and the group-count orders (the caller's on ties).
static std::vector<int> best_constraint_order(const std::vector<std::vector<int>>& groups, int m,
                                              long long* pairs_natural, long long* pairs_best)
{
  std::vector<int> ident(m), pos(m);
  std::iota(ident.begin(), ident.end(), 0);
  const long long nat = symbolic_tile_pairs(groups, ident, m);
  std::vector<int> best = ident;
  long long bp = nat;
  for (int cand = 0; cand < 2; ++cand) {
    std::vector<int> o = cand == 0 ? min_degree_order(groups, m) : group_count_order(groups, m);
    if ((int)o.size() != m) continue;
    for (int q = 0; q < m; ++q) pos[o[q]] = q;
    const long long pr = symbolic_tile_pairs(groups, pos, m);
    if (pr < bp) {
      bp = pr;
      best = o;
    }
  }
  if (pairs_natural) *pairs_natural = nat;
  if (pairs_best) *pairs_best = bp;
  return best;
}

int Solver::setup(const ProblemData& p, const Params& prm, double kappa)
{
  perm_.clear();
  const char* env = getenv("SDPAB_ORDER");
  const bool natural = env && std::string(env) == "natural";
  int nsdp = 0;
  for (int b : p.blockStruct) nsdp += (b > 1) ? 1 : 0;
  // a fill-reducing order pays only where the Schur pattern can be sparse:
  // several SDP blocks and at least four 128-constraint tiles
  if (!natural && nsdp >= 2 && p.m >= 4 * NBG && p.m <= 65536) {
    const std::vector<std::vector<int>> groups = constraint_groups(p);
    long long nat = 0, best = 0;
    std::vector<int> order = best_constraint_order(groups, p.m, &nat, &best);
    {
      std::vector<int> pos(p.m);
      for (int i = 0; i < p.m; ++i) pos[order[i]] = i;
      if (best < nat) {
        ProblemData q = p;
        for (Entry& e : q.entries)
          if (e.k >= 1 && e.k <= p.m) e.k = pos[e.k - 1] + 1;
        for (int i = 0; i < p.m; ++i) q.c[i] = p.c[order[i]];
        const int rc = setup_ordered(q, prm, kappa);
        if (rc == SDPAB_OK) perm_ = order;
        return rc;
      }
    }
  }
  return setup_ordered(p, prm, kappa);
}

int Solver::setup_ordered(const ProblemData& p, const Params& prm, double kappa)
{
  release();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDPAB_ENODEV, "no CUDA device");
  d_ = new DevState();
  DevState& S = *d_;
  S.m = p.m;
  S.prm = prm;
  const int m = p.m;
  if (m < 1) return set_error(SDPAB_EINVAL, "constraint number must be positive");
  // BlockStruct::makeInternalStructure (sdpa_block.cpp:66-95)
  const int nb = (int)p.blockStruct.size();
  S.blockStruct.assign(nb, 0);
  S.blockKind.assign(nb, 0);
  S.blockIndex.assign(nb, 0);
  int nsdp = 0, nlp = 0;
  for (int l = 0; l < nb; ++l) {
    int s = p.blockStruct[l];
    int t = (l < (int)p.blockType.size()) ? p.blockType[l] : 0;
    if (t == 1) return set_error(SDPAB_EINVAL, "SOCP blocks are not supported (as in the reference)");
    if (s >= 2 && t == 0) {
      S.blockKind[l] = 0; S.blockIndex[l] = nsdp++; S.blockStruct[l] = s;
    } else if (s < 0 || t == 2) {
      S.blockKind[l] = 2; S.blockIndex[l] = nlp; S.blockStruct[l] = std::abs(s); nlp += std::abs(s);
    } else if (s == 1) {
      S.blockKind[l] = 2; S.blockIndex[l] = nlp; S.blockStruct[l] = 1; nlp += 1;
    } else {
      return set_error(SDPAB_EINVAL, "invalid block struct");
    }
  }
  S.nlp = nlp;
  S.sdp.resize(nsdp);
  S.nDim = nlp;
  for (int l = 0; l < nb; ++l)
    if (S.blockKind[l] == 0) {
      SdpBlock& B = S.sdp[S.blockIndex[l]];
      B.n = S.blockStruct[l];
      B.fileBlock = l + 1;
      S.nDim += B.n;
    }
  // sort entries by (k, l, i, j) and split per block / constraint
  std::vector<Entry> E = p.entries;
  for (Entry& e : E)
    if (e.i > e.j) std::swap(e.i, e.j);
  std::stable_sort(E.begin(), E.end(), [](const Entry& a, const Entry& b) {
    if (a.k != b.k) return a.k < b.k;
    if (a.l != b.l) return a.l < b.l;
    if (a.i != b.i) return a.i < b.i;
    return a.j < b.j;
  });
  std::vector<std::vector<double>> Ch(nsdp);
  for (int q = 0; q < nsdp; ++q) Ch[q].assign((size_t)S.sdp[q].n * S.sdp[q].n, 0.0);
  std::vector<double> Clp(nlp, 0.0);
  // per block: constraint -> entries
  std::vector<std::vector<std::vector<int>>> per(nsdp);  // [block][k] -> entry indices
  for (int q = 0; q < nsdp; ++q) per[q].assign(m, {});
  std::vector<std::vector<std::pair<int, double>>> lpk(m);  // constraint -> (t, v)
  for (size_t q = 0; q < E.size(); ++q) {
    const Entry& e = E[q];
    if (e.k < 0 || e.k > m || e.l < 1 || e.l > nb) return set_error(SDPAB_EINVAL, "entry index out of range");
    const int l = e.l - 1;
    const int dim = S.blockStruct[l];
    if (e.i < 1 || e.j < 1 || e.i > dim || e.j > dim) return set_error(SDPAB_EINVAL, "entry outside its block");
    if (S.blockKind[l] == 0) {
      const int bi = S.blockIndex[l];
      const int n = S.sdp[bi].n;
      if (e.k == 0) {
        // C = -F0 (sdpa_io.cpp:511); duplicates accumulate
        Ch[bi][(e.i - 1) + (size_t)n * (e.j - 1)] -= e.v;
        if (e.i != e.j) Ch[bi][(e.j - 1) + (size_t)n * (e.i - 1)] -= e.v;
      } else {
        per[bi][e.k - 1].push_back((int)q);
      }
    } else {
      if (e.i != e.j) return set_error(SDPAB_EINVAL, "LP block entries must be diagonal");
      const int t = S.blockIndex[l] + e.i - 1;
      if (e.k == 0) Clp[t] -= e.v;
      else lpk[e.k - 1].push_back({t, e.v});
    }
  }
  // device allocations per SDP block
  for (int q = 0; q < nsdp; ++q) {
    SdpBlock& B = S.sdp[q];
    const size_t nn = (size_t)B.n * B.n;
    B.C = S.upload(Ch[q]);
    double** mats[] = {&B.X, &B.Z, &B.Zi, &B.LXi, &B.LZi, &B.D, &B.XDZ, &B.R, &B.dX, &B.dZ, &B.W1, &B.W2,
                       &B.X0, &B.Z0, &B.Lt};
    for (double** mp : mats) {
      *mp = S.alloc(nn);
      if (!*mp) return set_error(SDPAB_ECUDA, "device allocation failed (block matrices)");
    }
    // constraint index (InputData::initialize_index_SDP, sdpa_dataset.cpp:268-305)
    B.hptr.push_back(0);
    for (int k = 0; k < m; ++k) {
      if (per[q][k].empty()) continue;
      B.hcons.push_back(k);
      int eff = 0;
      for (int ei : per[q][k]) {
        const Entry& e = E[ei];
        B.hrow.push_back(e.i - 1);
        B.hcol.push_back(e.j - 1);
        B.hval.push_back(e.v);
        eff += (e.i == e.j) ? 1 : 2;  // NonZeroEffect (sdpa_struct.cpp:1339-1341)
      }
      B.hnnz.push_back(eff);
      B.hptr.push_back((long long)B.hrow.size());
    }
    B.nc = (int)B.hcons.size();
  }
  // formula choice: Newton::computeFormula_SDP (sdpa_newton.cpp:515-695)
  for (int q = 0; q < nsdp; ++q) {
    SdpBlock& B = S.sdp[q];
    const double n = B.n;
    B.hform.assign(B.nc, F3);
    for (int jl = 0; jl < B.nc; ++jl) {
      const double jnz = B.hnnz[jl];
      double up = jnz;
      for (int il = 0; il < B.nc; ++il) {
        const int inz = B.hnnz[il];
        if (inz < jnz) up += inz;
        else if (inz == jnz && B.hcons[il] > B.hcons[jl]) up += inz;
      }
      const double f1 = kappa * n * jnz + n * n * n + kappa * up;
      const double f2 = kappa * n * jnz + kappa * (n + 1) * up;
      const double f3 = kappa * (2 * kappa * jnz + 1) * up;
      const long long count = B.hptr[jl + 1] - B.hptr[jl];
      const bool dense = count >= (long long)(n * n * 0.20);  // SparseMatrix::changeToDense threshold
      int f;
      if (dense) {
        f = (f1 < f2) ? F1 : F2;
      } else if (f1 < f2 && f1 < f3) {
        f = (n <= 200 && 2.0 * n >= jnz) ? F3 : F1;
      } else if (f2 < f3) {
        f = F2;
      } else {
        f = F3;
      }
      B.hform[jl] = f;
      if (f != F3) B.hf1.push_back(jl);
    }
  }
  // device copies of the constraint index + F1 column structures
  size_t Tneed = 0;
  for (int q = 0; q < nsdp; ++q) {
    SdpBlock& B = S.sdp[q];
    B.cons = S.upload(B.hcons);
    B.nnz = S.upload(B.hnnz);
    B.form = S.upload(B.hform);
    B.ptr = S.upload(B.hptr);
    B.row = S.upload(B.hrow);
    B.col = S.upload(B.hcol);
    B.val = S.upload(B.hval);
    B.f1 = S.upload(B.hf1);
    if (!B.hf1.empty()) {
      // symmetric CSC of each F1 constraint, indexed by local constraint id
      std::vector<long long> cptr((size_t)B.nc * (B.n + 1), 0), eptr(B.nc + 1, 0);
      std::vector<int> crow;
      std::vector<double> cval;
      for (int jl = 0; jl < B.nc; ++jl) {
        eptr[jl] = (long long)crow.size();
        if (B.hform[jl] == F3) { eptr[jl + 1] = eptr[jl]; continue; }
        std::vector<std::vector<std::pair<int, double>>> cols(B.n);
        for (long long e = B.hptr[jl]; e < B.hptr[jl + 1]; ++e) {
          cols[B.hcol[e]].push_back({B.hrow[e], B.hval[e]});
          if (B.hrow[e] != B.hcol[e]) cols[B.hrow[e]].push_back({B.hcol[e], B.hval[e]});
        }
        long long base = (long long)crow.size();
        for (int c = 0; c < B.n; ++c) {
          cptr[(size_t)jl * (B.n + 1) + c] = (long long)crow.size() - base;
          for (auto& pr : cols[c]) { crow.push_back(pr.first); cval.push_back(pr.second); }
        }
        cptr[(size_t)jl * (B.n + 1) + B.n] = (long long)crow.size() - base;
      }
      eptr[B.nc] = (long long)crow.size();
      B.csc_cptr = S.upload(cptr);
      B.csc_ptr = S.upload(eptr);
      B.csc_row = S.upload(crow);
      B.csc_val = S.upload(cval);
      std::vector<int> hpos(B.hrow.size());
      for (size_t e = 0; e < hpos.size(); ++e) {
        const long long r = std::min(B.hrow[e], B.hcol[e]), c = std::max(B.hrow[e], B.hcol[e]);
        hpos[e] = (int)(c * (c + 1) / 2 + r);
      }
      B.pos = S.upload(hpos);
      // T holds the chunk's X A_j and then its packed H (n(n+1)/2 rows of 32);
      // G follows it
      Tneed = std::max(Tneed, (size_t)2 * F1_CHUNK * B.n * B.n);
    }
  }
  // LP data (lp_by_t: the constraints of each LP coordinate, kept for the
  // Schur pattern below)
  std::vector<std::vector<std::pair<int, double>>> lp_by_t(nlp);
  {
    std::vector<long long> ptr(m + 1, 0);
    std::vector<int> idx;
    std::vector<double> val;
    std::vector<std::vector<std::pair<int, double>>>& byT = lp_by_t;
    for (int k = 0; k < m; ++k) {
      for (auto& pr : lpk[k]) {
        idx.push_back(pr.first);
        val.push_back(pr.second);
        byT[pr.first].push_back({k, pr.second});
      }
      ptr[k + 1] = (long long)idx.size();
    }
    std::vector<long long> tptr(nlp + 1, 0);
    std::vector<int> tk;
    std::vector<double> tv;
    for (int t = 0; t < nlp; ++t) {
      for (auto& pr : byT[t]) { tk.push_back(pr.first); tv.push_back(pr.second); }
      tptr[t + 1] = (long long)tk.size();
    }
    S.lp_ptr = S.upload(ptr);
    S.lp_idx = S.upload(idx);
    S.lp_val = S.upload(val);
    S.lpT_ptr = S.upload(tptr);
    S.lpT_k = S.upload(tk);
    S.lpT_v = S.upload(tv);
    S.lpC = S.upload(Clp);
    double** lps[] = {&S.lpx, &S.lpz, &S.lpzi, &S.lplx, &S.lplz, &S.lpD, &S.lpR, &S.lpXDZ, &S.lpdx,
                      &S.lpdz, &S.lpW, &S.lpx0, &S.lpz0, &S.lptmp};
    for (double** pp : lps) *pp = S.alloc(nlp);
  }
  // Schur pattern at the tile level (Chordal::ordering_bMat decides between
  // the dense and the MUMPS sparse factorisation from the aggregate pattern,
  // sdpa_chordal.cpp:365-524): B_ij is nonzero only if constraints i and j
  // share an SDP block or an LP coordinate.  Tiles (128 x 128) that hold
  // such pairs, closed under the fill of a symbolic tile Cholesky, give the
  // trailing tile pairs of every panel; the factorisation skips the rest
  // when they are few enough.  SDPAB_SCHUR=dense or =sparse forces a mode.
  {
    const int nt = (m + NBG - 1) / NBG;
    std::vector<std::vector<char>> P(nt, std::vector<char>(nt, 0));
    auto mark = [&](const std::vector<int>& cons) {
      std::vector<int> t;
      for (int k : cons) t.push_back(k / NBG);
      std::sort(t.begin(), t.end());
      t.erase(std::unique(t.begin(), t.end()), t.end());
      for (size_t a = 0; a < t.size(); ++a)
        for (size_t b = 0; b <= a; ++b) P[t[a]][t[b]] = 1;
    };
    for (const SdpBlock& B : S.sdp) mark(B.hcons);
    for (int t = 0; t < nlp; ++t) {
      std::vector<int> c;
      for (auto& pr : lp_by_t[t]) c.push_back(pr.first);
      mark(c);
    }
    for (int i = 0; i < nt; ++i) P[i][i] = 1;
    S.pair_off.assign(nt + 1, 0);
    std::vector<int> hp;
    S.dense_pairs = S.sparse_pairs = 0;
    for (int k = 0; k < nt; ++k) {
      std::vector<int> R;
      for (int i = k + 1; i < nt; ++i)
        if (P[i][k]) R.push_back(i);
      for (size_t a = 0; a < R.size(); ++a)
        for (size_t b = 0; b <= a; ++b) {
          P[R[a]][R[b]] = 1;  // fill
          if (R[b] >= k + 2) {
            hp.push_back(R[a]);
            hp.push_back(R[b]);
          }
        }
      S.pair_off[k + 1] = (long long)hp.size() / 2;
      const long long rest = std::max(0, nt - k - 2);
      S.dense_pairs += rest * (rest + 1) / 2;
    }
    S.sparse_pairs = S.pair_off[nt];
    const char* env = getenv("SDPAB_SCHUR");
    const std::string mode = env ? env : "";
    if (mode == "dense" || nt < 3) S.sparse = false;
    else if (mode == "sparse") S.sparse = true;
    else S.sparse = nt >= 4 && (double)S.sparse_pairs < 0.6 * (double)S.dense_pairs;
    if (S.sparse) S.pairs = S.upload(hp);
  }
  S.b = S.upload(p.c);
  S.y = S.alloc(m);
  S.dy = S.alloc(m);
  S.g = S.alloc(m);
  S.rp = S.alloc(m);
  S.ytmp = S.alloc(m);
  S.B = S.alloc((size_t)m * m);
  S.Linv = S.alloc((size_t)NBG * NBG);
  if (m > SMALL_SOLVE) S.dinv = S.alloc((size_t)((m + NBG - 1) / NBG) * NBG * NBG);
  int nmaxb = 1;
  for (auto& B : S.sdp) nmaxb = std::max(nmaxb, B.n);
  Tneed = std::max(Tneed, (size_t)std::max(m, nmaxb) * NBG);
  S.T = S.alloc(Tneed);
  S.Tsize = Tneed;
  S.part = S.alloc(256);
  S.sc = S.alloc(64);
  {
    std::vector<BlockPtrs> hb;
    S.small_idx.clear();
    S.large_idx.clear();
    for (int q = 0; q < nsdp; ++q) {
      SdpBlock& B = S.sdp[q];
      if (B.n <= SMALL_BLOCK) {
        S.small_idx.push_back(q);
        BlockPtrs d{};
        d.X = B.X; d.Z = B.Z; d.Zi = B.Zi; d.LXi = B.LXi; d.LZi = B.LZi; d.W1 = B.W1; d.W2 = B.W2;
        d.R = B.R; d.XDZ = B.XDZ; d.dX = B.dX; d.dZ = B.dZ; d.D = B.D;
        d.cons = B.cons; d.ptr = B.ptr; d.row = B.row; d.col = B.col; d.val = B.val;
        d.n = B.n;
        d.nc = B.nc;
        hb.push_back(d);
        S.small_nmax = std::max(S.small_nmax, B.n);
      } else {
        S.large_idx.push_back(q);
      }
    }
    if (!hb.empty()) {
      void* pp = nullptr;
      if (cudaMalloc(&pp, hb.size() * sizeof(BlockPtrs)) != cudaSuccess)
        return set_error(SDPAB_ECUDA, "device allocation failed (block descriptors)");
      S.allocs.push_back(pp);
      cudaMemcpy(pp, hb.data(), hb.size() * sizeof(BlockPtrs), cudaMemcpyHostToDevice);
      S.small_ptrs = (BlockPtrs*)pp;
      const int sm = (int)small_block_smem(S.small_nmax);
      cudaFuncSetAttribute(k_blocks_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      cudaFuncSetAttribute(k_blocks_step, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      cudaFuncSetAttribute(k_blocks_direction, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
      cudaFuncSetAttribute(k_blocks_corrector, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    }
    S.blk_mins = S.alloc(2 * (size_t)std::max(nsdp, 1));
    std::vector<F3Desc> fd;
    std::vector<long long> fo(1, 0);
    for (SdpBlock& B : S.sdp) {
      if (!B.nc) continue;
      fd.push_back({B.cons, B.ptr, B.row, B.col, B.val, B.nnz, B.form, B.X, B.Zi, B.nc, B.n});
      fo.push_back(fo.back() + (long long)B.nc * B.nc);
    }
    S.f3_total = fo.back();
    S.f3_nb = (int)fd.size();
    S.f3_direct_block = -1;
    if (nsdp == 1 && nlp == 0 && S.sdp[0].nc == m) {
      const SdpBlock& B0 = S.sdp[0];
      bool direct = true;
      for (int l = 0; l < B0.nc && direct; ++l) direct = B0.hcons[l] == l && B0.hform[l] == F3;
      if (direct) {
        S.f3_direct_block = 0;
        // every pair whose entry counts multiply to more than F3_HEAVY (the
        // test k_f3_tiles applies): one of the two has more than
        // sqrt(F3_HEAVY) = 32 entries, so only those need pairing with all
        auto cnt = [&](int l) { return B0.hptr[l + 1] - B0.hptr[l]; };
        std::vector<int> hp;
        for (int a = 0; a < B0.nc; ++a) {
          if (cnt(a) <= 32) continue;
          for (int j = 0; j < B0.nc; ++j) {
            if (cnt(a) * cnt(j) <= F3_HEAVY) continue;
            if (cnt(j) > 32 && j > a) continue;  // listed once, from the larger index
            hp.push_back(a);
            hp.push_back(j);
          }
        }
        S.f3_nheavy = (int)(hp.size() / 2);
        if (S.f3_nheavy) S.f3_heavy = S.upload(hp);
      }
    }
    if (!fd.empty()) {
      void* pp = nullptr;
      if (cudaMalloc(&pp, fd.size() * sizeof(F3Desc)) != cudaSuccess)
        return set_error(SDPAB_ECUDA, "device allocation failed (F3 descriptors)");
      S.allocs.push_back(pp);
      cudaMemcpy(pp, fd.data(), fd.size() * sizeof(F3Desc), cudaMemcpyHostToDevice);
      S.f3_desc = (F3Desc*)pp;
      S.f3_off = S.upload(fo);
    }
    std::vector<F1Desc> f1d;
    std::vector<long long> f1o(1, 0);
    for (SdpBlock& B : S.sdp) {
      if (!B.nc || B.hf1.empty() || B.n > SMALL_F1) continue;
      f1d.push_back({B.f1, B.csc_cptr, B.csc_ptr, B.csc_row, B.csc_val, B.cons, B.ptr, B.row, B.col, B.val, B.nnz,
                     B.X, B.Zi, B.nc, B.n});
      f1o.push_back(f1o.back() + (long long)B.hf1.size());
      S.f1_nmax = std::max(S.f1_nmax, B.n);
    }
    S.f1_total = f1o.back();
    S.f1_nb = (int)f1d.size();
    if (!f1d.empty()) {
      void* pp = nullptr;
      if (cudaMalloc(&pp, f1d.size() * sizeof(F1Desc)) != cudaSuccess)
        return set_error(SDPAB_ECUDA, "device allocation failed (F1 descriptors)");
      S.allocs.push_back(pp);
      cudaMemcpy(pp, f1d.data(), f1d.size() * sizeof(F1Desc), cudaMemcpyHostToDevice);
      S.f1_desc = (F1Desc*)pp;
      S.f1_off = S.upload(f1o);
      cudaFuncSetAttribute(k_f1_small, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(2 * (size_t)S.f1_nmax * S.f1_nmax * sizeof(double)));
    }
    if (nsdp) {
      std::vector<double*> tab((size_t)MB_KINDS * nsdp);
      std::vector<long long> eoff(1, 0), coff(1, 0);
      std::vector<int> nq;
      std::vector<MbSparse> sp;
      for (int q = 0; q < nsdp; ++q) {
        SdpBlock& B = S.sdp[q];
        double* k[MB_KINDS] = {B.X, B.Z, B.dX, B.dZ, B.C, B.X0, B.Z0, B.D, B.R, B.W1, B.W2, B.Zi};
        for (int u = 0; u < MB_KINDS; ++u) tab[(size_t)u * nsdp + q] = k[u];
        eoff.push_back(eoff.back() + (long long)B.n * B.n);
        nq.push_back(B.n);
        if (B.nc) {
          sp.push_back({B.cons, B.ptr, B.row, B.col, B.val, B.n, q});
          coff.push_back(coff.back() + B.nc);
        }
      }
      S.mb_tab = S.upload(tab);
      S.mb_eoff = S.upload(eoff);
      S.mb_nq = S.upload(nq);
      S.mb_total = eoff.back();
      S.mb_sp = S.upload(sp);
      S.mb_coff = S.upload(coff);
      S.mb_ctotal = coff.back();
      S.mb_ns = (int)sp.size();
      if (!S.mb_tab || !S.mb_eoff || !S.mb_nq || !S.mb_sp || !S.mb_coff)
        return set_error(SDPAB_ECUDA, "device allocation failed (block tables)");
    }
  }
  void* fp = nullptr;
  if (cudaMalloc(&fp, 256) != cudaSuccess) return set_error(SDPAB_ECUDA, "device allocation failed");
  S.allocs.push_back(fp);
  S.flag = (int*)fp;
  S.tc_err = S.flag + 16;
  S.tc_f1_err = S.flag + 20;
  if (!S.B || !S.T || !S.b) return set_error(SDPAB_ECUDA, "device allocation failed (Schur matrix)");
  // shared memory limits of the block-level kernels
  cudaFuncSetAttribute(k_min_eig, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "setup");
  return SDPAB_OK;
}

int Solver::solve(const InitPoint* init, const Params* prm)
{
  // in a fill-reducing constraint order: the initial x in that order, the
  // result x back in the caller's
  if (!perm_.empty()) {
    InitPoint ip;
    const InitPoint* ini = init;
    if (init) {
      ip = *init;
      ip.xvec.assign(perm_.size(), 0.0);
      for (size_t i = 0; i < perm_.size(); ++i)
        if (perm_[i] < (int)init->xvec.size()) ip.xvec[i] = init->xvec[perm_[i]];
      ini = &ip;
    }
    const std::vector<int> order = perm_;
    perm_.clear();
    const int rc = solve(ini, prm);
    perm_ = order;
    if (xvec_.size() == order.size()) {
      std::vector<double> x(order.size());
      for (size_t i = 0; i < order.size(); ++i) x[order[i]] = xvec_[i];
      xvec_.swap(x);
    }
    return rc;
  }
  if (d_ && prm) d_->prm = *prm;
  if (!d_) return set_error(SDPAB_ESTATE, "solve before initializeSolve");
  DevState& S = *d_;
  const Params& P = S.prm;
  const int m = S.m, nlp = S.nlp;
  const double lam = P.lambdaStar;
  auto t_start = std::chrono::steady_clock::now();
  stats_ = SolveStats();
  stats_.schur_sparse = S.sparse ? 1 : 0;
  stats_.schur_sparse_pairs = S.sparse_pairs;
  stats_.schur_dense_pairs = S.dense_pairs;
  const int nsdp = (int)S.sdp.size();
  S.mixed = (precision_ == SDPAB_PREC_MIXED || precision_ == SDPAB_PREC_MIXED_SIMT) ? 1 : 0;
  // tensor-core trailing updates pay from a few panels on
  S.tc = precision_ == SDPAB_PREC_MIXED && m >= 256;
  S.mu_switch = (mu_switch_ > 0.0) ? mu_switch_ : 1.0e-2;
  S.tc_wait = tc_wait_;
  if (S.mixed && !S.B32) {
    void* p = nullptr;
    const size_t fl = (size_t)m * m + (size_t)NBG * NBG + (size_t)m * NBG + m;
    if (cudaMalloc(&p, fl * sizeof(float)) != cudaSuccess)
      return set_error(SDPAB_ECUDA, "device allocation failed (FP32 Schur factor)");
    S.allocs.push_back(p);
    S.B32 = (float*)p;
    if (S.tc) {  // split operands of the tensor-core trailing updates
      void* w = nullptr;
      if (cudaMalloc(&w, (size_t)syrk_tf32x3_work_bytes(m, NBG)) == cudaSuccess) {
        S.allocs.push_back(w);
        S.tc_work = w;
      }
    }
    // split operands of the tensor-core F1 products (X A_j) Z^-1, one chunk
    long long f1w = 0;
    for (const SdpBlock& B : S.sdp)
      if (!B.hf1.empty()) f1w = std::max(f1w, gemm_tf32x3_work_bytes(B.n, B.n, B.n, F1_CHUNK));
    if (precision_ == SDPAB_PREC_MIXED && f1w > 0) {
      void* w = nullptr;
      if (cudaMalloc(&w, (size_t)f1w) == cudaSuccess) {
        S.allocs.push_back(w);
        S.tc_f1_work = w;
      }
    }
    S.Linv32 = S.B32 + (size_t)m * m;
    S.T32 = S.Linv32 + (size_t)NBG * NBG;
    S.v32 = S.T32 + (size_t)m * NBG;
    S.res = S.alloc(2 * (size_t)m);
    if (m > SMALL_SOLVE) {
      void* q = nullptr;
      if (cudaMalloc(&q, (size_t)((m + NBG - 1) / NBG) * NBG * NBG * sizeof(float)) != cudaSuccess)
        return set_error(SDPAB_ECUDA, "device allocation failed (FP32 block inverses)");
      S.allocs.push_back(q);
      S.dinv32 = (float*)q;
    }
  }

  // ------------------------------------------------ initial point
  bool warm = init != nullptr;
  if (warm) {
    // user X -> internal Z, user Y -> internal X, x -> y = -x (sdpa_call.cpp:343-434)
    std::vector<double> ny(m);
    for (int k = 0; k < m; ++k) ny[k] = (k < (int)init->xvec.size()) ? -init->xvec[k] : 0.0;
    cudaMemcpy(S.y, ny.data(), m * sizeof(double), cudaMemcpyHostToDevice);
    std::vector<double> hx(nlp, 0.0), hz(nlp, 0.0);
    for (int l = 0; l < (int)S.blockKind.size(); ++l) {
      const std::vector<double>& Xu = init->X[l];
      const std::vector<double>& Yu = init->Y[l];
      if (S.blockKind[l] == 0) {
        SdpBlock& B = S.sdp[S.blockIndex[l]];
        const size_t nn = (size_t)B.n * B.n;
        if (Xu.size() != nn || Yu.size() != nn) return set_error(SDPAB_EINVAL, "init point block size");
        cudaMemcpy(B.Z, Xu.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
        cudaMemcpy(B.X, Yu.data(), nn * sizeof(double), cudaMemcpyHostToDevice);
      } else {
        for (int t = 0; t < S.blockStruct[l]; ++t) {
          hz[S.blockIndex[l] + t] = Xu[t];
          hx[S.blockIndex[l] + t] = Yu[t];
        }
      }
    }
    if (nlp) {
      cudaMemcpy(S.lpx, hx.data(), nlp * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(S.lpz, hz.data(), nlp * sizeof(double), cudaMemcpyHostToDevice);
    }
  }
  // Solutions::computeInverse (sdpa_dataset.cpp:117-142); returns false on failure
  auto compute_inverse = [&]() -> bool {
    bool ok = true;
    if (!S.small_idx.empty()) {
      cudaMemset(S.flag + 28, 0, sizeof(int));
      k_blocks_inverse<<<(unsigned)S.small_idx.size(), NT, small_block_smem(S.small_nmax)>>>(S.small_ptrs,
                                                                                          S.flag + 28);
      int bad = 0;
      cudaMemcpy(&bad, S.flag + 28, sizeof(int), cudaMemcpyDeviceToHost);
      if (bad) return false;
    }
    for (int q : S.large_idx) {
      SdpBlock& B = S.sdp[q];
      const long long nn = (long long)B.n * B.n;
      k_axpby<<<nblk(nn), 256>>>(nn, B.W1, 1.0, B.X, 0.0, nullptr);
      if (cholesky_grid(S, B.W1, B.n, false)) { ok = false; break; }
      k_tri_inv<double><<<1, NT, chol_smem()>>>(B.n, B.W1, B.n, B.LXi, B.n, nullptr);
      k_axpby<<<nblk(nn), 256>>>(nn, B.W2, 1.0, B.Z, 0.0, nullptr);
      if (cholesky_grid(S, B.W2, B.n, false)) { ok = false; break; }
      k_tri_inv<double><<<1, NT, chol_smem()>>>(B.n, B.W2, B.n, B.LZi, B.n, nullptr);
      gemm(S, B.n, B.n, B.n, true, B.LZi, B.n, false, B.LZi, B.n, B.Zi, B.n, 1.0, 0.0);
    }
    if (ok && nlp) {
      cudaMemset(S.flag, 0, sizeof(int));
      k_lp_inv<<<nblk(nlp), 256>>>(nlp, S.lpx, S.lplx, nullptr, S.flag);
      k_lp_inv<<<nblk(nlp), 256>>>(nlp, S.lpz, S.lplz, S.lpzi, S.flag);
      int bad = 0;
      cudaMemcpy(&bad, S.flag, sizeof(int), cudaMemcpyDeviceToHost);
      if (bad) ok = false;
    }
    return ok;
  };
  if (warm) {
    // this solver checks strict interiority of the given point and falls
    // back to the standard start (the reference ignores the failure here,
    // sdpa_solve.cpp:63)
    if (!compute_inverse()) {
      warm = false;
      stats_.warm_start_rejected = 1;
    }
  }
  if (!warm) {
    // Solutions::initialize (sdpa_dataset.cpp:47-74)
    for (SdpBlock& B : S.sdp) {
      const long long nn = (long long)B.n * B.n;
      k_set_identity<<<nblk(nn), 256>>>(B.n, B.X, lam);
      k_set_identity<<<nblk(nn), 256>>>(B.n, B.Z, lam);
      k_set_identity<<<nblk(nn), 256>>>(B.n, B.LXi, 1.0 / sqrt(lam));
      k_set_identity<<<nblk(nn), 256>>>(B.n, B.LZi, 1.0 / sqrt(lam));
      k_set_identity<<<nblk(nn), 256>>>(B.n, B.Zi, 1.0 / lam);
    }
    if (nlp) {
      std::vector<double> v(nlp, lam), v2(nlp, 1.0 / sqrt(lam)), v3(nlp, 1.0 / lam);
      cudaMemcpy(S.lpx, v.data(), nlp * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(S.lpz, v.data(), nlp * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(S.lplx, v2.data(), nlp * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(S.lplz, v2.data(), nlp * sizeof(double), cudaMemcpyHostToDevice);
      cudaMemcpy(S.lpzi, v3.data(), nlp * sizeof(double), cudaMemcpyHostToDevice);
    }
    cudaMemset(S.y, 0, m * sizeof(double));
  }
  if (warm) {
    for (SdpBlock& B : S.sdp) {
      const long long nn = (long long)B.n * B.n;
      k_axpby<<<nblk(nn), 256>>>(nn, B.X0, 1.0, B.X, 0.0, nullptr);
      k_axpby<<<nblk(nn), 256>>>(nn, B.Z0, 1.0, B.Z, 0.0, nullptr);
    }
    if (nlp) {
      k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpx0, 1.0, S.lpx, 0.0, nullptr);
      k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpz0, 1.0, S.lpz, 0.0, nullptr);
    }
  }

  // ------------------------------------------------ helpers
  // reductions and element-wise updates over every SDP block at once
  // (k_mb_*; kinds MB_*): sc[slot] (+)= scale * reduction, mode as k_mb_reduce
  auto mb_reduce = [&](int ka, int kb, int mode, int slot, bool acc, double scale) {
    const int g = (int)std::min<long long>(256, std::max<long long>(1, (S.mb_total + 2047) / 2048));
    const long long chunk = (S.mb_total + g - 1) / g;
    k_mb_reduce<<<g, 256>>>(S.mb_tab, ka, kb, S.mb_eoff, S.mb_nq, nsdp, chunk, S.part, mode);
    k_dot_final<<<1, 32>>>(g, S.part, S.sc + slot, mode == 1 ? 1 : 0, acc ? 1 : 0, scale);
  };
  auto mb_axpby = [&](int ko, double a, int kx, double b, int ky) {
    const long long chunk = 2048;
    k_mb_axpby<<<(unsigned)((S.mb_total + chunk - 1) / chunk), 256>>>(S.mb_tab, ko, a, kx, b, ky, S.mb_eoff,
                                                                        S.mb_nq, nsdp, chunk);
  };
  // out[k] = base[k] + sign * sum_blocks A_k . W   (W = matrix kind kw of
  // each block; LP vector wl)
  auto a_dot = [&](double* out, const double* base, double sign, int kw, const double* wl) {
    if (base) cudaMemcpy(out, base, m * sizeof(double), cudaMemcpyDeviceToDevice);
    else cudaMemset(out, 0, m * sizeof(double));
    if (S.mb_ctotal)
      k_mb_sp_dot<<<nblk(S.mb_ctotal * 32), 256>>>(S.mb_sp, S.mb_coff, S.mb_ns, S.mb_tab, kw, nsdp, sign, out);
    if (nlp) k_lp_dot<<<nblk(m), 256>>>(m, S.lp_ptr, S.lp_idx, S.lp_val, wl, sign, out);
  };
  // residuals (Residuals::compute, sdpa_dataset.cpp:585-608): rp = b - A.X,
  // D = C - Z - sum y_k A_k; sc[0] = |rp|max, sc[1] = |D|max
  auto residuals = [&]() {
    a_dot(S.rp, S.b, -1.0, MB_X, S.lpx);
    dot(S, m, S.rp, nullptr, 0, false, 1);
    bool first = true;
    if (nsdp) {
      mb_axpby(MB_D, 1.0, MB_C, -1.0, MB_Z);
      if (S.mb_ctotal)
        k_mb_sp_scatter<<<nblk(S.mb_ctotal * 32), 256>>>(S.mb_sp, S.mb_coff, S.mb_ns, S.mb_tab, MB_D, nsdp, S.y,
                                                         -1.0);
      mb_reduce(MB_D, MB_D, 1, 1, false, 1.0);
      first = false;
    }
    if (nlp) {
      k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpD, 1.0, S.lpC, -1.0, S.lpz);
      k_lp_scatter<<<nblk(nlp), 256>>>(nlp, S.lpT_ptr, S.lpT_k, S.lpT_v, S.y, -1.0, S.lpD);
      dot(S, nlp, S.lpD, nullptr, 1, !first, 1);
      first = false;
    }
    if (first) cudaMemset(S.sc + 1, 0, sizeof(double));
  };
  // sum over blocks of <A, B> (full Frobenius) + LP into sc[slot]
  auto ip = [&](int slot, int ka, int kb, const double* al, const double* bl) {
    bool acc = false;
    if (nsdp) {
      mb_reduce(ka, kb, 0, slot, false, 1.0);
      acc = true;
    }
    if (nlp) { dot(S, nlp, al, bl, slot, acc); acc = true; }
    if (!acc) cudaMemset(S.sc + slot, 0, sizeof(double));
  };

  residuals();
  ip(2, MB_C, MB_X, S.lpC, S.lpx);  // objP = C.X
  dot(S, m, S.b, S.y, 3, false);          // objD = b.y
  if (warm) ip(4, MB_X, MB_Z, S.lpx, S.lpz);  // X.Z
  double h[16];
  read_scalars(S, h, 5);
  Scalars sc;
  const double mu0 = warm ? h[4] / S.nDim : lam * lam;
  init_scalars(sc, P, S.nDim, mu0, h[0], h[1], h[2], h[3]);
  update_check(sc, P);

  // Per-phase device time (the reference's ComputeTime categories,
  // sdpa_parts.h:48-86), recorded with CUDA events on the solver's stream.
  enum { T_RMAT, T_BMAT, T_CHOL, T_SOLVE, T_DXDZ, T_STEP, T_UPDATE, T_RES, T_N };
  std::vector<cudaEvent_t> evs;
  std::vector<int> evphase;
  auto mark = [&](int ph) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e);
    evs.push_back(e);
    evphase.push_back(ph);
  };
  int iter = 0;
  while (true) {
    if (!update_check(sc, P) || iter >= P.maxIteration) break;
    mark(T_RMAT);
    predictor_setup(sc, P);
    const bool dinf = dual_infeasible(sc);
    const bool lowp = S.mixed && mixed_gap(sc) >= S.mu_switch;
    // ---- predictor rMat / gVec (Newton::compute_rMat, Make_gVec)
    if (nsdp) mb_axpby(MB_R, sc.beta * sc.mu, MB_ZI, -1.0, MB_X);
    if (dinf) {
      for (SdpBlock& B : S.sdp) {
        const long long nn = (long long)B.n * B.n;
        gemm(S, B.n, B.n, B.n, false, B.X, B.n, false, B.D, B.n, B.W1, B.n, 1.0, 0.0, false, 1, 0, 0, 0, lowp);
        gemm(S, B.n, B.n, B.n, false, B.W1, B.n, false, B.Zi, B.n, B.XDZ, B.n, 1.0, 0.0, false, 1, 0, 0, 0, lowp);
        k_axpby<<<nblk(nn), 256>>>(nn, B.W2, 1.0, B.R, -1.0, B.XDZ);
      }
    }
    const double* Wl = S.lpR;
    if (nlp) {
      k_lp_ops<<<nblk(nlp), 256>>>(0, nlp, sc.beta * sc.mu, 0, S.lpR, S.lpzi, S.lpx, nullptr, nullptr);
      if (dinf) {
        k_lp_ops<<<nblk(nlp), 256>>>(2, nlp, 0, 0, S.lpXDZ, S.lpx, S.lpD, S.lpzi, nullptr);
        k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpW, 1.0, S.lpR, -1.0, S.lpXDZ);
        Wl = S.lpW;
      }
    }
    a_dot(S.g, S.rp, -1.0, dinf ? MB_W2 : MB_R, Wl);
    mark(T_BMAT);
    // ---- Schur complement (Newton::Make_bMat).  In the FP32 phase of the
    // mixed mode the F1 products (X A_j) Z^-1 run on the tensor cores in
    // split TF32 (gemm_tf32x3); a tensor-core block that gave up waiting
    // leaves its tile unwritten, and the matrix is then built again with the
    // SIMT products.
    auto build_bmat = [&](bool use_tc) {
      if (S.f3_direct_block >= 0) {
        // one source: every entry written once, no zero fill, no atomics
        const SdpBlock& B0 = S.sdp[S.f3_direct_block];
        const long long T = (m + F3T - 1) / F3T;
        k_f3_tiles<<<(unsigned)(T * (T + 1) / 2), 256>>>(m, B0.ptr, B0.row, B0.col, B0.val, B0.nnz, B0.X, B0.Zi,
                                                          B0.n, S.B);
        if (S.f3_nheavy)
          k_f3_heavy<<<(unsigned)S.f3_nheavy, 1024>>>(m, S.f3_heavy, B0.ptr, B0.row, B0.col, B0.val, B0.nnz, B0.X,
                                                     B0.Zi, B0.n, S.B);
        return;
      }
      cudaMemset(S.B, 0, (size_t)m * m * sizeof(double));
      if (S.f3_total > 0)
        k_f3_all<<<(unsigned)nblk(S.f3_total), 256>>>(S.f3_desc, S.f3_off, S.f3_nb, S.B, m);
      if (S.f1_total > 0)
        k_f1_small<<<(unsigned)S.f1_total, 256, 2 * (size_t)S.f1_nmax * S.f1_nmax * sizeof(double)>>>(
            S.f1_desc, S.f1_off, S.f1_nb, S.B, m);
      for (SdpBlock& B : S.sdp) {
        if (!B.nc || B.n <= SMALL_F1) continue;
        const int nf = (int)B.hf1.size();
        for (int q0 = 0; q0 < nf; q0 += F1_CHUNK) {
          const int cnt = std::min(F1_CHUNK, nf - q0);
          const size_t nn = (size_t)B.n * B.n;
          double* T = S.T;
          double* G = S.T + (size_t)F1_CHUNK * nn;
          k_f1_left<<<dim3(B.n, cnt), 256>>>(B.n, q0, B.f1, B.csc_cptr, B.csc_ptr, B.csc_row, B.csc_val, B.X, T);
          const bool tc_done = use_tc && gemm_tf32x3(B.n, B.n, B.n, cnt, T, B.n, nn, B.Zi, B.n, G, B.n, nn,
                                                     S.tc_f1_work, S.tc_f1_err, 0, S.tc_wait) == 0;
          if (!tc_done)
            gemm(S, B.n, B.n, B.n, false, T, B.n, false, B.Zi, B.n, G, B.n, 1.0, 0.0, false, cnt, nn, 0, nn, lowp);
          static std::atomic<unsigned long long> pack_attr{0};
          smem_attr_per_device((const void*)k_f1_pack, (int)F1_PACK_SMEM, pack_attr);
          const long long nt = (B.n + F1_PACK_T - 1) / F1_PACK_T;
          k_f1_pack<<<(unsigned)(nt * (nt + 1) / 2), 256, F1_PACK_SMEM>>>(B.n, cnt, G, T);
          k_f1_spmm<<<dim3((B.nc + 7) / 8, 4), 256>>>(B.nc, q0, cnt, B.f1, B.cons, B.ptr, B.pos, B.val, B.nnz, T,
                                                      S.B, m);
        }
      }
      if (nlp) k_lp_bmat<<<nlp, 256>>>(S.lpT_ptr, S.lpT_k, S.lpT_v, S.lpx, S.lpzi, S.B, m);
    };
    const bool tc_f1 = lowp && S.tc_f1_work;
    if (tc_f1) cudaMemset(S.tc_f1_err, 0, sizeof(int));
    build_bmat(tc_f1);
    if (tc_f1) {
      int te = 0;
      cudaMemcpy(&te, S.tc_f1_err, sizeof(int), cudaMemcpyDeviceToHost);
      if (te) {
        stats_.tc_timeouts += 1;
        build_bmat(false);
      }
    }
    mark(T_CHOL);
    // ---- Cholesky with adjustment + solve (Newton::compute_DyVec).  Mixed
    // precision while mixed_gap >= mu_switch: FP32 factor of the FP64 Schur matrix
    // with FP64 iterative refinement of dy; FP64 factor otherwise (and when
    // the FP32 factorisation fails).
    bool fp32_factor = false;
    if (lowp) {
      k_convert<float, double><<<nblk((long long)m * m), 256>>>((long long)m * m, S.B32, S.B);
      if (S.tc) cudaMemset(S.tc_err, 0, sizeof(int));
      fp32_factor = cholesky_grid_t<float>(S, S.B32, m, true, S.Linv32, S.T32, S.dinv32) == 0;
      if (S.tc) {  // a tensor-core block that gave up leaves the factor incomplete: use FP64
        int te = 0;
        cudaMemcpy(&te, S.tc_err, sizeof(int), cudaMemcpyDeviceToHost);
        if (te) {
          fp32_factor = false;
          stats_.tc_timeouts += 1;
        }
      }
    }
    if (!fp32_factor && cholesky_grid(S, S.B, m, true, S.dinv)) {
      stats_.cholesky_failed = 1;
      break;
    }
    auto solve64 = [&](double* x) {
      if (m > SMALL_SOLVE) chol_solve_graph<double>(S, m, S.B, S.dinv, x);
      else k_chol_solve<double><<<1, NT, cta::SD_DOUBLES * sizeof(double)>>>(m, S.B, x);
    };
    auto solve32 = [&](float* x) {
      if (m > SMALL_SOLVE) chol_solve_graph<float>(S, m, S.B32, S.dinv32, x);
      else k_chol_solve<float><<<1, NT, cta::SD_DOUBLES * sizeof(float)>>>(m, S.B32, x);
    };
    auto schur_solve = [&](double* x) {
      if (!fp32_factor) {
        solve64(x);
        return;
      }
      double* rhs = S.res;
      double* r = S.res + m;
      cudaMemcpy(rhs, x, m * sizeof(double), cudaMemcpyDeviceToDevice);
      k_convert<float, double><<<nblk(m), 256>>>(m, S.v32, x);
      solve32(S.v32);
      k_convert<double, float><<<nblk(m), 256>>>(m, x, S.v32);
      for (int it = 0; it < 2; ++it) {  // x += B^{-1} (rhs - B x), correction in FP32
        k_residual<<<nblk((long long)m * 32), 256>>>(m, S.B, x, rhs, r);
        k_convert<float, double><<<nblk(m), 256>>>(m, S.v32, r);
        solve32(S.v32);
        k_add_f32<<<nblk(m), 256>>>(m, x, S.v32);
      }
    };
    mark(T_SOLVE);
    cudaMemcpy(S.dy, S.g, m * sizeof(double), cudaMemcpyDeviceToDevice);
    schur_solve(S.dy);
    mark(T_DXDZ);

    // ---- dZ and dX (compute_DzMat / compute_DxMat)
    auto direction = [&]() {
      if (!S.small_idx.empty())
        k_blocks_direction<<<(unsigned)S.small_idx.size(), NT, small_block_smem(S.small_nmax)>>>(
            S.small_ptrs, S.dy, dinf ? 1 : 0, lowp ? 1 : 0);
      for (int q : S.large_idx) {
        SdpBlock& B = S.sdp[q];
        const long long nn = (long long)B.n * B.n;
        if (dinf) k_axpby<<<nblk(nn), 256>>>(nn, B.dZ, 1.0, B.D, 0.0, nullptr);
        else cudaMemset(B.dZ, 0, nn * sizeof(double));
        if (B.nc) k_sp_scatter<<<nblk((long long)B.nc * 32), 256>>>(B.nc, B.cons, B.ptr, B.row, B.col, B.val,
                                                                    S.dy, -1.0, B.dZ, B.n);
        gemm(S, B.n, B.n, B.n, false, B.X, B.n, false, B.dZ, B.n, B.W1, B.n, 1.0, 0.0, false, 1, 0, 0, 0, lowp);
        gemm(S, B.n, B.n, B.n, false, B.W1, B.n, false, B.Zi, B.n, B.W2, B.n, 1.0, 0.0, false, 1, 0, 0, 0, lowp);
        k_sym_diff<<<nblk(nn), 256>>>(B.n, B.dX, B.R, B.W2);
      }
      if (nlp) {
        if (dinf) k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpdz, 1.0, S.lpD, 0.0, nullptr);
        else cudaMemset(S.lpdz, 0, nlp * sizeof(double));
        k_lp_scatter<<<nblk(nlp), 256>>>(nlp, S.lpT_ptr, S.lpT_k, S.lpT_v, S.dy, -1.0, S.lpdz);
        k_lp_ops<<<nblk(nlp), 256>>>(3, nlp, 0, 0, S.lpdx, S.lpR, S.lpx, S.lpdz, S.lpzi);
      }
    };
    direction();
    auto step_products = [&]() {
      ip(5, MB_C, MB_DX, S.lpC, S.lpdx);   // C.dX
      dot(S, m, S.b, S.dy, 6, false);            // b.dy
      ip(7, MB_X, MB_DZ, S.lpx, S.lpdz);   // X.dZ
      ip(8, MB_DX, MB_Z, S.lpdx, S.lpz);   // dX.Z
      ip(9, MB_DX, MB_DZ, S.lpdx, S.lpdz);  // dX.dZ
    };
    step_products();
    read_scalars(S, h, 10);
    predictor_step(sc, h[5], h[6]);
    corrector_beta(sc, P, h[7], h[8], h[9]);

    // ---- corrector
    if (!S.small_idx.empty())
      k_blocks_corrector<<<(unsigned)S.small_idx.size(), NT, small_block_smem(S.small_nmax)>>>(
          S.small_ptrs, sc.beta * sc.mu, dinf ? 1 : 0, lowp ? 1 : 0);
    for (SdpBlock& B : S.sdp) {
      const long long nn = (long long)B.n * B.n;
      if (B.n <= SMALL_BLOCK) continue;
      gemm(S, B.n, B.n, B.n, false, B.dX, B.n, false, B.dZ, B.n, B.W1, B.n, 1.0, 0.0, false, 1, 0, 0, 0, lowp);
      gemm(S, B.n, B.n, B.n, false, B.W1, B.n, false, B.Zi, B.n, B.W2, B.n, 1.0, 0.0, false, 1, 0, 0, 0, lowp);
      k_axpby_sub<<<nblk(nn), 256>>>(nn, B.R, sc.beta * sc.mu, B.Zi, -1.0, B.X, B.W2);
      if (dinf) k_axpby<<<nblk(nn), 256>>>(nn, B.W1, 1.0, B.R, -1.0, B.XDZ);
    }
    Wl = S.lpR;
    if (nlp) {
      k_lp_ops<<<nblk(nlp), 256>>>(1, nlp, sc.beta * sc.mu, 0, S.lpR, S.lpzi, S.lpx, S.lpdx, S.lpdz);
      if (dinf) {
        k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpW, 1.0, S.lpR, -1.0, S.lpXDZ);
        Wl = S.lpW;
      }
    }
    a_dot(S.dy, S.rp, -1.0, dinf ? MB_W1 : MB_R, Wl);
    mark(T_SOLVE);
    schur_solve(S.dy);
    mark(T_DXDZ);
    direction();
    mark(T_STEP);

    // ---- step length (StepLength::MehrotraCorrector)
    double minX = 1.0e50, minZ = 1.0e50;
    const int nsmall = (int)S.small_idx.size();
    if (nsmall)
      k_blocks_step<<<(unsigned)nsmall, NT, small_block_smem(S.small_nmax)>>>(S.small_ptrs, S.small_nmax,
                                                                              S.blk_mins);
    for (size_t u = 0; u < S.large_idx.size(); ++u) {
      SdpBlock& B = S.sdp[S.large_idx[u]];
      double* out = S.blk_mins + 2 * (nsmall + u);
      const size_t shm = (size_t)eig_scratch_doubles(B.n, 1) * sizeof(double);
      gemm(S, B.n, B.n, B.n, false, B.dX, B.n, true, B.LXi, B.n, B.W1, B.n, 1.0, 0.0);
      gemm(S, B.n, B.n, B.n, false, B.LXi, B.n, false, B.W1, B.n, B.W2, B.n, 1.0, 0.0);
      k_min_eig<<<1, NT, shm>>>(B.n, B.W2, out);
      gemm(S, B.n, B.n, B.n, false, B.dZ, B.n, true, B.LZi, B.n, B.W1, B.n, 1.0, 0.0);
      gemm(S, B.n, B.n, B.n, false, B.LZi, B.n, false, B.W1, B.n, B.W2, B.n, 1.0, 0.0);
      k_min_eig<<<1, NT, shm>>>(B.n, B.W2, out + 1);
    }
    if (nsdp) {
      std::vector<double> mm(2 * (size_t)nsdp);
      cudaMemcpy(mm.data(), S.blk_mins, mm.size() * sizeof(double), cudaMemcpyDeviceToHost);
      for (int q = 0; q < nsdp; ++q) {
        minX = std::min(minX, mm[2 * q]);
        minZ = std::min(minZ, mm[2 * q + 1]);
      }
    }
    if (nlp) {
      // LP part of Jal::getMinEigen (sdpa_jordan.cpp:99-105): dx_t / x_t
      std::vector<double> a(nlp), bb(nlp), cc(nlp), dd(nlp);
      cudaMemcpy(a.data(), S.lpdx, nlp * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(bb.data(), S.lplx, nlp * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(cc.data(), S.lpdz, nlp * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(dd.data(), S.lplz, nlp * sizeof(double), cudaMemcpyDeviceToHost);
      for (int t = 0; t < nlp; ++t) {
        minX = std::min(minX, a[t] * bb[t] * bb[t]);
        minZ = std::min(minZ, cc[t] * dd[t] * dd[t]);
      }
    }
    step_products();
    read_scalars(S, h, 10);
    corrector_step(sc, P, minX, minZ, h[5], h[6], h[7], h[8], h[9], sc.objD, sc.objP);
    {
      double row[8] = {sc.mu, sc.thetaP, sc.thetaD, sc.objP, sc.objD, sc.alphaP, sc.alphaD, sc.beta};
      stats_.trace.insert(stats_.trace.end(), row, row + 8);
    }

    mark(T_UPDATE);
    // ---- update (Solutions::update)
    if (nsdp) {
      mb_axpby(MB_X, 1.0, MB_X, sc.alphaP, MB_DX);
      mb_axpby(MB_Z, 1.0, MB_Z, sc.alphaD, MB_DZ);
    }
    if (nlp) {
      k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpx, 1.0, S.lpx, sc.alphaP, S.lpdx);
      k_axpby<<<nblk(nlp), 256>>>(nlp, S.lpz, 1.0, S.lpz, sc.alphaD, S.lpdz);
    }
    k_axpby<<<nblk(m), 256>>>(m, S.y, 1.0, S.y, sc.alphaD, S.dy);
    if (cannot_move(sc)) break;
    if (!compute_inverse()) break;
    mark(T_RES);
    // ---- residuals, mu, objectives, rho
    residuals();
    ip(2, MB_C, MB_X, S.lpC, S.lpx);
    dot(S, m, S.b, S.y, 3, false);
    ip(4, MB_X, MB_Z, S.lpx, S.lpz);
    if (warm) {
      ip(13, MB_X0, MB_Z, S.lpx0, S.lpz);
      ip(14, MB_X, MB_Z0, S.lpx, S.lpz0);
    } else {
      if (nsdp) {
        mb_reduce(MB_Z, MB_Z, 2, 13, false, lam);
        mb_reduce(MB_X, MB_X, 2, 14, false, lam);
      } else {
        cudaMemset(S.sc + 13, 0, 2 * sizeof(double));
      }
    }
    read_scalars(S, h, 16);
    double x0zM = h[13], xMz0 = h[14];
    if (!warm && nlp) {
      std::vector<double> a(nlp), bb(nlp);
      cudaMemcpy(a.data(), S.lpz, nlp * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(bb.data(), S.lpx, nlp * sizeof(double), cudaMemcpyDeviceToHost);
      for (int t = 0; t < nlp; ++t) { x0zM += lam * a[t]; xMz0 += lam * bb[t]; }
    }
    after_update(sc, P, h[4], h[0], h[1], h[2], h[3], x0zM, xMz0);
    ++iter;
  }
  mark(T_N);
  // final residuals (sdpa_solve.cpp:204), results
  residuals();
  read_scalars(S, h, 2);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_error(e, "solve");
  stats_.iterations = iter;
  stats_.internal_phase = sc.phase;
  stats_.phase = user_phase(sc.phase);
  stats_.primal_obj = -sc.objD;
  stats_.dual_obj = -sc.objP;
  stats_.objValPrimal = sc.objP;
  stats_.objValDual = sc.objD;
  stats_.primal_error = h[1];
  stats_.dual_error = h[0];
  stats_.mu = sc.mu;
  {
    const double row[8] = {sc.mu, sc.thetaP, sc.thetaD, sc.objP, sc.objD, sc.alphaP, sc.alphaD, sc.beta};
    for (int q = 0; q < 8; ++q) stats_.final_row[q] = row[q];
  }
  xvec_.assign(m, 0.0);
  cudaMemcpy(xvec_.data(), S.y, m * sizeof(double), cudaMemcpyDeviceToHost);
  for (double& v : xvec_) v = -v;
  const int nb = (int)S.blockKind.size();
  Xres_.assign(nb, {});
  Yres_.assign(nb, {});
  std::vector<double> hx(nlp), hz(nlp);
  if (nlp) {
    cudaMemcpy(hx.data(), S.lpx, nlp * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(hz.data(), S.lpz, nlp * sizeof(double), cudaMemcpyDeviceToHost);
  }
  for (int l = 0; l < nb; ++l) {
    if (S.blockKind[l] == 0) {
      SdpBlock& B = S.sdp[S.blockIndex[l]];
      const size_t nn = (size_t)B.n * B.n;
      Xres_[l].resize(nn);
      Yres_[l].resize(nn);
      cudaMemcpy(Xres_[l].data(), B.Z, nn * sizeof(double), cudaMemcpyDeviceToHost);
      cudaMemcpy(Yres_[l].data(), B.X, nn * sizeof(double), cudaMemcpyDeviceToHost);
    } else {
      const int off = S.blockIndex[l], len = S.blockStruct[l];
      Xres_[l].assign(hz.begin() + off, hz.begin() + off + len);
      Yres_[l].assign(hx.begin() + off, hx.begin() + off + len);
    }
  }
  stats_.solve_seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
  stats_.phase_seconds.assign(T_N, 0.0);
  for (size_t q = 0; q + 1 < evs.size(); ++q) {
    float ms = 0.0f;
    if (evphase[q] < T_N && cudaEventElapsedTime(&ms, evs[q], evs[q + 1]) == cudaSuccess)
      stats_.phase_seconds[evphase[q]] += ms / 1e3;
  }
  for (cudaEvent_t e : evs) cudaEventDestroy(e);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "solve");
  return SDPAB_OK;
}

}  // namespace sdpab

// The constraint order Solver::setup would use (host only, no device work):
// order[position] = constraint (0-based), or the identity when the natural
// order is kept; pairs[0] / pairs[1] = the symbolic tile pairs of the Schur
// factorisation in the natural / the returned order.  Entries as for
// sdpab_sdpa_input_problem (1-based k, l, i, j; k = 0 is F0).
extern "C" SDPAB_API int sdpab_constraint_order(int m, int nblock, const int* block_struct, long long nnz,
                                                const int* k, const int* l, const int* i, const int* j,
                                                int* order, long long* pairs)
{
  if (m < 1 || nblock < 1 || nnz < 0 || !block_struct || !order || !pairs || (nnz > 0 && (!k || !l || !i || !j)))
    return sdpab::set_error(SDPAB_EINVAL, "constraint_order: invalid arguments");
  sdpab::ProblemData p;
  p.m = m;
  p.blockStruct.assign(block_struct, block_struct + nblock);
  p.c.assign(m, 0.0);
  for (long long t = 0; t < nnz; ++t) p.entries.push_back({k[t], l[t], i[t], j[t], 1.0});
  const auto groups = sdpab::constraint_groups(p);
  std::vector<int> ident(m);
  for (int q = 0; q < m; ++q) ident[q] = q;
  pairs[0] = sdpab::symbolic_tile_pairs(groups, ident, m);
  int nsdp = 0;
  for (int b : p.blockStruct) nsdp += (b > 1) ? 1 : 0;
  std::vector<int> ord = ident;
  pairs[1] = pairs[0];
  if (nsdp >= 2 && m >= 4 * sdpab::NBG && m <= 65536) ord = sdpab::best_constraint_order(groups, m, nullptr, &pairs[1]);
  std::copy(ord.begin(), ord.end(), order);
  return SDPAB_OK;
}
