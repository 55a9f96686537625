// CTA-cooperative dense linear algebra for one small SDP block (order n up to
// a few hundred), the building blocks of the batched persistent solver.
// Every routine is called by ALL threads of the block with identical
// arguments; matrices are column-major FP64 in global memory (the block's
// L2-resident workspace) and tiles are staged through shared memory.
// Factorisations and triangular solves are blocked by 32: the 32 x 32
// diagonal block is handled by one warp with shuffles, everything else is a
// block-wide tile update, so the number of block barriers grows with n/32,
// not with n.  Nothing here waits on another thread block.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include <type_traits>

namespace sdpab {
namespace cta {

constexpr int NB = 32;      // blocking of factorisations / solves
constexpr int LDD = 33;     // leading dimension of the shared diagonal block
// Shared diagonal-block buffer: NB x NB block (leading dimension LDD) followed
// by the NB reciprocals of its diagonal.
constexpr int SD_DOUBLES = NB * LDD + NB;

// ------------------------------------------------------------ reductions
// Block reductions with ONE barrier: partials go to one of two alternating
// shared slots, so a fast thread entering the next reduction cannot overwrite
// a slot that a slow thread is still reading (that thread must first pass
// the next reduction's barrier).  All threads must call in the same order.
struct Reducer {
  double* buf;  // 4 * (NT/32) doubles: two parities of 2 * (NT/32) slots
  int parity;
};

template <int NT>
__device__ __forceinline__ double block_sum(double v, Reducer& R)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  double* slot = R.buf + R.parity * (2 * (NT / 32));
  R.parity ^= 1;
  if ((threadIdx.x & 31) == 0) slot[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < NT / 32; ++w) s += slot[w];
  return s;
}

// K <= 2 sums with one barrier (same slot discipline as block_sum).
template <int NT, int K>
__device__ __forceinline__ void block_sum_n(const double* v, double* out, Reducer& R)
{
  static_assert(K >= 1 && K <= 2, "block_sum_n: K <= 2");
  double* slot = R.buf + R.parity * (2 * (NT / 32));
  R.parity ^= 1;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double x = v[j];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) slot[j * (NT / 32) + (threadIdx.x >> 5)] = x;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) s += slot[j * (NT / 32) + w];
    out[j] = s;
  }
}

// K <= 2 maxima with one barrier (same slot discipline as block_sum).
template <int NT, int K>
__device__ __forceinline__ void block_max_n(const double* v, double* out, Reducer& R)
{
  static_assert(K >= 1 && K <= 2, "block_max_n: K <= 2");
  double* slot = R.buf + R.parity * (2 * (NT / 32));
  R.parity ^= 1;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double x = v[j];
    for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
    if ((threadIdx.x & 31) == 0) slot[j * (NT / 32) + (threadIdx.x >> 5)] = x;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double s = slot[j * (NT / 32)];
#pragma unroll
    for (int w = 1; w < NT / 32; ++w) s = fmax(s, slot[j * (NT / 32) + w]);
    out[j] = s;
  }
}

template <int NT>
__device__ __forceinline__ double block_max(double v, Reducer& R)
{
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  double* slot = R.buf + R.parity * (2 * (NT / 32));
  R.parity ^= 1;
  if ((threadIdx.x & 31) == 0) slot[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = slot[0];
#pragma unroll
  for (int w = 1; w < NT / 32; ++w) s = fmax(s, slot[w]);
  return s;
}

// Full Frobenius inner product of two n x n column-major matrices.
template <int NT>
__device__ double dot_mat(int n, const double* A, const double* B, Reducer& R)
{
  double s = 0.0;
  const int tot = n * n;
  for (int t = threadIdx.x; t < tot; t += NT) s += A[t] * B[t];
  return block_sum<NT>(s, R);
}

template <int NT>
__device__ double trace(int n, const double* A, Reducer& R)
{
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) s += A[i + (size_t)n * i];
  return block_sum<NT>(s, R);
}

template <int NT>
__device__ double dot_vec(int n, const double* a, const double* b, Reducer& R)
{
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) s += a[i] * b[i];
  return block_sum<NT>(s, R);
}

// Asynchronous global -> shared copy of one element of 4 or 8 bytes
// (cp.async; zero fill when `valid` is false, the source pointer must still
// be a valid address), and the group fences around it.
template <typename T>
__device__ __forceinline__ void cp_async_el(void* smem_dst, const T* gsrc, bool valid)
{
  static_assert(sizeof(T) == 4 || sizeof(T) == 8, "cp_async_el: 4- or 8-byte elements");
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(gsrc), "r"(valid ? 8 : 0));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(gsrc), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc, bool valid)
{
  cp_async_el<double>(smem_dst, (const double*)gsrc, valid);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ------------------------------------------------------------ GEMM
// All GEMM / factorisation routines are templated on the matrix storage type
// TM and the compute type TC (TC = float with TM = double is the mixed
// precision path: operands are rounded to FP32 when staged in shared memory,
// products accumulate in FP32, results are stored back in FP64), and on the
// number of threads NT of the calling block (256 or 128; 8 or 4 warps).
//
// 64 x 64 output tiles, K staged in chunks of gk<NT>() (16 with 256
// threads, 8 with 128: a 128-thread block shares its SM with three others
// and stages half as much).
constexpr int GT = 64, GK = 16;
template <int NT>
__host__ __device__ constexpr int gk() { return NT >= 256 ? 16 : 8; }
// shared memory (elements) a gemm_rect call may use: two stages of A and B
constexpr int GTP = GT + 4;  // staged row stride (bank spread of the FP64 MMA fragment loads)
constexpr int GEMM_RECT_SMEM = 4 * GK * GTP;  // 256 threads
template <int NT>
__host__ __device__ constexpr int gemm_rect_smem() { return 4 * gk<NT>() * GTP; }

// One FP64 tensor-core MMA, D = A B + D with A 8 x 4, B 4 x 8, D 8 x 8
// (mma.sync m8n8k4 .f64; per lane one element of A and of B, two of D).
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// gemm_rect with double-buffered cp.async staging (storage type = compute
// type): the (tile, K chunk) steps form one pipeline, chunk s+1 (of this or
// the next live tile) is copied while chunk s is multiplied, one barrier per
// step.  FP64: the warps as 2 x (NT / 64) over the 8 x 8 blocks of the tile
// on the FP64 MMA; FP32: the threads as 16 x (NT / 16), each 64 / (NT / 16)
// rows x 4 columns.  smem: 4 * gk<NT>() * GTP elements of T.
template <int NT, typename T>
__device__ __noinline__ void gemm_rect_db(int M, int N, int K, bool tA, const T* A, int lda, bool tB, const T* B,
                                          int ldb, T* C, int ldc, double alpha, double beta, void* smem_v,
                                          bool lower, int diag_off)
{
  constexpr int G = gk<NT>();
  T* buf = (T*)smem_v;  // [2][As: G*GTP | Bs: G*GTP]
  const int tm = (M + GT - 1) / GT, tn = (N + GT - 1) / GT, ntile = tm * tn;
  const int nk = (K + G - 1) / G;
  auto live = [&](int tile) {
    const int r0 = (tile % tm) * GT, c0 = (tile / tm) * GT;
    return !(lower && r0 + GT - 1 + diag_off < c0);
  };
  auto next_live = [&](int tile) {
    while (tile < ntile && !live(tile)) ++tile;
    return tile;
  };
  auto issue = [&](int tile, int k0, int which) {
    const int r0 = (tile % tm) * GT, c0 = (tile / tm) * GT;
    T* As = buf + which * 2 * G * GTP;
    T* Bs = As + G * GTP;
    for (int t = threadIdx.x; t < G * GT; t += NT) {
      int r, k;
      if (!tA) { r = t % GT; k = t / GT; } else { k = t % G; r = t / G; }
      const int gr = r0 + r, gk2 = k0 + k;
      const bool va = gr < M && gk2 < K;
      cp_async_el<T>(&As[k * GTP + r], va ? (tA ? A + gk2 + (size_t)lda * gr : A + gr + (size_t)lda * gk2) : A, va);
      int c;
      if (!tB) { k = t % G; c = t / G; } else { c = t % GT; k = t / GT; }
      const int gc = c0 + c, gk3 = k0 + k;
      const bool vb = gc < N && gk3 < K;
      cp_async_el<T>(&Bs[k * GTP + c], vb ? (tB ? B + gc + (size_t)ldb * gk3 : B + gk3 + (size_t)ldb * gc) : B, vb);
    }
    cp_async_commit();
  };
  int tile = next_live(0);
  if (tile >= ntile) {
    __syncthreads();
    return;
  }
  int it_tile = tile, it_k = 0;  // the next (tile, chunk) to copy
  auto advance = [&]() {
    if (++it_k == nk) {
      it_k = 0;
      it_tile = next_live(it_tile + 1);
    }
  };
  issue(it_tile, 0, 0);
  advance();
  int which = 0;
  while (tile < ntile) {
    const int r0 = (tile % tm) * GT, c0 = (tile / tm) * GT;
    if constexpr (std::is_same<T, double>::value) {
      // FP64 MMA (m8n8k4): warps as 2 x WC over the 8 x 8 blocks of the
      // tile, warp (wr, wc) owning blocks (wr + 2 i, wc + WC j), i < 4,
      // j < 8 / WC; lane l holds A(l / 4, l % 4), B(l % 4, l / 4),
      // C(l / 4, 2 (l % 4) + h)
      constexpr int WC = NT / 64, JB = 8 / WC;
      const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wr = w & 1, wc = w >> 1;
      const int q = lane & 3, p = lane >> 2;
      double acc[4][JB][2];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < JB; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
      for (int kc = 0; kc < nk; ++kc) {
        cp_async_wait_all();
        __syncthreads();  // this step's chunk is visible; the other buffer is free
        if (it_tile < ntile) {
          issue(it_tile, it_k * G, which ^ 1);
          advance();
        }
        const double* As = buf + which * 2 * G * GTP;
        const double* Bs = As + G * GTP;
        // rows k >= K of the last chunk are zero-filled: whole steps of 4
        const int kmax = min(G, K - kc * G);
        for (int kk = 0; kk < kmax; kk += 4) {
          double a[4], b[JB];
#pragma unroll
          for (int i = 0; i < 4; ++i) a[i] = As[(kk + q) * GTP + (wr + 2 * i) * 8 + p];
#pragma unroll
          for (int j = 0; j < JB; ++j) b[j] = Bs[(kk + q) * GTP + (wc + WC * j) * 8 + p];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < JB; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        which ^= 1;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int gr = r0 + (wr + 2 * i) * 8 + p;
        if (gr >= M) continue;
#pragma unroll
        for (int j = 0; j < JB; ++j) {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int gc = c0 + (wc + WC * j) * 8 + 2 * q + h;
            if (gc >= N) continue;
            if (lower && gr + diag_off < gc) continue;
            double* cp = C + gr + (size_t)ldc * gc;
            *cp = (beta == 0.0) ? alpha * acc[i][j][h] : alpha * acc[i][j][h] + beta * (*cp);
          }
        }
      }
    } else {
    constexpr int TY = NT / 16, IR = GT / TY;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    T acc[IR][4];
#pragma unroll
    for (int i = 0; i < IR; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = (T)0;
    for (int kc = 0; kc < nk; ++kc) {
      cp_async_wait_all();
      __syncthreads();  // this step's chunk is visible; the other buffer is free
      if (it_tile < ntile) {
        issue(it_tile, it_k * G, which ^ 1);
        advance();
      }
      const T* As = buf + which * 2 * G * GTP;
      const T* Bs = As + G * GTP;
      const int kmax = min(G, K - kc * G);
      for (int k = 0; k < kmax; ++k) {
        T a[IR], b[4];
#pragma unroll
        for (int i = 0; i < IR; ++i) a[i] = As[k * GTP + ty + TY * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[k * GTP + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < IR; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      which ^= 1;
    }
#pragma unroll
    for (int i = 0; i < IR; ++i) {
      const int gr = r0 + ty + TY * i;
      if (gr >= M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int gc = c0 + tx + 16 * j;
        if (gc >= N) continue;
        if (lower && gr + diag_off < gc) continue;
        T* cp = C + gr + (size_t)ldc * gc;
        *cp = (T)((beta == 0.0) ? alpha * (double)acc[i][j] : alpha * (double)acc[i][j] + beta * (double)(*cp));
      }
    }
    }
    tile = next_live(tile + 1);
  }
  __syncthreads();
}

// gemm_rect: C[M x N] = alpha * op(A)[M x K] * op(B)[K x N] + beta * C.
// 64 x 64 output tiles, K staged in chunks of gk<NT>().  When the storage
// and compute types agree the staging is gemm_rect_db's (cp.async, two
// stages); the mixed FP64-storage / FP32-compute form prefetches the next
// chunk into registers and converts while storing, with the threads as
// 16 x (NT / 16), each 64 / (NT / 16) rows x 4 columns (rows ty + (NT / 16) i,
// columns tx + 16 j).  lower = true updates only entries with
// (row + diag_off >= col) and skips tiles entirely above that diagonal
// (trailing updates of factorisations).  smem: gemm_rect_smem<NT>()
// elements of TC.  Ends with a barrier.
template <int NT, typename TM, typename TC>
__device__ __noinline__ void gemm_rect(int M, int N, int K, bool tA, const TM* A, int lda, bool tB,
                                       const TM* B, int ldb, TM* C, int ldc, double alpha, double beta,
                                       void* smem_v, bool lower = false, int diag_off = 0)
{
  static_assert(NT == 256 || NT == 128, "gemm tile mappings for 256 or 128 threads");
  if constexpr (std::is_same<TM, TC>::value) {
    if (K > 0) {
      gemm_rect_db<NT, TM>(M, N, K, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem_v, lower, diag_off);
      return;
    }
  }
  constexpr int G = gk<NT>();
  constexpr int PER = G * GT / NT;  // staged elements per thread and operand
  constexpr int TY = NT / 16, IR = GT / TY;
  TC* As = (TC*)smem_v;          // [G][GT]  As[k*GT + r]
  TC* Bs = As + G * GT;          // [G][GT]  Bs[k*GT + c]
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int tm = (M + GT - 1) / GT, tn = (N + GT - 1) / GT;
  TC ra[PER], rb[PER];
  auto fetch = [&](int r0, int c0, int k0) {
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int t = threadIdx.x + u * NT;
      int r, k;
      if (!tA) { r = t % GT; k = t / GT; } else { k = t % G; r = t / G; }
      const int gr = r0 + r, gk2 = k0 + k;
      ra[u] = (gr < M && gk2 < K) ? (TC)(tA ? A[gk2 + (size_t)lda * gr] : A[gr + (size_t)lda * gk2]) : (TC)0;
      int c;
      if (!tB) { k = t % G; c = t / G; } else { c = t % GT; k = t / GT; }
      const int gc = c0 + c, gk3 = k0 + k;
      rb[u] = (gc < N && gk3 < K) ? (TC)(tB ? B[gc + (size_t)ldb * gk3] : B[gk3 + (size_t)ldb * gc]) : (TC)0;
    }
  };
  auto store = [&]() {
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int t = threadIdx.x + u * NT;
      int r, k;
      if (!tA) { r = t % GT; k = t / GT; } else { k = t % G; r = t / G; }
      As[k * GT + r] = ra[u];
      int c;
      if (!tB) { k = t % G; c = t / G; } else { c = t % GT; k = t / GT; }
      Bs[k * GT + c] = rb[u];
    }
  };
  auto tile_live = [&](int tile) {
    const int r0 = (tile % tm) * GT, c0 = (tile / tm) * GT;
    return !(lower && r0 + GT - 1 + diag_off < c0);
  };
  int tile = 0;
  while (tile < tm * tn && !tile_live(tile)) ++tile;
  if (tile < tm * tn) fetch((tile % tm) * GT, (tile / tm) * GT, 0);
  while (tile < tm * tn) {
    const int r0 = (tile % tm) * GT, c0 = (tile / tm) * GT;
    TC acc[IR][4];
#pragma unroll
    for (int i = 0; i < IR; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = (TC)0;
    int next = tile + 1;
    while (next < tm * tn && !tile_live(next)) ++next;
    for (int k0 = 0; k0 < K; k0 += G) {
      store();
      __syncthreads();
      if (k0 + G < K) fetch(r0, c0, k0 + G);
      else if (next < tm * tn) fetch((next % tm) * GT, (next / tm) * GT, 0);
      const int kmax = min(G, K - k0);
      for (int k = 0; k < kmax; ++k) {
        TC a[IR], b[4];
#pragma unroll
        for (int i = 0; i < IR; ++i) a[i] = As[k * GT + ty + TY * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[k * GT + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < IR; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < IR; ++i) {
      const int gr = r0 + ty + TY * i;
      if (gr >= M) continue;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int gc = c0 + tx + 16 * j;
        if (gc >= N) continue;
        if (lower && gr + diag_off < gc) continue;
        TM* cp = C + gr + (size_t)ldc * gc;
        *cp = (TM)((beta == 0.0) ? alpha * (double)acc[i][j] : alpha * (double)acc[i][j] + beta * (double)(*cp));
      }
    }
    tile = next;
  }
  __syncthreads();
}

// Square n x n product as ONE output tile of (16 R) x (16 R), R = ceil(n/16)
// (n <= 96): the threads as 16 x (NT / 16); thread (tx, ty) owns rows
// ty + (NT / 16) i and columns tx + 16 j, so no padding beyond the next
// multiple of 16 is computed.  K is staged in chunks of 16 (smem
// 2 * 16 * 16R elements of TC).
template <int NT, int R, typename TM, typename TC>
__device__ __noinline__ void gemm_tile(int n, bool tA, const TM* A, int lda, bool tB, const TM* B, int ldb,
                                       TM* C, int ldc, double alpha, double beta, void* smem_v)
{
  constexpr int T = 16 * R, KC = 16, TY = NT / 16, RI = T / TY;
  TC* As = (TC*)smem_v;         // [KC][T]
  TC* Bs = As + KC * T;         // [KC][T]
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  TC acc[RI][R];
#pragma unroll
  for (int i = 0; i < RI; ++i)
#pragma unroll
    for (int j = 0; j < R; ++j) acc[i][j] = (TC)0;
  for (int k0 = 0; k0 < n; k0 += KC) {
    for (int t = threadIdx.x; t < KC * T; t += NT) {
      int r, k;
      if (!tA) { r = t % T; k = t / T; } else { k = t % KC; r = t / KC; }
      const int gk2 = k0 + k;
      As[k * T + r] = (r < n && gk2 < n) ? (TC)(tA ? A[gk2 + (size_t)lda * r] : A[r + (size_t)lda * gk2]) : (TC)0;
      int c;
      if (!tB) { k = t % KC; c = t / KC; } else { c = t % T; k = t / T; }
      const int gk3 = k0 + k;
      Bs[k * T + c] = (c < n && gk3 < n) ? (TC)(tB ? B[c + (size_t)ldb * gk3] : B[gk3 + (size_t)ldb * c]) : (TC)0;
    }
    __syncthreads();
    const int kmax = min(KC, n - k0);
    for (int k = 0; k < kmax; ++k) {
      TC a[RI], b[R];
#pragma unroll
      for (int i = 0; i < RI; ++i) a[i] = As[k * T + ty + TY * i];
#pragma unroll
      for (int j = 0; j < R; ++j) b[j] = Bs[k * T + tx + 16 * j];
#pragma unroll
      for (int i = 0; i < RI; ++i)
#pragma unroll
        for (int j = 0; j < R; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < RI; ++i) {
    const int gr = ty + TY * i;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int gc = tx + 16 * j;
      if (gr < n && gc < n) {
        TM* cp = C + gr + (size_t)ldc * gc;
        *cp = (TM)((beta == 0.0) ? alpha * (double)acc[i][j] : alpha * (double)acc[i][j] + beta * (double)(*cp));
      }
    }
  }
  __syncthreads();
}

// FP64 tile GEMM for n <= 96 on the FP64 tensor-core MMA
// (mma.sync m8n8k4 .f64: one 8 x 8 x 4 product, 256 FMAs, per warp
// instruction): one exact-size tile T x T (T = 16 R >= n) of 2R x 2R blocks
// of 8 x 8.  The warps as 2 x WC (WC = NT / 64), warp (wr, wc) owning the
// row blocks wr + 2 i (i < R) and, in each of NPASS column passes (1 with
// 256 threads, 2 with 128, so that a warp's accumulators stay at
// R x ceil(R / 2) blocks), the column blocks pbase + wc + WC j of the pass.
// K is staged in chunks of KC (16 with 256 threads, 8 with 128) by cp.async
// into two buffers ([k][r] with a row stride of T + 4 doubles, so each
// half-warp's fragment loads fall on distinct banks); a pass stages A
// whole and B's columns of the pass.  Fragments (PTX m8n8k4 .f64): lane l
// holds A(l / 4, l % 4), B(l % 4, l / 4) and C(l / 4, 2 (l % 4) + {0, 1}).
// smem: 4 * KC * (T + 4) doubles.
template <int NT>
__host__ __device__ constexpr int mma_kc() { return NT >= 256 ? 16 : 8; }

template <int NT, int R>
__device__ __noinline__ void gemm_tile_mma(int n, bool tA, const double* A, int lda, bool tB, const double* B,
                                           int ldb, double* C, int ldc, double alpha, double beta, void* smem_v)
{
  static_assert(NT == 256 || NT == 128, "gemm_tile_mma: 8 or 4 warps");
  constexpr int T = 16 * R, TP = T + 4, KC = mma_kc<NT>(), NB = T / 8;
  constexpr int WC = NT / 64, NPASS = (NT == 256) ? 1 : 2;
  constexpr int PB = (NB + NPASS - 1) / NPASS;  // column blocks per pass
  constexpr int CB = (PB + WC - 1) / WC;        // column blocks per warp and pass
  double* buf = (double*)smem_v;  // [2][As: KC*TP | Bs: KC*TP]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, wr = w & 1, wc = w >> 1;
  const int q = lane & 3, p = lane >> 2;
  const int nch = (n + KC - 1) / KC;
  for (int pass = 0; pass < NPASS; ++pass) {
    const int pbase = pass * PB;
    const int pcols = min(PB, NB - pbase) * 8;  // columns of this pass
    const int c0 = pbase * 8;
    auto issue = [&](int k0, int which) {
      double* As = buf + which * 2 * KC * TP;
      double* Bs = As + KC * TP;
      for (int t = threadIdx.x; t < KC * T; t += NT) {
        int r, k;
        if (!tA) { r = t % T; k = t / T; } else { k = t % KC; r = t / KC; }
        const int gk2 = k0 + k;
        const bool va = r < n && gk2 < n;
        cp_async8(&As[k * TP + r], va ? (tA ? A + gk2 + (size_t)lda * r : A + r + (size_t)lda * gk2) : A, va);
      }
      for (int t = threadIdx.x; t < KC * pcols; t += NT) {
        int c, k;
        if (!tB) { k = t % KC; c = t / KC; } else { c = t % pcols; k = t / pcols; }
        const int gc = c0 + c, gk3 = k0 + k;
        const bool vb = gc < n && gk3 < n;
        cp_async8(&Bs[k * TP + c], vb ? (tB ? B + gc + (size_t)ldb * gk3 : B + gk3 + (size_t)ldb * gc) : B, vb);
      }
      cp_async_commit();
    };
    double acc[R][CB][2];
#pragma unroll
    for (int i = 0; i < R; ++i)
#pragma unroll
      for (int j = 0; j < CB; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    issue(0, 0);
    for (int ch = 0; ch < nch; ++ch) {
      cp_async_wait_all();
      __syncthreads();  // chunk ch visible; every thread is done with chunk ch-1's buffer
      if (ch + 1 < nch) issue((ch + 1) * KC, (ch + 1) & 1);
      const double* As = buf + (ch & 1) * 2 * KC * TP;
      const double* Bs = As + KC * TP;
      // rows k >= n of the last chunk are zero-filled: whole steps of 4
      const int kmax = min(KC, n - ch * KC);
      for (int kk = 0; kk < kmax; kk += 4) {
        double a[R], b[CB];
#pragma unroll
        for (int i = 0; i < R; ++i) a[i] = As[(kk + q) * TP + (wr + 2 * i) * 8 + p];
#pragma unroll
        for (int j = 0; j < CB; ++j) {
          const int lb = wc + WC * j;  // column block within the pass
          b[j] = (lb < PB && pbase + lb < NB) ? Bs[(kk + q) * TP + lb * 8 + p] : 0.0;
        }
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
          for (int j = 0; j < CB; ++j)
            if (wc + WC * j < PB && pbase + wc + WC * j < NB) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const int gr = (wr + 2 * i) * 8 + p;
#pragma unroll
      for (int j = 0; j < CB; ++j) {
        const int lb = wc + WC * j;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int gc = (pbase + lb) * 8 + 2 * q + h;
          if (lb < PB && pbase + lb < NB && gr < n && gc < n) {
            double* cp = C + gr + (size_t)ldc * gc;
            *cp = (beta == 0.0) ? alpha * acc[i][j][h] : alpha * acc[i][j][h] + beta * (*cp);
          }
        }
      }
    }
    __syncthreads();
  }
}

// Shared memory (doubles) the square GEMM dispatch below needs with NT threads.
template <int NT>
__host__ __device__ constexpr int gemm_smem_min() { return 4 * mma_kc<NT>() * (96 + 4); }

// Square GEMM dispatch: one exact-size tile for n <= 96 (FP64: on the FP64
// MMA, double-buffered), 64 x 64 tiles above.  The FP32 form (lowp) with
// 128 threads keeps the exact tile to n <= 64 (the accumulators of larger
// ones would not stay in registers).  smem must hold gemm_smem_min<NT>()
// doubles.
template <int NT, typename TM>
__device__ __forceinline__ void gemm_prec(int n, bool tA, const TM* A, int lda, bool tB, const TM* B, int ldb,
                                          TM* C, int ldc, double alpha, double beta, void* smem, bool lowp)
{
  if (lowp) {
    if (n <= 32) gemm_tile<NT, 2, TM, float>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else if (n <= 48) gemm_tile<NT, 3, TM, float>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else if (n <= 64) gemm_tile<NT, 4, TM, float>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else {
      if constexpr (NT == 256) {
        if (n <= 80) {
          gemm_tile<NT, 5, TM, float>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
          return;
        }
        if (n <= 96) {
          gemm_tile<NT, 6, TM, float>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
          return;
        }
      }
      gemm_rect<NT, TM, float>(n, n, n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    }
  } else {
    if (n <= 32) gemm_tile_mma<NT, 2>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else if (n <= 48) gemm_tile_mma<NT, 3>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else if (n <= 64) gemm_tile_mma<NT, 4>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else if (n <= 80) gemm_tile_mma<NT, 5>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else if (n <= 96) gemm_tile_mma<NT, 6>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
    else gemm_rect<NT, TM, TM>(n, n, n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem);
  }
}

template <int NT>
__device__ __forceinline__ void gemm(int n, bool tA, const double* A, int lda, bool tB, const double* B, int ldb,
                                     double* C, int ldc, double alpha, double beta, double* smem)
{
  gemm_prec<NT, double>(n, tA, A, lda, tB, B, ldb, C, ldc, alpha, beta, smem, false);
}

// ------------------------------------------------------------ warp Cholesky
// Pivot rules: adjust = true is the reference's Schur-complement rule
// (rATL_dpotrfL, sdpa_dpotrf.cpp:31-33): pivot < -1e-6 fails, pivot < 1e-14
// is replaced by a huge value (1e100 in FP64; in FP32, where 1e100 is not
// representable, 1e30, which likewise makes the column vanish).  adjust =
// false is LAPACK dpotrf's rule (pivot <= 0 fails).  NaN fails under both.
template <typename T>
__device__ __forceinline__ T adjust_huge();
template <>
__device__ __forceinline__ double adjust_huge<double>() { return 1.0e100; }
template <>
__device__ __forceinline__ float adjust_huge<float>() { return 1.0e30f; }

// Factors the bs x bs (bs <= 32) lower triangle held in sD (leading
// dimension ld, LDD by default) in place with one warp: lane r keeps row r in
// registers and the column of each step is broadcast with shuffles (no
// shared-memory traffic inside the factorisation).  kb is the block's
// offset, used in the returned failing column (0 = success).
template <typename T>
static __device__ __noinline__ int warp_potrf32(int bs, T* sD, bool adjust, int kb, int ld = LDD)
{
  const int lane = threadIdx.x & 31;
  T a[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) a[c] = (c <= lane && lane < bs) ? sD[lane + ld * c] : (T)0;
  int fail = 0;
#pragma unroll
  for (int j = 0; j < 32; ++j) {
    if (j < bs && !fail) {
      T d = __shfl_sync(0xffffffffu, a[j], j);
      if (adjust) {
        if (d < (T)-1.0e-6 || d != d) fail = kb + j + 1;
        else if (d < (T)1.0e-14) d = adjust_huge<T>();
      } else if (!(d > (T)0)) {
        fail = kb + j + 1;
      }
      if (!fail) {
        const T ljj = sqrt(d);
        const T inv = (T)1 / ljj;
        if (lane == j) a[j] = ljj;
        else if (lane > j) a[j] *= inv;
        const T lrj = a[j];
#pragma unroll
        for (int c = j + 1; c < 32; ++c) {
          const T lcj = __shfl_sync(0xffffffffu, lrj, c);
          if (lane >= c) a[c] -= lrj * lcj;
        }
      }
    }
  }
  if (!fail && lane < bs) {
#pragma unroll
    for (int c = 0; c < 32; ++c)
      if (c <= lane) sD[lane + ld * c] = a[c];
  }
  return fail;
}

// ------------------------------------------------------------ Cholesky
// Shared memory (elements of T) cholesky_smem needs for order n.
__host__ __device__ constexpr long long cholesky_smem_elems(int n) { return (long long)n * (n + 1) + NB; }

// The pieces of a factorisation held entirely in shared memory: S is the
// n x n matrix column-major with leading dimension n + 1 (so the rows of a
// column and the columns of a row spread over the banks), followed by NB
// elements of scratch (the reciprocals of the current diagonal block).

// S = lower triangle of A (type TA, converted to T).  Ends with a barrier.
template <int NT, typename T, typename TA>
__device__ void smem_load_lower(int n, const TA* A, int lda, T* S)
{
  const int ld = n + 1;
  for (int t = threadIdx.x; t < n * n; t += NT) {
    const int i = t % n, j = t / n;
    if (i >= j) S[i + ld * j] = (T)A[i + (size_t)lda * j];
  }
  __syncthreads();
}

// Out = lower triangle of S (strict upper zeroed when zero_upper).  Ends
// with a barrier.
template <int NT, typename T>
__device__ void smem_store_lower(int n, const T* S, T* Out, int ldo, bool zero_upper)
{
  const int ld = n + 1;
  for (int t = threadIdx.x; t < n * n; t += NT) {
    const int i = t % n, j = t / n;
    if (i >= j) Out[i + (size_t)ldo * j] = S[i + ld * j];
    else if (zero_upper) Out[i + (size_t)ldo * j] = (T)0;
  }
  __syncthreads();
}

// In-place lower Cholesky of S, blocked by 32 (the diagonal block by one
// warp with shuffles, the panel by the warps four rows at a time, the
// trailing update by all threads in 2 x 2 register tiles), three barriers
// per block column.  Pivot rules and return value as cholesky.
template <int NT, typename T>
__device__ int smem_potrf(int n, T* S, bool adjust, int* s_flag)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int ld = n + 1;
  T* rcp = S + (size_t)n * ld;  // reciprocals of the current diagonal block
  for (int kb = 0; kb < n; kb += NB) {
    const int bs = min(NB, n - kb);
    T* Dg = S + kb * (ld + 1);
    if (wid == 0) {
      const int fail = warp_potrf32<T>(bs, Dg, adjust, kb, ld);
      if (lane == 0) *s_flag = fail;
      if (!fail && lane < bs) rcp[lane] = (T)1 / Dg[lane + ld * lane];
    }
    __syncthreads();
    const int f = *s_flag;
    if (f) { __syncthreads(); return f; }
    const int r0 = kb + bs, rem = n - r0;
    if (rem <= 0) break;
    // panel: S[r, kb:kb+bs] := S[r, kb:kb+bs] L_bb^{-T}, four rows per warp
    for (int rb = r0 + 4 * wid; rb < n; rb += 4 * (NT / 32)) {
      T x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) x[u] = (lane < bs && rb + u < n) ? S[(rb + u) + ld * (kb + lane)] : (T)0;
      for (int c = 0; c < bs; ++c) {
        const T dinv = rcp[c];
        const T lc = (lane > c && lane < bs) ? Dg[lane + ld * c] : (T)0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (lane == c) x[u] *= dinv;
          const T xc = __shfl_sync(0xffffffffu, x[u], c);
          x[u] -= xc * lc;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (lane < bs && rb + u < n) S[(rb + u) + ld * (kb + lane)] = x[u];
    }
    __syncthreads();
    // trailing: S22 -= P P^T on and below the diagonal, P = S[r0:, kb:kb+bs],
    // in 2 x 2 tiles (tile rows I >= tile columns J)
    const int T2 = (rem + 1) / 2;
    const int ntile = T2 * (T2 + 1) / 2;
    for (int q = tid; q < ntile; q += NT) {
      int I = (int)((sqrtf(8.0f * (float)q + 1.0f) - 1.0f) * 0.5f);
      while ((I + 1) * (I + 2) / 2 <= q) ++I;
      while (I * (I + 1) / 2 > q) --I;
      const int J = q - I * (I + 1) / 2;
      const int i0 = r0 + 2 * I, j0 = r0 + 2 * J;
      const bool i1ok = i0 + 1 < n, j1ok = j0 + 1 < n;
      T s00 = 0, s01 = 0, s10 = 0, s11 = 0;
      const T* P = S + ld * kb;
      for (int k = 0; k < bs; ++k) {
        const T a0 = P[i0 + ld * k], a1 = i1ok ? P[i0 + 1 + ld * k] : (T)0;
        const T b0 = P[j0 + ld * k], b1 = j1ok ? P[j0 + 1 + ld * k] : (T)0;
        s00 += a0 * b0;
        s01 += a0 * b1;
        s10 += a1 * b0;
        s11 += a1 * b1;
      }
      S[i0 + ld * j0] -= s00;
      if (i1ok) S[i0 + 1 + ld * j0] -= s10;
      if (j1ok && i0 >= j0 + 1) S[i0 + ld * (j0 + 1)] -= s01;
      if (i1ok && j1ok) S[i0 + 1 + ld * (j0 + 1)] -= s11;
    }
    __syncthreads();
  }
  return 0;
}

// Lower Cholesky of an n x n matrix factored entirely in shared memory: the
// lower triangle of A (type TA) is loaded once into S, factored in place
// (smem_potrf), and the factor is stored to the lower triangle of Out (type
// T); no global traffic between the load and the store.  Pivot rules,
// return value and failure behaviour as cholesky (Out is then not written).
// S: cholesky_smem_elems(n) elements of T.
template <int NT, typename T, typename TA>
__device__ int cholesky_smem(int n, const TA* A, int lda, T* Out, int ldo, bool adjust, T* S, int* s_flag)
{
  smem_load_lower<NT, T, TA>(n, A, lda, S);
  const int f = smem_potrf<NT, T>(n, S, adjust, s_flag);
  if (f) return f;
  smem_store_lower<NT, T>(n, S, Out, ldo, false);
  return 0;
}

// In-place lower Cholesky, right-looking, blocked by 32, pivot rules as
// warp_potrf32.  Returns 0 on success, else the failing column + 1.  The
// strict upper triangle is zeroed on success when zero_upper is set (callers
// that only read the lower triangle skip that pass).  sD: SD_DOUBLES
// elements of T; smem: GEMM staging.
template <int NT, typename T>
__device__ int cholesky(int n, T* A, int lda, bool adjust, T* sD, void* smem, int* s_flag, bool zero_upper = true)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int kb = 0; kb < n; kb += NB) {
    const int bs = min(NB, n - kb);
    // (a) diagonal block: staged by all threads, factored by warp 0
    for (int t = tid; t < NB * NB; t += NT) {
      const int r = t % NB, c = t / NB;
      if (r < bs && c <= r) sD[r + LDD * c] = A[(kb + r) + (size_t)lda * (kb + c)];
    }
    __syncthreads();
    if (wid == 0) {
      const int fail = warp_potrf32<T>(bs, sD, adjust, kb);
      if (lane == 0) *s_flag = fail;
      if (!fail && lane < bs) sD[NB * LDD + lane] = (T)1 / sD[lane + LDD * lane];
    }
    __syncthreads();
    const int f = *s_flag;
    if (f) { __syncthreads(); return f; }
    for (int t = tid; t < NB * NB; t += NT) {
      const int r = t % NB, c = t / NB;
      if (r < bs && c <= r) A[(kb + r) + (size_t)lda * (kb + c)] = sD[r + LDD * c];
    }
    const int r0 = kb + bs, rem = n - r0;
    if (rem > 0) {
      // (b) panel: A[r, kb:kb+bs] := A[r, kb:kb+bs] L_bb^{-T}; each warp solves
      //     four rows at a time (four independent shuffle chains)
      for (int rb = r0 + 4 * wid; rb < n; rb += 4 * (NT / 32)) {
        T x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          x[u] = (lane < bs && rb + u < n) ? A[(rb + u) + (size_t)lda * (kb + lane)] : (T)0;
        for (int c = 0; c < bs; ++c) {
          const T dinv = sD[NB * LDD + c];
          const T lc = (lane > c && lane < bs) ? sD[lane + LDD * c] : (T)0;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (lane == c) x[u] *= dinv;
            const T xc = __shfl_sync(0xffffffffu, x[u], c);
            x[u] -= xc * lc;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (lane < bs && rb + u < n) A[(rb + u) + (size_t)lda * (kb + lane)] = x[u];
      }
      __syncthreads();
      // (c) trailing: A22 -= P P^T (lower triangle), P = A[r0:, kb:kb+bs]
      const T* P = A + r0 + (size_t)lda * kb;
      gemm_rect<NT, T, T>(rem, rem, bs, false, P, lda, true, P, lda, A + r0 + (size_t)lda * r0, lda, -1.0, 1.0,
                          smem, true, 0);
    }
  }
  if (zero_upper) {
    for (int t = tid; t < n * n; t += NT) {
      const int i = t % n, k = t / n;
      if (i < k) A[i + (size_t)lda * k] = (T)0;
    }
    __syncthreads();
  }
  return 0;
}

// Li = L^{-1} for lower-triangular L: solves L Li = I blocked by 32
// (diagonal block substitution four columns per warp, trailing GEMM update).
// Li must not alias L.
template <int NT, typename T>
__device__ void tri_inverse(int n, const T* L, int ldl, T* Li, int ldi, T* sD, void* smem)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int t = tid; t < n * n; t += NT) {
    const int i = t % n, j = t / n;
    Li[i + (size_t)ldi * j] = (i == j) ? (T)1 : (T)0;
  }
  for (int kb = 0; kb < n; kb += NB) {
    const int bs = min(NB, n - kb);
    for (int t = tid; t < NB * NB; t += NT) {
      const int r = t % NB, c = t / NB;
      if (r < bs && c <= r) sD[r + LDD * c] = L[(kb + r) + (size_t)ldl * (kb + c)];
    }
    for (int r = tid; r < bs; r += NT) sD[NB * LDD + r] = (T)1 / L[(kb + r) + (size_t)ldl * (kb + r)];
    __syncthreads();
    for (int cb = 4 * wid; cb < kb + bs; cb += 4 * (NT / 32)) {
      T x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        x[u] = (lane < bs && cb + u < kb + bs) ? Li[(kb + lane) + (size_t)ldi * (cb + u)] : (T)0;
      for (int p = 0; p < bs; ++p) {
        const T dinv = sD[NB * LDD + p];
        const T lp = (lane > p && lane < bs) ? sD[lane + LDD * p] : (T)0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (lane == p) x[u] *= dinv;
          const T xp = __shfl_sync(0xffffffffu, x[u], p);
          x[u] -= lp * xp;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (lane < bs && cb + u < kb + bs) Li[(kb + lane) + (size_t)ldi * (cb + u)] = x[u];
    }
    __syncthreads();
    const int r0 = kb + bs, rem = n - r0;
    if (rem > 0)
      gemm_rect<NT, T, T>(rem, kb + bs, bs, false, L + r0 + (size_t)ldl * kb, ldl, false, Li + kb, ldi, Li + r0,
                          ldi, -1.0, 1.0, smem);
  }
  __syncthreads();
}

// Two independent Cholesky factorisations (LAPACK pivot rule, as cholesky
// with adjust = false) in lockstep: the diagonal blocks of A0 and A1 are
// factored concurrently by warps 0 and 1, the panels share one barrier, and
// the trailing updates follow each other.  Used for X and Z in the update
// step.  sD0, sD1: SD_DOUBLES elements of T each.  Returns 0 when both
// succeed, else nonzero (both matrices are then left partially factored).
// The strict upper triangles are zeroed when zero_upper is set.
template <int NT, typename T>
__device__ int cholesky_pair(int n, T* A0, T* A1, int lda, T* sD0, T* sD1, void* smem, int* s_flag2,
                             bool zero_upper = true)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  T* Am[2] = {A0, A1};
  T* sDm[2] = {sD0, sD1};
  for (int kb = 0; kb < n; kb += NB) {
    const int bs = min(NB, n - kb);
    for (int t = tid; t < 2 * NB * NB; t += NT) {
      const int mtx = t / (NB * NB), u = t % (NB * NB);
      const int r = u % NB, c = u / NB;
      if (r < bs && c <= r) sDm[mtx][r + LDD * c] = Am[mtx][(kb + r) + (size_t)lda * (kb + c)];
    }
    __syncthreads();
    if (wid < 2) {
      T* sD = sDm[wid];
      const int fail = warp_potrf32<T>(bs, sD, false, kb);
      if (lane == 0) s_flag2[wid] = fail;
      if (!fail && lane < bs) sD[NB * LDD + lane] = (T)1 / sD[lane + LDD * lane];
    }
    __syncthreads();
    const int f = s_flag2[0] | s_flag2[1];
    if (f) { __syncthreads(); return 1; }
    for (int t = tid; t < 2 * NB * NB; t += NT) {
      const int mtx = t / (NB * NB), u = t % (NB * NB);
      const int r = u % NB, c = u / NB;
      if (r < bs && c <= r) Am[mtx][(kb + r) + (size_t)lda * (kb + c)] = sDm[mtx][r + LDD * c];
    }
    const int r0 = kb + bs, rem = n - r0;
    if (rem > 0) {
      // panels of both matrices: A[r, kb:kb+bs] := A[r, kb:kb+bs] L_bb^{-T},
      // four rows per warp at a time
      const int rows4 = (rem + 3) / 4;
      for (int job = wid; job < 2 * rows4; job += NT / 32) {
        const int mtx = job / rows4, rb = r0 + 4 * (job % rows4);
        T* A = Am[mtx];
        const T* sD = sDm[mtx];
        T x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          x[u] = (lane < bs && rb + u < n) ? A[(rb + u) + (size_t)lda * (kb + lane)] : (T)0;
        for (int c = 0; c < bs; ++c) {
          const T dinv = sD[NB * LDD + c];
          const T lc = (lane > c && lane < bs) ? sD[lane + LDD * c] : (T)0;
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (lane == c) x[u] *= dinv;
            const T xc = __shfl_sync(0xffffffffu, x[u], c);
            x[u] -= xc * lc;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (lane < bs && rb + u < n) A[(rb + u) + (size_t)lda * (kb + lane)] = x[u];
      }
      __syncthreads();
      for (int mtx = 0; mtx < 2; ++mtx) {
        const T* P = Am[mtx] + r0 + (size_t)lda * kb;
        gemm_rect<NT, T, T>(rem, rem, bs, false, P, lda, true, P, lda, Am[mtx] + r0 + (size_t)lda * r0, lda, -1.0,
                            1.0, smem, true, 0);
      }
    }
  }
  if (zero_upper) {
    for (int t = tid; t < 2 * n * n; t += NT) {
      const int mtx = t / (n * n), u = t % (n * n);
      const int i = u % n, k = u / n;
      if (i < k) Am[mtx][i + (size_t)lda * k] = (T)0;
    }
    __syncthreads();
  }
  return 0;
}

// Li0 = L0^{-1} and Li1 = L1^{-1} in lockstep (tri_inverse for two lower
// triangles): one staging barrier and one substitution barrier per block
// column for both.  Li must not alias L.
template <int NT, typename T>
__device__ void tri_inverse_pair(int n, const T* L0, const T* L1, int ldl, T* Li0, T* Li1, int ldi, T* sD0, T* sD1,
                                 void* smem)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const T* Lm[2] = {L0, L1};
  T* Lim[2] = {Li0, Li1};
  T* sDm[2] = {sD0, sD1};
  for (int t = tid; t < 2 * n * n; t += NT) {
    const int mtx = t / (n * n), u = t % (n * n);
    const int i = u % n, j = u / n;
    Lim[mtx][i + (size_t)ldi * j] = (i == j) ? (T)1 : (T)0;
  }
  for (int kb = 0; kb < n; kb += NB) {
    const int bs = min(NB, n - kb);
    for (int t = tid; t < 2 * NB * NB; t += NT) {
      const int mtx = t / (NB * NB), u = t % (NB * NB);
      const int r = u % NB, c = u / NB;
      if (r < bs && c <= r) sDm[mtx][r + LDD * c] = Lm[mtx][(kb + r) + (size_t)ldl * (kb + c)];
    }
    for (int t = tid; t < 2 * NB; t += NT) {
      const int mtx = t / NB, r = t % NB;
      if (r < bs) sDm[mtx][NB * LDD + r] = (T)1 / Lm[mtx][(kb + r) + (size_t)ldl * (kb + r)];
    }
    __syncthreads();
    const int cols4 = (kb + bs + 3) / 4;
    for (int job = wid; job < 2 * cols4; job += NT / 32) {
      const int mtx = job / cols4, cb = 4 * (job % cols4);
      T* Li = Lim[mtx];
      const T* sD = sDm[mtx];
      T x[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        x[u] = (lane < bs && cb + u < kb + bs) ? Li[(kb + lane) + (size_t)ldi * (cb + u)] : (T)0;
      for (int p = 0; p < bs; ++p) {
        const T dinv = sD[NB * LDD + p];
        const T lp = (lane > p && lane < bs) ? sD[lane + LDD * p] : (T)0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (lane == p) x[u] *= dinv;
          const T xp = __shfl_sync(0xffffffffu, x[u], p);
          x[u] -= lp * xp;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (lane < bs && cb + u < kb + bs) Li[(kb + lane) + (size_t)ldi * (cb + u)] = x[u];
    }
    __syncthreads();
    const int r0 = kb + bs, rem = n - r0;
    if (rem > 0)
      for (int mtx = 0; mtx < 2; ++mtx)
        gemm_rect<NT, T, T>(rem, kb + bs, bs, false, Lm[mtx] + r0 + (size_t)ldl * kb, ldl, false, Lim[mtx] + kb,
                            ldi, Lim[mtx] + r0, ldi, -1.0, 1.0, smem);
  }
  __syncthreads();
}

// x = L^{-T} L^{-1} x for a Cholesky factor L (lower).  Blocked by 32: each
// diagonal block is staged in shared memory by all threads and solved by
// warp 0 with shuffles; the other rows are updated block-wide.
// sD: SD_DOUBLES elements of T.
template <int NT, typename T>
__device__ void chol_solve(int n, const T* L, int ldl, T* x, T* sD)
{
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  auto stage = [&](int kb, int bs) {
    for (int t = tid; t < NB * NB; t += NT) {
      const int r = t % NB, c = t / NB;
      if (r < bs && c <= r) sD[r + LDD * c] = L[(kb + r) + (size_t)ldl * (kb + c)];
    }
    for (int r = tid; r < bs; r += NT) sD[NB * LDD + r] = (T)1 / L[(kb + r) + (size_t)ldl * (kb + r)];
    __syncthreads();
  };
  for (int kb = 0; kb < n; kb += NB) {
    const int bs = min(NB, n - kb);
    stage(kb, bs);
    if (wid == 0) {
      T v = (lane < bs) ? x[kb + lane] : (T)0;
      for (int p = 0; p < bs; ++p) {
        if (lane == p) v *= sD[NB * LDD + p];
        const T vp = __shfl_sync(0xffffffffu, v, p);
        if (lane > p && lane < bs) v -= sD[lane + LDD * p] * vp;
      }
      if (lane < bs) x[kb + lane] = v;
    }
    __syncthreads();
    for (int i = kb + bs + tid; i < n; i += NT) {
      T s = (T)0;
#pragma unroll 8
      for (int p = 0; p < bs; ++p) s += L[i + (size_t)ldl * (kb + p)] * x[kb + p];
      x[i] -= s;
    }
    __syncthreads();
  }
  const int nblk = (n + NB - 1) / NB;
  for (int b = nblk - 1; b >= 0; --b) {
    const int kb = b * NB, bs = min(NB, n - kb);
    stage(kb, bs);
    if (wid == 0) {
      T v = (lane < bs) ? x[kb + lane] : (T)0;
      for (int p = bs - 1; p >= 0; --p) {
        if (lane == p) v *= sD[NB * LDD + p];
        const T vp = __shfl_sync(0xffffffffu, v, p);
        if (lane < p) v -= sD[p + LDD * lane] * vp;
      }
      if (lane < bs) x[kb + lane] = v;
    }
    __syncthreads();
    for (int i = wid; i < kb; i += NT / 32) {
      T s = (lane < bs) ? L[(kb + lane) + (size_t)ldl * i] * x[kb + lane] : (T)0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) x[i] -= s;
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------ eigenvalues
// Number of eigenvalues < x of a symmetric tridiagonal of order k given as
// its diagonal ds and squared off-diagonal e2 (e2[i] couples i and i+1),
// scaled so that every entry is at most 1 in magnitude: sign changes of the
// leading principal minors p_i(x) of T - xI (Sturm sequence), by the
// division-free recurrence p_{i+1} = (d_i - x) p_i - e_{i-1}^2 p_{i-1}.
// With the scaling a minor grows at most 5x per step for x inside the
// Gershgorin interval, so the pair is checked for rescaling every 8 steps
// only; sign changes are counted from the sign bits.
__device__ __forceinline__ int sturm_count(int k, const double* ds, const double* e2, double x)
{
  double pm = 1.0, p = ds[0] - x;
  int cnt = (p < 0.0) ? 1 : 0;
  for (int i = 1; i < k; ++i) {
    double pn = fma(ds[i] - x, p, -e2[i - 1] * pm);
    if (pn == 0.0) pn = (p < 0.0) ? 1.0e-300 : -1.0e-300;  // a zero minor counts as a sign change
    cnt += (int)(((unsigned)__double2hiint(pn) ^ (unsigned)__double2hiint(p)) >> 31);
    pm = p;
    p = pn;
    if ((i & 7) == 0) {
      const double big = fmax(fabs(p), fabs(pm));
      if (big > 1.0e100 || big < 1.0e-100) {
        const int ex = ilogb(big);
        p = scalbn(p, -ex);
        pm = scalbn(pm, -ex);
      }
    }
  }
  return cnt;
}

// Smallest eigenvalue of a symmetric tridiagonal (d, e) of order k <= 64,
// and the magnitude of the last component of its unit eigenvector (the
// Lanczos error estimate).
// * The matrix is scaled by its Gershgorin radius (lane-parallel bounds)
//   into `work` (2 * 64 doubles: diagonal, squared off-diagonal).
// * Warp multisection (33 points per round) until the bracket is narrow,
//   then Newton steps on f(x) = det(T - xI), whose smallest root is
//   approached monotonically from the left; each step is kept inside the
//   bracket, until the step is below one ulp of the result (or of 1e-2 of
//   the matrix scale for a result near zero).
// * The eigenvector component comes from the same recurrences: for an
//   eigenvalue lam of an unreduced tridiagonal,
//   u_k^2 = -P_{k-1}(lam) / P_k'(lam), with P_j the leading principal minors
//   of T - lam I, which Newton has just evaluated.
// * `upper` is a known upper bound of the result (the smallest Ritz value of
//   a leading principal submatrix, by interlacing; 1e300 for none).  The
//   first round then probes geometrically spaced points below it, which
//   brackets the value in one round when it has moved little.
// Called by one full warp; every lane returns the same values.
static __device__ double tridiag_min_eig_warp(int k, const double* d, const double* e, double upper,
                                              double* ulast, double* work)
{
  const int lane = threadIdx.x & 31;
  // Gershgorin interval, lane-parallel (k <= 64: two entries per lane)
  double lo = 1.0e300, hi = -1.0e300;
  for (int i = lane; i < k; i += 32) {
    const double r = ((i > 0) ? fabs(e[i - 1]) : 0.0) + ((i < k - 1) ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const double sc = fmax(fabs(lo), fabs(hi));
  if (!(sc > 0.0)) {  // the zero matrix
    *ulast = (k > 1) ? 0.0 : 1.0;
    return 0.0;
  }
  const double inv = 1.0 / sc;
  double* ds = work;
  double* e2 = work + 64;
  for (int i = lane; i < k; i += 32) {
    ds[i] = d[i] * inv;
    const double es = (i < k - 1) ? e[i] * inv : 0.0;
    e2[i] = es * es;
  }
  __syncwarp();
  lo = lo * inv - 1.0e-15;  // |lo|, |hi| <= 1 after scaling
  hi = hi * inv + 1.0e-15;
  const double up = upper * inv;
  if (up < hi && up > lo) {
    // probes p_0 = up + h (above the value), p_l = up + h - h 4^l
    const double h = 1.0e-12 * fmax(fabs(up), 1.0e-3) + 1.0e-300;
    const double x = (lane == 0) ? up + h : up + h - h * exp2(2.0 * lane);
    const bool below = (x > lo) && sturm_count(k, ds, e2, x) >= 1;
    const unsigned ball = __ballot_sync(0xffffffffu, below);
    if (ball & 1u) {  // the bound holds: bracket between the last probe with
                      // an eigenvalue below it and the next one
      const int f = (ball == 0xffffffffu) ? 32 : __ffs(~ball) - 1;  // first probe without (32: none)
      const double xhi = __shfl_sync(0xffffffffu, x, (f > 0 && f < 32) ? f - 1 : 31);
      const double xlo = __shfl_sync(0xffffffffu, x, (f < 32) ? f : 31);
      hi = fmin(hi, xhi);
      if (f < 32) lo = fmax(lo, xlo);
    }
  }
  for (int round = 0; round < 24; ++round) {
    if (hi - lo <= 1.0e-7 * fmax(fabs(lo), fabs(hi)) + 1.0e-12) break;
    const double w = (hi - lo) / 33.0;
    const double x = lo + w * (lane + 1);
    const int c = sturm_count(k, ds, e2, x);
    const unsigned ball = __ballot_sync(0xffffffffu, c >= 1);
    const int f = ball ? (__ffs(ball) - 1) : 32;  // first point with an eigenvalue below it
    const double nlo = lo + w * f;
    const double nhi = (f < 32) ? lo + w * (f + 1) : hi;
    lo = nlo;
    hi = nhi;
  }
  // Newton on f(x) = det(T - xI) from the left end of the bracket, with
  // P_{i+1} = (d_i - x) P_i - e^2 P_{i-1} and its derivative
  // D_{i+1} = -P_i + (d_i - x) D_i - e^2 D_{i-1}, rescaled together.
  double x = lo, Plast = 0.0, Dlast = 0.0;
  for (int it = 0; it < 20; ++it) {
    double Pm = 1.0, P = ds[0] - x, Dm = 0.0, Dv = -1.0;
    for (int i = 1; i < k; ++i) {
      const double dx = ds[i] - x, ee = e2[i - 1];
      const double Pn = fma(dx, P, -ee * Pm);
      const double Dn = fma(dx, Dv, -fma(ee, Dm, P));
      Pm = P; P = Pn; Dm = Dv; Dv = Dn;
      if ((i & 7) == 0) {
        const double big = fmax(fmax(fabs(P), fabs(Dv)), fmax(fabs(Pm), fabs(Dm)));
        if (big > 1.0e100 || big < 1.0e-100) {
          const int ex = ilogb(big);
          P = scalbn(P, -ex); Pm = scalbn(Pm, -ex); Dv = scalbn(Dv, -ex); Dm = scalbn(Dm, -ex);
        }
      }
    }
    Plast = Pm;  // P_{k-1}(x) and P_k'(x), same scale
    Dlast = Dv;
    if (!(Dv != 0.0) || P != P || Dv != Dv) break;
    const double xn = x - P / Dv;
    if (!(xn >= lo) || !(xn <= hi)) break;
    if (fabs(xn - x) <= fmax(2.2e-16 * fabs(xn), 2.2e-18)) { x = xn; break; }
    x = xn;
  }
  double u2 = 1.0;
  if (k > 1) {
    u2 = (Dlast != 0.0) ? -Plast / Dlast : 1.0;
    if (!(u2 >= 0.0)) u2 = 0.0;  // rounding (or NaN) below zero
    if (u2 > 1.0) u2 = 1.0;
  }
  *ulast = sqrt(u2);
  return x * sc;
}

}  // namespace cta
}  // namespace sdpab
