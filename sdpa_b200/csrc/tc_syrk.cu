// Tensor-core (tcgen05) symmetric rank-k update for the FP32 Schur
// factorisation of the mixed-precision path: C -= P P^T on the lower
// triangle of an M x M FP32 matrix, P M x K (K <= a Cholesky panel), both
// column-major.  This is the trailing update of the right-looking blocked
// Cholesky (rATL_dpotrfL's dsyrk step, sdpa_dpotrf.cpp:218-265), the bulk of
// the Schur factorisation's work for large m.
//
// FP32 accuracy from TF32 tensor cores: each operand is split as
// a = hi + lo with hi = tf32(a) and lo = tf32(a - hi), and
// P P^T = Phi Phi^T + Phi Plo^T + Plo Phi^T (+ Plo Plo^T, 2^-22 relative,
// dropped), all accumulated in FP32 in tensor memory.  The factor is then
// refined in FP64 by the caller, as for the SIMT FP32 factor.
//
// The same split-TF32 pipeline also forms the mixed-precision F1 products
// of the Schur assembly, G_q = T_q Z^-1 for a chunk of constraints
// (k_gemm_tf32x3, FP64 in and out).
//
// Two kernels for the update:
//  * k_split_tf32 writes P's hi and lo parts once per panel, already in the
//    MMA's shared-memory layout: for every 128-row block and 16-wide K chunk
//    an 8 KB tile in the canonical K-major no-swizzle layout (8-row x
//    16-byte core matrices; core (row group g, K group q) at byte
//    (q * 16 + g) * 128), hi and lo tiles side by side;
//  * k_syrk_tf32x3: one 128-thread block per 128 x 128 tile of the lower
//    triangle.  Thread 0 streams the four operand tiles of a K chunk into
//    one of two shared-memory stages (64 KB in all, so that three blocks
//    share an SM) with bulk asynchronous copies that complete on the
//    stage's "full" mbarrier, issues 3 x 2 MMAs
//    (M = N = 128, K = 8 each) into a 128-column FP32 accumulator in tensor
//    memory and commits them to the stage's "empty" mbarrier; once chunk
//    k-1's MMAs are done its stage is refilled with chunk k+1 while chunk
//    k's MMAs run.  The four warps then read the
//    accumulator (warp w: lanes 32w..32w+31 = tile rows) and update C,
//    16 columns per round of loads.
// Every wait is bounded: on time-out the block records an error, waits
// (bounded) for the MMAs it committed, frees its tensor memory and skips the
// update; the caller then falls back.
#include <cuda_runtime.h>
#include <stdint.h>

#include "sdpa_b200.h"
#include "sdpab_internal.h"

namespace sdpab {
namespace tc {

constexpr int TILE = 128;        // M = N of the MMA and of a block's tile
constexpr int KC = 16;           // K per stage
constexpr int THREADS = 128;
constexpr int OPER_BYTES = TILE * KC * 4;          // one operand tile (8 KB)
constexpr int OPER_WORDS = OPER_BYTES / 4;
constexpr int STAGE_BYTES = 4 * OPER_BYTES;        // A_hi, A_lo, B_hi, B_lo
constexpr int SMEM_BYTES = 2 * STAGE_BYTES + 128;  // two stages + barriers + TMEM address
constexpr uint32_t TMEM_COLS = 128;
constexpr long long WAIT_LIMIT = 1LL << 22;        // mbarrier polls before giving up

// Instruction descriptor: D F32, A and B TF32, both K-major, N = 128, M = 128.
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TILE >> 3) << 17) |
                           ((uint32_t)(TILE >> 4) << 24);

__host__ __device__ inline long long split_words(int M, int K)
{
  const long long T = (M + TILE - 1) / TILE, nk = (K + KC - 1) / KC;
  return T * nk * 2 * OPER_WORDS;
}

// Shared-memory matrix descriptor, canonical K-major layout without swizzle:
// start address, leading byte offset (between the two 16-byte K halves of an
// MMA), stride byte offset (between 8-row core groups), version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ uint32_t to_tf32(float a)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return r;
}

// Polls an mbarrier phase at most `limit` times (limit <= 0: none); true once
// the phase has completed.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = WAIT_LIMIT)
{
  for (long long it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
      "l"(da), "l"(db), "r"(IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

// P (M x K) -> hi / lo TF32 tiles in the MMA layout (zero outside M x K).
// One thread per (row, group of four K values); consecutive threads take
// consecutive rows, so the loads of P are coalesced.
__global__ void k_split_tf32(int M, int K, const float* __restrict__ P, int ldp, uint32_t* __restrict__ S)
{
  const int T = (M + TILE - 1) / TILE, nk = (K + KC - 1) / KC;
  const long long rows = (long long)T * TILE;
  const long long n = rows * nk * (KC / 4);
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= n) return;
  const int row = (int)(id % rows);
  const int qq = (int)(id / rows);  // K group of four, over all chunks
  const int b = row / TILE, t = row % TILE, c = qq / (KC / 4), q = qq % (KC / 4);
  uint32_t h[4], l[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int k = c * KC + 4 * q + u;
    const float a = (row < M && k < K) ? P[row + (size_t)ldp * k] : 0.0f;
    h[u] = to_tf32(a);
    l[u] = to_tf32(a - __uint_as_float(h[u]));
  }
  uint32_t* base = S + ((size_t)b * nk + c) * 2 * OPER_WORDS;
  const int w = (q * (TILE / 8) + (t >> 3)) * 32 + (t & 7) * 4;  // core (t / 8, q), row t % 8
  *reinterpret_cast<uint4*>(base + w) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(base + OPER_WORDS + w) = make_uint4(l[0], l[1], l[2], l[3]);
}

// Bulk asynchronous global -> shared copy (no multicast) completing on an
// mbarrier's transaction count.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// The MMA pipeline shared by the kernels below.  Shared memory: two stages
// of four operand tiles (A_hi, A_lo, B_hi, B_lo), then the full[2] and
// empty[2] mbarriers, the tensor-memory address and two state words.
struct Pipe {
  uint32_t full[2], empty[2];
  uint32_t tmem;
  int* state;  // [0] ok, [1] last committed chunk
};

// Barrier initialisation and the 128-column tensor-memory allocation (warp 0).
__device__ __forceinline__ Pipe pipe_open(unsigned char* smem)
{
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * STAGE_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem + 2 * STAGE_BYTES + 64);
  Pipe p;
  p.state = reinterpret_cast<int*>(smem + 2 * STAGE_BYTES + 80);
  for (int s = 0; s < 2; ++s) {
    p.full[s] = (uint32_t)__cvta_generic_to_shared(&bars[s]);
    p.empty[s] = (uint32_t)__cvta_generic_to_shared(&bars[2 + s]);
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < 2; ++s) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(p.full[s]), "r"(1));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(p.empty[s]), "r"(1));
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    p.state[0] = 1;
    p.state[1] = -1;
  }
  if ((threadIdx.x >> 5) == 0) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst), "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  p.tmem = *tmem_slot;
  return p;
}

// Thread 0: streams the nk chunks of the A row block `a` and the B row block
// `b` (hi and lo tiles adjacent per chunk) through the two stages and issues
// 3 x 2 MMAs per chunk into the accumulator; a stage is refilled with chunk
// k+1 once chunk k-1's MMAs have completed.  Every wait is bounded: the
// waits that advance the pipeline give up after `limit` polls (the caller's
// choice; WAIT_LIMIT in normal use, small in the tests of the fall-back),
// the waits that drain copies still in flight after giving up use
// WAIT_LIMIT, so the block's shared memory is quiet when it is released.
__device__ __forceinline__ void pipe_issue(const Pipe& p, unsigned char* smem, const uint32_t* a, const uint32_t* b,
                                           int nk, long long limit)
{
  const uint32_t st0 = (uint32_t)__cvta_generic_to_shared(smem);
  auto load_stage = [&](int s, int c) {
    const uint32_t dst = st0 + (uint32_t)(s * STAGE_BYTES);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(p.full[s]), "r"(STAGE_BYTES)
                 : "memory");
    bulk_load(dst, a + (size_t)c * 2 * OPER_WORDS, 2 * OPER_BYTES, p.full[s]);
    bulk_load(dst + 2 * OPER_BYTES, b + (size_t)c * 2 * OPER_WORDS, 2 * OPER_BYTES, p.full[s]);
  };
  bool ok = true;
  int committed = -1;
  int in_flight[2] = {-1, -1};  // chunk being copied into each stage (not yet waited for)
  for (int s = 0; s < 2 && s < nk; ++s) {
    load_stage(s, s);
    in_flight[s] = s;
  }
  for (int kc = 0; kc < nk && ok; ++kc) {
    const int s = kc & 1;
    ok = mbar_wait(p.full[s], (kc >> 1) & 1, limit);
    if (!ok) break;
    in_flight[s] = -1;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t base = st0 + (uint32_t)(s * STAGE_BYTES);
    const uint32_t lbo = (TILE / 8) * 128, sbo = 128;
#pragma unroll
    for (int j = 0; j < KC / 8; ++j) {
      const uint32_t off = (uint32_t)j * 2 * (TILE / 8) * 128;  // two K groups of 4 per MMA
      const uint64_t ahi = smem_desc(base + off, lbo, sbo);
      const uint64_t alo = smem_desc(base + OPER_BYTES + off, lbo, sbo);
      const uint64_t bhi = smem_desc(base + 2 * OPER_BYTES + off, lbo, sbo);
      const uint64_t blo = smem_desc(base + 3 * OPER_BYTES + off, lbo, sbo);
      mma_tf32(p.tmem, ahi, bhi, (kc > 0 || j > 0) ? 1u : 0u);
      mma_tf32(p.tmem, ahi, blo, 1u);
      mma_tf32(p.tmem, alo, bhi, 1u);
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(p.empty[s])
                 : "memory");
    committed = kc;
    // refill the stage of chunk kc-1 with chunk kc+1 once its MMAs are done
    // (chunk kc's MMAs keep the tensor cores busy meanwhile)
    if (kc >= 1 && kc + 1 < nk) {
      const int sp = (kc - 1) & 1;
      ok = mbar_wait(p.empty[sp], ((kc - 1) >> 1) & 1, limit);
      if (ok) {
        load_stage(sp, kc + 1);
        in_flight[sp] = kc + 1;
      }
    }
  }
  if (!ok)  // let copies still in flight land before the block's shared memory is released
    for (int s2 = 0; s2 < 2; ++s2)
      if (in_flight[s2] >= 0) (void)mbar_wait(p.full[s2], (in_flight[s2] >> 1) & 1);
  p.state[0] = ok ? 1 : 0;
  p.state[1] = committed;
}

// All threads: true when every chunk's MMAs completed (the last commit
// completes after all of them, and is waited for with WAIT_LIMIT also after
// a give-up, so no MMA still writes the accumulator when it is freed); on
// failure the error flag is set.
__device__ __forceinline__ bool pipe_wait(const Pipe& p, int nk, int* err)
{
  __syncthreads();
  const int last = p.state[1];
  bool ok = p.state[0] != 0 && last == nk - 1;
  if (last >= 0) ok = (__syncthreads_and(mbar_wait(p.empty[last & 1], (last >> 1) & 1)) != 0) && ok;
  if (!ok && threadIdx.x == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  return ok;
}

// Accumulator columns 16 grp .. 16 grp + 15 of this thread's row (warp w
// reads tile rows 32 w .. 32 w + 31).
__device__ __forceinline__ void tmem_row16(uint32_t tmem, int grp, uint32_t* v)
{
  const int wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const uint32_t taddr = tmem + ((uint32_t)(32 * wid) << 16) + (uint32_t)(16 * grp + 8 * j);
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[8 * j + 0]), "=r"(v[8 * j + 1]), "=r"(v[8 * j + 2]), "=r"(v[8 * j + 3]),
                   "=r"(v[8 * j + 4]), "=r"(v[8 * j + 5]), "=r"(v[8 * j + 6]), "=r"(v[8 * j + 7])
                 : "r"(taddr));
  }
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void pipe_close(const Pipe& p)
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(p.tmem), "r"(TMEM_COLS));
}

__global__ void __launch_bounds__(THREADS, 3)
k_syrk_tf32x3(int M, int K, const uint32_t* __restrict__ S, float* __restrict__ C, int ldc, int* err,
              long long limit)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
  // lower-triangular tile (ti >= tj) of this block
  const long long t = blockIdx.x;
  int ti = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
  while ((long long)(ti + 1) * (ti + 2) / 2 <= t) ++ti;
  while ((long long)ti * (ti + 1) / 2 > t) --ti;
  const int tj = (int)(t - (long long)ti * (ti + 1) / 2);
  const int r0 = ti * TILE, c0 = tj * TILE;
  const int nk = (K + KC - 1) / KC;

  const Pipe p = pipe_open(smem);
  if (tid == 0)
    pipe_issue(p, smem, S + (size_t)ti * nk * 2 * OPER_WORDS, S + (size_t)tj * nk * 2 * OPER_WORDS, nk, limit);
  if (pipe_wait(p, nk, err)) {
    const int gr = r0 + 32 * wid + lane;
    for (int grp = 0; grp < TILE / 16; ++grp) {
      float cv[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int gc = c0 + 16 * grp + u;
        cv[u] = (gr < M && gc <= gr) ? C[gr + (size_t)ldc * gc] : 0.0f;
      }
      uint32_t v[16];
      tmem_row16(p.tmem, grp, v);
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int gc = c0 + 16 * grp + u;
        if (gr < M && gc <= gr) C[gr + (size_t)ldc * gc] = cv[u] - __uint_as_float(v[u]);
      }
    }
  }
  pipe_close(p);
}

// FP64 operands (batched: matrix q at P + q sP) -> hi / lo TF32 tiles in the
// MMA layout, split q at S + q * split_words(M, K); the values are first
// rounded to FP32.  Same thread mapping as k_split_tf32.
__global__ void k_split_tf32_f64(int M, int K, const double* __restrict__ P, int ldp, long long sP,
                                 uint32_t* __restrict__ S)
{
  const int T = (M + TILE - 1) / TILE, nk = (K + KC - 1) / KC;
  const long long rows = (long long)T * TILE;
  const long long n = rows * nk * (KC / 4);
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= n) return;
  const double* Pq = P + (size_t)blockIdx.y * sP;
  uint32_t* Sq = S + (size_t)blockIdx.y * split_words(M, K);
  const int row = (int)(id % rows);
  const int qq = (int)(id / rows);
  const int b = row / TILE, t = row % TILE, c = qq / (KC / 4), q = qq % (KC / 4);
  uint32_t h[4], l[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int k = c * KC + 4 * q + u;
    const float a = (row < M && k < K) ? (float)Pq[row + (size_t)ldp * k] : 0.0f;
    h[u] = to_tf32(a);
    l[u] = to_tf32(a - __uint_as_float(h[u]));
  }
  uint32_t* base = Sq + ((size_t)b * nk + c) * 2 * OPER_WORDS;
  const int w = (q * (TILE / 8) + (t >> 3)) * 32 + (t & 7) * 4;
  *reinterpret_cast<uint4*>(base + w) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(base + OPER_WORDS + w) = make_uint4(l[0], l[1], l[2], l[3]);
}

// C_q = A_q B^T (M x N, FP64, column-major, C_q at C + q sC) from split
// operands: A_q (M x K) at Sa + q * split_words(M, K), B (N x K) at Sb,
// shared by the batch.  Block (tile of M x N, q).
__global__ void __launch_bounds__(THREADS, 3)
k_gemm_tf32x3(int M, int N, int K, const uint32_t* __restrict__ Sa, const uint32_t* __restrict__ Sb,
              double* __restrict__ C, int ldc, long long sC, int* err, long long limit)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
  const int TM = (M + TILE - 1) / TILE;
  const int ti = blockIdx.x % TM, tj = blockIdx.x / TM;
  const int r0 = ti * TILE, c0 = tj * TILE;
  const int nk = (K + KC - 1) / KC;
  const uint32_t* a = Sa + (size_t)blockIdx.y * split_words(M, K) + (size_t)ti * nk * 2 * OPER_WORDS;
  const uint32_t* b = Sb + (size_t)tj * nk * 2 * OPER_WORDS;
  double* Cq = C + (size_t)blockIdx.y * sC;

  const Pipe p = pipe_open(smem);
  if (tid == 0) pipe_issue(p, smem, a, b, nk, limit);
  if (pipe_wait(p, nk, err)) {
    const int gr = r0 + 32 * wid + lane;
    for (int grp = 0; grp < TILE / 16; ++grp) {
      uint32_t v[16];
      tmem_row16(p.tmem, grp, v);
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int gc = c0 + 16 * grp + u;
        if (gr < M && gc < N) Cq[gr + (size_t)ldc * gc] = (double)__uint_as_float(v[u]);
      }
    }
  }
  pipe_close(p);
}

}  // namespace tc

long long syrk_tf32x3_work_bytes(int M, int K) { return M > 0 && K > 0 ? tc::split_words(M, K) * 4 : 0; }

long long gemm_tf32x3_work_bytes(int M, int N, int K, int batch)
{
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return 0;
  return ((long long)batch * tc::split_words(M, K) + tc::split_words(N, K)) * 4;
}

// C_q = A_q B^T for q < batch (FP64 in and out, column-major; A_q M x K at
// A + q sA, B N x K shared, C_q at C + q sC), on tensor cores in split TF32
// with FP32 accumulation; `work` holds gemm_tf32x3_work_bytes bytes
// (16-byte aligned).  Returns a CUDA status; *err (device) is set when a
// block timed out waiting.
int gemm_tf32x3(int M, int N, int K, int batch, const double* A, int lda, long long sA, const double* B, int ldb,
                double* C, int ldc, long long sC, void* work, int* err, cudaStream_t st, long long wait_polls)
{
  const long long limit = (wait_polls < 0) ? tc::WAIT_LIMIT : wait_polls;
  if (M <= 0 || N <= 0 || K <= 0 || batch <= 0) return 0;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_per_device((const void*)tc::k_gemm_tf32x3, tc::SMEM_BYTES, attr);
  if (e != cudaSuccess) return (int)e;
  uint32_t* Sa = (uint32_t*)work;
  uint32_t* Sb = Sa + (size_t)batch * tc::split_words(M, K);
  const long long nk = (K + tc::KC - 1) / tc::KC;
  const long long TMt = (M + tc::TILE - 1) / tc::TILE, TNt = (N + tc::TILE - 1) / tc::TILE;
  const long long ta = TMt * tc::TILE * nk * (tc::KC / 4), tb = TNt * tc::TILE * nk * (tc::KC / 4);
  tc::k_split_tf32_f64<<<dim3((unsigned)((ta + 255) / 256), (unsigned)batch), 256, 0, st>>>(M, K, A, lda, sA, Sa);
  tc::k_split_tf32_f64<<<dim3((unsigned)((tb + 255) / 256), 1), 256, 0, st>>>(N, K, B, ldb, 0, Sb);
  tc::k_gemm_tf32x3<<<dim3((unsigned)(TMt * TNt), (unsigned)batch), tc::THREADS, tc::SMEM_BYTES, st>>>(
      M, N, K, Sa, Sb, C, ldc, sC, err, limit);
  return (int)cudaGetLastError();
}

// C -= P P^T on the lower triangle (M x M, FP32), P M x K; `work` holds
// syrk_tf32x3_work_bytes(M, K) bytes (16-byte aligned).  Returns a CUDA
// status; *err (device) is set when a block timed out waiting.
int syrk_tf32x3(int M, int K, const float* P, int ldp, float* C, int ldc, void* work, int* err, cudaStream_t st,
                long long wait_polls)
{
  const long long limit = (wait_polls < 0) ? tc::WAIT_LIMIT : wait_polls;
  if (M <= 0 || K <= 0) return 0;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = smem_attr_per_device((const void*)tc::k_syrk_tf32x3, tc::SMEM_BYTES, attr);
  if (e != cudaSuccess) return (int)e;
  const long long T = (M + tc::TILE - 1) / tc::TILE, nk = (K + tc::KC - 1) / tc::KC;
  const long long threads = T * tc::TILE * nk * (tc::KC / 4);
  tc::k_split_tf32<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(M, K, P, ldp, (uint32_t*)work);
  const long long tiles = T * (T + 1) / 2;
  tc::k_syrk_tf32x3<<<(unsigned)tiles, tc::THREADS, tc::SMEM_BYTES, st>>>(M, K, (const uint32_t*)work, C, ldc,
                                                                          err, limit);
  return (int)cudaGetLastError();
}

}  // namespace sdpab

namespace {
__device__ int g_tc_err;  // time-out flag of the stand-alone entry below
}

extern "C" SDPAB_API long long sdpab_tc_syrk_work_bytes(int M, int K) { return sdpab::syrk_tf32x3_work_bytes(M, K); }

// Stand-alone form (device pointers; no counterpart in the reference): the
// tensor-core update on `stream`, synchronised, with SDPAB_ECUDA when a
// block gave up waiting for its MMAs.  wait_polls < 0: the default bound of
// the pipeline's waits; >= 0: that many polls (a block that runs out leaves
// its tile of C unchanged).
extern "C" SDPAB_API int sdpab_tc_syrk(int M, int K, const float* P, int ldp, float* C, int ldc, void* work,
                                       long long wait_polls, void* stream)
{
  if (M < 0 || K < 0 || !P || !C || !work || ldp < M || ldc < M)
    return sdpab::set_error(SDPAB_EINVAL, "tc_syrk: bad arguments");
  if (((uintptr_t)work & 15) != 0) return sdpab::set_error(SDPAB_EINVAL, "tc_syrk: work must be 16-byte aligned");
  int* err = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void**)&err, g_tc_err);
  if (e != cudaSuccess) return sdpab::cuda_error(e, "tc_syrk: cudaGetSymbolAddress");
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return sdpab::cuda_error(e, "tc_syrk: cudaMemsetAsync");
  const int rc = sdpab::syrk_tf32x3(M, K, P, ldp, C, ldc, work, err, st, wait_polls);
  if (rc != 0) return sdpab::cuda_error((cudaError_t)rc, "tc_syrk: launch");
  int h = 0;
  e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return sdpab::cuda_error(e, "tc_syrk");
  return h ? sdpab::set_error(SDPAB_ECUDA, "tc_syrk: a block timed out waiting for its MMAs") : SDPAB_OK;
}

extern "C" SDPAB_API long long sdpab_tc_gemm_work_bytes(int M, int N, int K, int batch)
{
  return sdpab::gemm_tf32x3_work_bytes(M, N, K, batch);
}

// Stand-alone form of the F1 product kernel (device pointers; no counterpart
// in the reference, whose F1 products are dgemm calls, sdpa_newton.cpp:
// 885-889): C_q = A_q B^T on `stream`, synchronised, SDPAB_ECUDA when a block
// gave up waiting for its MMAs (wait_polls as for sdpab_tc_syrk).
extern "C" SDPAB_API int sdpab_tc_gemm(int M, int N, int K, int batch, const double* A, int lda, long long sA,
                                       const double* B, int ldb, double* C, int ldc, long long sC, void* work,
                                       long long wait_polls, void* stream)
{
  if (M < 0 || N < 0 || K < 0 || batch < 0 || !A || !B || !C || !work || lda < M || ldb < N || ldc < M)
    return sdpab::set_error(SDPAB_EINVAL, "tc_gemm: bad arguments");
  if (((uintptr_t)work & 15) != 0) return sdpab::set_error(SDPAB_EINVAL, "tc_gemm: work must be 16-byte aligned");
  int* err = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void**)&err, g_tc_err);
  if (e != cudaSuccess) return sdpab::cuda_error(e, "tc_gemm: cudaGetSymbolAddress");
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemsetAsync(err, 0, sizeof(int), st);
  if (e != cudaSuccess) return sdpab::cuda_error(e, "tc_gemm: cudaMemsetAsync");
  const int rc = sdpab::gemm_tf32x3(M, N, K, batch, A, lda, sA, B, ldb, C, ldc, sC, work, err, st, wait_polls);
  if (rc != 0) return sdpab::cuda_error((cudaError_t)rc, "tc_gemm: launch");
  int h = 0;
  e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return sdpab::cuda_error(e, "tc_gemm");
  return h ? sdpab::set_error(SDPAB_ECUDA, "tc_gemm: a block timed out waiting for its MMAs") : SDPAB_OK;
}
