// Low-rank factor of the dual of a MaxCut-type SDP, the input of the
// SDPAB_INIT_FACTOR start (no counterpart in the reference solver).
//
// For an instance whose constraints are X_ii = b_i (F_i = e_i e_i^T, one
// SDP block, m = n, b > 0) the user's dual problem is
//   max <F0, Y>  s.t.  Y_ii = b_i,  Y >= 0,
// and in the Burer-Monteiro form Y = V V^T (V: n x r, row i of norm
// sqrt(b_i)) block-coordinate ascent over the rows has a closed-form step:
//   v_i <- sqrt(b_i) g_i / |g_i|,   g_i = sum_{j != i} F0_ij v_j
// (the mixing method, Wang, Chang and Kolter, "The Mixing method: low-rank
// coordinate descent for semidefinite programming with diagonal
// constraints", 2017).  With r(r+1)/2 > n its fixed points are, generically,
// the global optimum; a few hundred sweeps reach the accuracy at which the
// interior-point method can start close to the central path.
//
// Layout and schedule.  One warp (one block of 32 threads) per instance,
// instances taken largest first from a work queue.  The warp keeps V in
// shared memory (n rows of RL = 16 or 32 doubles) and F0's off-diagonal
// entries in a global scratch laid out as 16-byte records (offset of the
// neighbour's V row, weight), built per instance from the packed entries in
// a deterministic order.  The rows are greedily coloured (no two neighbours
// share a colour) and updated colour by colour, in groups of up to H rows of
// one colour at once: such rows do not read one another, so a group's
// updates give exactly what updating its rows one after the other gives.
// The groups' records, sweep after sweep, form one periodic stream that the
// warp copies (cp.async, 32 records at a time) into a ring in shared memory
// ahead of the group being updated.  Each group of RL / 2 lanes updates one
// row, two components per lane: its neighbours one after another in two
// FMA chains, then the norm by shuffles within the group and a reciprocal
// square root.  An instance is a chain of about n / H group updates per
// sweep; instances run concurrently.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "sdpab_internal.h"

namespace sdpab {


namespace {

constexpr int LR_MAX_RANK = 32;

// splitmix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", 2014) of a per-entry counter, mapped to [-1, 1).
__device__ __forceinline__ double lr_uniform(unsigned long long seed, long long q, int i, int k)
{
  unsigned long long z = seed + 0x9E3779B97F4A7C15ull *
                                    ((unsigned long long)q * 65536ull * 64ull + (unsigned long long)i * 64ull +
                                     (unsigned long long)k + 1ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// One off-diagonal entry of F0 in row layout: the neighbour's V row as an
// offset in doubles (column * RL) and the weight F0_ij.
struct __align__(16) LrRec {
  int off;
  int pad;
  double w;
};

// The ring: LR_SLOTS chunks of 32 records.
constexpr int LR_SLOTS = 8;
constexpr int LR_RING = 32 * LR_SLOTS;

// Shared memory of one warp for instances of order <= nmax with RL-wide
// rows: V (nmax RL doubles), the ring (LR_RING records), sqrt(b) per row
// (nmax doubles), record offsets by row, fill cursors / colours, the update
// order, the group starts and the record offsets by position (5 (nmax + 1)
// ints, rounded up to 16 bytes).
__host__ __device__ inline size_t lr_warp_bytes(int nmax, int RL)
{
  const size_t ints = (5 * ((size_t)nmax + 1) + 3) / 4 * 4;
  return ((size_t)nmax * RL + nmax) * sizeof(double) + LR_RING * sizeof(LrRec) + ints * sizeof(int);
}

__device__ __forceinline__ void lr_cp16(void* dst, const void* src)
{
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void lr_commit() { asm volatile("cp.async.commit_group;\n" ::); }
// Waits until at most `pending` (0 .. LR_SLOTS - 1) of this thread's most
// recent copy groups are still in flight.
__device__ __forceinline__ void lr_wait(int pending)
{
  if (pending >= 7) asm volatile("cp.async.wait_group 7;\n" ::: "memory");
  else if (pending == 6) asm volatile("cp.async.wait_group 6;\n" ::: "memory");
  else if (pending == 5) asm volatile("cp.async.wait_group 5;\n" ::: "memory");
  else if (pending == 4) asm volatile("cp.async.wait_group 4;\n" ::: "memory");
  else if (pending == 3) asm volatile("cp.async.wait_group 3;\n" ::: "memory");
  else if (pending == 2) asm volatile("cp.async.wait_group 2;\n" ::: "memory");
  else if (pending == 1) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
  else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

// 1 / sqrt(x) for x > 0 (normal): the single-precision hardware estimate
// refined by two Newton-Raphson steps y <- y (3 - x y^2) / 2 (the standard
// iteration for the reciprocal square root; each step squares the relative
// error, 2^-23 -> 2^-46 -> below double rounding).  The factor only needs
// the row's norm to a few ulps.
__device__ __forceinline__ double lr_rsqrt(double x)
{
  if (!(x > 1.0e-30 && x < 1.0e30)) return rsqrt(x);  // outside float's comfortable range
  double y = (double)rsqrtf((float)x);
  y = y * fma(-0.5 * x * y, y, 1.5);
  y = y * fma(-0.5 * x * y, y, 1.5);
  return y;
}

// Columns instance q uses: r(r+1)/2 > n with one to spare.
__host__ __device__ inline int lr_rank_for(int n, int R)
{
  int r = (int)ceil(sqrt(2.0 * (double)n)) + 1;
  return r < R ? r : R;
}

template <int RL>
__global__ void __launch_bounds__(32) k_mixing(sdpab_batch p, int R, int max_sweeps, double tol,
                                               long long sweep_work, unsigned long long seed,
                                               long long num_entries, LrRec* csr,
                                               double* V, int* sweeps, const int* order, int* queue)
{
  extern __shared__ __align__(16) unsigned char lr_smem[];
  constexpr unsigned FULL = 0xffffffffu;
  constexpr int LPV = RL / 2;   // lanes per row vector, two components each
  constexpr int H = 32 / LPV;   // lane groups: one row of a group each
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  double* Vs = (double*)lr_smem;                 // n x RL, rows in the instance's order
  LrRec* ring = (LrRec*)(Vs + (size_t)p.nmax * RL);
  double* sb = (double*)(ring + LR_RING);        // sqrt(b_i) by row
  int* rp = (int*)(sb + p.nmax);                 // record offsets (n + 1): by row, then by position
  int* cur = rp + p.nmax + 1;                    // counts, fill cursors, then colours (n + 1)
  int* perm = cur + p.nmax + 1;                  // the rows in update order (n)
  int* gs = perm + p.nmax;                       // group starts, in positions (n + 1)
  for (;;) {
    int qi = 0;
    if (lane == 0) qi = atomicAdd(queue, 1);
    qi = __shfl_sync(FULL, qi, 0);
    if (qi >= p.count) break;
    const long long q = order ? order[qi] : qi;
    const int n = p.n[q], m = p.m[q];
    const long long* mp = p.mat_ptr + p.mat_off[q];
    const double* bq = p.b + p.vec_off[q];
    // ---- the form X_ii = b_i: one SDP block, m = n, constraint k one entry
    // (r, r) of value 1, b_k > 0, every row once
    int bad = (m != n || n > p.nmax || n < 2 || mp[m + 1] > num_entries) ? 1 : 0;
    if (!bad && p.nblock) bad = (p.nblock[q] != 1 || p.blk_size[p.blk_off[q]] < 2) ? 1 : 0;
    if (!bad) {
      for (int i = lane; i < n; i += 32) cur[i] = 0;
      __syncwarp();
      for (int k = lane; k < m; k += 32) {
        const long long e0 = mp[k + 1];
        if (mp[k + 2] - e0 != 1) { bad = 1; continue; }
        const int r = p.row[e0];
        const double bk = bq[k];
        if (r != p.col[e0] || r < 0 || r >= n || p.val[e0] != 1.0 || !(bk > 0.0)) { bad = 1; continue; }
        atomicAdd(&cur[r], 1);
        sb[r] = sqrt(bk);
      }
      __syncwarp();
      for (int i = lane; i < n; i += 32) bad |= (cur[i] != 1) ? 1 : 0;
    }
    const long long f0 = mp[0], f1 = mp[1];
    if (!__any_sync(FULL, bad)) {
      // ---- F0's off-diagonal entries by rows: counts, exclusive scan, fill
      __syncwarp();
      for (int i = lane; i < n; i += 32) cur[i] = 0;
      __syncwarp();
      for (long long e = f0 + lane; e < f1; e += 32) {
        const int r = p.row[e], c = p.col[e];
        if (r < 0 || c < 0 || r >= n || c >= n) { bad = 1; continue; }
        if (r != c && p.val[e] != 0.0) {
          atomicAdd(&cur[r], 1);
          atomicAdd(&cur[c], 1);
        }
      }
    }
    if (__any_sync(FULL, bad)) {
      if (lane == 0) sweeps[q] = -1;
      __syncwarp();
      continue;
    }
    __syncwarp();
    // exclusive scan of cur[0 .. cnt) into dst[0 .. cnt], the total in dst[cnt]
    auto scan = [&](const int* src, int* dst, int cnt) {
      int carry = 0;
      for (int i0 = 0; i0 < cnt; i0 += 32) {
        const int i = i0 + lane;
        const int v = (i < cnt) ? src[i] : 0;
        int s = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int t = __shfl_up_sync(FULL, s, o);
          if (lane >= o) s += t;
        }
        if (i < cnt) dst[i] = carry + s - v;
        carry += __shfl_sync(FULL, s, 31);
      }
      if (lane == 0) dst[cnt] = carry;
      __syncwarp();
    };
    scan(cur, rp, n);
    for (int i = lane; i < n; i += 32) cur[i] = rp[i];
    __syncwarp();
    // each 32-entry chunk places its entries in lane order (ranks among the
    // lanes with the same target row), so the layout does not depend on
    // timing; records by row go to region A (2 f0 ..), by update position to
    // region B (2 num_entries + 2 f0 ..)
    LrRec* recA = csr + 2 * f0;
    LrRec* recB = csr + 2 * num_entries + 2 * f0;
    for (long long c0 = f0; c0 < f1; c0 += 32) {
      const long long e = c0 + lane;
      int r = -1, c = -1;
      double v = 0.0;
      if (e < f1) {
        r = p.row[e];
        c = p.col[e];
        v = p.val[e];
      }
      const bool ok = e < f1 && r != c && v != 0.0;
      const unsigned act = __ballot_sync(FULL, ok);
#pragma unroll
      for (int dir = 0; dir < 2; ++dir) {
        const int key = dir ? c : r, other = dir ? r : c;
        unsigned peers = 0;
        if (ok) {
          peers = __match_any_sync(act, key);
          LrRec rec;
          rec.off = other * RL;
          rec.pad = 0;
          rec.w = v;
          recA[cur[key] + __popc(peers & lt)] = rec;
        }
        __syncwarp();
        if (ok && (peers & lt) == 0) cur[key] += __popc(peers);
        __syncwarp();
      }
    }
    __threadfence_block();
    // ---- greedy colouring in row order: row i takes the smallest colour
    // below 64 that no neighbour coloured before it has (64 + i when none is
    // free); rows of one colour are not neighbours, so their updates commute
    int* col = cur;
    for (int i = lane; i < n; i += 32) col[i] = -1;
    __syncwarp();
    for (int i = 0; i < n; ++i) {
      unsigned lo = 0, hi = 0;
      for (int t = rp[i] + lane; t < rp[i + 1]; t += 32) {
        const int cj = col[recA[t].off / RL];
        if (cj >= 0 && cj < 32) lo |= 1u << cj;
        else if (cj >= 32 && cj < 64) hi |= 1u << (cj - 32);
      }
      lo = __reduce_or_sync(FULL, lo);
      hi = __reduce_or_sync(FULL, hi);
      const int c = (~lo) ? __ffs(~lo) - 1 : ((~hi) ? 31 + __ffs(~hi) : 64 + i);
      if (lane == 0) col[i] = c;
      __syncwarp();
    }
    // ---- update order: the rows by colour, in row order within a colour
    {
      int np = 0;
      for (int c = 0; c < 65 && np < n; ++c) {
        for (int i0 = 0; i0 < n; i0 += 32) {
          const int i = i0 + lane;
          const bool in = i < n && (c < 64 ? col[i] == c : col[i] >= 64);
          const unsigned bal = __ballot_sync(FULL, in);
          if (in) perm[np + __popc(bal & lt)] = i;
          np += __popc(bal);
        }
      }
    }
    __syncwarp();
    // ---- records in update order (region B) and their offsets pp by position
    int* pp = gs + p.nmax + 1;
    for (int k = lane; k < n; k += 32) pp[k] = rp[perm[k] + 1] - rp[perm[k]];
    __syncwarp();
    scan(pp, pp, n);
    for (int k = 0; k < n; ++k) {
      const int src = rp[perm[k]], dst = pp[k], cnt = pp[k + 1] - pp[k];
      for (int t = lane; t < cnt; t += 32) recB[dst + t] = recA[src + t];
    }
    // ---- groups of up to H consecutive positions of one colour whose
    // records fit the ring together (a longer row is a group of its own)
    int ng = 0;
    if (lane == 0) {
      int k = 0;
      while (k < n) {
        const int start = k, c = col[perm[k]];
        int tot = pp[k + 1] - pp[k];
        ++k;
        while (k < n && k - start < H && col[perm[k]] == c && tot + pp[k + 1] - pp[k] <= LR_RING - 32) {
          tot += pp[k + 1] - pp[k];
          ++k;
        }
        gs[ng++] = start;
      }
      gs[ng] = n;
    }
    ng = __shfl_sync(FULL, ng, 0);
    __threadfence_block();
    __syncwarp();
    // ---- seeded start, rows scaled to norm sqrt(b_i)
    const int rq = lr_rank_for(n, R);
    for (int t = lane; t < n * RL; t += 32) {
      const int i = t / RL, k = t - i * RL;
      Vs[t] = (k < rq) ? lr_uniform(seed, q, i, k) : 0.0;
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      double ss = 0.0;
      for (int k = 0; k < rq; ++k) ss += Vs[i * RL + k] * Vs[i * RL + k];
      const double sc = (ss > 0.0) ? sb[i] / sqrt(ss) : 0.0;
      for (int k = 0; k < rq; ++k) Vs[i * RL + k] *= sc;
    }
    __syncwarp();
    // ---- sweeps, one group of rows at a time: lane group h (LPV lanes, two
    // components each) updates the group's h-th row.  The groups' records,
    // sweep after sweep, are one periodic stream of L = pp[n] records; the
    // warp copies it 32 records at a time into the ring, up to LR_SLOTS
    // chunks ahead of the group being updated.
    const int h = lane / LPV, kk = lane % LPV;
    const bool act0 = 2 * kk < rq, act1 = 2 * kk + 1 < rq;
    const int L = pp[n];
    int issued = 0;   // chunks of the stream issued
    int pos = 0;      // stream position of the current group's first record
    int src = 0;      // this lane's record of the next chunk: (32 issued + lane) mod L
    auto issue = [&]() {
      if (L > 0) {
        lr_cp16(&ring[(issued & (LR_SLOTS - 1)) * 32 + lane], recB + src);
        src += 32;
        while (src >= L) src -= L;
      }
      lr_commit();
      ++issued;
    };
    __threadfence();  // region B's records are written before the ring copies read them
    __syncwarp();
    if (L > 0) {
      src = lane;
      while (src >= L) src -= L;
      while (issued < LR_SLOTS) issue();
    }
    double fold = 0.0;
    int s = 0;
    // at most max_sweeps sweeps, and at most sweep_work / (n + L) when set
    int cap = max_sweeps;
    if (sweep_work > 0) cap = (int)min((long long)cap, max(1LL, sweep_work / ((long long)n + L)));
    while (s < cap) {
      double fl = 0.0;  // this lane's share of sum_i sqrt(b_i) |g_i|
      for (int g = 0; g < ng; ++g) {
        const int k0 = gs[g], k1 = gs[g + 1];
        const int tot = pp[k1] - pp[k0];
        const bool inring = tot <= LR_RING - 32;
        if (inring && tot > 0) {
          lr_wait(issued - 1 - ((pos + tot - 1) >> 5));  // the chunk of the group's last record
          __syncwarp();
        }
        const int k = k0 + h;
        const bool mine = k < k1;
        double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
        int row = 0;
        if (mine) {
          row = perm[k];
          const int d = pp[k + 1] - pp[k];
          if (inring) {
            const int rb = pos + pp[k] - pp[k0];
            int t = 0;
#pragma unroll 2
            for (; t + 1 < d; t += 2) {
              const LrRec r0 = ring[(rb + t) & (LR_RING - 1)];
              const LrRec r1 = ring[(rb + t + 1) & (LR_RING - 1)];
              const double2 v0 = *(const double2*)(Vs + r0.off + 2 * kk);
              const double2 v1 = *(const double2*)(Vs + r1.off + 2 * kk);
              a0 = fma(r0.w, v0.x, a0);
              a1 = fma(r0.w, v0.y, a1);
              b0 = fma(r1.w, v1.x, b0);
              b1 = fma(r1.w, v1.y, b1);
            }
            if (t < d) {
              const LrRec r0 = ring[(rb + t) & (LR_RING - 1)];
              const double2 v0 = *(const double2*)(Vs + r0.off + 2 * kk);
              a0 = fma(r0.w, v0.x, a0);
              a1 = fma(r0.w, v0.y, a1);
            }
          } else {
            const LrRec* rr = recB + pp[k];
            for (int t = 0; t < d; ++t) {
              const LrRec r0 = rr[t];
              const double2 v0 = *(const double2*)(Vs + r0.off + 2 * kk);
              a0 = fma(r0.w, v0.x, a0);
              a1 = fma(r0.w, v0.y, a1);
            }
          }
        }
        const double g0 = (mine && act0) ? a0 + b0 : 0.0, g1 = (mine && act1) ? a1 + b1 : 0.0;
        double ss = g0 * g0 + g1 * g1;
#pragma unroll
        for (int o = LPV / 2; o > 0; o >>= 1) ss += __shfl_xor_sync(FULL, ss, o);
        if (mine && ss > 0.0) {
          const double sc = sb[row] * lr_rsqrt(ss);
          if (act0) Vs[row * RL + 2 * kk] = g0 * sc;
          if (act1) Vs[row * RL + 2 * kk + 1] = g1 * sc;
          if (kk == 0) fl += sc * ss;
        }
        pos += tot;
        __syncwarp();  // the group's ring records are read, its V rows written
        while (issued < (pos >> 5) + LR_SLOTS) issue();
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) fl += __shfl_xor_sync(FULL, fl, o);
      ++s;
      if (s > 1 && fabs(fl - fold) <= tol * fabs(fl)) break;
      fold = fl;
    }
    lr_wait(0);
    __syncwarp();
    double* Vq = V + p.vec_off[q] * R;
    for (int t = lane; t < n * R; t += 32) {
      const int i = t / R, k = t - i * R;
      Vq[t] = Vs[i * RL + k];
    }
    if (lane == 0) sweeps[q] = s;
    __syncwarp();
  }
}

// Row-layout records of F0's entries and the work-queue counter, per
// device, kept between calls.
// Each call takes the next of LR_QUEUES work-queue counters, so calls that
// run concurrently on different streams (on disjoint instances) do not share
// one.
constexpr int LR_QUEUES = 1024;
struct LrScratch {
  LrRec* rec = nullptr;
  int* queue = nullptr;
  long long cap = 0;
  unsigned calls = 0;
  void release()
  {
    if (rec) cudaFree(rec);
    if (queue) cudaFree(queue);
    rec = nullptr;
    queue = nullptr;
    cap = 0;
  }
};
constexpr int LR_MAX_DEVICES = 64;
LrScratch g_lr[LR_MAX_DEVICES];

}  // namespace

void lowrank_release()
{
  int dev = 0;
  cudaGetDevice(&dev);
  g_lr[(dev >= 0 && dev < LR_MAX_DEVICES) ? dev : 0].release();
}

}  // namespace sdpab

using namespace sdpab;

// The default rank: each instance's own ceil(sqrt(2 n)) + 1, capped at 16
// (row vectors of 16 doubles) while 16 still satisfies r (r + 1) / 2 > n,
// the rank above which the factored problem's fixed points are generically
// the SDP's optimum; 32 at most.
extern "C" int sdpab_lowrank_default_rank(int nmax)
{
  nmax = std::max(nmax, 1);
  const int r = lr_rank_for(nmax, LR_MAX_RANK);
  return (r > 16 && 16 * 17 / 2 > nmax) ? 16 : r;
}

extern "C" int sdpab_lowrank_factor(const sdpab_batch* prob, long long num_entries, int rank, int max_sweeps,
                                    double tol, long long sweep_work, unsigned long long seed, double* V,
                                    int* sweeps, const int* order, void* stream)
{
  if (!prob || !V || !sweeps || prob->count < 0 || num_entries < 0 || rank < 0 || rank > LR_MAX_RANK ||
      max_sweeps < 0 || !(tol >= 0.0) || sweep_work < 0)
    return set_error(SDPAB_EINVAL, "lowrank_factor: invalid arguments");
  if (prob->count == 0) return SDPAB_OK;
  if (prob->nmax < 1) return set_error(SDPAB_EINVAL, "lowrank_factor: nmax must be positive");
  const int R = rank > 0 ? rank : sdpab_lowrank_default_rank(prob->nmax);
  const int RL = (R <= 16) ? 16 : 32;
  const size_t smem = lr_warp_bytes(prob->nmax, RL);
  if (smem > 227 * 1024) return set_error(SDPAB_ESIZE, "lowrank_factor: nmax * rank too large for shared memory");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDPAB_ENODEV, "lowrank_factor: no CUDA device");
  LrScratch& S = g_lr[(dev >= 0 && dev < LR_MAX_DEVICES) ? dev : 0];
  const long long need = std::max<long long>(4 * num_entries, 32);  // records by row, then by position
  if (S.cap < need) {
    S.release();
    if (cudaMalloc((void**)&S.rec, need * sizeof(LrRec)) != cudaSuccess ||
        cudaMalloc((void**)&S.queue, LR_QUEUES * sizeof(int)) != cudaSuccess) {
      S.release();
      return set_error(SDPAB_ECUDA, "lowrank_factor: scratch allocation failed");
    }
    S.cap = need;
  }
  int* queue = S.queue + (S.calls++ % LR_QUEUES);
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_error(e, "lowrank_factor: clearing the queue");
  auto kern = (RL == 16) ? k_mixing<16> : k_mixing<32>;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_error(e, "lowrank_factor: cudaFuncSetAttribute");
  int sms = 0, bps = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 32, smem);
  if (e != cudaSuccess) return cuda_error(e, "lowrank_factor: occupancy");
  if (bps < 1) return set_error(SDPAB_ESIZE, "lowrank_factor: the block does not fit on an SM");
  const int grid = (int)std::min<long long>(prob->count, (long long)sms * bps);
  kern<<<grid, 32, smem, (cudaStream_t)stream>>>(*prob, R, max_sweeps, tol, sweep_work, seed, num_entries, S.rec, V,
                                                 sweeps, order, queue);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "lowrank_factor: launch");
  return SDPAB_OK;
}
