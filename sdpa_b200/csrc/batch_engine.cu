// Batched persistent SDP solver: one launch solves a whole batch of small
// SDPs.  An instance is one SDP block, or several SDP blocks and LP entries
// laid along the diagonal of one n x n matrix: the HKM iterates of a
// block-diagonal start stay block-diagonal (every product and inverse of
// block-diagonal matrices is), so the dense steps run on the whole matrix,
// and the step length takes each block's minimum eigenvalue as the
// reference does.  Each thread block repeatedly takes the next instance
// from a device work queue (atomic counter over a largest-first order) and
// runs SDPA's complete Mehrotra predictor-corrector loop for it
// (SDPA::solve, sdpa_solve.cpp:59-233), with every dense step executed
// cooperatively by the block on an L2-resident per-block workspace.
//
// Per iteration (reference operation sequence, sdpa_newton.cpp:2755-2809):
//   predictor: R = beta mu Z^-1 - X; [X D Z^-1]; g = -A.(R - XDZ^-1) + r_p;
//              Schur B by formula F3 (calF3_thread_2, sdpa_newton.cpp:1319-1403);
//              adjusted Cholesky (sdpa_dpotrf.cpp:31-33); dy; dZ; dX (symmetrised)
//   corrector: R -= dX dZ Z^-1; g; dy (same factor); dZ; dX
//   step:      Lanczos (n > 20) or dense eigenvalue (n <= 20) minimum
//              eigenvalue of L^-1 dX L^-T (sdpa_linear.cpp:29-182)
//   update:    X, y, Z; Cholesky + inverse of X and Z, Z^-1 (sdpa_dataset.cpp:117-171)
//   residuals, mu, objectives (sdpa_dataset.cpp:585-608, sdpa_parts.cpp:914-1060)
// The scalar rules live in ipm_control.h, shared with the host-driven solver.
// There are no inter-block waits: the only synchronisation is __syncthreads.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <numeric>
#include <vector>

#include "cta_linalg.cuh"
#include "eig.cuh"
#include "ipm_control.h"
#include "sdpa_b200.h"
#include "sdpab_internal.h"

namespace sdpab {

// Dynamic shared memory of the solver block (bt threads), in doubles /
// bytes, given the staging area `gsm` (doubles) for GEMM tiles, Lanczos
// matrices and the diagonal blocks of the factorisations.
static __host__ __device__ long long fixed_smem_doubles(int nmax, int mmax, int bt)
{
  return 4 * (bt / 32) + 6LL * mmax + 4LL * nmax + eig_scratch_doubles(nmax);
}

static size_t smem_bytes_for(int nmax, int mmax, long long gsm, int bt)
{
  return (size_t)(gsm + fixed_smem_doubles(nmax, mmax, bt)) * sizeof(double) +
         (size_t)(2 * mmax + nmax) * sizeof(int) + 64;
}

// Shared memory of one SM, what the system reserves per resident block, and
// an allowance for the solver kernel's static shared memory (under 1 KB).
constexpr long long SM_SMEM_BYTES = 228LL * 1024, BLOCK_RESERVED_BYTES = 1024, STATIC_SMEM_BYTES = 1024;

// Staging area for `per_sm` resident blocks of bt threads: at least the
// square GEMM's double-buffered tiles (cta::gemm_smem_min) and the two
// diagonal blocks; `want` doubles when given, by default both Lanczos
// matrices (2 n^2) when they fit in LANCZOS_SMEM_DOUBLES, else one, else
// the minimum; capped at what per_sm blocks of this size can have.  (Shared
// memory beyond that is taken from the L1 cache the workspace loads use.)
static long long staging_min(int bt)
{
  const long long g = (bt >= 256) ? cta::gemm_smem_min<256>() : cta::gemm_smem_min<128>();
  return std::max<long long>(g, 2 * cta::SD_DOUBLES);
}

static long long staging_doubles(int nmax, int mmax, int want, int bt, int per_sm)
{
  const long long g = staging_min(bt);
  const long long m2 = (long long)nmax * nmax;
  long long s;
  if (want > 0) s = want;
  else if (2 * m2 <= LANCZOS_SMEM_DOUBLES) s = 2 * m2;
  else if (m2 <= LANCZOS_SMEM_DOUBLES) s = m2;
  else s = g;
  const long long per_block = std::min<long long>(227LL * 1024, SM_SMEM_BYTES / std::max(per_sm, 1) -
                                                                    BLOCK_RESERVED_BYTES) -
                              STATIC_SMEM_BYTES;
  const long long cap = (per_block - (long long)smem_bytes_for(nmax, mmax, 0, bt)) / (long long)sizeof(double);
  if (s > cap) s = cap;
  s = s / 32 * 32;
  return s > g ? s : g;
}

struct BatchArgs {
  sdpab_batch p;
  sdpab_batch_init init;
  sdpab_batch_result r;
  Params prm;
  const int* order;
  int gsm_doubles;        // staging area (doubles) at the head of dynamic shared memory
  int mixed;             // SDPAB_PREC_MIXED: FP32 Schur factor + FP64 refinement while mixed_gap >= mu_switch
  int mixed_products;    // mixed mode: the n^3 products in FP32 as well (else on the FP64 MMA)
  double mu_switch;
  double refine_tol;     // mixed mode: refinement stops once the correction is below this times |dy|
  int factor_smem;       // the Schur factorisation in shared memory when the staging area holds it
  double* ws;
  long long ws_stride;  // doubles per block
  int* queue;
};

// Sparse helpers over one matrix's entry range -----------------------------

// A . W for a symmetric A stored as upper-triangle entries and a general W
// (Lal::getInnerProduct(Sparse, Dense), sdpa_linear.cpp:318-460).
__device__ __forceinline__ double sp_dot(const int* row, const int* col, const double* val,
                                         long long beg, long long end, const double* W, int ld)
{
  double s = 0.0;
  for (long long e = beg; e < end; ++e) {
    int r = row[e], c = col[e];
    double v = val[e];
    s += (r == c) ? v * W[r + (size_t)ld * r] : v * (W[r + (size_t)ld * c] + W[c + (size_t)ld * r]);
  }
  return s;
}

// W += scale * A (both triangles), block-parallel over entries.
template <int BT>
__device__ __forceinline__ void sp_axpy_block(const int* row, const int* col, const double* val,
                                              long long beg, long long end, double scale, double* W,
                                              int ld)
{
  for (long long e = beg + threadIdx.x; e < end; e += BT) {
    int r = row[e], c = col[e];
    double v = scale * val[e];
    atomicAdd(&W[r + (size_t)ld * c], v);
    if (r != c) atomicAdd(&W[c + (size_t)ld * r], v);
  }
}

// W += scale * sum_k coef[k] A_k, one thread per constraint
// (InputData::multi_plusToA, sdpa_dataset.cpp:427-433).  mp points at the
// instance's F0 pointer; A_k is matrix k+1.
template <int BT>
__device__ __forceinline__ void sp_axpy_constraints(const int* row, const int* col,
                                                    const double* val, const long long* mp, int m,
                                                    const double* coef, double scale, double* W,
                                                    int ld)
{
  for (int k = threadIdx.x; k < m; k += BT) {
    const double s = scale * coef[k];
    for (long long e = mp[k + 1]; e < mp[k + 2]; ++e) {
      int r = row[e], c = col[e];
      double v = s * val[e];
      atomicAdd(&W[r + (size_t)ld * c], v);
      if (r != c) atomicAdd(&W[c + (size_t)ld * r], v);
    }
  }
}

// calF3_thread_2 (sdpa_newton.cpp:1319-1403): Tr(A_i X A_j Z^-1) with A_j
// outer (its entries alpha,beta) and A_i inner (gamma,delta).
__device__ __forceinline__ double f3_value(const int* row, const int* col, const double* val,
                                           long long jb, long long je, long long ib, long long ie,
                                           const double* X, const double* Zi, int n)
{
  double ret = 0.0;
  for (long long e1 = jb; e1 < je; ++e1) {
    const int al = row[e1], be = col[e1];
    const double v1 = val[e1];
    const double* Xa = X + (size_t)n * al;
    const double* Xb = X + (size_t)n * be;
    const double* Za = Zi + (size_t)n * al;
    const double* Zb = Zi + (size_t)n * be;
    double sum = 0.0;
    if (al != be) {
      for (long long e2 = ib; e2 < ie; ++e2) {
        const int ga = row[e2], de = col[e2];
        double plu = (ga != de)
                         ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] + Za[de] * Xb[ga] + Za[ga] * Xb[de]
                         : Zb[de] * Xa[ga] + Za[de] * Xb[ga];
        sum += val[e2] * plu;
      }
    } else {
      for (long long e2 = ib; e2 < ie; ++e2) {
        const int ga = row[e2], de = col[e2];
        double plu = (ga != de) ? Zb[de] * Xa[ga] + Zb[ga] * Xa[de] : Zb[de] * Xa[ga];
        sum += val[e2] * plu;
      }
    }
    ret += v1 * sum;
  }
  return ret;
}

// F1 columns of the Schur complement (compute_bMat_dense_SDP with calF1,
// sdpa_newton.cpp:885-889, :1827-1922): for every constraint j flagged in
// `form`, G = X A_j Z^-1 and B_ij = A_i . G for each i that j dominates.
// T, G: n x n scratch.  With a block structure (nb > 0 blocks at boff of
// signed orders bsz; bid = SDP block of each row, -1 for LP entries) X, A_j
// and Z^-1 are block-diagonal, so T = X A_j and G are formed one block at a
// time, only for the blocks A_j touches (G is zero elsewhere), and LP
// entries are diagonal products.  Not inlined: only instances with F1
// constraints call it.
//
// T = X A_j with A_j symmetric, stored as upper entries (r, c, v).  Blocks
// of order <= 64: A_j's block is scattered into the scratch Ad as a dense
// k x k matrix and T = X_b A_b is a tiled block product like G = T Z^-1.
// Larger blocks and a single block: one thread per row of T, accumulating
// over the entries.
template <int BT>
static __device__ void f1_rows(int n, int r0, int k, long long jb, long long je, const int* er, const int* ec,
                               const double* ev, const double* X, double* T)
{
  for (int i = r0 + (int)threadIdx.x; i < r0 + k; i += BT) {
    for (int c = r0; c < r0 + k; ++c) T[i + (size_t)n * c] = 0.0;
    for (long long e = jb; e < je; ++e) {
      const int r = er[e], c = ec[e];
      if (r < r0 || r >= r0 + k) continue;
      const double v = ev[e];
      T[i + (size_t)n * c] += v * X[i + (size_t)n * r];
      if (r != c) T[i + (size_t)n * r] += v * X[i + (size_t)n * c];
    }
  }
}

template <int BT>
static __device__ __noinline__ void schur_f1(int n, int m, const long long* mp, const int* er, const int* ec,
                                             const double* ev, const double* X, const double* Zi, double* T,
                                             double* G, double* Ad, double* B, const int* nnz, const int* form,
                                             int nb, const int* boff, const int* bsz, const int* bid, double* gsm)
{
  __shared__ unsigned long long s_touch;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int j = 0; j < m; ++j) {
    if (!form[j]) continue;
    const long long jb = mp[j + 1], je = mp[j + 2];
    if (nb <= 0) {
      f1_rows<BT>(n, 0, n, jb, je, er, ec, ev, X, T);
      __syncthreads();
      cta::gemm<BT>(n, false, T, n, false, Zi, n, G, n, 1.0, 0.0, gsm);
    } else {
      // blocks touched by A_j
      if (tid == 0) s_touch = 0ull;
      __syncthreads();
      unsigned long long mine = 0ull;
      for (long long e = jb + tid; e < je; e += BT) {
        const int b = bid[er[e]];
        if (b >= 0) mine |= 1ull << b;
      }
      if (mine) atomicOr(&s_touch, mine);
      __syncthreads();
      const unsigned long long touch = s_touch;
      for (int l = 0; l < nb; ++l) {
        const int k = bsz[l], o = boff[l];
        if (k >= 2) {
          if (!((touch >> l) & 1ull)) continue;
          if (k > 64) {
            f1_rows<BT>(n, o, k, jb, je, er, ec, ev, X, T);
            continue;
          }
          for (int t = tid; t < k * k; t += BT) Ad[t] = 0.0;
          __syncthreads();
          for (long long e = jb + tid; e < je; e += BT) {
            const int r = er[e] - o, c = ec[e] - o;
            if (r < 0 || r >= k) continue;
            Ad[r + k * c] = ev[e];
            Ad[c + k * r] = ev[e];
          }
          __syncthreads();
          const size_t od = (size_t)o * (n + 1);
          cta::gemm<BT>(k, false, X + od, n, false, Ad, k, T + od, n, 1.0, 0.0, gsm);
        } else {
          // LP entries: G_tt = (sum of A_j's entries at (t, t)) X_tt Z^-1_tt
          for (int t = tid; t < -k; t += BT) {
            const int d = o + t;
            double a = 0.0;
            for (long long e = jb; e < je; ++e) a += (er[e] == d) ? ev[e] : 0.0;
            const size_t dd = (size_t)d * (n + 1);
            G[dd] = a * X[dd] * Zi[dd];
          }
        }
      }
      __syncthreads();
      // G = T Z^-1 block by block; zero where A_j does not reach
      for (int l = 0; l < nb; ++l) {
        const int k = bsz[l];
        if (k < 2) continue;
        const size_t o = (size_t)boff[l] * (n + 1);
        if ((touch >> l) & 1ull) {
          cta::gemm<BT>(k, false, T + o, n, false, Zi + o, n, G + o, n, 1.0, 0.0, gsm);
        } else {
          for (int t = tid; t < k * k; t += BT) G[o + (size_t)(t % k) + (size_t)n * (t / k)] = 0.0;
        }
      }
    }
    __syncthreads();
    // B_ij = A_i . G for the i dominated by j, one warp per i
    const int jnz = nnz[j];
    for (int i = wid; i < m; i += BT / 32) {
      const int inz = nnz[i];
      if (jnz < inz || (inz == jnz && i < j)) continue;
      double s = 0.0;
      for (long long e = mp[i + 1] + lane; e < mp[i + 2]; e += 32) {
        const int r = er[e], c = ec[e];
        const double v = ev[e];
        s += (r == c) ? v * G[r + (size_t)n * r] : v * (G[r + (size_t)n * c] + G[c + (size_t)n * r]);
      }
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) {
        B[i + (size_t)m * j] = s;
        B[j + (size_t)m * i] = s;
      }
    }
    __syncthreads();
  }
}

// The solver -----------------------------------------------------------------

// GENERAL: the batch carries a block structure (sdpab_batch.nblock; one
// block of order n counts), and the solver supports several blocks and F1
// Schur columns for constraints with many entries.  The other instantiation
// (single SDP block, every Schur entry by F3) has none of that bookkeeping,
// so the MaxCut-like common case keeps its register allocation.
template <bool GENERAL, int BT>
__global__ void __launch_bounds__(BT, 512 / BT) batch_ipm_fp64(BatchArgs a)
{
  extern __shared__ double smem[];
  const int nmax = a.p.nmax, mmax = a.p.mmax;
  const int gsm_doubles = a.gsm_doubles;
  // GEMM staging / Lanczos matrices; the diagonal blocks of the blocked
  // factorisations and solves share it (they are dead while a GEMM or a
  // Lanczos process uses it: every such call starts and ends at a barrier)
  double* gsm = smem;
  double* sD = gsm;                                     // diagonal block NB*LDD
  double* sD2 = sD + cta::SD_DOUBLES;                   // second diagonal block (paired X / Z steps)
  double* redbuf = gsm + gsm_doubles;                   // 4 * BT/32
  double* vy = redbuf + 4 * (BT / 32);                  // y   (mmax)
  double* vdy = vy + mmax;                              // dy  (mmax)
  double* vg = vdy + mmax;                              // g   (mmax)
  double* vrp = vg + mmax;                              // r_p (mmax)
  double* vdz = vrp + mmax;                             // dZ when it is diagonal (nmax)
  double* vres = vdz + nmax;                            // refinement residual (mmax)
  float* x32 = (float*)(vres + mmax);                   // FP32 solve vector (mmax floats)
  double* vX0d = vres + 2 * mmax;                       // diagonals of X0, Z0 and C (nmax each)
  double* vZ0d = vX0d + nmax;
  double* vCd = vZ0d + nmax;
  cta::Reducer RD{redbuf, 0};
  EigScratch es;
  eig_scratch_carve(es, vCd + nmax, nmax, &RD);          // eig_scratch_doubles(nmax)
  int* s_nnz = (int*)(vCd + nmax + eig_scratch_doubles(nmax));  // mmax ints
  int* s_bid = s_nnz + mmax;  // nmax ints: block of each row (-1 = LP entry)
  int* s_form = s_bid + nmax;  // mmax ints: 1 = constraint's Schur column by F1

  __shared__ int s_inst, s_flag, s_flag2[2];
  __shared__ int s_nb, s_boff[SDPAB_BATCH_MAX_BLOCKS], s_bsz[SDPAB_BATCH_MAX_BLOCKS];
  __shared__ Scalars S;
  const int tid = threadIdx.x;
  const Params& P = a.prm;

  double* wsb = a.ws + (size_t)blockIdx.x * a.ws_stride;
  const size_t nn = (size_t)nmax * nmax;
  double* X = wsb;
  double* Z = X + nn;
  double* Zi = Z + nn;
  double* LXi = Zi + nn;
  double* LZi = LXi + nn;
  double* D = LZi + nn;
  double* XDZ = D + nn;
  double* R = XDZ + nn;
  double* dX = R + nn;
  double* dZ = dX + nn;
  double* W1 = dZ + nn;
  double* W2 = W1 + nn;
  double* X0 = W2 + nn;
  double* Z0 = X0 + nn;
  double* B = Z0 + nn;  // mmax * mmax
  float* B32 = (float*)(B + (size_t)mmax * mmax);  // mixed mode: FP32 factor of B (mmax * mmax floats)

  for (;;) {
    if (tid == 0) s_inst = atomicAdd(a.queue, 1);
    __syncthreads();
    const int q = s_inst;
    __syncthreads();
    if (q >= a.p.count) break;
    const int inst = a.order ? a.order[q] : q;
    const int n = a.p.n[inst], m = a.p.m[inst];
    if (n < 1 || m < 1 || n > nmax || m > mmax) {
      if (tid == 0) a.r.status[inst] = SDPAB_ESIZE;
      continue;
    }
    const long long* mp = a.p.mat_ptr + a.p.mat_off[inst];  // m+2 pointers
    const int* er = a.p.row;
    const int* ec = a.p.col;
    const double* ev = a.p.val;
    const double* bv = a.p.b + a.p.vec_off[inst];
    const double lam = P.lambdaStar;
    const int nn_i = n * n;

    // block structure (SDPA's bLOCKsTRUCT): blocks along the diagonal in
    // file order; s_bid[t] = the SDP block holding row t, -1 for LP entries
    bool blocked = false;
    if constexpr (GENERAL) {
      if (tid == 0) {
        const int nb = a.p.nblock[inst];
        int bad = (nb < 1 || nb > SDPAB_BATCH_MAX_BLOCKS), off = 0;
        for (int l = 0; l < nb && !bad; ++l) {
          const int sz = a.p.blk_size[a.p.blk_off[inst] + l];
          bad = (sz == 0);
          s_boff[l] = off;
          s_bsz[l] = (sz == 1) ? -1 : sz;  // order 1 is an LP entry (sdpa_block.cpp:80-91)
          off += (sz < 0) ? -sz : sz;
        }
        s_nb = (bad || off != n) ? -1 : nb;
      }
      __syncthreads();
      if (s_nb < 0) {
        if (tid == 0) a.r.status[inst] = SDPAB_EINVAL;
        continue;
      }
      for (int l = 0; l < s_nb; ++l) {
        const int sz = s_bsz[l], cnt = (sz < 0) ? -sz : sz;
        for (int t = tid; t < cnt; t += BT) s_bid[s_boff[l] + t] = (sz >= 2) ? l : -1;
      }
      __syncthreads();
      blocked = !(s_nb == 1 && s_bsz[0] == n);
    }
    // entries must index inside one block (LP: its diagonal): reject the
    // instance otherwise
    {
      int bad = 0;
      for (long long e = mp[0] + tid; e < mp[m + 1]; e += BT) {
        const int r = er[e], c = ec[e];
        const bool out = (r < 0 || c < 0 || r >= n || c >= n);
        bad |= out;
        if (!out && blocked) bad |= (s_bid[r] != s_bid[c]) || (s_bid[r] < 0 && r != c);
      }
      if (__syncthreads_or(bad)) {
        if (tid == 0) a.r.status[inst] = SDPAB_EINVAL;
        continue;
      }
    }
    // all constraint entries on the diagonal?
    int offdiag = 0;
    for (long long e = mp[1] + tid; e < mp[m + 1]; e += BT) offdiag |= (er[e] != ec[e]);
    const bool diag_cons = !__syncthreads_or(offdiag);
    // NonZeroEffect per constraint (diagonal 1, off-diagonal 2; sdpa_struct.cpp:1339-1341)
    for (int k = tid; k < m; k += BT) {
      int c = 0;
      for (long long e = mp[k + 1]; e < mp[k + 2]; ++e) c += (er[e] == ec[e]) ? 1 : 2;
      s_nnz[k] = c;
    }
    // Schur formula per constraint j, in the manner of the reference's
    // choice (Newton::computeFormula_SDP, sdpa_newton.cpp:515-695) but with
    // the costs of this solver's two implementations: F3 costs about four
    // gathers per entry pair, 4 nnz_j up_j; F1 costs the block GEMMs of
    // X A_j Z^-1 (sum of k^3), forming X A_j (2 n nnz_j) and one pass over
    // the dominated entries (up_j), where up_j sums the NonZeroEffect of the
    // constraints j dominates.  The formulas give the same values up to
    // rounding.  Single-block batches (MaxCut-like) use F3 only.
    bool any_f1 = false;
    if constexpr (GENERAL) {
      __syncthreads();
      double kcube = 0.0;
      if (blocked) {
        for (int l = 0; l < s_nb; ++l)
          if (s_bsz[l] >= 2) kcube += (double)s_bsz[l] * s_bsz[l] * s_bsz[l];
      } else {
        kcube = (double)n * n * n;
      }
      int anyf1 = 0;
      for (int j = tid; j < m; j += BT) {
        const int jnz = s_nnz[j];
        double up = 0.0;
        for (int i = 0; i < m; ++i) {
          const int inz = s_nnz[i];
          if (!(jnz < inz || (inz == jnz && i < j))) up += inz;
        }
        const int use = kcube + 2.0 * n * jnz + up < 4.0 * jnz * up;
        s_form[j] = use;
        anyf1 |= use;
      }
      any_f1 = __syncthreads_or(anyf1);
    }

    // A warm-started or mixed-precision solve that ends outside pdOPT is
    // solved again from the standard start in FP64 (status 2); iterations
    // count both attempts.
    int status = 0, iter_total = 0;
    double nrp, nrd;
    // residuals: r_p = b - A.X, D = C - Z - sum y_k A_k (Residuals::compute).
    // D is formed in the scratch W1 (free wherever this runs) and kept (in D)
    // only when the point is dual infeasible, the one case in which the next
    // iteration reads it; a dual-feasible solve never touches D's slot.
    auto residuals = [&](double& nrp, double& nrd) {
      double mx = 0.0;
      for (int k = tid; k < m; k += BT) {
        double r = bv[k] - sp_dot(er, ec, ev, mp[k + 1], mp[k + 2], X, n);
        vrp[k] = r;
        mx = fmax(mx, fabs(r));
      }
      nrp = cta::block_max<BT>(mx, RD);
      for (int t = tid; t < nn_i; t += BT) W1[t] = -Z[t];
      __syncthreads();
      sp_axpy_block<BT>(er, ec, ev, mp[0], mp[1], -1.0, W1, n);  // C = -F0
      sp_axpy_constraints<BT>(er, ec, ev, mp, m, vy, -1.0, W1, n);
      __syncthreads();
      mx = 0.0;
      for (int t = tid; t < nn_i; t += BT) mx = fmax(mx, fabs(W1[t]));
      nrd = cta::block_max<BT>(mx, RD);
      if (nrd > P.epsilonDash) {  // dual infeasible (Phase::updateCheck): the next predictor reads D
        for (int t = tid; t < nn_i; t += BT) D[t] = W1[t];
        __syncthreads();
      }
    };
    // C . W with C = -F0
    auto c_dot = [&](const double* W) {
      double s = 0.0;
      for (long long e = mp[0] + tid; e < mp[1]; e += BT) {
        int r = er[e], c = ec[e];
        double v = -ev[e];
        s += (r == c) ? v * W[r + (size_t)n * r] : v * (W[r + (size_t)n * c] + W[c + (size_t)n * r]);
      }
      return cta::block_sum<BT>(s, RD);
    };

    for (int attempt = 0; attempt < 2; ++attempt) {
    // ---------------- initial point
    const int wmode = (attempt == 0 && a.init.flag) ? a.init.flag[inst] : SDPAB_INIT_NONE;
    bool warm = false;
    if (wmode == SDPAB_INIT_POINT) {
      warm = true;
      const double* Xu = a.init.X + a.p.dense_off[inst];
      const double* Yu = a.init.Y + a.p.dense_off[inst];
      const double* xv = a.init.xvec + a.p.vec_off[inst];
      // only the diagonal blocks of a block-structured point are used
      for (int t = tid; t < nn_i; t += BT) {
        const int i = t % n, j = t / n;
        const bool keep = !blocked || (s_bid[i] == s_bid[j] && (s_bid[i] >= 0 || i == j));
        const double xu = keep ? Xu[t] : 0.0, yu = keep ? Yu[t] : 0.0;
        Z[t] = xu; X[t] = yu; W1[t] = xu; W2[t] = yu;
      }
      for (int k = tid; k < m; k += BT) vy[k] = -xv[k];
      __syncthreads();
      // strict interiority check (the reference ignores computeInverse's
      // failure here, sdpa_solve.cpp:63; this solver falls back instead)
      int fx = cta::cholesky<BT, double>(n, W2, n, false, sD, gsm, &s_flag);
      int fz = fx ? 1 : cta::cholesky<BT, double>(n, W1, n, false, sD, gsm, &s_flag);
      if (fx || fz) { warm = false; status = 1; }
      else {
        cta::tri_inverse<BT, double>(n, W2, n, LXi, n, sD, gsm);
        cta::tri_inverse<BT, double>(n, W1, n, LZi, n, sD, gsm);
        cta::gemm<BT>(n, true, LZi, n, false, LZi, n, Zi, n, 1.0, 0.0, gsm);
      }
    } else if (wmode == SDPAB_INIT_DUAL) {
      // Proposed x only.  Applicable when the constraints are X_ii = b_i
      // (F_i = e_i e_i^T, m = n, b > 0): then sum_i F_i = I, so shifting x by
      // s adds s I to X = sum F_i x_i - F0, and Y = D X^{-1} D with
      // D_ii = sqrt(b_i / (X^{-1})_ii) satisfies the constraints exactly.
      int bad = (m != n);
      for (int k = tid; k < m && !bad; k += BT) {
        if (mp[k + 2] - mp[k + 1] != 1) { bad = 1; break; }
        const long long e = mp[k + 1];
        if (er[e] != ec[e] || ev[e] != 1.0 || !(bv[k] > 0.0)) bad = 1;
      }
      // every diagonal position covered exactly once
      for (int t = tid; t < n; t += BT) W1[t] = 0.0;
      __syncthreads();
      for (int k = tid; k < m && !bad; k += BT) atomicAdd(&W1[er[mp[k + 1]]], 1.0);
      __syncthreads();
      for (int t = tid; t < n && !bad; t += BT) bad |= (W1[t] != 1.0);
      bad = __syncthreads_or(bad);
      if (!bad) {
        const double* xv = a.init.xvec + a.p.vec_off[inst];
        for (int k = tid; k < m; k += BT) vy[k] = -xv[k];
        for (int t = tid; t < nn_i; t += BT) Z[t] = 0.0;
        __syncthreads();
        sp_axpy_block<BT>(er, ec, ev, mp[0], mp[1], -1.0, Z, n);  // C = -F0
        __syncthreads();
        double cs = 0.0;
        for (int t = tid; t < n; t += BT) cs += fabs(Z[t + (size_t)n * t]);
        cs = cta::block_sum<BT>(cs, RD) / n;
        const double margin = ((a.init.init_margin > 0.0) ? a.init.init_margin : 0.02) * ((cs > 0.0) ? cs : 1.0);
        sp_axpy_constraints<BT>(er, ec, ev, mp, m, vy, -1.0, Z, n);  // Z = C - sum y_k A_k
        __syncthreads();
        double lmin;
        if (n > 20) lmin = lanczos_min_eig<BT>(n, Z, es);
        else lmin = dense_min_eig<BT>(n, Z, es);
        double shift = (lmin < margin) ? margin - lmin : 0.0;
        int ok = 0;
        for (int attempt = 0; attempt < 8 && !ok; ++attempt) {
          for (int t = tid; t < nn_i; t += BT) W1[t] = Z[t] + (((t % n) == (t / n)) ? shift : 0.0);
          __syncthreads();
          if (cta::cholesky<BT, double>(n, W1, n, false, sD, gsm, &s_flag) == 0) ok = 1;
          else shift = 2.0 * shift + margin;
        }
        if (ok) {
          for (int k = tid; k < m; k += BT) vy[k] -= shift;
          for (int t = tid; t < nn_i; t += BT) if ((t % n) == (t / n)) Z[t] += shift;
          cta::tri_inverse<BT, double>(n, W1, n, LZi, n, sD, gsm);
          cta::gemm<BT>(n, true, LZi, n, false, LZi, n, Zi, n, 1.0, 0.0, gsm);
          // X = D Z^-1 D with X_kk = b_k
          for (int t = tid; t < n; t += BT) {
            const int r = er[mp[t + 1]];
            W1[r] = sqrt(bv[t] / Zi[r + (size_t)n * r]);
          }
          __syncthreads();
          for (int t = tid; t < nn_i; t += BT) {
            const int i = t % n, j = t / n;
            X[t] = W1[i] * Zi[t] * W1[j];
          }
          __syncthreads();
          for (int t = tid; t < nn_i; t += BT) W2[t] = X[t];
          __syncthreads();
          if (cta::cholesky<BT, double>(n, W2, n, false, sD, gsm, &s_flag) == 0) {
            cta::tri_inverse<BT, double>(n, W2, n, LXi, n, sD, gsm);
            warm = true;
          }
        }
      }
      if (!warm) status = 1;
    } else if (wmode == SDPAB_INIT_FACTOR) {
      // A low-rank factor V of the user Y (row i of norm sqrt(b_i)) for
      // constraints X_ii = b_i: Y = V V^T, multipliers x_i = (F0 Y)_ii / b_i,
      // internal Z = sum F_i x_i - F0 (Z Y = 0 at the optimum), and a start
      // on the central path's equation X Z = mu I: with s = mean |F0_ii|,
      // mu = max(init_mu, 3 |Z V| / (|V| s)) s and tau = 0.3 sqrt(mu s)
      //   Z0 = Z + mu (Y + tau I)^-1 + delta I,   X0 = mu Z0^-1,
      // delta the first of 0, mu/n, 4 mu/n, ... that makes Z0 positive
      // definite (X0 = Y + mu (Z + tau I)^-1 instead when delta > 0).  Near
      // the path, Z ~ Z* + mu Y*^+ and X ~ Y* + mu Z*^+: the added term is the
      // first-order correction on the range of Y, where it makes mu Z0^-1 ~ Y;
      // tau keeps it bounded in the directions where Y is (nearly) singular
      // and is far above the factor's own error.  X0 is primal feasible to
      // O(mu), Z0 dual feasible to O(mu / tau).
      const int R = a.init.rank;
      int bad = (m != n || blocked || !a.init.V || R < 1 || R > 32 || R > nmax) ? 1 : 0;  // n x R scratch in nmax^2 slots
      for (int k = tid; k < m && !bad; k += BT) {
        if (mp[k + 2] - mp[k + 1] != 1) { bad = 1; break; }
        const long long e = mp[k + 1];
        if (er[e] != ec[e] || ev[e] != 1.0 || !(bv[k] > 0.0)) bad = 1;
      }
      for (int t = tid; t < n; t += BT) W1[t] = 0.0;
      __syncthreads();
      for (int k = tid; k < m && !bad; k += BT) atomicAdd(&W1[er[mp[k + 1]]], 1.0);
      __syncthreads();
      for (int t = tid; t < n && !bad; t += BT) bad |= (W1[t] != 1.0);
      bad = __syncthreads_or(bad);
      if (!bad) {
        const double* Vq = a.init.V + a.p.vec_off[inst] * R;
        // C = -F0 and its scale s
        for (int t = tid; t < nn_i; t += BT) Z[t] = 0.0;
        __syncthreads();
        sp_axpy_block<BT>(er, ec, ev, mp[0], mp[1], -1.0, Z, n);
        __syncthreads();
        double cs = 0.0;
        for (int t = tid; t < n; t += BT) cs += fabs(Z[t + (size_t)n * t]);
        cs = cta::block_sum<BT>(cs, RD) / n;
        if (!(cs > 0.0)) cs = 1.0;
        // C V (n x R, in dX; V row-major n x R = column-major R x n, ld R):
        // (F0 Y)_ii = -<v_i, (C V)_i> with Y = V V^T, so x_i = (F0 Y)_ii / b_i
        // per row (in W1) and y_k = -x_{row(k)}
        cta::gemm_rect<BT, double, double>(n, R, n, false, Z, n, true, Vq, R, dX, n, 1.0, 0.0, gsm);
        for (int i = tid; i < n; i += BT) {
          double acc = 0.0;
          for (int k = 0; k < R; ++k) acc += Vq[(size_t)i * R + k] * dX[i + (size_t)n * k];
          W2[i] = -acc;
        }
        __syncthreads();
        for (int k = tid; k < m; k += BT) {
          const int r = er[mp[k + 1]];
          const double xr = W2[r] / bv[k];
          vy[k] = -xr;
          W1[r] = xr;
        }
        __syncthreads();
        sp_axpy_constraints<BT>(er, ec, ev, mp, m, vy, -1.0, Z, n);  // Z = C - sum y_k A_k
        __syncthreads();
        // the factor's stationarity residual rho = |Z V| / (|V| s) (0 at the
        // optimum; Z V = C V + diag(x) V) sets mu: a start closer than the
        // factor's own error stalls
        double zv = 0.0, vv = 0.0;
        for (int t = tid; t < n * R; t += BT) {
          const int i = t % n, k = t / n;
          const double v = Vq[(size_t)i * R + k];
          const double r = dX[t] + W1[i] * v;
          zv += r * r;
          vv += v * v;
        }
        zv = cta::block_sum<BT>(zv, RD);
        vv = cta::block_sum<BT>(vv, RD);
        const double rho = (vv > 0.0) ? sqrt(zv / vv) / cs : 0.0;
        const double mu_s = fmax((a.init.init_mu > 0.0) ? a.init.init_mu : 3.0e-6, 3.0 * rho) * cs;
        const double tau = 0.3 * sqrt(mu_s * cs);
        // (Y + tau I)^-1 = (I - V M^-1 V^T) / tau, M = tau I + V^T V (R x R):
        // M = L L^T in W1, Li = L^-1 in LXi, U = V Li^T (n x R) in dX,
        // Z0 = Z + (mu / tau) (I - U U^T)
        cta::gemm_rect<BT, double, double>(R, R, n, false, Vq, R, true, Vq, R, W1, R, 1.0, 0.0, gsm);
        for (int t = tid; t < R; t += BT) W1[t + R * t] += tau;
        __syncthreads();
        if (cta::cholesky<BT, double>(R, W1, R, false, sD, gsm, &s_flag) == 0) {
          cta::tri_inverse<BT, double>(R, W1, R, LXi, R, sD, gsm);
          cta::gemm_rect<BT, double, double>(n, R, R, true, Vq, R, true, LXi, R, dX, n, 1.0, 0.0, gsm);
          cta::gemm_rect<BT, double, double>(n, n, R, false, dX, n, true, dX, n, W2, n, 1.0, 0.0, gsm);
          const double sc = mu_s / tau;
          for (int t = tid; t < nn_i; t += BT) Z[t] += sc * ((((t % n) == (t / n)) ? 1.0 : 0.0) - W2[t]);
          __syncthreads();
          // the smallest shift of the ladder that leaves Z0 positive definite
          double delta = 0.0;
          int ok = 0;
          for (int step = 0; step < 12 && !ok; ++step) {
            for (int t = tid; t < nn_i; t += BT) W1[t] = Z[t] + (((t % n) == (t / n)) ? delta : 0.0);
            __syncthreads();
            if (cta::cholesky<BT, double>(n, W1, n, false, sD, gsm, &s_flag) == 0) ok = 1;
            else delta = mu_s / n * (double)(1 << (2 * step));
          }
          if (ok) {
            // Z0 shifted by delta (x with it) and Z0^-1.  X0 = mu Z0^-1 (X0 Z0
            // = mu I, the central path's equation) when no shift was needed;
            // a shift means Z has negative curvature beyond the factor's
            // correction, where mu Z0^-1 would be large, and then
            // X0 = Y + mu (Z + tau I)^-1, bounded by tau, with Y = V V^T.
            for (int k = tid; k < m; k += BT) vy[k] -= delta;
            for (int t = tid; t < nn_i; t += BT) if ((t % n) == (t / n)) Z[t] += delta;
            cta::tri_inverse<BT, double>(n, W1, n, LZi, n, sD, gsm);
            cta::gemm<BT>(n, true, LZi, n, false, LZi, n, Zi, n, 1.0, 0.0, gsm);
            if (delta == 0.0) {
              // X0 = mu Z0^-1 = (sqrt(mu) L^-T)(sqrt(mu) L^-T)^T with Z0 = L L^T
              // (L in W1), so L^T / sqrt(mu) is the inverse of a factor of X0:
              // upper triangular, which serves as LXi (the step length's
              // L^-1 dX L^-T has the same spectrum for any factor of X)
              const double ism = 1.0 / sqrt(mu_s);
              for (int t = tid; t < nn_i; t += BT) {
                const int i = t % n, j = t / n;
                X[t] = mu_s * Zi[t];
                LXi[t] = W1[j + (size_t)n * i] * ism;
              }
              __syncthreads();
              warm = true;
            } else {
              // Z + tau I = (Z0 - delta I - mu (Y + tau I)^-1) + tau I, from
              // the unshifted parts still at hand: W2 = U U^T, sc = mu / tau
              for (int t = tid; t < nn_i; t += BT) {
                const bool dg = (t % n) == (t / n);
                W1[t] = Z[t] - sc * ((dg ? 1.0 : 0.0) - W2[t]) + (dg ? tau - delta : 0.0);
              }
              __syncthreads();
              if (cta::cholesky<BT, double>(n, W1, n, false, sD, gsm, &s_flag) != 0) ok = 0;
              if (ok) {
                cta::tri_inverse<BT, double>(n, W1, n, LXi, n, sD, gsm);
                cta::gemm<BT>(n, true, LXi, n, false, LXi, n, D, n, 1.0, 0.0, gsm);
                cta::gemm_rect<BT, double, double>(n, n, R, true, Vq, R, false, Vq, R, X, n, 1.0, 0.0, gsm);
                for (int t = tid; t < nn_i; t += BT) {
                  X[t] += mu_s * D[t];
                  W2[t] = X[t];
                }
              }
            }
            __syncthreads();
            if (!warm && ok && cta::cholesky<BT, double>(n, W2, n, false, sD, gsm, &s_flag) == 0) {
              cta::tri_inverse<BT, double>(n, W2, n, LXi, n, sD, gsm);
              warm = true;
            }
          }
        }
      }
      if (!warm) status = 1;
    }
    if (!warm) {
      for (int t = tid; t < nn_i; t += BT) {
        bool dg = (t % n) == (t / n);
        X[t] = dg ? lam : 0.0;
        Z[t] = dg ? lam : 0.0;
        LXi[t] = dg ? 1.0 / sqrt(lam) : 0.0;
        LZi[t] = dg ? 1.0 / sqrt(lam) : 0.0;
        Zi[t] = dg ? 1.0 / lam : 0.0;
      }
      for (int k = tid; k < m; k += BT) vy[k] = 0.0;
    }
    __syncthreads();
    if (warm) {
      for (int t = tid; t < nn_i; t += BT) { X0[t] = X[t]; Z0[t] = Z[t]; }
      __syncthreads();
    }
    // A start from a proposed x (SDPAB_INIT_DUAL) has Z0 = C - sum y0_k A_k
    // with every A_k diagonal; while every step's dZ stays diagonal, Z - Z0
    // is diagonal and Z0's off-diagonal is C's, so the inner products with
    // the initial point reduce to diagonals:
    //   X0 . Z = X0 . Z0 + sum_i X0_ii (Z_ii - Z0_ii),
    //   X . Z0 = C . X + sum_i X_ii (Z0_ii - C_ii),
    // and X0, Z0 are not read again (their slots leave L2).
    bool diag_track = warm && wmode == SDPAB_INIT_DUAL;
    double x0z0 = 0.0;
    if (diag_track) {
      for (int t = tid; t < n; t += BT) {
        vX0d[t] = X[t * (n + 1)];
        vZ0d[t] = Z[t * (n + 1)];
        vCd[t] = 0.0;
      }
      __syncthreads();
      for (long long e = mp[0] + tid; e < mp[1]; e += BT)
        if (er[e] == ec[e]) atomicAdd(&vCd[er[e]], -ev[e]);  // C = -F0
      __syncthreads();
    }

    residuals(nrp, nrd);
    double mu0;
    if (warm) {
      x0z0 = cta::dot_mat<BT>(n, X, Z, RD);
      mu0 = x0z0 / n;
    } else {
      mu0 = lam * lam;
    }
    {
      double objP = c_dot(X);
      double objD = cta::dot_vec<BT>(m, bv, vy, RD);
      if (tid == 0) {
        init_scalars(S, P, n, mu0, nrp, nrd, objP, objD);
        update_check(S, P);
      }
    }
    __syncthreads();

    // mixed mode: once an FP32 factor fails or its refinement stalls, the
    // rest of the solve factors in FP64
    bool fp64_only = false;
    // x = B^-1 rhs with the FP32 factor in B32 and FP64 iterative refinement
    // against B (full, FP64): x <- x + L32^-T L32^-1 (rhs - B x) until the
    // correction is below REFINE_TOL |x| (the error left is then that times
    // the FP32 solve's own contraction, about cond(B) 6e-8); at most REFINE
    // steps, so a B too ill-conditioned for the FP32 factor returns false (x
    // is then not used) and the solve continues with the FP64 factor.
    auto solve_refined = [&](const double* rhs, double* x) -> bool {
      constexpr int REFINE = 3;
      for (int k = tid; k < m; k += BT) x32[k] = (float)rhs[k];
      __syncthreads();
      cta::chol_solve<BT, float>(m, B32, m, x32, (float*)sD);
      for (int k = tid; k < m; k += BT) x[k] = (double)x32[k];
      __syncthreads();
      const int lane = tid & 31, wid = tid >> 5;
      for (int step = 0; step < REFINE; ++step) {
        // residual rhs - B x, one warp per row (B symmetric: row i = column i)
        for (int i = wid; i < m; i += BT / 32) {
          double acc = 0.0;
          for (int j = lane; j < m; j += 32) acc += B[j + (size_t)m * i] * x[j];
          for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
          if (lane == 0) {
            const double r = rhs[i] - acc;
            vres[i] = r;
            x32[i] = (float)r;
          }
        }
        __syncthreads();
        cta::chol_solve<BT, float>(m, B32, m, x32, (float*)sD);
        double cmax = 0.0, xmax = 0.0;
        for (int k = tid; k < m; k += BT) {
          const double c = (double)x32[k];
          const double xn = x[k] + c;
          x[k] = xn;
          cmax = fmax(cmax, fabs(c));
          xmax = fmax(xmax, fabs(xn));
        }
        double v2[2] = {cmax, xmax}, mx2[2];
        cta::block_max_n<BT, 2>(v2, mx2, RD);
        if (!(mx2[0] == mx2[0])) return false;  // NaN
        if (mx2[0] <= a.refine_tol * mx2[1]) return true;
      }
      return false;
    };
    // adjusted FP64 Cholesky of B in place (solves read the lower triangle):
    // in shared memory when the staging area holds it, else blocked from L2
    auto factor_fp64 = [&]() -> int {
      if (a.factor_smem && cta::cholesky_smem_elems(m) <= (long long)gsm_doubles)
        return cta::cholesky_smem<BT, double, double>(m, B, m, B, m, true, gsm, &s_flag);
      return cta::cholesky<BT, double>(m, B, m, true, sD, gsm, &s_flag, false);
    };
    int iter = 0;
    for (;;) {
      if (tid == 0) s_flag = update_check(S, P) ? 1 : 0;
      __syncthreads();
      if (!s_flag || iter >= P.maxIteration) break;
      if (tid == 0) predictor_setup(S, P);
      __syncthreads();
      const bool dinf = dual_infeasible(S);
      const double bm = S.beta * S.mu;
      // mixed precision: FP32 products while mu is above the switch point
      const bool lowp = a.mixed && attempt == 0 && !fp64_only && mixed_gap(S) >= a.mu_switch;
      const bool lowp_prod = lowp && a.mixed_products;
      // every constraint diagonal and the point dual feasible: dZ is diagonal,
      // so products with dZ are column scalings (exactly what the GEMM with a
      // diagonal factor computes)
      const bool dz_diag = diag_cons && !dinf;

      // ---- predictor: rMat and gVec (sdpa_newton.cpp:793-883)
      for (int t = tid; t < nn_i; t += BT) R[t] = bm * Zi[t] - X[t];
      __syncthreads();
      const double* G = R;
      if (dinf) {
        cta::gemm_prec<BT, double>(n, false, X, n, false, D, n, W1, n, 1.0, 0.0, gsm, lowp_prod);
        cta::gemm_prec<BT, double>(n, false, W1, n, false, Zi, n, XDZ, n, 1.0, 0.0, gsm, lowp_prod);
        for (int t = tid; t < nn_i; t += BT) W2[t] = R[t] - XDZ[t];
        __syncthreads();
        G = W2;
      }
      for (int k = tid; k < m; k += BT) vg[k] = -sp_dot(er, ec, ev, mp[k + 1], mp[k + 2], G, n) + vrp[k];
      // ---- Schur complement by F3 (compute_bMat_dense_SDP3, sdpa_newton.cpp:2019-2125)
      // for the pairs whose dominant constraint is F3, then the F1 columns
      for (int t = tid; t < m * m; t += BT) {
        const int i = t % m, j = t / m;
        const int inz = s_nnz[i], jnz = s_nnz[j];
        if (jnz < inz || (inz == jnz && i < j)) continue;
        if (GENERAL && any_f1 && s_form[j]) continue;
        double v = f3_value(er, ec, ev, mp[j + 1], mp[j + 2], mp[i + 1], mp[i + 2], X, Zi, n);
        B[i + (size_t)m * j] = v;
        B[j + (size_t)m * i] = v;
      }
      __syncthreads();
      if (GENERAL && any_f1) {
        if (blocked)
          schur_f1<BT>(n, m, mp, er, ec, ev, X, Zi, W1, W2, dX, B, s_nnz, s_form, s_nb, s_boff, s_bsz, s_bid, gsm);
        else
          schur_f1<BT>(n, m, mp, er, ec, ev, X, Zi, W1, W2, dX, B, s_nnz, s_form, 0, nullptr, nullptr, nullptr, gsm);
      }
      // ---- adjusted Cholesky and solve (compute_DyVec, sdpa_newton.cpp:2672-2716).
      // Mixed mode (FP32 phase): the factor in FP32 (the same adjust rule) of
      // an FP32 copy of B, each solve refined in FP64 against B; a factor
      // that fails, or a solve whose refinement does not converge, sends this
      // iteration and the rest of the solve to the FP64 factor.
      bool f32 = false;
      if (lowp) {
        if (a.factor_smem && cta::cholesky_smem_elems(m) <= 2LL * gsm_doubles) {
          f32 = cta::cholesky_smem<BT, float, double>(m, B, m, B32, m, true, (float*)gsm, &s_flag) == 0;
        } else {
          for (int t = tid; t < m * m; t += BT) B32[t] = (float)B[t];
          __syncthreads();
          f32 = cta::cholesky<BT, float>(m, B32, m, true, (float*)sD, gsm, &s_flag, false) == 0;
        }
        if (f32) f32 = solve_refined(vg, vdy);
        if (!f32) fp64_only = true;
      }
      if (!f32) {
        if (factor_fp64()) break;
        for (int k = tid; k < m; k += BT) vdy[k] = vg[k];
        __syncthreads();
        cta::chol_solve<BT, double>(m, B, m, vdy, sD);
      }

      // ---- dZ, dX (compute_DzMat / compute_DxMat, sdpa_newton.cpp:2718-2752).
      // With every constraint diagonal and the point dual feasible, dZ =
      // -sum dy_k A_k is diagonal: it is kept as the vector vdz (the full
      // matrix dZ is not written), X dZ is a column scaling, and the inner
      // products and the update with dZ touch the diagonal only.
      auto direction = [&]() {
        if (dz_diag) {
          for (int t = tid; t < n; t += BT) vdz[t] = 0.0;
          __syncthreads();
          for (int k = tid; k < m; k += BT) {
            const double s = -vdy[k];
            for (long long e = mp[k + 1]; e < mp[k + 2]; ++e) atomicAdd(&vdz[er[e]], s * ev[e]);
          }
          __syncthreads();
          for (int t = tid; t < nn_i; t += BT) W1[t] = X[t] * vdz[t / n];
          __syncthreads();
        } else {
          for (int t = tid; t < nn_i; t += BT) dZ[t] = dinf ? D[t] : 0.0;
          __syncthreads();
          sp_axpy_constraints<BT>(er, ec, ev, mp, m, vdy, -1.0, dZ, n);
          __syncthreads();
          cta::gemm_prec<BT, double>(n, false, X, n, false, dZ, n, W1, n, 1.0, 0.0, gsm, lowp_prod);
        }
        cta::gemm_prec<BT, double>(n, false, W1, n, false, Zi, n, W2, n, 1.0, 0.0, gsm, lowp_prod);
        for (int t = tid; t < nn_i; t += BT) {
          const int i = t % n, j = t / n;
          if (i >= j) {
            double lo = R[i + n * j] - W2[i + n * j];
            double up = R[j + n * i] - W2[j + n * i];
            double s = 0.5 * (lo + up);
            dX[i + n * j] = s;
            dX[j + n * i] = s;
          }
        }
        __syncthreads();
      };
      // A . dZ (A = X or dX): the diagonal only when dZ is diagonal
      auto dot_dz = [&](const double* A) {
        if (!dz_diag) return cta::dot_mat<BT>(n, A, dZ, RD);
        double s = 0.0;
        for (int t = tid; t < n; t += BT) s += A[t * (n + 1)] * vdz[t];
        return cta::block_sum<BT>(s, RD);
      };
      direction();
      {
        double CdX = c_dot(dX);
        double bdy = cta::dot_vec<BT>(m, bv, vdy, RD);
        double xdz = dot_dz(X);
        double dxz = cta::dot_mat<BT>(n, dX, Z, RD);
        double dxdz = dot_dz(dX);
        if (tid == 0) {
          predictor_step(S, CdX, bdy);
          corrector_beta(S, P, xdz, dxz, dxdz);
        }
        __syncthreads();
      }

      // ---- corrector (Newton::Mehrotra(CORRECTOR))
      {
        const double bm2 = S.beta * S.mu;
        if (dz_diag) {
          for (int t = tid; t < nn_i; t += BT) W1[t] = dX[t] * vdz[t / n];
          __syncthreads();
        } else {
          cta::gemm_prec<BT, double>(n, false, dX, n, false, dZ, n, W1, n, 1.0, 0.0, gsm, lowp_prod);
        }
        cta::gemm_prec<BT, double>(n, false, W1, n, false, Zi, n, W2, n, 1.0, 0.0, gsm, lowp_prod);
        for (int t = tid; t < nn_i; t += BT) {
          double rr = bm2 * Zi[t] - X[t];
          rr = rr - W2[t];
          R[t] = rr;
          W1[t] = dinf ? rr - XDZ[t] : rr;
        }
        __syncthreads();
        for (int k = tid; k < m; k += BT) vg[k] = -sp_dot(er, ec, ev, mp[k + 1], mp[k + 2], W1, n) + vrp[k];
        __syncthreads();
        bool refined = f32 && solve_refined(vg, vdy);
        if (f32 && !refined) {
          // the FP32 factor does not carry this right-hand side: FP64 factor
          // (B is intact: the FP32 path never factors it in place)
          fp64_only = true;
          if (factor_fp64()) break;
        }
        if (!refined) {
          for (int k = tid; k < m; k += BT) vdy[k] = vg[k];
          __syncthreads();
          cta::chol_solve<BT, double>(m, B, m, vdy, sD);
        }
        direction();
      }

      // ---- step length (StepLength::MehrotraCorrector)
      {
        // R and XDZ are free here (both are rebuilt by the next predictor)
        double mins[2];
        const double* DZ = dz_diag ? vdz : dZ;  // the diagonal vector when dZ is diagonal
        if (GENERAL && blocked)
          min_eig_pair_blocks<BT>(n, s_nb, s_boff, s_bsz, LXi, dX, LZi, DZ, W1, W2, R, XDZ, gsm, gsm_doubles, es,
                              mins, dz_diag);
        else
          min_eig_pair<BT>(n, LXi, dX, LZi, DZ, W1, W2, R, XDZ, gsm, gsm_doubles, es, mins, dz_diag);
        const double minX = mins[0], minZ = mins[1];
        double CdX = c_dot(dX);
        double bdy = cta::dot_vec<BT>(m, bv, vdy, RD);
        double xdz = dot_dz(X);
        double dxz = cta::dot_mat<BT>(n, dX, Z, RD);
        double dxdz = dot_dz(dX);
        if (tid == 0) corrector_step(S, P, minX, minZ, CdX, bdy, xdz, dxz, dxdz, S.objD, S.objP);
        __syncthreads();
      }

      // ---- update (Solutions::update, sdpa_dataset.cpp:145-171)
      {
        const double ap = S.alphaP, ad = S.alphaD;
        diag_track = diag_track && dz_diag;
        // X += ap dX, Z += ad dZ, and the copies the factorisations work on
        for (int t = tid; t < nn_i; t += BT) {
          const double x = X[t] + ap * dX[t];
          double z = Z[t];
          if (!dz_diag) z += ad * dZ[t];
          else if ((t % n) == (t / n)) z += ad * vdz[t / n];
          X[t] = x;
          Z[t] = z;
          W2[t] = x;
          W1[t] = z;
        }
        for (int k = tid; k < m; k += BT) vy[k] += ad * vdy[k];
        __syncthreads();
        if (cannot_move(S)) break;
        // X and Z factored and inverted in lockstep (either failing ends the loop)
        if (cta::cholesky_pair<BT, double>(n, W2, W1, n, sD, sD2, gsm, s_flag2, false))
          break;  // the inverses read the lower triangles only
        cta::tri_inverse_pair<BT, double>(n, W2, W1, n, LXi, LZi, n, sD, sD2, gsm);
        cta::gemm<BT>(n, true, LZi, n, false, LZi, n, Zi, n, 1.0, 0.0, gsm);
      }
      // ---- residuals and scalars
      {
        double xz = cta::dot_mat<BT>(n, X, Z, RD);
        residuals(nrp, nrd);
        double objP = c_dot(X);
        double objD = cta::dot_vec<BT>(m, bv, vy, RD);
        double x0zM, xMz0;
        if (diag_track) {
          double v2[2] = {0.0, 0.0};
          for (int t = tid; t < n; t += BT) {
            v2[0] += vX0d[t] * (Z[t * (n + 1)] - vZ0d[t]);
            v2[1] += X[t * (n + 1)] * (vZ0d[t] - vCd[t]);
          }
          double s2[2];
          cta::block_sum_n<BT, 2>(v2, s2, RD);
          x0zM = x0z0 + s2[0];
          xMz0 = objP + s2[1];
        } else if (warm) {
          x0zM = cta::dot_mat<BT>(n, X0, Z, RD);
          xMz0 = cta::dot_mat<BT>(n, X, Z0, RD);
        } else {
          x0zM = lam * cta::trace<BT>(n, Z, RD);
          xMz0 = lam * cta::trace<BT>(n, X, RD);
        }
        if (tid == 0) after_update(S, P, xz, nrp, nrd, objP, objD, x0zM, xMz0);
        __syncthreads();
      }
      ++iter;
    }
    iter_total += iter;
    if (attempt == 0 && (warm || a.mixed) && S.phase != pdOPT) {
      status = 2;
      __syncthreads();
      continue;
    }
    break;
    }  // attempts
    // final residuals (sdpa_solve.cpp:204) and results
    residuals(nrp, nrd);
    if (tid == 0) {
      a.r.primal_obj[inst] = -S.objD;
      a.r.dual_obj[inst] = -S.objP;
      a.r.mu[inst] = S.mu;
      a.r.primal_error[inst] = nrd;
      a.r.dual_error[inst] = nrp;
      a.r.iterations[inst] = iter_total;
      a.r.phase[inst] = user_phase(S.phase);
      a.r.status[inst] = status;
    }
    if (a.r.xvec) {
      double* xo = a.r.xvec + a.p.vec_off[inst];
      for (int k = tid; k < m; k += BT) xo[k] = -vy[k];
    }
    if (a.r.X) {
      double* o = a.r.X + a.p.dense_off[inst];
      for (int t = tid; t < nn_i; t += BT) o[t] = Z[t];
    }
    if (a.r.Y) {
      double* o = a.r.Y + a.p.dense_off[inst];
      for (int t = tid; t < nn_i; t += BT) o[t] = X[t];
    }
    __syncthreads();
  }
}

// Host side -----------------------------------------------------------------

// The instantiation for a batch: block-aware only when it carries a
// structure; 256 or 128 threads per instance.
static void* solver_kernel(const sdpab_batch* prob, int bt)
{
  if (bt == 128)
    return prob->nblock ? (void*)batch_ipm_fp64<true, 128> : (void*)batch_ipm_fp64<false, 128>;
  return prob->nblock ? (void*)batch_ipm_fp64<true, 256> : (void*)batch_ipm_fp64<false, 256>;
}

// Launch shape of the solver: threads per block (instance), resident blocks
// per SM, staging doubles and dynamic shared memory bytes.
struct LaunchShape {
  int bt, per_sm;
  long long gsm;
  size_t shm;
};

// Threads per block from the configuration (256 by default, or 128), and
// the blocks per SM it asks for (default: 2 of 256 threads, 4 of 128); the
// staging area is sized for that many, and the occupancy the device reports
// caps it.
static int launch_shape(const sdpab_batch* prob, int want_bt, int want_per_sm, int want_staging, int dev,
                        LaunchShape& L, const char* who)
{
  L.bt = (want_bt == 128) ? 128 : 256;
  const int per_sm_req = (want_per_sm > 0) ? want_per_sm : (L.bt == 128 ? 4 : 2);
  L.gsm = staging_doubles(prob->nmax, prob->mmax, want_staging, L.bt, per_sm_req);
  void* k = solver_kernel(prob, L.bt);
  int per_sm = 0;
  // the default staging is the budget of per_sm_req blocks; should the
  // device fit fewer of that size, it shrinks (1 KB at a time) to the size
  // that fits them
  for (;;) {
    L.shm = smem_bytes_for(prob->nmax, prob->mmax, L.gsm, L.bt);
    if (L.shm > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.shm);
      if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute");
    }
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, L.bt, L.shm);
    if (e != cudaSuccess) return cuda_error(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (per_sm >= per_sm_req || want_staging > 0 || L.gsm - 128 < staging_min(L.bt)) break;
    L.gsm -= 128;
  }
  if (per_sm < 1) {
    char msg[160];
    snprintf(msg, sizeof(msg), "%s: the solver block does not fit on an SM", who);
    return set_error(SDPAB_ESIZE, msg);
  }
  L.per_sm = std::min(per_sm, per_sm_req);
  (void)dev;
  return SDPAB_OK;
}

static void launch_solver(const sdpab_batch* prob, const LaunchShape& L, int grid, const BatchArgs& a,
                          cudaStream_t stream)
{
  if (L.bt == 128) {
    if (prob->nblock) batch_ipm_fp64<true, 128><<<grid, 128, L.shm, stream>>>(a);
    else batch_ipm_fp64<false, 128><<<grid, 128, L.shm, stream>>>(a);
  } else {
    if (prob->nblock) batch_ipm_fp64<true, 256><<<grid, 256, L.shm, stream>>>(a);
    else batch_ipm_fp64<false, 256><<<grid, 256, L.shm, stream>>>(a);
  }
}

static long long ws_doubles(int nmax, int mmax, bool mixed)
{
  long long nn = (long long)nmax * nmax;
  const long long mm = (long long)mmax * mmax;
  // 14 n x n, the Schur matrix and, in mixed precision, its FP32 factor (last)
  long long s = 14 * nn + mm + (mixed ? (mm + 1) / 2 : 0);
  return (s + 31) / 32 * 32;  // 256-byte aligned per block
}

int batch_solve_device(const sdpab_batch* prob, const sdpab_batch_init* init,
                       const sdpab_params* prm, const sdpab_batch_config* cfg,
                       sdpab_batch_result* res, const int* order, cudaStream_t stream)
{
  if (!prob || !prm || !res || prob->count < 0 || prob->nmax < 1 || prob->mmax < 1)
    return set_error(SDPAB_EINVAL, "batch_solve: invalid arguments");
  if (prob->count == 0) return SDPAB_OK;
  if (prob->nmax > 1024 || prob->mmax > 2048)
    return set_error(SDPAB_ESIZE, "batch_solve: nmax <= 1024 and mmax <= 2048 are supported");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDPAB_ENODEV, "no CUDA device");
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  LaunchShape L;
  int rc = launch_shape(prob, cfg ? cfg->block_threads : 0, cfg ? cfg->ctas_per_sm : 0,
                        cfg ? cfg->staging_doubles : 0, dev, L, "batch_solve");
  if (rc != SDPAB_OK) return rc;
  int grid = std::min(prob->count, sms * L.per_sm);
  const long long stride = ws_doubles(prob->nmax, prob->mmax, cfg && cfg->precision == SDPAB_PREC_MIXED);
  Workspace& W = workspace();
  double* ws = (double*)W.get((size_t)grid * stride * sizeof(double) + 256);
  if (!ws) return set_error(SDPAB_ECUDA, "workspace allocation failed");
  int* queue = W.counter();
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
  if (e != cudaSuccess) return cuda_error(e, "cudaMemsetAsync");
  BatchArgs a;
  a.p = *prob;
  if (init) a.init = *init; else memset(&a.init, 0, sizeof(a.init));
  a.r = *res;
  memcpy(&a.prm, prm, sizeof(Params));
  a.order = order;
  a.gsm_doubles = (int)L.gsm;
  a.mixed = (cfg && cfg->precision == SDPAB_PREC_MIXED) ? 1 : 0;
  a.mixed_products = (cfg && cfg->mixed_products) ? 1 : 0;
  a.mu_switch = (cfg && cfg->mixed_switch_gap > 0.0) ? cfg->mixed_switch_gap : 1.0e-2;
  a.refine_tol = (cfg && cfg->refine_tol > 0.0) ? cfg->refine_tol : 1.0e-8;
  a.factor_smem = (cfg && cfg->factor_smem) ? 1 : 0;
  a.ws = ws;
  a.ws_stride = stride;
  a.queue = queue;
  launch_solver(prob, L, grid, a, stream);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "batch_ipm_fp64 launch");
  return SDPAB_OK;
}

// No-allocation variant of the batched solve ---------------------------------
//
// Some callers cannot call cudaMalloc once they are running: a process whose
// own memory pool has already reserved the device's memory, or a service that
// must not allocate after start-up because cudaMalloc synchronises the device
// and can fail when memory is tight or fragmented.  For them the batched
// solver can run on a fixed scratch region that is part of this library
// instead of the growable workspace.  The region is a file-scope device
// array, so every GPU that loads the library holds it until the process
// exits.  Host code must not use the array's name as a device address: the
// address is looked up with cudaGetSymbolAddress on every call, on the
// device that is current (a cached address would go stale after
// cudaDeviceReset; the lookup allocates nothing), and the first call on a
// device also loads the module there, so make that first call before any
// stream capture.  All calls share the one region and it keeps the previous
// call's contents; the work-queue counter is cleared on every call, and two
// calls that overlap on the GPU race on the region.
static __device__ __align__(256) double g_noalloc_scratch[SDPAB_NOALLOC_SCRATCH_BYTES / sizeof(double)];

int batch_solve_noalloc(const sdpab_batch* prob, const sdpab_batch_init* init,
                        const sdpab_params* prm, sdpab_batch_result* res, const int* order,
                        cudaStream_t stream)
{
  if (!prob || !prm || !res || prob->count < 0 || prob->nmax < 1 || prob->mmax < 1)
    return set_error(SDPAB_EINVAL, "batch_solve_noalloc: invalid arguments");
  if (prob->count == 0) return SDPAB_OK;
  if (prob->nmax > 1024 || prob->mmax > 2048)
    return set_error(SDPAB_ESIZE, "batch_solve_noalloc: nmax <= 1024 and mmax <= 2048 are supported");
  const long long stride = ws_doubles(prob->nmax, prob->mmax, false);  // FP64 only: no FP32 factor
  const long long head = 32;  // doubles reserved for the work-queue counter
  const long long capacity = ((long long)(SDPAB_NOALLOC_SCRATCH_BYTES / sizeof(double)) - head) / stride;
  if (capacity < 1) {
    char msg[200];
    snprintf(msg, sizeof(msg),
             "batch_solve_noalloc: one block's workspace (14*nmax^2 + mmax^2 doubles) exceeds the "
             "%llu MiB scratch region; use sdpab_batch_solve",
             (unsigned long long)(SDPAB_NOALLOC_SCRATCH_BYTES >> 20));
    return set_error(SDPAB_ESIZE, msg);
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDPAB_ENODEV, "batch_solve_noalloc: no CUDA device");
  void* sym = nullptr;
  {
    cudaError_t e = cudaGetSymbolAddress(&sym, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "batch_solve_noalloc: cudaGetSymbolAddress");
  }
  double* base = (double*)sym;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  LaunchShape L;
  int rc = launch_shape(prob, 256, 2, 0, dev, L, "batch_solve_noalloc");
  if (rc != SDPAB_OK) return rc;
  const long long grid = std::min<long long>(std::min<long long>(prob->count, (long long)sms * L.per_sm),
                                             capacity);
  int* queue = (int*)base;
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int), stream);
  if (e != cudaSuccess) return cuda_error(e, "batch_solve_noalloc: clearing the queue counter");
  BatchArgs a;
  a.p = *prob;
  if (init) a.init = *init; else memset(&a.init, 0, sizeof(a.init));
  a.r = *res;
  memcpy(&a.prm, prm, sizeof(Params));
  a.order = order;
  a.gsm_doubles = (int)L.gsm;
  a.mixed = 0;
  a.mixed_products = 0;
  a.mu_switch = 1.0e-2;
  a.refine_tol = 1.0e-8;
  a.factor_smem = 0;
  a.ws = base + head;
  a.ws_stride = stride;
  a.queue = queue;
  launch_solver(prob, L, (int)grid, a, stream);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_error(e, "batch_solve_noalloc: launch");
  return SDPAB_OK;
}

}  // namespace sdpab

extern "C" int sdpab_batch_solve_noalloc(const sdpab_batch* prob, const sdpab_batch_init* init,
                                         const sdpab_params* prm, sdpab_batch_result* res,
                                         const int* order, void* stream)
{
  return sdpab::batch_solve_noalloc(prob, init, prm, res, order, (cudaStream_t)stream);
}
