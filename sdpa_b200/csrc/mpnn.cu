// Message-passing network that proposes the dual vector x of a MaxCut SDP
// from its graph (the learned warm start; no counterpart in the reference).
//
//   h0 = node features (F0)
//   h_{l+1} = relu(h_l Ws_l^T + (A h_l) Wn_l^T + b_l),  l = 0, 1, 2  (hidden H)
//   r = h_3 w_o + b_o          (per node: x_i = r_i * d_i / 4)
// A is the row-normalised weighted adjacency a_ij = w_ij / (d_i + 1).
// Weights are used in BF16 (a master FP32 copy is kept for the optimiser);
// every product accumulates in FP32.  Forward, backward (loss = mean squared
// error over masked nodes) and Adam are hand-written SIMT kernels in FP32
// (a layer over a 4096-graph batch is ~14 GFLOP and ~0.3 GB of activations,
// a fraction of a millisecond either way).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "sdpa_b200.h"
#include "sdpab_internal.h"

namespace sdpab {

constexpr int H = SDPAB_MPNN_HIDDEN;
constexpr int F0 = SDPAB_MPNN_FEATURES;
constexpr int L = SDPAB_MPNN_LAYERS;

__host__ __device__ inline int fin_of(int l) { return l == 0 ? F0 : H; }
// flat parameter offsets: per layer Ws (H x Fin), Wn (H x Fin), b (H); then w_o (H), b_o (1)
__host__ __device__ inline long long off_ws(int l)
{
  long long o = 0;
  for (int q = 0; q < l; ++q) o += 2LL * H * fin_of(q) + H;
  return o;
}
__host__ __device__ inline long long off_wn(int l) { return off_ws(l) + (long long)H * fin_of(l); }
__host__ __device__ inline long long off_b(int l) { return off_wn(l) + (long long)H * fin_of(l); }
__host__ __device__ inline long long off_out() { return off_ws(L); }
__host__ __device__ inline long long n_params() { return off_out() + H + 1; }

// Y[i, :] = sum_e val[e] X[col[e], :]   (one thread per (node, feature))
__global__ void k_spmm(int N, int F, const int* rowptr, const int* col, const float* val, const float* X,
                       float* Y)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)N * F) return;
  const int i = (int)(t / F), f = (int)(t % F);
  float s = 0.0f;
  for (int e = rowptr[i]; e < rowptr[i + 1]; ++e) s = fmaf(val[e], X[(long long)col[e] * F + f], s);
  Y[t] = s;
}

// z = h Ws^T + agg Wn^T + b; hout = relu(z).  A block covers FWD_NODES
// nodes: the layer's weights are staged transposed (k-major, so the 32
// lanes of a warp read 32 consecutive output features: no bank conflicts)
// and the nodes' h and agg rows are staged once; thread (j, g) computes
// output feature j of nodes g, g + 4, ... from registers.  The products are
// accumulated in the same order for every node (per k: agg term, then h
// term), FP32 throughout.
constexpr int FWD_NODES = 32;
constexpr int FWD_PER = FWD_NODES / 4;  // nodes per thread (256 threads = 64 features x 4)
__global__ void __launch_bounds__(256) k_dense_fwd(int N, int Fin, const float* h, const float* agg,
                                                   const __nv_bfloat16* Ws, const __nv_bfloat16* Wn,
                                                   const __nv_bfloat16* b, float* z, float* hout)
{
  __shared__ float sWs[H * H], sWn[H * H];                        // [k][j]
  __shared__ __align__(16) float sh[FWD_NODES * H], sa[FWD_NODES * H];  // [node][k]
  for (int t = threadIdx.x; t < H * Fin; t += blockDim.x) {
    const int jj = t / Fin, k = t % Fin;  // source layout [j][k]
    sWs[k * H + jj] = __bfloat162float(Ws[t]);
    sWn[k * H + jj] = __bfloat162float(Wn[t]);
  }
  const int i0 = blockIdx.x * FWD_NODES;
  const int cnt = min(FWD_NODES, N - i0);
  for (int t = threadIdx.x; t < FWD_NODES * Fin; t += blockDim.x) {
    const int r = t / Fin;
    const bool ok = r < cnt;
    sh[t] = ok ? h[(long long)i0 * Fin + t] : 0.0f;
    sa[t] = ok ? agg[(long long)i0 * Fin + t] : 0.0f;
  }
  __syncthreads();
  const int j = threadIdx.x % H, g = threadIdx.x / H;
  const float bj = __bfloat162float(b[j]);
  float acc[FWD_PER];
#pragma unroll
  for (int u = 0; u < FWD_PER; ++u) acc[u] = bj;
  for (int k = 0; k < Fin; ++k) {
    const float ws = sWs[k * H + j], wn = sWn[k * H + j];
#pragma unroll
    for (int u = 0; u < FWD_PER; ++u) {
      const int r = g + 4 * u;
      acc[u] = fmaf(sh[r * Fin + k], ws, fmaf(sa[r * Fin + k], wn, acc[u]));
    }
  }
#pragma unroll
  for (int u = 0; u < FWD_PER; ++u) {
    const int r = g + 4 * u;
    if (r < cnt) {
      const long long o = (long long)(i0 + r) * H + j;
      z[o] = acc[u];
      hout[o] = acc[u] > 0.0f ? acc[u] : 0.0f;
    }
  }
}

// readout, loss and its gradient: r_i = h_i . w_o + b_o;
// loss = sum_i mask_i (r_i - t_i)^2 / cnt; dr_i = 2 mask_i (r_i - t_i) / cnt
__global__ void k_readout(int N, const float* h, const __nv_bfloat16* wo, const float* target,
                          const float* mask, float inv_cnt, float* r, float* dr, float* loss)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float s = __bfloat162float(wo[H]);
  for (int j = 0; j < H; ++j) s = fmaf(h[(long long)i * H + j], __bfloat162float(wo[j]), s);
  r[i] = s;
  if (target) {
    const float m = mask ? mask[i] : 1.0f;
    const float d = (s - target[i]) * m;
    dr[i] = 2.0f * d * inv_cnt;
    atomicAdd(loss, d * d * inv_cnt);
  }
}

// dh3 = dr (x) w_o ; grads of w_o, b_o (per-block partial sums, then atomics)
__global__ void k_readout_bwd(int N, const float* h, const float* dr, const __nv_bfloat16* wo, float* dh,
                              float* gwo)
{
  __shared__ float part[H + 1];
  for (int t = threadIdx.x; t <= H; t += blockDim.x) part[t] = 0.0f;
  __syncthreads();
  const int j = threadIdx.x % H;
  const int per = blockDim.x / H;
  float acc = 0.0f, accb = 0.0f;
  for (int i = blockIdx.x * per + threadIdx.x / H; i < N; i += gridDim.x * per) {
    dh[(long long)i * H + j] = dr[i] * __bfloat162float(wo[j]);
    acc = fmaf(dr[i], h[(long long)i * H + j], acc);
    if (j == 0) accb += dr[i];
  }
  atomicAdd(&part[j], acc);
  if (j == 0) atomicAdd(&part[H], accb);
  __syncthreads();
  for (int t = threadIdx.x; t <= H; t += blockDim.x) atomicAdd(&gwo[t], part[t]);
}

// dz = dh * (z > 0)
__global__ void k_relu_bwd(long long n, const float* z, const float* dh, float* dz)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) dz[t] = z[t] > 0.0f ? dh[t] : 0.0f;
}

// weight gradients: gWs += dz^T h, gWn += dz^T agg, gb += sum dz.  Each block
// reduces a chunk of nodes for all (j, k) pairs, then adds atomically.
__global__ void k_dense_bwd_w(int N, int Fin, const float* dz, const float* h, const float* agg, float* gWs,
                              float* gWn, float* gb)
{
  constexpr int CH = 64;
  __shared__ float sdz[CH][H], sh[CH][H], sa[CH][H];
  const int pairs = H * Fin;
  float accs[16], accn[16], accb = 0.0f;
  for (int u = 0; u < 16; ++u) accs[u] = accn[u] = 0.0f;
  for (int i0 = blockIdx.x * CH; i0 < N; i0 += gridDim.x * CH) {
    __syncthreads();
    for (int t = threadIdx.x; t < CH * H; t += blockDim.x) {
      const int r = t / H, c = t % H, i = i0 + r;
      sdz[r][c] = (i < N) ? dz[(long long)i * H + c] : 0.0f;
      if (c < Fin) {
        sh[r][c] = (i < N) ? h[(long long)i * Fin + c] : 0.0f;
        sa[r][c] = (i < N) ? agg[(long long)i * Fin + c] : 0.0f;
      }
    }
    __syncthreads();
    for (int u = 0; u < 16; ++u) {
      const int p = threadIdx.x + u * blockDim.x;
      if (p >= pairs) break;
      const int j = p / Fin, k = p % Fin;
      float s = 0.0f, sn = 0.0f;
      for (int r = 0; r < CH; ++r) {
        s = fmaf(sdz[r][j], sh[r][k], s);
        sn = fmaf(sdz[r][j], sa[r][k], sn);
      }
      accs[u] += s;
      accn[u] += sn;
    }
    if (threadIdx.x < H)
      for (int r = 0; r < CH; ++r) accb += sdz[r][threadIdx.x];
  }
  for (int u = 0; u < 16; ++u) {
    const int p = threadIdx.x + u * blockDim.x;
    if (p >= pairs) break;
    atomicAdd(&gWs[p], accs[u]);
    atomicAdd(&gWn[p], accn[u]);
  }
  if (threadIdx.x < H) atomicAdd(&gb[threadIdx.x], accb);
}

// dh_self = dz Ws ; dagg = dz Wn   (one thread per (node, k))
__global__ void k_dense_bwd_x(int N, int Fin, const float* dz, const __nv_bfloat16* Ws, const __nv_bfloat16* Wn,
                              float* dh, float* dagg)
{
  __shared__ float sWs[H * H], sWn[H * H];
  for (int t = threadIdx.x; t < H * Fin; t += blockDim.x) {
    sWs[t] = __bfloat162float(Ws[t]);
    sWn[t] = __bfloat162float(Wn[t]);
  }
  __syncthreads();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)N * Fin) return;
  const int i = (int)(t / Fin), k = (int)(t % Fin);
  float s = 0.0f, sn = 0.0f;
  for (int j = 0; j < H; ++j) {
    const float d = dz[(long long)i * H + j];
    s = fmaf(d, sWs[j * Fin + k], s);
    sn = fmaf(d, sWn[j * Fin + k], sn);
  }
  dh[t] = s;
  dagg[t] = sn;
}

__global__ void k_add(long long n, float* a, const float* b)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) a[t] += b[t];
}

// Adam on the FP32 master weights; the BF16 working copy is refreshed.
__global__ void k_adam(long long n, float* w, __nv_bfloat16* wb, const float* g, float* m1, float* m2, float lr,
                       float b1, float b2, float eps, float c1, float c2, float wd)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gr = g[t] + wd * w[t];
  m1[t] = b1 * m1[t] + (1.0f - b1) * gr;
  m2[t] = b2 * m2[t] + (1.0f - b2) * gr * gr;
  const float mh = m1[t] / c1, vh = m2[t] / c2;
  w[t] -= lr * mh / (sqrtf(vh) + eps);
  wb[t] = __float2bfloat16(w[t]);
}

__global__ void k_to_bf16(long long n, const float* w, __nv_bfloat16* wb)
{
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < n) wb[t] = __float2bfloat16(w[t]);
}

static inline int nb(long long n, int t = 256) { return (int)((n + t - 1) / t); }

// x_i = r_i d_i / 4 (nodes with edges), fallback_i otherwise
__global__ void k_propose(int n, const float* r, const double* degree, const double* fallback, double* x)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x[i] = (degree[i] > 1.0e-9) ? (double)r[i] * degree[i] * 0.25 : fallback[i];
}

// Activation layout inside act: per layer l: h_l (N x Fin_l), agg_l (N x Fin_l),
// z_l (N x H); then h_L (N x H), r (N).
struct Act {
  float *h[L + 1], *agg[L], *z[L], *r;
};
static Act carve(float* act, int N)
{
  Act a;
  float* p = act;
  for (int l = 0; l < L; ++l) {
    a.h[l] = p; p += (long long)N * fin_of(l);
    a.agg[l] = p; p += (long long)N * fin_of(l);
    a.z[l] = p; p += (long long)N * H;
  }
  a.h[L] = p; p += (long long)N * H;
  a.r = p;
  return a;
}

static long long act_floats(int N)
{
  long long s = 0;
  for (int l = 0; l < L; ++l) s += 2LL * N * fin_of(l) + (long long)N * H;
  return s + (long long)N * H + N;
}

static long long scratch_floats(int N) { return 4LL * N * H + N; }

static void forward(const sdpab_graph_batch* g, const __nv_bfloat16* wb, const Act& a, cudaStream_t st)
{
  const int N = g->num_nodes;
  cudaMemcpyAsync(a.h[0], g->feat, sizeof(float) * (size_t)N * F0, cudaMemcpyDeviceToDevice, st);
  for (int l = 0; l < L; ++l) {
    const int Fin = fin_of(l);
    k_spmm<<<nb((long long)N * Fin), 256, 0, st>>>(N, Fin, g->rowptr, g->col, g->aval, a.h[l], a.agg[l]);
    k_dense_fwd<<<nb(N, FWD_NODES), 256, 0, st>>>(N, Fin, a.h[l], a.agg[l], wb + off_ws(l), wb + off_wn(l), wb + off_b(l),
                                          a.z[l], a.h[l + 1]);
  }
}

}  // namespace sdpab

using namespace sdpab;

extern "C" {

SDPAB_API long long sdpab_mpnn_num_params(void) { return n_params(); }
SDPAB_API long long sdpab_mpnn_act_floats(int num_nodes) { return act_floats(num_nodes); }
SDPAB_API long long sdpab_mpnn_scratch_floats(int num_nodes) { return scratch_floats(num_nodes); }

SDPAB_API int sdpab_mpnn_forward(const sdpab_graph_batch* g, const unsigned short* weights_bf16, float* act,
                                 float* out, void* stream)
{
  if (!g || !weights_bf16 || !act || !out || g->num_nodes < 1) return set_error(SDPAB_EINVAL, "mpnn_forward: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const __nv_bfloat16* wb = (const __nv_bfloat16*)weights_bf16;
  Act a = carve(act, g->num_nodes);
  forward(g, wb, a, st);
  k_readout<<<nb(g->num_nodes), 256, 0, st>>>(g->num_nodes, a.h[L], wb + off_out(), nullptr, nullptr, 0.0f,
                                             out, nullptr, nullptr);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SDPAB_OK : cuda_error(e, "mpnn_forward");
}

SDPAB_API int sdpab_mpnn_loss_grad(const sdpab_graph_batch* g, const unsigned short* weights_bf16, float* act,
                                   float* scratch, const float* target, const float* mask, float* grads,
                                   float* loss, void* stream)
{
  if (!g || !weights_bf16 || !act || !scratch || !target || !grads || !loss || g->num_nodes < 1)
    return set_error(SDPAB_EINVAL, "mpnn_loss_grad: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int N = g->num_nodes;
  const __nv_bfloat16* wb = (const __nv_bfloat16*)weights_bf16;
  Act a = carve(act, N);
  forward(g, wb, a, st);
  float cnt = (float)N;
  if (mask) cnt = g->mask_count > 0 ? (float)g->mask_count : (float)N;
  cudaMemsetAsync(grads, 0, sizeof(float) * n_params(), st);
  cudaMemsetAsync(loss, 0, sizeof(float), st);
  float* dr = scratch;
  float* dh = scratch + N;
  float* dz = dh + (long long)N * H;
  float* dself = dz + (long long)N * H;
  float* dagg = dself + (long long)N * H;
  k_readout<<<nb(N), 256, 0, st>>>(N, a.h[L], wb + off_out(), target, mask, 1.0f / cnt, a.r, dr, loss);
  k_readout_bwd<<<std::min(nb(N, 4), 1024), 256, 0, st>>>(N, a.h[L], dr, wb + off_out(), dh, grads + off_out());
  for (int l = L - 1; l >= 0; --l) {
    const int Fin = fin_of(l);
    k_relu_bwd<<<nb((long long)N * H), 256, 0, st>>>((long long)N * H, a.z[l], dh, dz);
    k_dense_bwd_w<<<std::min(nb(N, 64), 1024), 256, 0, st>>>(N, Fin, dz, a.h[l], a.agg[l], grads + off_ws(l),
                                                              grads + off_wn(l), grads + off_b(l));
    if (l > 0) {
      k_dense_bwd_x<<<nb((long long)N * Fin), 256, 0, st>>>(N, Fin, dz, wb + off_ws(l), wb + off_wn(l), dself, dagg);
      // dh_l = dself + A^T dagg   (transpose adjacency values aval_t)
      k_spmm<<<nb((long long)N * Fin), 256, 0, st>>>(N, Fin, g->rowptr, g->col, g->aval_t, dagg, dh);
      k_add<<<nb((long long)N * Fin), 256, 0, st>>>((long long)N * Fin, dh, dself);
    }
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SDPAB_OK : cuda_error(e, "mpnn_loss_grad");
}

SDPAB_API int sdpab_mpnn_adam(float* master, unsigned short* weights_bf16, const float* grads, float* m1, float* m2,
                              int step, float lr, float beta1, float beta2, float eps, float weight_decay,
                              void* stream)
{
  if (!master || !weights_bf16 || !grads || !m1 || !m2 || step < 1) return set_error(SDPAB_EINVAL, "mpnn_adam: bad arguments");
  const long long n = n_params();
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<nb(n), 256, 0, (cudaStream_t)stream>>>(n, master, (__nv_bfloat16*)weights_bf16, grads, m1, m2, lr,
                                                  beta1, beta2, eps, c1, c2, weight_decay);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SDPAB_OK : cuda_error(e, "mpnn_adam");
}

SDPAB_API int sdpab_mpnn_propose_x(int num_nodes, const float* r, const double* degree, const double* fallback,
                                   double* xvec, void* stream)
{
  if (num_nodes < 1 || !r || !degree || !fallback || !xvec) return set_error(SDPAB_EINVAL, "mpnn_propose_x: bad arguments");
  k_propose<<<nb(num_nodes), 256, 0, (cudaStream_t)stream>>>(num_nodes, r, degree, fallback, xvec);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SDPAB_OK : cuda_error(e, "mpnn_propose_x");
}

SDPAB_API int sdpab_mpnn_to_bf16(const float* master, unsigned short* weights_bf16, void* stream)
{
  const long long n = n_params();
  k_to_bf16<<<nb(n), 256, 0, (cudaStream_t)stream>>>(n, master, (__nv_bfloat16*)weights_bf16);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SDPAB_OK : cuda_error(e, "mpnn_to_bf16");
}

}  // extern "C"
