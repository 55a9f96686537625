// extern "C" entry points of include/sdpa_b200.h that are not tied to one
// solver engine: parameters, errors, workspace, and the host-pointer batch
// path (copies in, one persistent launch, copies out).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "ipm_control.h"
#include "sdpa_b200.h"
#include "sdpab_internal.h"

namespace sdpab {

static thread_local char g_err[512] = "";

int set_error(int code, const char* msg)
{
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}

int cuda_error(cudaError_t e, const char* where)
{
  snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
  return SDPAB_ECUDA;
}

void* Workspace::get(size_t bytes)
{
  if (bytes <= bytes_ && ptr_) return ptr_;
  if (ptr_) cudaFree(ptr_);
  ptr_ = nullptr;
  bytes_ = 0;
  if (cudaMalloc(&ptr_, bytes) != cudaSuccess) { ptr_ = nullptr; return nullptr; }
  bytes_ = bytes;
  return ptr_;
}

int* Workspace::counter()
{
  if (!counter_) {
    if (cudaMalloc((void**)&counter_, 256) != cudaSuccess) counter_ = nullptr;
  }
  return counter_;
}

void Workspace::release()
{
  if (ptr_) cudaFree(ptr_);
  if (counter_) cudaFree(counter_);
  ptr_ = nullptr;
  counter_ = nullptr;
  bytes_ = 0;
}

static const int kMaxDevices = 64;
static Workspace g_ws[kMaxDevices];

Workspace& workspace()
{
  int dev = 0;
  cudaGetDevice(&dev);
  return g_ws[(dev >= 0 && dev < kMaxDevices) ? dev : 0];
}

// Growable device staging buffers of the host-pointer batch path.
struct Staging {
  void* p[24] = {nullptr};
  size_t sz[24] = {0};
  void* get(int slot, size_t bytes)
  {
    if (bytes == 0) bytes = 16;
    if (sz[slot] >= bytes) return p[slot];
    if (p[slot]) cudaFree(p[slot]);
    p[slot] = nullptr;
    sz[slot] = 0;
    if (cudaMalloc(&p[slot], bytes) != cudaSuccess) return nullptr;
    sz[slot] = bytes;
    return p[slot];
  }
  void release()
  {
    for (int i = 0; i < 24; ++i) {
      if (p[i]) cudaFree(p[i]);
      p[i] = nullptr;
      sz[i] = 0;
    }
  }
};
static Staging g_stage[kMaxDevices];
static std::mutex g_stage_mu;

}  // namespace sdpab

using namespace sdpab;

extern "C" {

const char* sdpab_last_error(void) { return sdpab::g_err; }

const char* sdpab_version(void) { return "sdpa_b200 0.1 (SDPA 7.4.4 semantics, sm_100a)"; }

int sdpab_default_params(int type, sdpab_params* p)
{
  if (!p || type < 0 || type > 2) return set_error(SDPAB_EINVAL, "default_params: bad type");
  Params q = default_params(type);
  memcpy(p, &q, sizeof(q));
  return SDPAB_OK;
}

int sdpab_read_params(const char* path, sdpab_params* p)
{
  if (!path || !p) return set_error(SDPAB_EINVAL, "read_params: null argument");
  FILE* f = fopen(path, "r");
  if (!f) return set_error(SDPAB_EIO, "read_params: cannot open parameter file");
  // Parameter::readFile (sdpa_parts.cpp:231-263): one leading number per line.
  double v[10];
  int got = 0;
  char line[4096];
  while (got < 10 && fgets(line, sizeof(line), f)) {
    double x;
    if (sscanf(line, "%lf", &x) == 1) v[got++] = x;
  }
  fclose(f);
  if (got < 10) return set_error(SDPAB_EIO, "read_params: fewer than 10 numeric lines");
  p->maxIteration = (int)v[0];
  p->epsilonStar = v[1];
  p->lambdaStar = v[2];
  p->omegaStar = v[3];
  p->lowerBound = v[4];
  p->upperBound = v[5];
  p->betaStar = v[6];
  p->betaBar = v[7];
  p->gammaStar = v[8];
  p->epsilonDash = v[9];
  return SDPAB_OK;
}

int sdpab_batch_solve(const sdpab_batch* prob, const sdpab_batch_init* init,
                      const sdpab_params* prm, const sdpab_batch_config* cfg,
                      sdpab_batch_result* res, const int* order, void* stream)
{
  return batch_solve_device(prob, init, prm, cfg, res, order, (cudaStream_t)stream);
}

long long sdpab_workspace_bytes(void) { return (long long)workspace().bytes(); }

int sdpab_release_workspace(void)
{
  int dev = 0;
  cudaGetDevice(&dev);
  workspace().release();
  lowrank_release();
  std::lock_guard<std::mutex> lk(g_stage_mu);
  if (dev >= 0 && dev < kMaxDevices) g_stage[dev].release();
  return SDPAB_OK;
}

int sdpab_batch_solve_host(const sdpab_batch* hp, const sdpab_batch_init* hinit,
                           const sdpab_params* prm, const sdpab_batch_config* cfg,
                           sdpab_batch_result* hr)
{
  if (!hp || !prm || !hr || hp->count < 0) return set_error(SDPAB_EINVAL, "batch_solve_host: null argument");
  const int N = hp->count;
  const bool want_init = hinit && hinit->flag;
  if (N == 0) return SDPAB_OK;
  if (!hp->n || !hp->m || !hp->vec_off || !hp->b || !hp->mat_off || !hp->mat_ptr || !hp->row ||
      !hp->col || !hp->val || !hp->dense_off || !hr->primal_obj || !hr->dual_obj || !hr->mu ||
      !hr->primal_error || !hr->dual_error || !hr->iterations || !hr->phase || !hr->status)
    return set_error(SDPAB_EINVAL, "batch_solve_host: a required array is NULL");
  // array extents from the offsets
  int nmax = 1, mmax = 1;
  long long nvec = 0, nptr = 0, nent = 0, nden = 0;
  for (int i = 0; i < N; ++i) {
    const int n = hp->n[i], m = hp->m[i];
    if (n < 1 || m < 1) return set_error(SDPAB_EINVAL, "batch_solve_host: n and m must be positive");
    nmax = std::max(nmax, n);
    mmax = std::max(mmax, m);
    nvec = std::max(nvec, hp->vec_off[i] + m);
    nptr = std::max(nptr, hp->mat_off[i] + m + 2);
    nent = std::max(nent, hp->mat_ptr[hp->mat_off[i] + m + 1]);
    nden = std::max(nden, hp->dense_off[i] + (long long)n * n);
  }
  // block structure: extent of blk_size, and each instance's orders add up to n
  long long nbs = 0;
  if (hp->nblock) {
    if (!hp->blk_off || !hp->blk_size) return set_error(SDPAB_EINVAL, "batch_solve_host: blk_off / blk_size NULL");
    for (int i = 0; i < N; ++i) {
      const int nb = hp->nblock[i];
      if (nb < 1 || nb > SDPAB_BATCH_MAX_BLOCKS || hp->blk_off[i] < 0)
        return set_error(SDPAB_EINVAL, "batch_solve_host: nblock out of range");
      long long tot = 0;
      for (int l = 0; l < nb; ++l) {
        const int sz = hp->blk_size[hp->blk_off[i] + l];
        if (sz == 0) return set_error(SDPAB_EINVAL, "batch_solve_host: block of order 0");
        tot += (sz < 0) ? -(long long)sz : sz;
      }
      if (tot != hp->n[i]) return set_error(SDPAB_EINVAL, "batch_solve_host: block orders do not add up to n");
      nbs = std::max(nbs, (long long)hp->blk_off[i] + nb);
    }
  }
  bool need_x = false, need_v = false;
  if (want_init) {
    bool need_xy = false;
    for (int i = 0; i < N; ++i) {
      need_xy |= (hinit->flag[i] == SDPAB_INIT_POINT);
      need_x |= (hinit->flag[i] == SDPAB_INIT_POINT || hinit->flag[i] == SDPAB_INIT_DUAL);
      need_v |= (hinit->flag[i] == SDPAB_INIT_FACTOR);
    }
    if (need_x && !hinit->xvec) return set_error(SDPAB_EINVAL, "batch_solve_host: init xvec is NULL");
    if (need_xy && (!hinit->X || !hinit->Y))
      return set_error(SDPAB_EINVAL, "batch_solve_host: SDPAB_INIT_POINT needs init X and Y");
    if (need_v && (!hinit->V || hinit->rank < 1 || hinit->rank > 32))
      return set_error(SDPAB_EINVAL, "batch_solve_host: SDPAB_INIT_FACTOR needs V and a rank of 1..32");
  }
  std::vector<int> order(N);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return (long long)hp->n[a] * hp->n[a] + hp->m[a] >
                                              (long long)hp->n[b] * hp->n[b] + hp->m[b]; });
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(SDPAB_ENODEV, "no CUDA device");
  std::lock_guard<std::mutex> lk(g_stage_mu);
  Staging& S = g_stage[(dev >= 0 && dev < kMaxDevices) ? dev : 0];
  cudaStream_t st = 0;
  struct Copy { int slot; const void* src; size_t bytes; };
  const Copy in[] = {
      {0, hp->n, N * sizeof(int)},          {1, hp->m, N * sizeof(int)},
      {2, hp->vec_off, N * sizeof(long long)}, {3, hp->b, nvec * sizeof(double)},
      {4, hp->mat_off, N * sizeof(long long)}, {5, hp->mat_ptr, nptr * sizeof(long long)},
      {6, hp->row, nent * sizeof(int)},      {7, hp->col, nent * sizeof(int)},
      {8, hp->val, nent * sizeof(double)},   {9, hp->dense_off, N * sizeof(long long)},
      {10, order.data(), N * sizeof(int)},
      {11, want_init ? hinit->flag : nullptr, want_init ? N * sizeof(int) : 0},
      {12, (want_init && hinit->xvec) ? hinit->xvec : nullptr, want_init ? nvec * sizeof(double) : 0},
      {13, want_init ? hinit->X : nullptr, want_init ? nden * sizeof(double) : 0},
      {14, want_init ? hinit->Y : nullptr, want_init ? nden * sizeof(double) : 0},
      {20, hp->nblock, hp->nblock ? N * sizeof(int) : 0},
      {21, hp->nblock ? hp->blk_off : nullptr, hp->nblock ? N * sizeof(int) : 0},
      {22, hp->nblock ? hp->blk_size : nullptr, nbs * sizeof(int)},
      {23, need_v ? hinit->V : nullptr, need_v ? nvec * hinit->rank * sizeof(double) : 0},
  };
  void* d[24] = {nullptr};
  for (const Copy& c : in) {
    if (!c.src) continue;
    d[c.slot] = S.get(c.slot, c.bytes);
    if (!d[c.slot]) return set_error(SDPAB_ECUDA, "batch_solve_host: device allocation failed");
    cudaError_t e = cudaMemcpyAsync(d[c.slot], c.src, c.bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_error(e, "batch_solve_host: H2D copy");
  }
  // results: one contiguous device region per kind
  struct Out { int slot; void* dst; size_t bytes; };
  const Out out[] = {
      {15, hr->xvec, hr->xvec ? nvec * sizeof(double) : 0},
      {16, hr->X, hr->X ? nden * sizeof(double) : 0},
      {17, hr->Y, hr->Y ? nden * sizeof(double) : 0},
      {18, hr->primal_obj, 5 * N * sizeof(double)},  // primal, dual, mu, perr, derr
      {19, hr->iterations, 3 * N * sizeof(int)},     // iterations, phase, status
  };
  for (const Out& o : out) {
    if (!o.dst) continue;
    d[o.slot] = S.get(o.slot, o.bytes);
    if (!d[o.slot]) return set_error(SDPAB_ECUDA, "batch_solve_host: device allocation failed");
  }
  sdpab_batch dp = *hp;
  dp.nmax = std::max(hp->nmax, nmax);
  dp.mmax = std::max(hp->mmax, mmax);
  dp.n = (const int*)d[0];
  dp.m = (const int*)d[1];
  dp.vec_off = (const long long*)d[2];
  dp.b = (const double*)d[3];
  dp.mat_off = (const long long*)d[4];
  dp.mat_ptr = (const long long*)d[5];
  dp.row = (const int*)d[6];
  dp.col = (const int*)d[7];
  dp.val = (const double*)d[8];
  dp.dense_off = (const long long*)d[9];
  dp.nblock = (const int*)d[20];
  dp.blk_off = (const int*)d[21];
  dp.blk_size = (const int*)d[22];
  sdpab_batch_init di;
  memset(&di, 0, sizeof(di));
  if (want_init) {
    di.init_margin = hinit->init_margin;
    di.flag = (const int*)d[11];
    di.xvec = (const double*)d[12];
    di.X = (const double*)d[13];
    di.Y = (const double*)d[14];
    di.V = (const double*)d[23];
    di.rank = hinit->rank;
    di.init_mu = hinit->init_mu;
  }
  sdpab_batch_result dr;
  double* sc = (double*)d[18];
  int* ic = (int*)d[19];
  dr.xvec = (double*)d[15];
  dr.X = (double*)d[16];
  dr.Y = (double*)d[17];
  dr.primal_obj = sc;
  dr.dual_obj = sc + N;
  dr.mu = sc + 2 * N;
  dr.primal_error = sc + 3 * N;
  dr.dual_error = sc + 4 * N;
  dr.iterations = ic;
  dr.phase = ic + N;
  dr.status = ic + 2 * N;
  int rc = batch_solve_device(&dp, want_init ? &di : nullptr, prm, cfg, &dr, (const int*)d[10], st);
  if (rc != SDPAB_OK) return rc;
  // copy back (scalar arrays are gathered per kind)
  double* hs[5] = {hr->primal_obj, hr->dual_obj, hr->mu, hr->primal_error, hr->dual_error};
  for (int q = 0; q < 5; ++q) {
    cudaError_t e = cudaMemcpyAsync(hs[q], sc + (size_t)q * N, N * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_error(e, "batch_solve_host: D2H copy");
  }
  int* hi[3] = {hr->iterations, hr->phase, hr->status};
  for (int q = 0; q < 3; ++q) {
    cudaError_t e = cudaMemcpyAsync(hi[q], ic + (size_t)q * N, N * sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_error(e, "batch_solve_host: D2H copy");
  }
  for (int q = 15; q <= 17; ++q) {
    const Out& o = out[q - 15];
    if (!o.dst) continue;
    cudaError_t e = cudaMemcpyAsync(o.dst, d[q], o.bytes, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return cuda_error(e, "batch_solve_host: D2H copy");
  }
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_error(e, "batch_solve_host: synchronize");
  return SDPAB_OK;
}

}  // extern "C"
