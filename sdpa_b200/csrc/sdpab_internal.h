// Internal helpers shared by the library's translation units: thread-local
// error text, CUDA error mapping and the per-device cached workspace.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

#include <atomic>

#include "sdpa_b200.h"

namespace sdpab {

int set_error(int code, const char* msg);
// Tensor-core (tcgen05, split TF32) lower update C -= P P^T of an M x M FP32
// matrix (tc_syrk.cu); `work` holds syrk_tf32x3_work_bytes(M, K) bytes.
// Returns a cudaError_t value; *err (device) is set when a block gave up
// waiting for its MMAs (the update is then incomplete).  wait_polls < 0: the
// default bound of the pipeline's waits; >= 0: that many polls (tests of
// the fall-back paths).
long long syrk_tf32x3_work_bytes(int M, int K);
int syrk_tf32x3(int M, int K, const float* P, int ldp, float* C, int ldc, void* work, int* err, cudaStream_t st,
                long long wait_polls = -1);
long long gemm_tf32x3_work_bytes(int M, int N, int K, int batch);
int gemm_tf32x3(int M, int N, int K, int batch, const double* A, int lda, long long sA, const double* B, int ldb,
                double* C, int ldc, long long sC, void* work, int* err, cudaStream_t st, long long wait_polls = -1);
int cuda_error(cudaError_t e, const char* where);

// Raises a kernel's dynamic shared-memory limit to `bytes` on the current
// device, once per device (the attribute is per device; `done` holds one bit
// per device ordinal, devices 64 and up are set on every call).
inline cudaError_t smem_attr_per_device(const void* kernel, int bytes, std::atomic<unsigned long long>& done)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ull << dev : 0ull;
  if (bit && (done.load() & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit);
  return e;
}

// Device memory kept between solver calls on the current device: the
// per-block workspace of the batched solver plus a small counter page.
// Grows on demand; sdpab_release_workspace frees it.
class Workspace {
 public:
  void* get(size_t bytes);
  int* counter();
  size_t bytes() const { return bytes_; }
  void release();

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
  int* counter_ = nullptr;
};

Workspace& workspace();

// Frees the low-rank factor routine's scratch on the current device.
void lowrank_release();

// IO::computeDimacs (sdpa_io.cpp:775-813) on the device: the final primal
// residual vector, dual residual matrices, X and Z of a finished solve
// (device pointers; SDP blocks as n x n column-major, LP blocks as vectors).
struct DimacsInput {
  int m;
  const double* rp;
  int nsdp;
  const int* n;
  const double* const* X;
  const double* const* Z;
  const double* const* D;
  int nlp;
  const double *lpx, *lpz, *lpD;
};
// out = {||rp||^2, ||D||^2, lambda_min(X), lambda_min(Z), X . Z} (dimacs.cu)
int dimacs_device(const DimacsInput& in, double* out, cudaStream_t st);
// Minimum eigenvalue of each of `count` symmetric matrices (device pointers,
// lower triangles referenced) into out_host (dimacs.cu)
int min_eigenvalues_device(int count, const int* n, const double* const* A, double* out_host, cudaStream_t st);

int batch_solve_device(const sdpab_batch* prob, const sdpab_batch_init* init,
                       const sdpab_params* prm, const sdpab_batch_config* cfg,
                       sdpab_batch_result* res, const int* order, cudaStream_t stream);

}  // namespace sdpab
