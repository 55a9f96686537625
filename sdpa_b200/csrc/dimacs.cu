// DIMACS error measures of a finished solve, computed on the device
// (IO::computeDimacs, sdpa_io.cpp:775-813): the two-norms of the final
// primal residual vector and dual residual matrix, X . Z, and the minimum
// eigenvalues of X and Z.  The reference takes each SDP block's minimum
// eigenvalue with LAPACK dsyev (Jal::getMinEigen(DenseLinearSpace&),
// sdpa_jordan.cpp:111-145, Lal::getMinEigenValue, sdpa_linear.cpp:145-182);
// here one block of threads per SDP block reduces its lower triangle to a
// symmetric tridiagonal matrix by Householder reflections and one warp then
// brackets the smallest eigenvalue by Sturm-count multisection.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "sdpab_internal.h"

namespace sdpab {

namespace {

constexpr int ENT = 1024;  // threads per eigenvalue block

struct EigJob {
  int n;
  const double* A;  // n x n column-major, lower triangle referenced
  double* work;     // n^2 + 4 n doubles
  double* out;      // the minimum eigenvalue
};

__device__ double block_sum_1024(double v, double* red)
{
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < ENT / 32; ++w) s += red[w];
  __syncthreads();
  return s;
}

// Number of eigenvalues of the symmetric tridiagonal (d, e) below sigma
// (Sturm count through the LDL^T pivots).
__device__ int sturm_count(int n, const double* d, const double* e, double sigma)
{
  int c = 0;
  double q = d[0] - sigma;
  const double tiny = 1.0e-300;
  if (q == 0.0) q = -tiny;
  c += q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = d[i] - sigma - e[i - 1] * e[i - 1] / q;
    if (q == 0.0) q = -tiny;
    c += q < 0.0;
  }
  return c;
}

__global__ void __launch_bounds__(ENT) k_sym_min_eig(const EigJob* jobs)
{
  __shared__ double red[ENT / 32];
  __shared__ double s_lohi[2];
  const EigJob J = jobs[blockIdx.x];
  const int n = J.n, tid = threadIdx.x;
  double* M = J.work;
  double* v = M + (size_t)n * n;
  double* p = v + n;
  double* d = p + n;
  double* e = d + n;
  // symmetric copy of the lower triangle (dsyev "Lower")
  for (size_t t = tid; t < (size_t)n * n; t += ENT) {
    const int i = (int)(t % n), j = (int)(t / n);
    M[t] = (i >= j) ? J.A[t] : J.A[j + (size_t)n * i];
  }
  for (int i = tid; i < n; i += ENT) e[i] = 0.0;
  __syncthreads();
  for (int k = 0; k + 2 < n; ++k) {
    const int len = n - k - 1;
    const double* x = M + (k + 1) + (size_t)n * k;
    double s = 0.0;
    for (int i = tid; i < len; i += ENT) s += x[i] * x[i];
    const double nrm2 = block_sum_1024(s, red);
    const double x0 = x[0];
    const double alpha = (x0 >= 0.0) ? -sqrt(nrm2) : sqrt(nrm2);
    const double vn2 = nrm2 - x0 * x0 + (x0 - alpha) * (x0 - alpha);
    if (tid == 0) e[k] = (nrm2 > 0.0) ? alpha : 0.0;
    if (!(vn2 > 0.0)) {
      __syncthreads();
      continue;
    }
    for (int i = tid; i < len; i += ENT) v[i] = (i == 0) ? x0 - alpha : x[i];
    __syncthreads();
    // p = (2 / vn2) S v over the trailing block S
    double kv = 0.0;
    const double* S = M + (k + 1) + (size_t)n * (k + 1);
    for (int i = tid; i < len; i += ENT) {
      double acc = 0.0;
      for (int c = 0; c < len; ++c) acc += S[i + (size_t)n * c] * v[c];
      acc *= 2.0 / vn2;
      p[i] = acc;
      kv += acc * v[i];
    }
    kv = block_sum_1024(kv, red) / vn2;
    // w = p - K v, then S -= v w^T + w v^T
    for (int i = tid; i < len; i += ENT) p[i] -= kv * v[i];
    __syncthreads();
    double* Sw = M + (k + 1) + (size_t)n * (k + 1);
    for (size_t t = tid; t < (size_t)len * len; t += ENT) {
      const int i = (int)(t % len), c = (int)(t / len);
      Sw[i + (size_t)n * c] -= v[i] * p[c] + p[i] * v[c];
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += ENT) d[i] = M[i + (size_t)n * i];
  if (tid == 0 && n >= 2) e[n - 2] = M[(n - 1) + (size_t)n * (n - 2)];
  __syncthreads();
  // Gershgorin interval
  double lo = 1.0e300, hi = -1.0e300;
  for (int i = tid; i < n; i += ENT) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - r);
    hi = fmax(hi, d[i] + r);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if ((tid & 31) == 0) red[tid >> 5] = lo;
  __syncthreads();
  if (tid == 0) {
    double m = red[0];
    for (int w = 1; w < ENT / 32; ++w) m = fmin(m, red[w]);
    s_lohi[0] = m;
  }
  __syncthreads();
  if ((tid & 31) == 0) red[tid >> 5] = hi;
  __syncthreads();
  if (tid == 0) {
    double m = red[0];
    for (int w = 1; w < ENT / 32; ++w) m = fmax(m, red[w]);
    s_lohi[1] = m;
  }
  __syncthreads();
  if (tid < 32) {
    const int lane = tid;
    double a = s_lohi[0], b = s_lohi[1];
    const double span = fmax(fabs(a), fabs(b));
    a -= 1.0e-14 * span + 1.0e-300;
    b += 1.0e-14 * span + 1.0e-300;
    // multisection: 32 interior points per round, the bracket keeps
    // count(a) = 0 and count(b) >= 1; it stops at the matrix's own rounding
    // level (about eps ||A||, as dsyev) or at a relative width of 4 eps
    const double tol = 1.0e-16 * span;
    for (int round = 0; round < 64; ++round) {
      const double w = b - a;
      if (!(w > tol) || !(w > 4.0e-16 * fmax(fabs(a), fabs(b))) || w <= 1.0e-300) break;
      const double h = (b - a) / 33.0;
      const double sig = a + h * (lane + 1);
      const int cnt = sturm_count(n, d, e, sig);
      const unsigned has = __ballot_sync(0xffffffffu, cnt >= 1);
      if (has) {
        const int j = __ffs(has) - 1;
        const double nb = a + h * (j + 1);
        a = (j == 0) ? a : a + h * j;
        b = nb;
      } else {
        a = a + h * 32;
      }
    }
    if (lane == 0) *J.out = 0.5 * (a + b);
  }
}

// out[slot] = sum a*b (b == nullptr: sum a^2) or min a, one block, fixed order
__global__ void __launch_bounds__(ENT) k_reduce(long long n, const double* a, const double* b, int mode,
                                                double* out, int accumulate)
{
  __shared__ double red[ENT / 32];
  double s = (mode == 1) ? 1.0e300 : 0.0;
  for (long long t = threadIdx.x; t < n; t += ENT) {
    if (mode == 1) s = fmin(s, a[t]);
    else s += a[t] * (b ? b[t] : a[t]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double y = __shfl_xor_sync(0xffffffffu, s, o);
    s = (mode == 1) ? fmin(s, y) : s + y;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = red[0];
    for (int w = 1; w < ENT / 32; ++w) r = (mode == 1) ? fmin(r, red[w]) : r + red[w];
    if (accumulate) r = (mode == 1) ? fmin(r, *out) : r + *out;
    *out = r;
  }
}

}  // namespace

// Minimum eigenvalues of `count` symmetric matrices (device pointers,
// column-major, lower triangles referenced) into out_host.
int min_eigenvalues_device(int count, const int* n, const double* const* A, double* out_host,
                           cudaStream_t st)
{
  if (count <= 0) return SDPAB_OK;
  std::vector<EigJob> jobs(count);
  size_t total = 0;
  for (int q = 0; q < count; ++q) {
    if (n[q] < 1) return set_error(SDPAB_EINVAL, "min_eigenvalue: order < 1");
    total += (size_t)n[q] * n[q] + 4 * (size_t)n[q];
  }
  double* work = nullptr;
  double* outs = nullptr;
  EigJob* djobs = nullptr;
  cudaError_t e = cudaMalloc(&work, total * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&outs, count * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&djobs, count * sizeof(EigJob));
  if (e == cudaSuccess) {
    size_t off = 0;
    for (int q = 0; q < count; ++q) {
      jobs[q] = EigJob{n[q], A[q], work + off, outs + q};
      off += (size_t)n[q] * n[q] + 4 * (size_t)n[q];
    }
    e = cudaMemcpyAsync(djobs, jobs.data(), count * sizeof(EigJob), cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) {
    k_sym_min_eig<<<count, ENT, 0, st>>>(djobs);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out_host, outs, count * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(work);
  cudaFree(outs);
  cudaFree(djobs);
  if (e != cudaSuccess) return cuda_error(e, "min_eigenvalue");
  return SDPAB_OK;
}

// The five device quantities of IO::computeDimacs: out = {||rp||^2,
// ||D||^2 (SDP blocks + LP), min eig X, min eig Z, X . Z}.
int dimacs_device(const DimacsInput& in, double* out, cudaStream_t st)
{
  double* acc = nullptr;
  cudaError_t e = cudaMalloc(&acc, 8 * sizeof(double));
  if (e != cudaSuccess) return cuda_error(e, "dimacs");
  // slots: 0 rp^2, 1 D^2, 2 X.Z, 3 min LP x, 4 min LP z
  cudaMemsetAsync(acc, 0, 8 * sizeof(double), st);
  if (in.m > 0) k_reduce<<<1, ENT, 0, st>>>(in.m, in.rp, nullptr, 0, acc + 0, 0);
  bool first = true;
  for (int q = 0; q < in.nsdp; ++q) {
    const long long nn = (long long)in.n[q] * in.n[q];
    k_reduce<<<1, ENT, 0, st>>>(nn, in.D[q], nullptr, 0, acc + 1, first ? 0 : 1);
    k_reduce<<<1, ENT, 0, st>>>(nn, in.X[q], in.Z[q], 0, acc + 2, first ? 0 : 1);
    first = false;
  }
  if (in.nlp > 0) {
    k_reduce<<<1, ENT, 0, st>>>(in.nlp, in.lpD, nullptr, 0, acc + 1, first ? 0 : 1);
    k_reduce<<<1, ENT, 0, st>>>(in.nlp, in.lpx, in.lpz, 0, acc + 2, first ? 0 : 1);
    k_reduce<<<1, ENT, 0, st>>>(in.nlp, in.lpx, nullptr, 1, acc + 3, 0);
    k_reduce<<<1, ENT, 0, st>>>(in.nlp, in.lpz, nullptr, 1, acc + 4, 0);
  }
  double h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, acc, 8 * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaFree(acc);
  if (e != cudaSuccess) return cuda_error(e, "dimacs");
  double xmin = (in.nlp > 0) ? h[3] : 1.0e50, zmin = (in.nlp > 0) ? h[4] : 1.0e50;
  if (in.nsdp > 0) {
    std::vector<double> ex(in.nsdp), ez(in.nsdp);
    int rc = min_eigenvalues_device(in.nsdp, in.n, in.X, ex.data(), st);
    if (rc == SDPAB_OK) rc = min_eigenvalues_device(in.nsdp, in.n, in.Z, ez.data(), st);
    if (rc != SDPAB_OK) return rc;
    for (int q = 0; q < in.nsdp; ++q) {
      xmin = fmin(xmin, ex[q]);
      zmin = fmin(zmin, ez[q]);
    }
  }
  out[0] = h[0];
  out[1] = h[1];
  out[2] = xmin;
  out[3] = zmin;
  out[4] = h[2];
  return SDPAB_OK;
}

}  // namespace sdpab

extern "C" SDPAB_API int sdpab_min_eigenvalue(int n, const double* A, double* out, void* stream)
{
  if (n < 1 || !A || !out) return sdpab::set_error(SDPAB_EINVAL, "sdpab_min_eigenvalue: invalid arguments");
  const double* Ap[1] = {A};
  return sdpab::min_eigenvalues_device(1, &n, Ap, out, (cudaStream_t)stream);
}
