// Kernel-level entry points mirroring the reference Backend
// (src/sovopt/core/backend.py:317-493): sparse products, the fused PDHG
// step kernels and the reductions, on device pointers and a caller stream.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>

#include "common.cuh"

namespace pdlp {
namespace {

constexpr int kT = 256;
constexpr unsigned kAll = 0xffffffffu;

int grid_1d(long long n, int per = kT) {
  long long g = (n + per - 1) / per;
  return (int)std::max(1LL, std::min(g, 1LL << 20));
}

// Lanes per row from the mean row length (power of two in [1, 32]).
int lanes_of(long long nnz, long long rows) {
  if (rows <= 0) return 1;
  const double avg = (double)nnz / (double)rows;
  int L = 1;
  while (L < 32 && L < avg) L <<= 1;
  return L;
}

// y = A x with L lanes per row: each lane sums its strided entries in order,
// a xor butterfly combines them (fixed order, so repeats are bitwise equal).
template <typename T, int L>
__global__ void __launch_bounds__(kT) spmv_kernel(int m, const int64_t* __restrict__ rp,
                                                  const int* __restrict__ ri,
                                                  const T* __restrict__ rx,
                                                  const T* __restrict__ x, T* __restrict__ y) {
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const int row = gtid / L;
  const int lane = threadIdx.x & (L - 1);
  T acc = T(0);
  if (row < m) {
    const int64_t p0 = __ldg(rp + row), p1 = __ldg(rp + row + 1);
    for (int64_t p = p0 + lane; p < p1; p += L) acc += __ldg(rx + p) * __ldg(x + __ldg(ri + p));
  }
#pragma unroll
  for (int off = L >> 1; off > 0; off >>= 1) acc += __shfl_xor_sync(kAll, acc, off);
  if (row < m && lane == 0) y[row] = acc;
}

// Lanes per row of a matrix, remembered by its row-pointer address: the
// entry point is given no nnz, so the first call on a matrix reads rp[m] back
// (one synchronisation) and later calls reuse the choice.  A stale entry (a
// freed and reused address) only changes the lane count, never the result
// beyond rounding order.
std::mutex lanes_mu;
std::unordered_map<const void*, std::pair<int, int>> lanes_cache;   // rp -> (m, L)

template <typename T>
int launch_spmv(int m, const int64_t* rp, const int* ri, const T* rx, const T* x, T* y,
                cudaStream_t st) {
  if (m < 0) return fail(PDLP_ERR_ARG, "m must be >= 0");
  if (m == 0) return PDLP_OK;
  if (!rp || !ri || !rx || !x || !y) return fail(PDLP_ERR_ARG, "NULL pointer");
  int L = 0;
  {
    std::lock_guard<std::mutex> lock(lanes_mu);
    auto it = lanes_cache.find(rp);
    if (it != lanes_cache.end() && it->second.first == m) L = it->second.second;
  }
  if (L == 0) {
    int64_t nnz = 0;
    PDLP_CUDA(cudaMemcpyAsync(&nnz, rp + m, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    PDLP_CUDA(cudaStreamSynchronize(st));
    L = lanes_of(nnz, m);
    std::lock_guard<std::mutex> lock(lanes_mu);
    if (lanes_cache.size() >= 256) lanes_cache.clear();
    lanes_cache[rp] = {m, L};
  }
  const long long threads = (long long)m * L;
  const int g = grid_1d(threads);
  switch (L) {
    case 1: spmv_kernel<T, 1><<<g, kT, 0, st>>>(m, rp, ri, rx, x, y); break;
    case 2: spmv_kernel<T, 2><<<g, kT, 0, st>>>(m, rp, ri, rx, x, y); break;
    case 4: spmv_kernel<T, 4><<<g, kT, 0, st>>>(m, rp, ri, rx, x, y); break;
    case 8: spmv_kernel<T, 8><<<g, kT, 0, st>>>(m, rp, ri, rx, x, y); break;
    case 16: spmv_kernel<T, 16><<<g, kT, 0, st>>>(m, rp, ri, rx, x, y); break;
    default: spmv_kernel<T, 32><<<g, kT, 0, st>>>(m, rp, ri, rx, x, y); break;
  }
  PDLP_CUDA(cudaGetLastError());
  count_launches(1);
  return PDLP_OK;
}

// Y = A X, X row-major (ncols, k): one thread per (row, column of X); the
// entries of a row are summed in storage order.
__global__ void __launch_bounds__(kT) spmm_kernel(int m, int k, const int64_t* __restrict__ rp,
                                                  const int* __restrict__ ri,
                                                  const double* __restrict__ rx,
                                                  const double* __restrict__ X,
                                                  double* __restrict__ Y) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long row = g / k;
  const int col = (int)(g - row * k);
  if (row >= m) return;
  double acc = 0.0;
  const int64_t p0 = rp[row], p1 = rp[row + 1];
  for (int64_t p = p0; p < p1; ++p) acc += rx[p] * X[(long long)ri[p] * k + col];
  Y[row * k + col] = acc;
}

__global__ void primal_step_kernel(int n, double* xnew, const double* x, const double* c,
                                   const double* aty, const double* lo, const double* hi,
                                   double tau) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xnew[i] = clip(x[i] - tau * (c[i] + aty[i]), lo[i], hi[i]);
}

__global__ void dual_step_kernel(int m, double* ynew, const double* y, const double* ax,
                                 const double* rl, const double* ru, double sigma) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double w = y[i] + sigma * ax[i];
  ynew[i] = w - sigma * clip(w / sigma, rl[i], ru[i]);
}

__global__ void pdhg_primal_kernel(int n, double* x, double* dx, const double* c,
                                   const double* aty, const double* lo, const double* hi,
                                   double tau) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xi = x[i];
  const double v = clip(xi - tau * (c[i] + aty[i]), lo[i], hi[i]);
  dx[i] = v - xi;
  x[i] = v;
}

__global__ void pdhg_dual_kernel(int m, double* y, double* dy, double* ax, const double* adx,
                                 const double* rl, const double* ru, double sigma) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const double a = adx[i];
  const double axn = ax[i] + a;
  ax[i] = axn;
  const double yo = y[i];
  const double w = yo + sigma * (axn + a);
  const double yn = w - sigma * clip(w / sigma, rl[i], ru[i]);
  dy[i] = yn - yo;
  y[i] = yn;
}

__global__ void pdhg_accum_kernel(int n, double* acc, const double* inc, double* run_sum,
                                  const double* v, double eta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  acc[i] += inc[i];
  run_sum[i] += eta * v[i];
}

enum { RED_DOT = 0, RED_SQ = 1, RED_ABSMAX = 2 };

__device__ __forceinline__ double red_combine(double a, double b, int op) {
  return op == RED_ABSMAX ? fmax(a, b) : a + b;
}

// Block-level partial of a reduction over [0, n) with a grid-stride loop of
// fixed shape: partials[blockIdx.x].  Deterministic for a given grid.
__global__ void __launch_bounds__(kT) reduce_partial_kernel(long long n, const double* a,
                                                            const double* b, int op,
                                                            double* partials) {
  __shared__ double sh[kT / 32];
  double acc = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double v = a[i];
    const double t = op == RED_DOT ? v * b[i] : (op == RED_SQ ? v * v : fabs(v));
    acc = red_combine(acc, t, op);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc = red_combine(acc, __shfl_down_sync(kAll, acc, off), op);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (kT / 32) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = red_combine(v, __shfl_down_sync(kAll, v, off), op);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
  }
}

__global__ void __launch_bounds__(kT) reduce_final_kernel(int nparts, const double* partials,
                                                          int op, double* out) {
  __shared__ double sh[kT / 32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc = red_combine(acc, partials[i], op);
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc = red_combine(acc, __shfl_down_sync(kAll, acc, off), op);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (kT / 32) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v = red_combine(v, __shfl_down_sync(kAll, v, off), op);
    if (threadIdx.x == 0) *out = v;
  }
}

constexpr int kRedBlocks = 592;   // 4 x 148 SMs: fixed, so results do not depend on the device

int reduce(long long n, const double* a, const double* b, int op, double* out, cudaStream_t st) {
  if (!out) return fail(PDLP_ERR_ARG, "out is NULL");
  if (n < 0) return fail(PDLP_ERR_ARG, "n must be >= 0");
  if (n == 0) { *out = 0.0; return PDLP_OK; }
  if (!a || (op == RED_DOT && !b)) return fail(PDLP_ERR_ARG, "NULL pointer");
  // scratch: block partials and the result, from the stream-ordered pool
  double* scratch = nullptr;
  PDLP_CUDA(cudaMallocAsync((void**)&scratch, sizeof(double) * (kRedBlocks + 1), st));
  reduce_partial_kernel<<<kRedBlocks, kT, 0, st>>>(n, a, b, op, scratch);
  reduce_final_kernel<<<1, kT, 0, st>>>(kRedBlocks, scratch, op, scratch + kRedBlocks);
  count_launches(2);
  cudaError_t e = cudaGetLastError();
  double h = 0.0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, scratch + kRedBlocks, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(scratch, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "reduction");
  *out = op == RED_SQ ? sqrt(h) : h;
  return PDLP_OK;
}

// ---- dot product with a fixed, statically allocated scratch ---------------
// pdlp_dot_noalloc serves callers that must not allocate device memory (a
// serving loop whose free memory is held by resident problems, a caller with
// a fixed device footprint).  It reduces chunks of kNaChunk elements, one
// block per chunk, into the partials at the head of noalloc_scratch; the
// final block sum goes to the slot after the largest partial count.  The
// array is one per device, 128 KiB, shared by every call on that device and
// left holding the last call's sums: calls that overlap in time race.
constexpr int kNaChunk = 16384;
constexpr int kNaMaxChunks = 16384;
constexpr long long kNaMaxN = (long long)kNaChunk * kNaMaxChunks;   // 2^28 elements
constexpr int kNaMaxDevices = 64;
static __device__ __align__(256) double noalloc_scratch[kNaMaxChunks + 1];

// partials[blockIdx.x] = sum of a[i] * b[i] over the block's chunk, in a fixed
// order (thread t takes elements t, t + kT, ... of the chunk; warp and block
// trees after), so repeated calls give the same bits.
__global__ void __launch_bounds__(kT) dot_chunk_kernel(long long n, const double* __restrict__ a,
                                                       const double* __restrict__ b,
                                                       double* __restrict__ partials) {
  __shared__ double sh[kT / 32];
  const long long base = (long long)blockIdx.x * kNaChunk;
  const long long end = min(n, base + kNaChunk);
  double acc = 0.0;
#pragma unroll 8
  for (long long i = base + threadIdx.x; i < end; i += kT) acc += a[i] * b[i];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(kAll, acc, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (kT / 32) ? sh[threadIdx.x] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kAll, v, off);
    if (threadIdx.x == 0) partials[blockIdx.x] = v;
  }
}

// Device address of noalloc_scratch, looked up once per device ordinal (with
// that device current) on the first call made there.
std::mutex noalloc_mu;
double* noalloc_ptr[kNaMaxDevices] = {};

int noalloc_scratch_ptr(double** out) {
  int dev = 0;
  PDLP_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices)
    return fail(PDLP_ERR_ARG, "pdlp_dot_noalloc: device ordinal " + std::to_string(dev) +
                                  " is beyond the " + std::to_string(kNaMaxDevices) +
                                  " devices it supports");
  std::lock_guard<std::mutex> lock(noalloc_mu);
  if (!noalloc_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(noalloc_scratch)");
    noalloc_ptr[dev] = static_cast<double*>(p);
  }
  *out = noalloc_ptr[dev];
  return PDLP_OK;
}

}  // namespace
}  // namespace pdlp

using namespace pdlp;

extern "C" {

int pdlp_spmv_f64(int32_t m, const int64_t* rp, const int32_t* ri, const double* rx,
                  const double* x, double* y, void* stream) {
  return launch_spmv<double>(m, rp, ri, rx, x, y, (cudaStream_t)stream);
}

int pdlp_spmv_f32(int32_t m, const int64_t* rp, const int32_t* ri, const float* rx,
                  const float* x, float* y, void* stream) {
  return launch_spmv<float>(m, rp, ri, rx, x, y, (cudaStream_t)stream);
}

int pdlp_spmm_f64(int32_t m, int32_t k, const int64_t* rp, const int32_t* ri,
                  const double* rx, const double* X, double* Y, void* stream) {
  if (m < 0 || k < 0) return fail(PDLP_ERR_ARG, "negative size");
  if (m == 0 || k == 0) return PDLP_OK;
  if (!rp || !ri || !rx || !X || !Y) return fail(PDLP_ERR_ARG, "NULL pointer");
  const long long threads = (long long)m * k;
  spmm_kernel<<<grid_1d(threads), kT, 0, (cudaStream_t)stream>>>(m, k, rp, ri, rx, X, Y);
  PDLP_CUDA(cudaGetLastError());
  count_launches(1);
  return PDLP_OK;
}

int pdlp_primal_step(int32_t n, double* xnew, const double* x, const double* c,
                     const double* aty, const double* lo, const double* hi, double tau,
                     void* stream) {
  if (n < 0) return fail(PDLP_ERR_ARG, "n must be >= 0");
  if (n == 0) return PDLP_OK;
  primal_step_kernel<<<grid_1d(n), kT, 0, (cudaStream_t)stream>>>(n, xnew, x, c, aty, lo, hi, tau);
  PDLP_CUDA(cudaGetLastError());
  count_launches(1);
  return PDLP_OK;
}

int pdlp_dual_step(int32_t m, double* ynew, const double* y, const double* ax,
                   const double* rl, const double* ru, double sigma, void* stream) {
  if (m < 0) return fail(PDLP_ERR_ARG, "m must be >= 0");
  if (m == 0) return PDLP_OK;
  dual_step_kernel<<<grid_1d(m), kT, 0, (cudaStream_t)stream>>>(m, ynew, y, ax, rl, ru, sigma);
  PDLP_CUDA(cudaGetLastError());
  count_launches(1);
  return PDLP_OK;
}

int pdlp_pdhg_primal(int32_t n, double* x, double* dx, const double* c, const double* aty,
                     const double* lo, const double* hi, double tau, void* stream) {
  if (n < 0) return fail(PDLP_ERR_ARG, "n must be >= 0");
  if (n == 0) return PDLP_OK;
  pdhg_primal_kernel<<<grid_1d(n), kT, 0, (cudaStream_t)stream>>>(n, x, dx, c, aty, lo, hi, tau);
  PDLP_CUDA(cudaGetLastError());
  count_launches(1);
  return PDLP_OK;
}

int pdlp_pdhg_dual(int32_t m, double* y, double* dy, double* ax, const double* adx,
                   const double* rl, const double* ru, double sigma, void* stream) {
  if (m < 0) return fail(PDLP_ERR_ARG, "m must be >= 0");
  if (m == 0) return PDLP_OK;
  pdhg_dual_kernel<<<grid_1d(m), kT, 0, (cudaStream_t)stream>>>(m, y, dy, ax, adx, rl, ru, sigma);
  PDLP_CUDA(cudaGetLastError());
  count_launches(1);
  return PDLP_OK;
}

int pdlp_pdhg_accum(int32_t n, double* acc, const double* inc, double* run_sum,
                    const double* v, double eta, void* stream) {
  if (n < 0) return fail(PDLP_ERR_ARG, "n must be >= 0");
  if (n == 0) return PDLP_OK;
  pdhg_accum_kernel<<<grid_1d(n), kT, 0, (cudaStream_t)stream>>>(n, acc, inc, run_sum, v, eta);
  PDLP_CUDA(cudaGetLastError());
  count_launches(1);
  return PDLP_OK;
}

int pdlp_dot(int64_t n, const double* a, const double* b, double* out, void* stream) {
  return reduce(n, a, b, RED_DOT, out, (cudaStream_t)stream);
}

int pdlp_nrm2(int64_t n, const double* a, double* out, void* stream) {
  return reduce(n, a, nullptr, RED_SQ, out, (cudaStream_t)stream);
}

int pdlp_nrm_inf(int64_t n, const double* a, double* out, void* stream) {
  return reduce(n, a, nullptr, RED_ABSMAX, out, (cudaStream_t)stream);
}

int pdlp_dot_noalloc(int64_t n, const double* a, const double* b, double* out, void* stream) {
  if (!out) return fail(PDLP_ERR_ARG, "out is NULL");
  if (n < 0) return fail(PDLP_ERR_ARG, "n must be >= 0");
  if (n > kNaMaxN)
    return fail(PDLP_ERR_ARG, "pdlp_dot_noalloc: n = " + std::to_string((long long)n) +
                                  " is above its fixed-scratch limit of " +
                                  std::to_string(kNaMaxN) + " elements; use pdlp_dot");
  double* scratch = nullptr;
  const int rc = noalloc_scratch_ptr(&scratch);
  if (rc != PDLP_OK) return rc;
  if (n == 0) { *out = 0.0; return PDLP_OK; }
  if (!a || !b) return fail(PDLP_ERR_ARG, "NULL pointer");
  cudaStream_t st = (cudaStream_t)stream;
  // every partial the final sum reads is written by this call first: nothing
  // in the scratch has to start at zero
  const int chunks = (int)((n + kNaChunk - 1) / kNaChunk);
  dot_chunk_kernel<<<chunks, kT, 0, st>>>(n, a, b, scratch);
  reduce_final_kernel<<<1, kT, 0, st>>>(chunks, scratch, RED_DOT, scratch + kNaMaxChunks);
  count_launches(2);
  cudaError_t e = cudaGetLastError();
  double h = 0.0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&h, scratch + kNaMaxChunks, sizeof(double), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_fail(e, "pdlp_dot_noalloc");
  *out = h;
  return PDLP_OK;
}

}  // extern "C"
