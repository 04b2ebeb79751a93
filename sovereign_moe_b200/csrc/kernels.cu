// Kernel-level entry points mirroring the reference Backend
// (src/sovopt/core/backend.py:317-493): sparse products, the fused PDHG
// step kernels and the reductions, on device pointers and a caller stream.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <map>
#include <string>
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

// y = A x in two launches, with a fixed summation order.
//
// spmv_rows32_kernel: one warp per block of 32 consecutive rows.  Rows with
// more than kLongRow entries are not summed here: the warp appends them to a
// list (order immaterial) and leaves them to the second launch.
//
// Streamed variant (the default): the warp splits its block's short rows into
// runs of consecutive rows whose entries fit its staging buffer
// (kStageEntries).  A run's entries are one contiguous range of the CSR
// arrays, so the warp loads indices and values with coalesced, mutually
// independent loads, gathers every x it needs at once, and stages the
// products in shared memory.  Each lane then sums one row from the buffer in
// storage order.  A run costs two memory round trips, however many rows it
// has.
//
// Row-group variant: the warp picks L lanes per row from the block's mean
// row length (a power of two, 1..32); each lane sums its strided entries in
// order, a xor butterfly over the L lanes combines them, and 32/L rows run
// side by side.
//
// spmv_long_rows_kernel: one block of 8 warps per listed long row (grid-
// stride).  Chunk c of the row goes to warp c mod 8, which keeps a per-lane
// running sum.  A warp tree and then the 8 warp sums in order give the row
// sum.  So the result of every row depends only on the matrix, not on the
// list order or the launch shape, and repeated calls give the same bits.
constexpr int kSpmvWarps = 8;
constexpr int kLongRow = 256;
constexpr int kStageEntries = 256;     // entries a warp stages for one run of rows
constexpr int kStageUnroll = 8;        // independent loads per lane in flight

// Variants of the row-block pass (pdlp_spmv_*_ex): streamed where a run of
// rows fits the staging buffer, or the row-group path for every block.
enum SpmvVariant : int { SPMV_AUTO = 0, SPMV_STREAMED = 1, SPMV_ROW_GROUPS = 2, SPMV_BANDED = 3 };
constexpr int kBandCap = 3072;         // x entries a block stages (banded variant)

// Streams the rows i0 .. i1-1 of the warp's block (rows r0 + i), whose
// entries are [p0, p0 + cnt), cnt <= kStageEntries: coalesced, independent
// loads of indices and values, every gather at once, products staged in
// shared memory; lane i then sums row i in storage order.
//
// With a band (banded variant), x[blo, blo + bcnt) is already in shared memory
// and the gathers that fall in it read from there.
template <typename T>
__device__ __forceinline__ void spmv_rows_staged(int r0, int i0, int i1, long long rs,
                                                 long long re, long long p0, int cnt, int lane,
                                                 const int* __restrict__ ri,
                                                 const T* __restrict__ rx,
                                                 const T* __restrict__ x, T* __restrict__ y,
                                                 T* __restrict__ prod,
                                                 const T* band = nullptr, int blo = 0,
                                                 int bcnt = 0) {
  for (int q0 = 0; q0 < cnt; q0 += kStageUnroll * 32) {
    int idx[kStageUnroll];
    T val[kStageUnroll];
#pragma unroll
    for (int u = 0; u < kStageUnroll; ++u) {
      const int q = q0 + u * 32 + lane;
      idx[u] = q < cnt ? __ldg(ri + p0 + q) : 0;
      val[u] = q < cnt ? __ldg(rx + p0 + q) : T(0);
    }
    T xv[kStageUnroll];
#pragma unroll
    for (int u = 0; u < kStageUnroll; ++u) {
      const int q = q0 + u * 32 + lane;
      const unsigned off = (unsigned)(idx[u] - blo);
      xv[u] = q < cnt ? (off < (unsigned)bcnt ? band[off] : __ldg(x + idx[u])) : T(0);
    }
#pragma unroll
    for (int u = 0; u < kStageUnroll; ++u) {
      const int q = q0 + u * 32 + lane;
      if (q < cnt) prod[q] = val[u] * xv[u];
    }
  }
  __syncwarp();
  if (lane >= i0 && lane < i1) {
    const int e = (int)(re - p0);
    int q = (int)(rs - p0);
    T a = T(0);
    for (; q + 3 < e; q += 4) {       // four loads in flight, the adds in storage order
      const T v0 = prod[q], v1 = prod[q + 1], v2 = prod[q + 2], v3 = prod[q + 3];
      a += v0;
      a += v1;
      a += v2;
      a += v3;
    }
    for (; q < e; ++q) a += prod[q];
    y[r0 + lane] = a;
  }
  __syncwarp();
}

// The run of rows that starts at row `start` of a warp's block (a short row):
// the consecutive short rows from there whose entries fit the staging buffer
// together.  Rows are contiguous in storage, so the run's entries are one
// range; a long row, the buffer's capacity or the block's end closes it.
// Returns the run's end (exclusive), the same in every lane.
__device__ __forceinline__ int spmv_next_run(int start, int nr, long long rs, long long re,
                                             unsigned long_mask, int lane) {
  const long long base = __shfl_sync(kAll, rs, start);
  const bool ok = lane >= start && lane < nr && !((long_mask >> lane) & 1u) &&
                  re - base <= kStageEntries;
  const unsigned fit = __ballot_sync(kAll, ok) >> start;    // bit 0: row `start`
  const unsigned gap = ~fit;
  const int len = gap ? __ffs(gap) - 1 : 32 - start;
  return start + len;
}

template <typename T, int L>
__device__ __forceinline__ void spmv_block_rows(int r0, int nr, long long rs, long long re,
                                                unsigned long_mask, int lane,
                                                const int* __restrict__ ri,
                                                const T* __restrict__ rx,
                                                const T* __restrict__ x, T* __restrict__ y) {
  constexpr int G = 32 / L;
  const int sub = lane & (L - 1), gi = lane / L;
  for (int g = 0; g < nr; g += G) {
    const int i = g + gi;                       // row of this lane's group, within the block
    const long long p0 = __shfl_sync(kAll, rs, i & 31);
    const long long p1 = __shfl_sync(kAll, re, i & 31);
    const bool active = i < nr && !((long_mask >> i) & 1u);
    T acc = T(0);
    if (active) {
#pragma unroll 4
      for (long long p = p0 + sub; p < p1; p += L) acc += __ldg(rx + p) * __ldg(x + __ldg(ri + p));
    }
#pragma unroll
    for (int off = L >> 1; off > 0; off >>= 1) acc += __shfl_xor_sync(kAll, acc, off);
    if (active && sub == 0) y[r0 + i] = acc;
  }
}

template <typename T>
__global__ void __launch_bounds__(kSpmvWarps * 32) spmv_rows32_kernel(
    int m, const int64_t* __restrict__ rp, const int* __restrict__ ri,
    const T* __restrict__ rx, const T* __restrict__ x, T* __restrict__ y,
    int* __restrict__ long_rows, int variant) {
  __shared__ T stage[kSpmvWarps][kStageEntries];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long nblk = ((long long)m + 31) / 32;
  const long long stride = (long long)gridDim.x * kSpmvWarps;
  for (long long b = (long long)blockIdx.x * kSpmvWarps + w; b < nblk; b += stride) {
    const int r0 = (int)(b * 32);
    const int nr = min(32, m - r0);
    const long long rs = lane < nr ? (long long)__ldg(rp + r0 + lane) : 0LL;
    const long long re = lane < nr ? (long long)__ldg(rp + r0 + lane + 1) : 0LL;
    const bool is_long = lane < nr && re - rs > kLongRow;
    if (is_long) {
      // a count left over by a failed earlier call cannot push a write past
      // the list (m + 2 entries): the slot is checked
      const int slot = atomicAdd(long_rows, 1);
      if (slot < m) long_rows[2 + slot] = r0 + lane;
    }
    const unsigned long_mask = __ballot_sync(kAll, is_long);
    const unsigned rows_mask = nr == 32 ? kAll : ((1u << nr) - 1u);
    unsigned skip = long_mask;                  // rows the row-group path leaves alone
    if (variant != SPMV_ROW_GROUPS) {
      // every short row, in runs that fit the buffer; long rows are left to
      // the second launch
      for (int start = 0; start < nr;) {
        if ((long_mask >> start) & 1u) { ++start; continue; }
        const int end = spmv_next_run(start, nr, rs, re, long_mask, lane);
        const long long qa = __shfl_sync(kAll, rs, start), qb = __shfl_sync(kAll, re, end - 1);
        spmv_rows_staged<T>(r0, start, end, rs, re, qa, (int)(qb - qa), lane, ri, rx, x, y,
                            stage[w]);
        start = end;
      }
      continue;
    }
    // mean length of the rows left -> lanes per row
    const bool mine = lane < nr && !((skip >> lane) & 1u);
    long long len = mine ? re - rs : 0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) len += __shfl_xor_sync(kAll, len, off);
    const int left = __popc(rows_mask & ~skip);
    const long long avg = left > 0 ? (len + left - 1) / left : 0;
    if (avg <= 1) spmv_block_rows<T, 1>(r0, nr, rs, re, skip, lane, ri, rx, x, y);
    else if (avg <= 2) spmv_block_rows<T, 2>(r0, nr, rs, re, skip, lane, ri, rx, x, y);
    else if (avg <= 4) spmv_block_rows<T, 4>(r0, nr, rs, re, skip, lane, ri, rx, x, y);
    else if (avg <= 8) spmv_block_rows<T, 8>(r0, nr, rs, re, skip, lane, ri, rx, x, y);
    else if (avg <= 16) spmv_block_rows<T, 16>(r0, nr, rs, re, skip, lane, ri, rx, x, y);
    else spmv_block_rows<T, 32>(r0, nr, rs, re, skip, lane, ri, rx, x, y);
  }
}

// Banded variant: one block per 256 consecutive rows (a warp per 32), no
// grid stride.  The block first reads the indices of its short rows (the
// entries the runs will stage) and reduces their smallest and largest; when
// that span fits kBandCap entries (3072), the block loads x over it into
// shared memory with coalesced loads, and the runs' gathers read from there
// instead of from L2.  Long rows go to the second launch, as in the other
// variants.
template <typename T>
__global__ void __launch_bounds__(kSpmvWarps * 32) spmv_band_kernel(
    int m, const int64_t* __restrict__ rp, const int* __restrict__ ri,
    const T* __restrict__ rx, const T* __restrict__ x, T* __restrict__ y,
    int* __restrict__ long_rows) {
  __shared__ T stage[kSpmvWarps][kStageEntries];
  __shared__ T band[kBandCap];
  __shared__ int wlo[kSpmvWarps], whi[kSpmvWarps];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const long long nblk = ((long long)m + 31) / 32;
  const long long b = (long long)blockIdx.x * kSpmvWarps + w;
  const bool have = b < nblk;                       // warp-uniform
  const int r0 = have ? (int)(b * 32) : 0;
  const int nr = have ? min(32, m - r0) : 0;
  const long long rs = lane < nr ? (long long)__ldg(rp + r0 + lane) : 0LL;
  const long long re = lane < nr ? (long long)__ldg(rp + r0 + lane + 1) : 0LL;
  const bool is_long = lane < nr && re - rs > kLongRow;
  if (is_long) {
    const int slot = atomicAdd(long_rows, 1);
    if (slot < m) long_rows[2 + slot] = r0 + lane;
  }
  const unsigned long_mask = __ballot_sync(kAll, is_long);
  // the span of the short rows' indices (the entries the runs will stage),
  // over the block
  int lo = 0x7fffffff, hi = -1;
  for (int start = 0; start < nr;) {
    if ((long_mask >> start) & 1u) { ++start; continue; }
    const int end = spmv_next_run(start, nr, rs, re, long_mask, lane);
    const long long qa = __shfl_sync(kAll, rs, start), qb = __shfl_sync(kAll, re, end - 1);
    for (long long q = qa + lane; q < qb; q += 32) {
      const int j = __ldg(ri + q);
      lo = min(lo, j);
      hi = max(hi, j);
    }
    start = end;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    lo = min(lo, __shfl_xor_sync(kAll, lo, off));
    hi = max(hi, __shfl_xor_sync(kAll, hi, off));
  }
  if (lane == 0) { wlo[w] = lo; whi[w] = hi; }
  __syncthreads();
  int blo = 0x7fffffff, bhi = -1;
  for (int k = 0; k < kSpmvWarps; ++k) { blo = min(blo, wlo[k]); bhi = max(bhi, whi[k]); }
  const int bcnt = (bhi >= blo && bhi - blo < kBandCap) ? bhi - blo + 1 : 0;   // block-uniform
  for (int i = threadIdx.x; i < bcnt; i += kSpmvWarps * 32) band[i] = __ldg(x + blo + i);
  __syncthreads();
  for (int start = 0; start < nr;) {
    if ((long_mask >> start) & 1u) { ++start; continue; }
    const int end = spmv_next_run(start, nr, rs, re, long_mask, lane);
    const long long qa = __shfl_sync(kAll, rs, start), qb = __shfl_sync(kAll, re, end - 1);
    spmv_rows_staged<T>(r0, start, end, rs, re, qa, (int)(qb - qa), lane, ri, rx, x, y, stage[w],
                        band, blo, bcnt);
    start = end;
  }
}

template <typename T>
__global__ void __launch_bounds__(kSpmvWarps * 32) spmv_long_rows_kernel(
    const int64_t* __restrict__ rp, const int* __restrict__ ri, const T* __restrict__ rx,
    const T* __restrict__ x, T* __restrict__ y, int m, int* __restrict__ long_rows) {
  __shared__ T part[kSpmvWarps];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int count = min(long_rows[0], m);
  for (int k = blockIdx.x; k < count; k += gridDim.x) {
    const int r = long_rows[2 + k];
    if (r < 0 || r >= m) continue;    // only after a failed earlier call (block-uniform)
    const long long p0 = __ldg(rp + r), p1 = __ldg(rp + r + 1);
    T sum = T(0);
    for (long long base = p0 + 128LL * w; base < p1; base += 128LL * kSpmvWarps) {
      int idx[4];
      T val[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const long long p = base + lane + 32 * u;
        idx[u] = p < p1 ? __ldg(ri + p) : 0;
        val[u] = p < p1 ? __ldg(rx + p) : T(0);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const long long p = base + lane + 32 * u;
        if (p < p1) sum += val[u] * __ldg(x + idx[u]);
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(kAll, sum, off);
    if (lane == 0) part[w] = sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      T t = T(0);
      for (int i = 0; i < kSpmvWarps; ++i) t += part[i];
      y[r] = t;
    }
    __syncthreads();
  }
  // the last block to finish clears the count and this counter for the next
  // call on the stream (every block read the count before it got here)
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(long_rows + 1, 1) == (int)gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    long_rows[0] = 0;
    long_rows[1] = 0;
  }
}

// The long-row list of each (device, stream): a count, a counter of finished
// blocks, then row indices.  It is kept between calls and grown when a larger
// m comes, so a call allocates nothing in the common case.  Both counters are
// zeroed when the list is allocated, and the long-row kernel zeroes them again
// at its end, so a call needs no reset of its own.  Calls on one stream are
// ordered by the stream; calls on different streams use different lists.
std::mutex spmv_mu;
std::map<std::pair<int, cudaStream_t>, std::pair<int*, size_t>> spmv_lists;

int long_row_list(cudaStream_t st, size_t entries, int** out) {
  int dev = 0;
  PDLP_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(spmv_mu);
  auto& slot = spmv_lists[{dev, st}];
  if (slot.second < entries) {
    if (slot.first) {
      PDLP_CUDA(cudaStreamSynchronize(st));
      cudaFree(slot.first);
      slot = {nullptr, 0};
    }
    const size_t n = std::max(entries, (size_t)1 << 16);
    PDLP_CUDA(cudaMalloc((void**)&slot.first, sizeof(int) * n));
    PDLP_CUDA(cudaMemsetAsync(slot.first, 0, 2 * sizeof(int), st));
    slot.second = n;
  }
  *out = slot.first;
  return PDLP_OK;
}

template <typename T>
int launch_spmv(int m, const int64_t* rp, const int* ri, const T* rx, const T* x, T* y,
                cudaStream_t st, int variant = SPMV_AUTO) {
  if (m < 0) return fail(PDLP_ERR_ARG, "m must be >= 0");
  if (variant < SPMV_AUTO || variant > SPMV_BANDED) return fail(PDLP_ERR_ARG, "unknown SpMV variant");
  if (m == 0) return PDLP_OK;
  if (!rp || !ri || !rx || !x || !y) return fail(PDLP_ERR_ARG, "NULL pointer");
  int* long_rows = nullptr;
  const int rc = long_row_list(st, (size_t)m + 2, &long_rows);
  if (rc != PDLP_OK) return rc;
  const long long nblk = ((long long)m + 31) / 32;
  const int g = (int)std::min((nblk + kSpmvWarps - 1) / kSpmvWarps, 1LL << 30);
  if (variant == SPMV_BANDED) {
    const long long gb = (nblk + kSpmvWarps - 1) / kSpmvWarps;
    if (gb > (1LL << 31) - 1) return fail(PDLP_ERR_ARG, "m too large for the banded variant");
    spmv_band_kernel<T><<<(int)gb, kSpmvWarps * 32, 0, st>>>(m, rp, ri, rx, x, y, long_rows);
  } else {
    spmv_rows32_kernel<T><<<g, kSpmvWarps * 32, 0, st>>>(m, rp, ri, rx, x, y, long_rows, variant);
  }
  spmv_long_rows_kernel<T><<<592, kSpmvWarps * 32, 0, st>>>(rp, ri, rx, x, y, m, long_rows);
  count_launches(2);
  PDLP_CUDA(cudaGetLastError());
  return PDLP_OK;
}

// The SpMV autotuner: times every variant of the row-block pass on the
// caller's matrix and vectors (one warm call each, then three interleaved
// rounds of `reps` calls per variant bracketed by CUDA events on the caller's
// stream, keeping each variant's fastest round, so that a passing change of
// the GPU's state does not decide the choice) and returns the fastest.  Its
// cost is about a hundred SpMVs; the caller keeps the choice for the matrix.
template <typename T>
int tune_spmv(int m, const int64_t* rp, const int* ri, const T* rx, const T* x, T* y,
              cudaStream_t st, int reps, int* best, double* ms_out) {
  if (!best) return fail(PDLP_ERR_ARG, "best is NULL");
  if (reps <= 0) reps = 10;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  PDLP_CUDA(cudaEventCreate(&e0));
  const cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) { cudaEventDestroy(e0); return cuda_fail(ce, "cudaEventCreate"); }
  constexpr int kRounds = 3;
  const int variants[3] = {SPMV_STREAMED, SPMV_ROW_GROUPS, SPMV_BANDED};
  double per_ms[3] = {0.0, 0.0, 0.0};
  int rc = PDLP_OK;
  for (int k = 0; k < 3 && rc == PDLP_OK; ++k) rc = launch_spmv<T>(m, rp, ri, rx, x, y, st, variants[k]);
  for (int round = 0; round < kRounds && rc == PDLP_OK; ++round) {
    for (int k = 0; k < 3 && rc == PDLP_OK; ++k) {
      cudaEventRecord(e0, st);
      for (int r = 0; r < reps && rc == PDLP_OK; ++r)
        rc = launch_spmv<T>(m, rp, ri, rx, x, y, st, variants[k]);
      cudaEventRecord(e1, st);
      const cudaError_t se = cudaEventSynchronize(e1);
      if (se != cudaSuccess) { rc = cuda_fail(se, "cudaEventSynchronize"); break; }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      const double per = (double)ms / reps;
      if (round == 0 || per < per_ms[k]) per_ms[k] = per;
    }
  }
  *best = SPMV_STREAMED;
  if (rc == PDLP_OK) {
    double best_ms = per_ms[0];
    for (int k = 0; k < 3; ++k) {
      if (ms_out) ms_out[k] = per_ms[k];
      if (per_ms[k] < best_ms) { best_ms = per_ms[k]; *best = variants[k]; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
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

int pdlp_spmv_ex_f64(int32_t variant, int32_t m, const int64_t* rp, const int32_t* ri,
                     const double* rx, const double* x, double* y, void* stream) {
  return launch_spmv<double>(m, rp, ri, rx, x, y, (cudaStream_t)stream, variant);
}

int pdlp_spmv_ex_f32(int32_t variant, int32_t m, const int64_t* rp, const int32_t* ri,
                     const float* rx, const float* x, float* y, void* stream) {
  return launch_spmv<float>(m, rp, ri, rx, x, y, (cudaStream_t)stream, variant);
}

int pdlp_spmv_tune_f64(int32_t m, const int64_t* rp, const int32_t* ri, const double* rx,
                       const double* x, double* y, void* stream, int32_t reps,
                       int32_t* best_variant, double* ms_per_variant) {
  return tune_spmv<double>(m, rp, ri, rx, x, y, (cudaStream_t)stream, reps, best_variant,
                           ms_per_variant);
}

int pdlp_spmv_tune_f32(int32_t m, const int64_t* rp, const int32_t* ri, const float* rx,
                       const float* x, float* y, void* stream, int32_t reps,
                       int32_t* best_variant, double* ms_per_variant) {
  return tune_spmv<float>(m, rp, ri, rx, x, y, (cudaStream_t)stream, reps, best_variant,
                          ms_per_variant);
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
