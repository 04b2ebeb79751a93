// Device code of the PDLP engine: tile passes, finishers, grid barrier.
//
// Algorithm: restarted averaged PDHG of src/sovopt/lp/pdlp.py:238-494 with
// the method="pdlp" preconditioner of src/sovopt/numerics/scaling.py:149-478,
// executed as a per-LP state machine (see engine.cuh).  Every arithmetic
// expression of the reference's iteration is kept (same operands, same
// order), in float64; sums over rows/columns use a fixed reduction tree, so a
// run is bitwise repeatable and independent of the other LPs in the batch.
#pragma once

#include "common.cuh"
#include "engine.cuh"

namespace pdlp {

constexpr int kBlock = 256;            // threads per block (all engine kernels)
constexpr int kMaxTileRows = 1024;     // rows per tile (shared-memory staging)
constexpr int kTileNnz = 4096;         // entries per normal tile (products staged in smem)
constexpr double kRuizTol = 1e-2;      // scaling.py:149
constexpr unsigned kFull = 0xffffffffu;

// Per-block shared memory (dynamic: larger than the 48 KB static limit).
struct Smem {
  double prod[kTileNnz];               // products of the tile's entries
  double s0[kMaxTileRows];             // row sums, first right-hand side
  double s1[kMaxTileRows];             // row sums, second right-hand side
  int ptr[kMaxTileRows + 1];           // the tile's row pointers
  double red[32 * kNP];
  double res[kNP];
  Inst inst;                           // cached descriptor of inst_id
  int inst_id;
  int flag;
};

// ---- reductions -----------------------------------------------------------

enum : int { OP_SUM = 0, OP_MAX = 1, OP_MIN = 2 };

__device__ __forceinline__ double combine(double a, double b, int op) {
  return op == OP_SUM ? a + b : (op == OP_MAX ? fmax(a, b) : fmin(a, b));
}

__device__ __forceinline__ double identity_of(int op) {
  return op == OP_MIN ? INFINITY : 0.0;
}

struct Ops {
  unsigned maxmask = 0, minmask = 0;
  __device__ __forceinline__ int op(int s) const {
    return (maxmask >> s & 1u) ? OP_MAX : ((minmask >> s & 1u) ? OP_MIN : OP_SUM);
  }
};

// Block-wide reduction of kNP slots; the result lands in sm.res (all threads
// may read it after the call).  Fixed shuffle tree: deterministic.
__device__ void block_reduce(double* v, Ops ops, Smem& sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
#pragma unroll
  for (int s = 0; s < kNP; ++s) {
    int op = ops.op(s);
    double a = v[s];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a = combine(a, __shfl_down_sync(kFull, a, off), op);
    if (lane == 0) sm.red[warp * kNP + s] = a;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int s = 0; s < kNP; ++s) {
      int op = ops.op(s);
      double a = lane < nwarps ? sm.red[lane * kNP + s] : identity_of(op);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a = combine(a, __shfl_down_sync(kFull, a, off), op);
      if (lane == 0) sm.res[s] = a;
    }
  }
  __syncthreads();
}

// ---- sparse row passes ----------------------------------------------------

// out[r - b] = sum over row r of term(r, p), rows [b, e), L lanes per row.
// Each lane sums its strided entries in storage order, then a xor butterfly
// combines the L lanes; with L == 1 the sum is fully sequential.
template <int NR, class F>
__device__ __forceinline__ void rows_spmv(const int* __restrict__ ptr, int b, int e, int L,
                                          F f, double* s0, double* s1) {
  const int tid = threadIdx.x;
  const int lane = tid & (L - 1);
  const int grp = tid / L, ngrp = blockDim.x / L;
  for (int rb = b; rb < e; rb += ngrp) {
    const int r = rb + grp;
    double a0 = 0.0, a1 = 0.0;
    if (r < e) {
      const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
      for (int p = p0 + lane; p < p1; p += L) f(r, p, a0, a1);
    }
    for (int off = L >> 1; off > 0; off >>= 1) {
      a0 += __shfl_xor_sync(kFull, a0, off);
      if (NR == 2) a1 += __shfl_xor_sync(kFull, a1, off);
    }
    if (r < e && lane == 0) {
      s0[r - b] = a0;
      if (NR == 2) s1[r - b] = a1;
    }
  }
}

// One long row reduced by the whole block (fixed tree); result in s0[0], s1[0].
template <int NR, class F>
__device__ __forceinline__ void heavy_spmv(const int* __restrict__ ptr, int r, F f,
                                           double* s0, double* s1, Smem& sm) {
  const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
  double v[kNP];
#pragma unroll
  for (int s = 0; s < kNP; ++s) v[s] = 0.0;
  for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) f(r, p, v[0], v[1]);
  block_reduce(v, Ops{}, sm);
  if (threadIdx.x == 0) {
    s0[0] = sm.res[0];
    if (NR == 2) s1[0] = sm.res[1];
  }
  __syncthreads();
}

// Row sums of a normal tile, CSR-stream style: every entry's product is
// computed first (all loads and gathers of the tile independent of each
// other), staged in shared memory, then each row is summed from there by L
// lanes (each lane its strided entries in storage order, then a xor
// butterfly; L == 1 is the sequential storage-order sum).  The order depends
// only on the row and on L, never on the tile or the batch.
// term(p, rhs) returns value[p] * x_rhs[index[p]].
template <int NR, class F>
__device__ __forceinline__ void stream_spmv(const Tile& t, int L, F term, Smem& sm) {
  const int tid = threadIdx.x, BT = blockDim.x;
  const int rows = t.end - t.begin;
  const int p0 = sm.ptr[0];
  const int cnt = sm.ptr[rows] - p0;
#pragma unroll 1
  for (int rhs = 0; rhs < NR; ++rhs) {
    for (int q0 = 0; q0 < cnt; q0 += 4 * BT) {
      double v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + u * BT + tid;
        v[u] = q < cnt ? term(p0 + q, rhs) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + u * BT + tid;
        if (q < cnt) sm.prod[q] = v[u];
      }
    }
    __syncthreads();
    double* out = rhs == 0 ? sm.s0 : sm.s1;
    const int lane = tid & (L - 1);
    const int grp = tid / L, ngrp = BT / L;
    for (int rb = 0; rb < rows; rb += ngrp) {
      const int li = rb + grp;
      double a = 0.0;
      if (li < rows) {
        const int e = sm.ptr[li + 1] - p0;
        for (int q = sm.ptr[li] - p0 + lane; q < e; q += L) a += sm.prod[q];
      }
      for (int off = L >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(kFull, a, off);
      if (li < rows && lane == 0) out[li] = a;
    }
    __syncthreads();
  }
}

// Loads the tile's row pointers into shared memory (normal tiles).
__device__ __forceinline__ void load_tile_ptr(const Tile& t, const int* ptr, Smem& sm) {
  if (t.heavy) return;
  const int rows = t.end - t.begin;
  for (int i = threadIdx.x; i <= rows; i += blockDim.x) sm.ptr[i] = ld_ro(ptr + t.begin + i);
  __syncthreads();
}

template <int NR, class F>
__device__ __forceinline__ void tile_spmv(const Tile& t, const int* ptr, int L, F term, Smem& sm) {
  if (t.heavy) {
    auto f = [&](int r, int p, double& a0, double& a1) {
      a0 += term(p, 0);
      if (NR == 2) a1 += term(p, 1);
    };
    heavy_spmv<NR>(ptr, t.begin, f, sm.s0, sm.s1, sm);
  } else {
    load_tile_ptr(t, ptr, sm);
    stream_spmv<NR>(t, L, term, sm);
  }
  __syncthreads();
}

// Max of |w| over each row after an optional in-place rescale (Ruiz pass).
template <class F>
__device__ __forceinline__ void tile_rowmax(const Tile& t, const int* ptr, int L, F f, Smem& sm) {
  if (t.heavy) {
    const int r = t.begin;
    const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
    double v[kNP];
#pragma unroll
    for (int s = 0; s < kNP; ++s) v[s] = 0.0;
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) v[0] = fmax(v[0], f(r, p));
    Ops o; o.maxmask = 1u;
    block_reduce(v, o, sm);
    if (threadIdx.x == 0) sm.s0[0] = sm.res[0];
  } else {
    const int tid = threadIdx.x;
    const int lane = tid & (L - 1), grp = tid / L, ngrp = blockDim.x / L;
    for (int rb = t.begin; rb < t.end; rb += ngrp) {
      const int r = rb + grp;
      double a = 0.0;
      if (r < t.end) {
        const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
        for (int p = p0 + lane; p < p1; p += L) a = fmax(a, f(r, p));
      }
      for (int off = L >> 1; off > 0; off >>= 1) a = fmax(a, __shfl_xor_sync(kFull, a, off));
      if (r < t.end && lane == 0) sm.s0[r - t.begin] = a;
    }
  }
  __syncthreads();
}

// Elementwise pass over the entries of the tile's rows.
template <class F>
__device__ __forceinline__ void tile_entries(const Tile& t, const int* ptr, F f) {
  if (t.heavy) {
    const int r = t.begin;
    const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
    for (int p = p0 + threadIdx.x; p < p1; p += blockDim.x) f(r, p);
  } else {
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    for (int r = t.begin + warp; r < t.end; r += nw) {
      const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
      for (int p = p0 + lane; p < p1; p += 32) f(r, p);
    }
  }
}

// Last row (exclusive) this thread visits in a thread-per-row loop over the
// tile: all rows of a normal tile, only thread 0 for a heavy (single-row) tile.
__device__ __forceinline__ int row_loop_end(const Tile& t) {
  return t.heavy ? (threadIdx.x == 0 ? t.begin + 1 : t.begin) : t.end;
}

// ---- small math shared by both sides -------------------------------------------

__device__ __forceinline__ double row_bound(double b, double s) {
  double o = b * s;
  if (b <= -kInf) o = -kInf;
  if (b >= kInf) o = kInf;
  return o;
}

__device__ __forceinline__ double col_bound(double b, double s) {
  double o = b / s;
  if (b <= -kInf) o = -kInf;
  if (b >= kInf) o = kInf;
  return o;
}

// Moreau prox of the row box (backend.py:217-231): w - sigma clip(w/sigma, rl, ru).
__device__ __forceinline__ double prox(double w, double sigma, double rl, double ru) {
  double t = w / sigma;
  return w - sigma * clip(t, rl, ru);
}

// distance of ax from [rl, ru] (pdlp.py:199)
__device__ __forceinline__ double pviol(double ax, double rl, double ru) {
  return fmax(rl - ax, 0.0) + fmax(ax - ru, 0.0);
}

// -delta*_C(y) term: y times the bound its sign selects (pdlp.py:213-214)
__device__ __forceinline__ double supp(double y, double rl, double ru) {
  double b = y > 0.0 ? (ru < kInf ? ru : 0.0) : (rl > -kInf ? rl : 0.0);
  return b * y;
}

// dual infeasibility of reduced cost d (pdlp.py:204-207)
__device__ __forceinline__ double dres(double d, double lo, double hi) {
  return (lo > -kInf ? 0.0 : fmax(d, 0.0)) + (hi < kInf ? 0.0 : fmax(-d, 0.0));
}

// bound term of the dual objective (pdlp.py:215-216)
__device__ __forceinline__ double bndterm(double d, double lo, double hi) {
  double b = d > 0.0 ? (lo > -kInf ? lo : 0.0) : (hi < kInf ? hi : 0.0);
  return b * d;
}

__device__ __forceinline__ double bviol(double x, double lo, double hi) {
  return fmax(lo - x, 0.0) + fmax(x - hi, 0.0);
}

// Deterministic standard normal for the device-generated power start vector.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ double gen_normal(unsigned long long i) {
  unsigned long long a = mix64(2 * i + 1), b = mix64(2 * i + 2);
  double u1 = ((a >> 11) + 1) * (1.0 / 9007199254740993.0);   // (0, 1]
  double u2 = (b >> 11) * (1.0 / 9007199254740992.0);         // [0, 1)
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

}  // namespace pdlp
