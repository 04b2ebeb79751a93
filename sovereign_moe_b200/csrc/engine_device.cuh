// Device helpers of the PDLP engine: warp-level tile passes and reductions.
//
// Algorithm: restarted averaged PDHG of src/sovopt/lp/pdlp.py:238-494 with
// the method="pdlp" preconditioner of src/sovopt/numerics/scaling.py:149-478,
// executed as a per-LP state machine (see engine.cuh).  Every arithmetic
// expression of the reference's iteration is kept (same operands, same
// order), in float64.  Every sum uses an order that depends only on the LP
// (its rows and the lanes-per-row choice), never on the batch, so a run is
// bitwise repeatable and independent of the other LPs that share a launch.
#pragma once

#include "common.cuh"
#include "engine.cuh"

namespace pdlp {

constexpr int kWarps = 4;              // warps per block (engine kernels)
constexpr int kBlock = 32 * kWarps;    // threads per block
constexpr int kWTileRows = 64;         // rows per normal tile
constexpr int kWTileNnz = 512;         // entries per normal tile
constexpr int kVecs = 7;               // vectors staged for a hot-mode epilogue
constexpr double kRuizTol = 1e-2;      // scaling.py:149
constexpr unsigned kFull = 0xffffffffu;

// Per-warp shared memory.  The s* arrays receive bulk asynchronous copies
// (whole 16-byte chunks) of a tile's row pointers, indices, values and
// epilogue vectors; each has room for the alignment offset of the copied
// range.  sval doubles as the products' staging area.  bar[0] tracks the
// matrix copies of the current tile, bar[1] its epilogue vectors.
struct __align__(16) WarpSmem {
  unsigned long long bar[2];
  int sptr[kWTileRows + 8];
  int sidx[kWTileNnz + 8];
  double sval[kWTileNnz + 4];
  double vec[kVecs][kWTileRows + 4];
  double s0[kWTileRows];               // row sums, first right-hand side
  double s1[kWTileRows];               // row sums, second right-hand side
  int inst_id;
  int pad[3];
  Inst inst;                           // cached descriptor of inst_id
};

// ---- bulk asynchronous staging (cp.async.bulk + mbarrier) --------------------
//
// One lane of a warp arms the warp's mbarrier with the byte count of a group
// of copies and issues them; the copy engine writes shared memory and
// completes the barrier's phase when every byte has landed.  Sources are
// 16-byte aligned (arena arrays start on 256 bytes and ranges are rounded
// down to a 16-byte chunk); sizes are whole 16-byte chunks, reading at most
// 15 bytes past a range, which stays inside the slot's arena (every array is
// followed by padding).

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this warp's earlier shared-memory accesses (generic proxy) before
// the copy engine's writes (async proxy) into the same buffers.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Orders global-memory writes this thread has observed through the generic
// proxy (ordinary stores, made visible by a grid barrier) before the bulk
// copies it issues afterwards, which read global memory through the async
// proxy.
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
  return ok != 0;
}

// Whole 16-byte chunks covering elements [first, first + count) of E-byte
// elements; the copy starts at element first rounded down to a chunk.
template <int E>
__device__ __forceinline__ unsigned bulk_bytes(int first, int count) {
  constexpr int per = 16 / E;
  if (count <= 0) return 0u;
  const int a = first & ~(per - 1);
  return (unsigned)((first + count - a + per - 1) / per) * 16u;
}

template <int E>
__device__ __forceinline__ int bulk_offset(int first) {
  return first & (16 / E - 1);
}

template <int E>
__device__ __forceinline__ void bulk_stage(void* dst, const void* base, int first, int count,
                                           unsigned long long* bar) {
  const unsigned bytes = bulk_bytes<E>(first, count);
  if (bytes == 0u) return;
  const char* src = reinterpret_cast<const char*>(base) + (size_t)(first & ~(16 / E - 1)) * E;
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Per-warp state kept in registers for the launch: the phase bits of the two
// copy barriers, and the tiles of the current reduction group whose
// completion the warp has not counted yet.  A warp counts the tiles of one
// group that it processes back to back with one atomic, when it leaves the
// group (`flush`: its next tile lies in another group, or it has none).
struct BulkPhase {
  unsigned m = 0, v = 0;
  unsigned pend = 0;
  bool flush = true;
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

// Warp-wide reduction of kNP slots with a fixed xor tree; every lane ends
// with the result.
__device__ __forceinline__ void warp_reduce(double* v, Ops ops) {
#pragma unroll
  for (int s = 0; s < kNP; ++s) {
    const int op = ops.op(s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[s] = combine(v[s], __shfl_xor_sync(kFull, v[s], off), op);
  }
}

// ---- sparse passes over one tile (one warp) ---------------------------------

// Row sums of the tile for NR right-hand sides into W.s0 (W.s1).
// Normal tile: every entry's product is computed first -- all loads and
// gathers of the tile independent of each other -- and staged in shared
// memory; each row is then summed by L lanes (each lane its strided entries in
// storage order, then a xor butterfly; L == 1 is the storage-order sum).
// Heavy tile (one row longer than a normal tile holds): the 32 lanes stride
// over the row, then a xor butterfly.  Either way the order depends only on
// the row and L.  term(p, rhs) returns value[p] * x_rhs[index[p]].
template <int NR, class F>
__device__ __forceinline__ void warp_spmv(const Tile& t, const int* ptr, const int* tptr, int L,
                                          F term, WarpSmem& W, int lane) {
  if (t.heavy) {
    const int p0 = ld_ro(ptr + t.begin), p1 = ld_ro(ptr + t.begin + 1);
    double a0 = 0.0, a1 = 0.0;
    for (int p = p0 + lane; p < p1; p += 32) {
      a0 += term(p, 0);
      if (NR == 2) a1 += term(p, 1);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a0 += __shfl_xor_sync(kFull, a0, off);
      if (NR == 2) a1 += __shfl_xor_sync(kFull, a1, off);
    }
    if (lane == 0) { W.s0[0] = a0; if (NR == 2) W.s1[0] = a1; }
    __syncwarp();
    return;
  }
  // tptr[0..rows] are the tile's row pointers (staged by the caller)
  const int rows = t.end - t.begin;
  const int p0 = tptr[0];
  const int cnt = tptr[rows] - p0;
#pragma unroll 1
  for (int rhs = 0; rhs < NR; ++rhs) {
    for (int q0 = 0; q0 < cnt; q0 += 8 * 32) {
      double v[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int q = q0 + u * 32 + lane;
        v[u] = q < cnt ? term(p0 + q, rhs) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int q = q0 + u * 32 + lane;
        if (q < cnt) W.sval[q] = v[u];
      }
    }
    __syncwarp();
    double* out = rhs == 0 ? W.s0 : W.s1;
    const int sub = lane & (L - 1);
    const int grp = lane / L, ngrp = 32 / L;
    for (int rb = 0; rb < rows; rb += ngrp) {
      const int li = rb + grp;
      double a = 0.0;
      if (li < rows) {
        const int e = tptr[li + 1] - p0;
        int q = tptr[li] - p0 + sub;
        for (; q + 7 * L < e; q += 8 * L) {
          double v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) v[u] = W.sval[q + u * L];
#pragma unroll
          for (int u = 0; u < 8; ++u) a += v[u];
        }
        for (; q < e; q += L) a += W.sval[q];
      }
      for (int off = L >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(kFull, a, off);
      if (li < rows && sub == 0) out[li] = a;
    }
    __syncwarp();
  }
}

// Row sums from staged products: prod[q] for the tile's entries, row li
// spanning tptr[li]-p0 .. tptr[li+1]-p0; L lanes per row as in warp_spmv.
__device__ __forceinline__ void staged_row_sums(const int* tptr, const double* prod, int rows,
                                                int L, double* out, int lane) {
  const int p0 = tptr[0];
  const int sub = lane & (L - 1);
  const int grp = lane / L, ngrp = 32 / L;
  for (int rb = 0; rb < rows; rb += ngrp) {
    const int li = rb + grp;
    double a = 0.0;
    if (li < rows) {
      const int e = tptr[li + 1] - p0;
      int q = tptr[li] - p0 + sub;
      // eight loads in flight, the adds still in storage order
      for (; q + 7 * L < e; q += 8 * L) {
        double v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = prod[q + u * L];
#pragma unroll
        for (int u = 0; u < 8; ++u) a += v[u];
      }
      for (; q < e; q += L) a += prod[q];
    }
    for (int off = L >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(kFull, a, off);
    if (li < rows && sub == 0) out[li] = a;
  }
  __syncwarp();
}

// The same in float32 (FP32-SpMV precision): products in float, each row's
// sum accumulated in float in storage order, written out as double.
__device__ __forceinline__ void staged_row_sums_f32(const int* tptr, const float* prod, int rows,
                                                    int L, double* out, int lane) {
  const int p0 = tptr[0];
  const int sub = lane & (L - 1);
  const int grp = lane / L, ngrp = 32 / L;
  for (int rb = 0; rb < rows; rb += ngrp) {
    const int li = rb + grp;
    float a = 0.0f;
    if (li < rows) {
      const int e = tptr[li + 1] - p0;
      int q = tptr[li] - p0 + sub;
      for (; q + 7 * L < e; q += 8 * L) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = prod[q + u * L];
#pragma unroll
        for (int u = 0; u < 8; ++u) a += v[u];
      }
      for (; q < e; q += L) a += prod[q];
    }
    for (int off = L >> 1; off > 0; off >>= 1) a += __shfl_xor_sync(kFull, a, off);
    if (li < rows && sub == 0) out[li] = (double)a;
  }
  __syncwarp();
}

// Per-row max of f(r, p) over the tile (Ruiz pass); result in W.s0.
template <class F>
__device__ __forceinline__ void warp_rowmax(const Tile& t, const int* ptr, int L, F f,
                                            WarpSmem& W, int lane) {
  if (t.heavy) {
    const int p0 = ld_ro(ptr + t.begin), p1 = ld_ro(ptr + t.begin + 1);
    double a = 0.0;
    for (int p = p0 + lane; p < p1; p += 32) a = fmax(a, f(t.begin, p));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a = fmax(a, __shfl_xor_sync(kFull, a, off));
    if (lane == 0) W.s0[0] = a;
  } else {
    const int sub = lane & (L - 1), grp = lane / L, ngrp = 32 / L;
    for (int rb = t.begin; rb < t.end; rb += ngrp) {
      const int r = rb + grp;
      double a = 0.0;
      if (r < t.end) {
        const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
        for (int p = p0 + sub; p < p1; p += L) a = fmax(a, f(r, p));
      }
      for (int off = L >> 1; off > 0; off >>= 1) a = fmax(a, __shfl_xor_sync(kFull, a, off));
      if (r < t.end && sub == 0) W.s0[r - t.begin] = a;
    }
  }
  __syncwarp();
}

// Elementwise pass over the entries of the tile's rows: f(r, p).
template <class F>
__device__ __forceinline__ void warp_entries(const Tile& t, const int* ptr, F f, int lane) {
  for (int r = t.begin; r < t.end; ++r) {
    const int p0 = ld_ro(ptr + r), p1 = ld_ro(ptr + r + 1);
    for (int p = p0 + lane; p < p1; p += 32) f(r, p);
  }
}

// Last row (exclusive) this lane visits in a lane-per-row loop over the tile:
// every row of a normal tile, only lane 0 for a heavy (single-row) tile.
__device__ __forceinline__ int row_loop_end(const Tile& t, int lane) {
  return t.heavy ? (lane == 0 ? t.begin + 1 : t.begin) : t.end;
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
