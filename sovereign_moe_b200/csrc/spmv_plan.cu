// Planned SpMV (pdlp_spmv_plan_*): y = A x for a CSR matrix whose structure
// is analysed once and whose products are then taken many times -- the
// PDHG loop multiplies by the same A and A^T at every iteration.  It does the
// reference Backend's spmv (src/sovopt/core/backend.py:373-384, the kernel at
// backend.py:118-152) on a fixed sparsity pattern.
//
// The plan (host code, once per matrix) cuts the rows into tiles of at most
// kPlanRows consecutive rows and kPlanNnz entries.  For each tile it picks
//   * a window of at most kPlanBand consecutive columns holding as many of the
//     tile's column indices as possible (a banded matrix, such as a
//     multi-period plan, has one per tile), and
//   * a halo: up to kHalo further columns, the ones the tile uses most often
//     outside the window (e.g. the coupling rows of a multi-period plan).
// It keeps its own copy of the column indices, rewritten per entry: an index
// into the tile's staged x (window or halo), or -(j + 1) for an entry whose x
// is gathered from global memory.  A row longer than kPlanNnz is a tile of
// its own ("huge").  The tiles are split into one contiguous range per CTA
// with about equal estimated time.
//
// The kernel is persistent: one CTA per SM around a ring of kPlanStages
// shared-memory stages, with three roles.
//   * The copy warp's elected lane issues, per tile, bulk asynchronous copies
//     (cp.async.bulk, completion counted on the stage's mbarrier) of the row
//     pointers, rewritten indices, values and x window.
//   * The halo warp gathers the tile's halo from x into the stage, one load
//     per lane, issuing the next tile's loads before it stores this tile's.
//   * kPlanCW consumer warps, in kGroups groups that take alternate tiles,
//     wait for the stage, sum the rows, and release it.
// So the matrix streams from HBM while earlier tiles are being summed, and
// the gathers of x read shared memory instead of one L1 wavefront each.
//
// Each product is launched as a programmatic dependent of the kernel before
// it in the stream.  Its CTAs take an SM as the previous kernel's CTAs leave
// it, fetch their tile descriptors and copy the plan's arrays (row order,
// row pointers, indices) of the first tile of each consumer group.  Only
// after the previous kernel has completed (griddepcontrol.wait) do they read
// the caller's values and x or write y.  In a loop of products this hides the
// launch and the first copies of each product behind the tail of the one
// before.
//
// Summation order (fixed by the matrix alone, so repeated calls give the same
// bits):
//   * a row of at most kLaneRow entries: one lane, storage order, each product
//     rounded before it is added -- the order of the reference's CPU kernel
//     (src/sovopt/core/sparse.py:50-58), so these rows equal it bit for bit
//     (the plan orders a tile's rows so that a warp's 32 rows start on
//     different shared-memory banks);
//   * a longer row of a normal tile: lane l sums entries l, l+32, ... in
//     order, then a xor butterfly over the warp;
//   * a huge row: one warp (the first of the group that takes the tile),
//     read from global memory, in the same lane-strided order as a longer
//     row.
//
// Every wait on an mbarrier is bounded in wall time (kPlanWaitNs).  A wait
// that runs out records PDLP_ERR_BARRIER_TIMEOUT in the plan's status word
// and that warp stops; the warps waiting on it then run out in turn (the
// consumers share no barrier among themselves), and the copy warp waits
// (again bounded) for the copies it has in flight before it exits.
// pdlp_spmv_plan_status reads the word.
#include <algorithm>
#include <chrono>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine_device.cuh"

#include <cstdint>

// The opaque handle of include/pdlp_b200.h.
struct pdlp_spmv_plan {
  int device = 0;
  int m = 0, n = 0;
  int64_t* rp = nullptr;        // copy of the row pointers, device
  int32_t* idx = nullptr;       // rewritten indices (tiles) or a copy of ri (row-block kernel)
  void* tiles = nullptr;        // PlanTile[ntiles], device
  int* cta_first = nullptr;     // [nctas + 1], device
  int* long_rows = nullptr;     // row (within its tile) of each row of 65..2048 entries
  int* halo_cols = nullptr;     // columns of each tile's halo, in tile order
  uint16_t* perm = nullptr;     // per row: the order in which a tile's short rows meet lanes
  int* status = nullptr;        // device word: 0 or the error of a wait that ran out
  int64_t base = 0;             // the caller's rp[0]: entry q of the plan is the caller's base + q
  int ntiles = 0, nctas = 0;
  pdlp_spmv_plan_info info{};
};

namespace pdlp {
namespace {

constexpr int kPlanRows = 512;        // rows per tile
constexpr int kPlanNnz = 2048;        // entries per tile
constexpr int kPlanBand = 3072;       // x window of a tile
constexpr int kHalo = 32;             // further x entries of a tile (one per halo-warp lane)
constexpr int kHaloAt = kPlanBand + 4;  // staged-x index of the first halo entry
constexpr int kLaneRow = 64;          // rows up to this length: one lane, storage order
constexpr int kPlanCW = 16;           // consumer warps
constexpr int kGroupW = 8;            // consumer warps per group: groups sum alternate tiles
constexpr int kGroups = kPlanCW / kGroupW;
constexpr int kCopyWarp = kPlanCW, kHaloWarp = kPlanCW + 1;
constexpr int kPlanThreads = (kPlanCW + 2) * 32;
constexpr int kPlanStages = 4;
// Consumers wait on a stage by phase parity, so each stage must always be
// consumed by the same group: tile k + kPlanStages is then the next tile of
// the group that consumed tile k, which waits for it only after it has
// released tile k.  With groups not dividing the stages, another group could
// reach the stage while tile k's phase is still open, match the parity of the
// phase before it, and read a stale stage.
static_assert(kPlanStages % kGroups == 0, "every stage consumed by one group");
constexpr int kChunk = 32;            // tile descriptors a warp fetches at once
constexpr long long kPlanWaitNs = 1000000000LL;
// cost model of the CTA balance (ns): a round trip to global memory, one to
// shared memory, the fixed cost of a tile, and one SM's share of HBM
// bandwidth in bytes per ns
constexpr double kGatherNs = 1500.0, kSharedNs = 150.0, kTileNs = 300.0, kSmBytesPerNs = 40.0;
constexpr unsigned kAllLanes = 0xffffffffu;

enum : int { TILE_NORMAL = 0, TILE_HUGE = 1 };

struct PlanTile {
  long long p0;    // first entry (absolute index into the entry arrays)
  long long cnt;   // entries
  int r0, nr;      // rows [r0, r0 + nr)
  int blo, bcnt;   // x window [blo, blo + bcnt) staged in shared memory; bcnt 0: none
  int kind;
  int nlong;       // rows of more than kLaneRow entries, listed from long_first
  int long_first;  // in the plan's long_rows array (row index within the tile)
  int nhalo;       // halo columns, listed from halo_first in halo_cols
  int halo_first;
  int staged;      // 1: every entry's x is staged (no gather from global memory)
  int nshort;      // rows of at most kLaneRow entries: perm[r0 .. r0 + nshort)
  int pad;
};
static_assert(sizeof(PlanTile) == 64, "PlanTile layout");

// Byte layout of one stage.  Each copied array has room for the copy's start
// being rounded down to a 16-byte chunk; every size is a multiple of 16, so
// every array starts on a 16-byte boundary.  The x region holds the window
// (staged-x indices 0 .. kPlanBand-1) and, from kHaloAt on, the halo; the
// halo lies past every byte the window's copy can write.
template <typename T>
struct StageLayout {
  static constexpr int kPer = 16 / (int)sizeof(T);
  static constexpr int desc_bytes = 64;                         // the tile's PlanTile
  static constexpr int perm_off = desc_bytes;
  static constexpr int perm_bytes = (kPlanRows + 8) * 2;
  static constexpr int rp_off = perm_off + perm_bytes;
  static constexpr int rp_bytes = (kPlanRows + 2) * 8;
  static constexpr int idx_off = rp_off + rp_bytes;
  static constexpr int idx_bytes = (kPlanNnz + 4) * 4;
  static constexpr int val_off = idx_off + idx_bytes;
  static constexpr int val_bytes = (kPlanNnz + kPer) * (int)sizeof(T);
  static constexpr int x_off = val_off + val_bytes;
  static constexpr int x_bytes = (kHaloAt + kHalo + kPer) * (int)sizeof(T);
  static constexpr int bytes = x_off + x_bytes;
};
static_assert(StageLayout<double>::bytes % 16 == 0 && StageLayout<float>::bytes % 16 == 0,
              "stage alignment");
static_assert(kHaloAt >= kPlanBand + 4 && kPlanBand % 4 == 0, "halo past the window's copy");
static_assert(kPlanStages * StageLayout<double>::bytes + 5 * 1024 <= 227 * 1024, "shared memory");

// Whole 16-byte chunks covering elements [first, first + count) of E-byte
// elements (64-bit entry offsets).
template <int E>
__device__ __forceinline__ unsigned lbulk_bytes(long long first, long long count) {
  constexpr long long per = 16 / E;
  if (count <= 0) return 0u;
  const long long a = first & ~(per - 1);
  return (unsigned)((first + count - a + per - 1) / per) * 16u;
}

template <int E>
__device__ __forceinline__ void lbulk_stage(void* dst, const void* base, long long first,
                                            unsigned bytes, unsigned long long* bar) {
  if (bytes == 0u) return;
  const char* src = reinterpret_cast<const char*>(base) + (first & ~(long long)(16 / E - 1)) * E;
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_init_count(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Programmatic dependent launch.  grid_dep_wait returns once the kernel
// before this one in the stream has completed and its writes are visible (at
// once when there is none); grid_dep_release lets the next kernel in the
// stream, if it was launched as a programmatic dependent, start its CTAs as
// this kernel's CTAs leave the SMs.
__device__ __forceinline__ void grid_dep_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

__device__ __forceinline__ void grid_dep_release() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Waits for the phase of `bar` with parity `parity`; false (and the status
// word set) once kPlanWaitNs of wall time have passed.
__device__ bool plan_wait(unsigned long long* bar, unsigned parity, int* status) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = global_ns();
  for (unsigned spins = 1;; ++spins) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((spins & 63u) == 0u && global_ns() - t0 > kPlanWaitNs) {
      atomicCAS(status, 0, PDLP_ERR_BARRIER_TIMEOUT);
      return false;
    }
  }
}

__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// Tile `j` of the 32 whose descriptors the lanes of a warp hold, one each.
__device__ __forceinline__ PlanTile shfl_tile(const PlanTile& mine, int j) {
  PlanTile t;
  const int* src = reinterpret_cast<const int*>(&mine);
  int* dst = reinterpret_cast<int*>(&t);
#pragma unroll
  for (int w = 0; w < (int)(sizeof(PlanTile) / 4); ++w) dst[w] = __shfl_sync(kAllLanes, src[w], j);
  return t;
}

// The rows of a normal tile, by the kGroupW warps of one group (gw is the
// warp's index in it).  STAGED: every entry's x is in the stage, so the
// gathers read shared memory only.
template <typename T, bool STAGED>
__device__ __forceinline__ void consume_tile(const PlanTile& t, const unsigned char* st,
                                             const T* __restrict__ x, T* __restrict__ y,
                                             const int* __restrict__ long_rows, long long base,
                                             int gw, int lane) {
  using L = StageLayout<T>;
  const long long* srp = reinterpret_cast<const long long*>(st + L::rp_off) + (t.r0 & 1);
  const int* sidx = reinterpret_cast<const int*>(st + L::idx_off) + (int)(t.p0 & 3);
  const T* sval =
      reinterpret_cast<const T*>(st + L::val_off) + (int)((base + t.p0) & (L::kPer - 1));
  const T* sx = reinterpret_cast<const T*>(st + L::x_off) + (t.blo & (L::kPer - 1));
  const uint16_t* sperm = reinterpret_cast<const uint16_t*>(st + L::perm_off) + (t.r0 & 7);
  // a rewritten index: staged x (window or halo), or -(column + 1)
  auto xval = [&](int jj) -> T {
    if (STAGED) return sx[jj];
    return jj >= 0 ? sx[jj] : __ldg(x + (-1 - jj));
  };
  // the short rows, one per lane, in the plan's order: the 32 rows of a warp
  // start at different banks, so the lanes' loads of indices and values do
  // not collide in shared memory
  for (int rb = gw * 32; rb < t.nshort; rb += kGroupW * 32) {
    if (rb + lane < t.nshort) {
      const int li = sperm[rb + lane];
      const int ps = (int)(srp[li] - t.p0), pe = (int)(srp[li + 1] - t.p0);
      T a = T(0);
      int q = ps;
      for (; q + 8 <= pe; q += 8) {         // eight entries' loads in flight
        T v[8], xv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          v[u] = sval[q + u];
          xv[u] = xval(sidx[q + u]);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) a = add_rn(a, mul_rn(v[u], xv[u]));
      }
      if (q < pe) {                          // the last 1..7 entries, loads in flight
        const int r = pe - q;
        T v[8], xv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          v[u] = u < r ? sval[q + u] : T(0);
          xv[u] = u < r ? xval(sidx[q + u]) : T(0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
          if (u < r) a = add_rn(a, mul_rn(v[u], xv[u]));
      }
      y[t.r0 + li] = a;
    }
  }
  // rows of more than kLaneRow entries, dealt round-robin to the group's
  // warps: lane l sums entries l, l+32, ... in order (eight loads in flight),
  // then a xor butterfly
  for (int kk = gw; kk < t.nlong; kk += kGroupW) {
    const int li = __ldg(long_rows + t.long_first + kk);
    const int qs = (int)(srp[li] - t.p0), qe = (int)(srp[li + 1] - t.p0);
    T a = T(0);
    for (int q = qs + lane; q < qe; q += 256) {
      T v[8], xv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const bool in = q + 32 * u < qe;
        v[u] = in ? sval[q + 32 * u] : T(0);
        xv[u] = in ? xval(sidx[q + 32 * u]) : T(0);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (q + 32 * u < qe) a = add_rn(a, mul_rn(v[u], xv[u]));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a = add_rn(a, __shfl_xor_sync(kAllLanes, a, off));
    if (lane == 0) y[t.r0 + li] = a;
  }
}

template <typename T>
__global__ void __launch_bounds__(kPlanThreads, 1) spmv_plan_kernel(

    const PlanTile* __restrict__ tiles, const int* __restrict__ cta_first,
    const int64_t* __restrict__ rp, const int* __restrict__ idx, const T* __restrict__ rx,
    const T* __restrict__ x, T* __restrict__ y, const int* __restrict__ long_rows,
    const int* __restrict__ halo_cols, const uint16_t* __restrict__ perm, long long base,
    int* status) {
  using L = StageLayout<T>;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ unsigned long long full[kPlanStages], empty[kPlanStages];
  __shared__ int hcols[kChunk][kHalo];
  __shared__ int abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t_begin = cta_first[blockIdx.x];
  const int count = cta_first[blockIdx.x + 1] - t_begin;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kPlanStages; ++s) {
      mbar_init_count(&full[s], 2);          // the copy warp and the halo warp
      mbar_init_count(&empty[s], kGroupW);   // the warps of the group that sums the tile
    }
    abort_flag = 0;
    mbar_init_fence();
  }
  __syncthreads();
  // Every CTA of this kernel is resident from here on, so the next product
  // may start its CTAs as these leave.  Until grid_dep_wait returns, a CTA
  // reads only the plan's own arrays (uploaded before plan creation
  // returned): the caller's values, x and y are touched after it.
  grid_dep_release();

  if (warp == kCopyWarp) {
    // lane 0 writes a tile's descriptor into its stage and issues its copies:
    // first those of the plan's arrays (row order, row pointers, indices),
    // then those of the caller's values and x window
    auto stage_plan = [&](const PlanTile& t, int s) {
      unsigned char* st = smem + s * L::bytes;
      *reinterpret_cast<PlanTile*>(st) = t;       // published by the arrive below
      // the consumers' reads of this stage (generic proxy) come before the
      // copy engine's writes into it (async proxy)
      fence_proxy_async();
      if (t.kind == TILE_HUGE) {                  // read from global memory by a consumer warp
        mbar_arrive(&full[s]);
        return;
      }
      const unsigned bperm = lbulk_bytes<2>(t.r0, t.nshort);
      const unsigned brp = lbulk_bytes<8>(t.r0, t.nr + 1);
      const unsigned bidx = lbulk_bytes<4>(t.p0, t.cnt);
      const unsigned bval = lbulk_bytes<(int)sizeof(T)>(base + t.p0, t.cnt);
      const unsigned bx = lbulk_bytes<(int)sizeof(T)>(t.blo, t.bcnt);
      // the phase completes when all five copies have landed
      mbar_arrive_tx(&full[s], bperm + brp + bidx + bval + bx);
      lbulk_stage<2>(st + L::perm_off, perm, t.r0, bperm, &full[s]);
      lbulk_stage<8>(st + L::rp_off, rp, t.r0, brp, &full[s]);
      lbulk_stage<4>(st + L::idx_off, idx, t.p0, bidx, &full[s]);
    };
    auto stage_caller = [&](const PlanTile& t, int s) {
      if (t.kind == TILE_HUGE) return;
      unsigned char* st = smem + s * L::bytes;
      lbulk_stage<(int)sizeof(T)>(st + L::val_off, rx, base + t.p0,
                                  lbulk_bytes<(int)sizeof(T)>(base + t.p0, t.cnt), &full[s]);
      lbulk_stage<(int)sizeof(T)>(st + L::x_off, x, t.blo,
                                  lbulk_bytes<(int)sizeof(T)>(t.blo, t.bcnt), &full[s]);
    };
    // the first tile of each consumer group (free stages): the plan's part
    // while the kernel before this one may still run, the caller's part after
    // it ends.  (Priming all kPlanStages stages put the plan's copies of
    // later tiles ahead of the first tile's values in a single call, about
    // 1 us later to its end.)
    PlanTile mine{};
    if (lane < count) mine = tiles[t_begin + lane];
    const int primed = min(count, kGroups);
    for (int j = 0; j < primed; ++j) {
      const PlanTile t = shfl_tile(mine, j);
      if (lane == 0) stage_plan(t, j);
    }
    grid_dep_wait();
    // the previous kernel's ordinary stores to the values and x come before
    // this lane's bulk (async proxy) reads of them
    if (lane == 0) fence_proxy_async_global();
    for (int j = 0; j < primed; ++j) {
      const PlanTile t = shfl_tile(mine, j);
      if (lane == 0) stage_caller(t, j);
    }
    // the rest: the lanes fetch 32 tile descriptors at once; lane 0 waits for
    // each stage to be free, then stages the tile
    int k = primed;
    bool stop = false;
    for (int c0 = 0; c0 < count && !stop; c0 += kChunk) {
      if (c0 > 0) {
        mine = PlanTile{};
        if (c0 + lane < count) mine = tiles[t_begin + c0 + lane];
      }
      const int cn = min(kChunk, count - c0);
      for (int j = c0 == 0 ? primed : 0; j < cn; ++j, ++k) {
        const int s = k % kPlanStages;
        int go = 1;
        if (lane == 0) {
          if (k >= kPlanStages && !plan_wait(&empty[s], ((k / kPlanStages) - 1) & 1u, status)) go = 0;
          if (*(volatile int*)&abort_flag) go = 0;
        }
        go = __shfl_sync(kAllLanes, go, 0);
        if (!go) { stop = true; break; }
        const PlanTile t = shfl_tile(mine, j);
        if (lane == 0) {
          stage_plan(t, s);
          stage_caller(t, s);
        }
      }
    }
    // every copy still in flight lands before the CTA exits (the phases the
    // consumers already saw complete return at once)
    if (lane == 0)
      for (int j = max(0, k - kPlanStages); j < k; ++j)
        plan_wait(&full[j % kPlanStages], (j / kPlanStages) & 1u, status);
    return;
  }

  if (warp == kHaloWarp) {
    // per chunk of 32 tiles: the halo columns into shared memory (lane l
    // holds column l of each tile), then per tile one gather of x per lane,
    // the next tile's gathers issued before this tile's values are stored
    int k = 0;
    bool stop = false;
    for (int c0 = 0; c0 < count && !stop; c0 += kChunk) {
      PlanTile mine{};
      if (c0 + lane < count) mine = tiles[t_begin + c0 + lane];
      const int cn = min(kChunk, count - c0);
#pragma unroll
      for (int j = 0; j < kChunk; ++j) {       // 32 independent loads per lane
        const int nh = __shfl_sync(kAllLanes, mine.nhalo, j);
        const int hf = __shfl_sync(kAllLanes, mine.halo_first, j);
        hcols[j][lane] = (j < cn && lane < nh) ? __ldg(halo_cols + hf + lane) : -1;
      }
      __syncwarp();
      if (c0 == 0) grid_dep_wait();          // x is the caller's
      int col = hcols[0][lane];
      T cur = col >= 0 ? __ldg(x + col) : T(0);
      for (int j = 0; j < cn; ++j, ++k) {
        const int nc = j + 1 < cn ? hcols[j + 1][lane] : -1;
        const T nxt = nc >= 0 ? __ldg(x + nc) : T(0);
        const int s = k % kPlanStages;
        int go = 1;
        if (lane == 0) {
          if (k >= kPlanStages && !plan_wait(&empty[s], ((k / kPlanStages) - 1) & 1u, status)) go = 0;
          if (*(volatile int*)&abort_flag) go = 0;
        }
        go = __shfl_sync(kAllLanes, go, 0);
        if (!go) { stop = true; break; }
        const int blo = __shfl_sync(kAllLanes, mine.blo, j);
        T* sx = reinterpret_cast<T*>(smem + s * L::bytes + L::x_off) + (blo & (L::kPer - 1));
        if (hcols[j][lane] >= 0) sx[kHaloAt + lane] = cur;
        __syncwarp();
        if (lane == 0) mbar_arrive(&full[s]);
        cur = nxt;
      }
      __syncwarp();                          // hcols is rewritten for the next chunk
    }
    return;
  }

  // consumer warps: group g sums tiles g, g + kGroups, ...  (A stage fills
  // only after the copy and halo warps' waits; the consumers wait too, since
  // they read x and the values of huge tiles from global memory and write y.)
  grid_dep_wait();
  const int group = warp / kGroupW, gw = warp % kGroupW;
  for (int k = group; k < count; k += kGroups) {
    const int s = k % kPlanStages;
    if (!plan_wait(&full[s], (k / kPlanStages) & 1u, status)) {
      abort_flag = 1;
      break;
    }
    const unsigned char* st = smem + s * L::bytes;
    const PlanTile t = *reinterpret_cast<const PlanTile*>(st);
    if (t.kind == TILE_HUGE) {
      if (gw == 0) {
        T a = T(0);
        const long long end = t.p0 + t.cnt;
        for (long long q = t.p0 + lane; q < end; q += 32)
          a = add_rn(a, mul_rn(__ldg(rx + base + q), __ldg(x + (-1 - __ldg(idx + q)))));
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a = add_rn(a, __shfl_xor_sync(kAllLanes, a, off));
        if (lane == 0) y[t.r0] = a;
      }
    } else if (t.staged) {
      consume_tile<T, true>(t, st, x, y, long_rows, base, gw, lane);
    } else {
      consume_tile<T, false>(t, st, x, y, long_rows, base, gw, lane);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
  }
}

// ---- host: the plan --------------------------------------------------------

// The window of at most kPlanBand columns that holds the most of a tile's
// column indices, trimmed to the span of the indices it holds.  The window is
// kept when it is used often enough to pay for staging it: at least one
// covered entry per 8 staged columns.
void choose_window(const int* idx, long long cnt, int* blo, int* bcnt, std::vector<int>& scratch) {
  *blo = 0;
  *bcnt = 0;
  if (cnt <= 0) return;
  int lo = idx[0], hi = idx[0];
  for (long long q = 1; q < cnt; ++q) {
    lo = std::min(lo, idx[q]);
    hi = std::max(hi, idx[q]);
  }
  int wlo = lo, whi = hi;
  long long cov = cnt;
  if ((long long)hi - lo + 1 > kPlanBand) {
    scratch.assign(idx, idx + cnt);
    std::sort(scratch.begin(), scratch.end());
    long long best = 0, bestA = 0, bestB = 0;
    long long b = 0;
    for (long long a = 0; a < cnt; ++a) {
      if (b < a) b = a;
      while (b < cnt && (long long)scratch[b] - scratch[a] < kPlanBand) ++b;
      if (b - a > best) { best = b - a; bestA = a; bestB = b; }
    }
    wlo = scratch[bestA];
    whi = scratch[bestB - 1];
    cov = best;
  }
  const long long width = (long long)whi - wlo + 1;
  if (cov * 8 < width) return;
  *blo = wlo;
  *bcnt = (int)width;
}

// The tile's halo -- its most used columns outside the window, at most kHalo
// (ties to the lower column) -- and its rewritten indices.  Returns the
// entries whose x is staged (window or halo).
long long rewrite_tile(const int* ri, long long cnt, int blo, int bcnt, int* out,
                       std::vector<int>& halo, std::vector<std::pair<int, int>>& scratch) {
  halo.clear();
  scratch.clear();
  for (long long q = 0; q < cnt; ++q) {
    const int j = ri[q];
    if (!(j >= blo && j < blo + bcnt)) scratch.push_back({j, 0});
  }
  if (!scratch.empty()) {
    std::sort(scratch.begin(), scratch.end());
    std::vector<std::pair<int, int>> uses;           // (-count, column)
    for (size_t a = 0; a < scratch.size();) {
      size_t b = a;
      while (b < scratch.size() && scratch[b].first == scratch[a].first) ++b;
      uses.push_back({-(int)(b - a), scratch[a].first});
      a = b;
    }
    std::sort(uses.begin(), uses.end());
    for (size_t h = 0; h < uses.size() && (int)h < kHalo; ++h) halo.push_back(uses[h].second);
    std::sort(halo.begin(), halo.end());
  }
  long long staged = 0;
  for (long long q = 0; q < cnt; ++q) {
    const int j = ri[q];
    if (j >= blo && j < blo + bcnt) {
      out[q] = j - blo;
      ++staged;
      continue;
    }
    const auto it = std::lower_bound(halo.begin(), halo.end(), j);
    if (it != halo.end() && *it == j) {
      out[q] = kHaloAt + (int)(it - halo.begin());
      ++staged;
    } else {
      out[q] = -1 - j;
    }
  }
  return staged;
}

template <typename T>
int set_smem_attr() {
  PDLP_CUDA(cudaFuncSetAttribute(spmv_plan_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 kPlanStages * StageLayout<T>::bytes));
  return PDLP_OK;
}

void free_plan(pdlp_spmv_plan* p) {
  cudaFree(p->rp);
  cudaFree(p->idx);
  cudaFree(p->tiles);
  cudaFree(p->cta_first);
  cudaFree(p->long_rows);
  cudaFree(p->halo_cols);
  cudaFree(p->perm);
  cudaFree(p->status);
  delete p;
}

// Copies n elements of a host vector to a new device array (at least one
// element is allocated, so every pointer of a plan is valid).
template <typename E>
cudaError_t upload(E** dst, const E* src, size_t n, cudaStream_t st) {
  cudaError_t e = cudaMalloc((void**)dst, sizeof(E) * std::max<size_t>(1, n));
  if (e == cudaSuccess && n > 0) e = cudaMemcpyAsync(*dst, src, sizeof(E) * n, cudaMemcpyHostToDevice, st);
  return e;
}

int plan_create(int32_t m, int32_t n, const int64_t* rp, const int32_t* ri, cudaStream_t st,
                pdlp_spmv_plan** out) {
  if (!out) return fail(PDLP_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (m < 0 || n < 0) return fail(PDLP_ERR_ARG, "m and n must be >= 0");
  if (m > 0 && !rp) return fail(PDLP_ERR_ARG, "NULL pointer");
  const auto t0 = std::chrono::steady_clock::now();
  int dev = 0, sms = 0;
  PDLP_CUDA(cudaGetDevice(&dev));
  PDLP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  std::vector<int64_t> hrp((size_t)m + 1, 0);
  if (m > 0) {
    PDLP_CUDA(cudaMemcpyAsync(hrp.data(), rp, sizeof(int64_t) * ((size_t)m + 1),
                              cudaMemcpyDeviceToHost, st));
    PDLP_CUDA(cudaStreamSynchronize(st));
  }
  const int64_t base = hrp[0];
  if (base < 0) return fail(PDLP_ERR_ARG, "rp[0] must be >= 0");
  for (int i = 0; i < m; ++i)
    if (hrp[i + 1] < hrp[i]) return fail(PDLP_ERR_ARG, "row pointers must not decrease (row " +
                                                           std::to_string(i) + ")");
  const int64_t nnz = hrp[m] - base;
  if (nnz > 0 && !ri) return fail(PDLP_ERR_ARG, "NULL pointer");
  std::vector<int32_t> hri((size_t)nnz);
  if (nnz > 0) {
    PDLP_CUDA(cudaMemcpyAsync(hri.data(), ri + base, sizeof(int32_t) * (size_t)nnz,
                              cudaMemcpyDeviceToHost, st));
    PDLP_CUDA(cudaStreamSynchronize(st));
    for (int64_t q = 0; q < nnz; ++q)
      if (hri[(size_t)q] < 0 || hri[(size_t)q] >= n)
        return fail(PDLP_ERR_ARG, "column index out of range at entry " + std::to_string(base + q));
  }
  for (auto& v : hrp) v -= base;                   // the plan's entries start at 0

  std::vector<PlanTile> tiles;
  std::vector<double> cost;                        // estimated ns of each tile on one SM
  std::vector<int> longs, halos, halo, scratch;
  std::vector<std::pair<int, int>> pairs;
  std::vector<int32_t> pidx((size_t)nnz);
  std::vector<uint16_t> hperm((size_t)m + 8, 0);
  std::vector<std::pair<int, int>> order;
  pdlp_spmv_plan_info info{};
  for (int i = 0; i < m;) {
    const long long len = hrp[i + 1] - hrp[i];
    if (len > kPlanNnz) {
      tiles.push_back(PlanTile{hrp[i], len, i, 1, 0, 0, TILE_HUGE, 0, 0, 0, (int)halos.size(), 0});
      for (long long q = hrp[i]; q < hrp[i + 1]; ++q) pidx[(size_t)q] = -1 - hri[(size_t)q];
      cost.push_back(kGatherNs * (double)((len + 255) / 256) + kTileNs);
      ++info.huge_rows;
      ++i;
      continue;
    }
    const int start = i;
    long long cnt = 0;
    while (i < m && i - start < kPlanRows) {
      const long long l = hrp[i + 1] - hrp[i];
      if (l > kPlanNnz || cnt + l > kPlanNnz) break;
      cnt += l;
      ++i;
    }
    PlanTile t{hrp[start], cnt, start, i - start, 0, 0, TILE_NORMAL, 0, (int)longs.size(), 0,
               (int)halos.size(), 0};
    long long max_short = 0, max_long = 0;
    for (int r = start; r < i; ++r) {
      const long long l = hrp[r + 1] - hrp[r];
      if (l > kLaneRow) {
        longs.push_back(r - start);
        max_long = std::max(max_long, l);
      } else {
        max_short = std::max(max_short, l);
      }
    }
    t.nlong = (int)longs.size() - t.long_first;
    // the short rows' order for the lanes: bucketed by the bank their first
    // index lands on in the stage ((p0 + row start) mod 32, p0 counted from
    // the 16-byte boundary the copy starts at), then taken one per bucket in
    // turn, so that each 32 consecutive rows start on different banks
    {
      order.clear();
      int rank[32] = {0};
      for (int r = start; r < i; ++r) {
        if (hrp[r + 1] - hrp[r] > kLaneRow) continue;
        const int bank = (int)(((hrp[start] & 3) + (hrp[r] - hrp[start])) & 31);
        order.push_back({rank[bank]++ * 32 + bank, r - start});
      }
      std::stable_sort(order.begin(), order.end(),
                       [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
                         return a.first < b.first;
                       });
      t.nshort = (int)order.size();
      for (int k = 0; k < t.nshort; ++k) hperm[(size_t)start + k] = (uint16_t)order[k].second;
    }
    const int* tri = hri.data() + hrp[start];
    choose_window(tri, cnt, &t.blo, &t.bcnt, scratch);
    const long long staged =
        rewrite_tile(tri, cnt, t.blo, t.bcnt, pidx.data() + hrp[start], halo, pairs);
    t.nhalo = (int)halo.size();
    t.staged = staged == cnt ? 1 : 0;
    halos.insert(halos.end(), halo.begin(), halo.end());
    if (t.bcnt > 0) ++info.banded_tiles;
    info.entries_in_band += staged;
    // the tile's time: its bytes at one SM's share of HBM bandwidth, or the
    // longest chain of dependent loads, whichever is longer -- a chain step
    // costs a global round trip when entries are gathered from global memory
    const double step = staged < cnt ? kGatherNs : kSharedNs;
    const double chain =
        step * (double)((max_short + 7) / 8) +
        step * (double)((t.nlong + kGroupW - 1) / kGroupW) * (double)((max_long + 255) / 256);
    const double bytes = 12.0 * (double)cnt + 8.0 * t.bcnt + 16.0 * t.nr;
    cost.push_back(std::max(bytes / kSmBytesPerNs, chain) + kTileNs);
    tiles.push_back(t);
  }
  info.tiles = (int32_t)tiles.size();
  info.entries = nnz;
  // with fewer than half the entries staged the gathers go to global memory
  // anyway, and the row-block kernel's many resident warps hide them better
  // than the persistent kernel's sixteen
  info.kernel = 2 * info.entries_in_band < nnz ? PDLP_SPMV_PLAN_STREAMED : PDLP_SPMV_PLAN_TILES;

  // contiguous tile ranges of about equal estimated time, one per CTA
  const int nctas = std::max(1, std::min(sms, std::max(1, (int)tiles.size())));
  double total = 0.0;
  for (double c : cost) total += c;
  std::vector<int> first((size_t)nctas + 1, (int)tiles.size());
  first[0] = 0;
  {
    double acc = 0.0;
    int c = 1;
    for (size_t k = 0; k < tiles.size() && c < nctas; ++k) {
      acc += cost[k];
      while (c < nctas && acc >= total * c / nctas) first[(size_t)c++] = (int)k + 1;
    }
  }
  info.ctas = nctas;

  auto* p = new pdlp_spmv_plan;
  p->device = dev;
  p->m = m;
  p->n = n;
  p->ntiles = (int)tiles.size();
  p->nctas = nctas;
  p->base = base;
  const std::vector<int32_t>& kept = info.kernel == PDLP_SPMV_PLAN_TILES ? pidx : hri;
  cudaError_t e = upload(&p->rp, hrp.data(), hrp.size(), st);
  if (e == cudaSuccess) e = upload(&p->idx, kept.data(), kept.size(), st);
  if (e == cudaSuccess) e = upload((PlanTile**)&p->tiles, tiles.data(), tiles.size(), st);
  if (e == cudaSuccess) e = upload(&p->cta_first, first.data(), first.size(), st);
  if (e == cudaSuccess) e = upload(&p->long_rows, longs.data(), longs.size(), st);
  if (e == cudaSuccess) e = upload(&p->halo_cols, halos.data(), halos.size(), st);
  if (e == cudaSuccess) e = upload(&p->perm, hperm.data(), hperm.size(), st);
  if (e == cudaSuccess) e = cudaMalloc((void**)&p->status, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(p->status, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // the host vectors go out of scope
  if (e != cudaSuccess) {
    free_plan(p);
    return cuda_fail(e, "planned SpMV set-up");
  }
  int rc = set_smem_attr<double>();
  if (rc == PDLP_OK) rc = set_smem_attr<float>();
  if (rc != PDLP_OK) {
    free_plan(p);
    return rc;
  }
  info.seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  p->info = info;
  *out = p;
  return PDLP_OK;
}

int spmv_streamed(pdlp_spmv_plan* p, const double* rx, const double* x, double* y,
                  cudaStream_t st) {
  return pdlp_spmv_ex_f64(PDLP_SPMV_STREAMED, p->m, p->rp, p->idx, rx, x, y, st);
}

int spmv_streamed(pdlp_spmv_plan* p, const float* rx, const float* x, float* y, cudaStream_t st) {
  return pdlp_spmv_ex_f32(PDLP_SPMV_STREAMED, p->m, p->rp, p->idx, rx, x, y, st);
}

template <typename T>
int plan_run(pdlp_spmv_plan* p, const T* rx, const T* x, T* y, cudaStream_t st) {
  if (!p) return fail(PDLP_ERR_ARG, "plan is NULL");
  if (p->m == 0) return PDLP_OK;
  if (!y || (p->info.entries > 0 && (!rx || !x))) return fail(PDLP_ERR_ARG, "NULL pointer");
  int dev = 0;
  PDLP_CUDA(cudaGetDevice(&dev));
  if (dev != p->device) return fail(PDLP_ERR_ARG, "the plan was made on another device");
  // the plan's entry q is the caller's entry base + q
  if (p->info.kernel == PDLP_SPMV_PLAN_STREAMED) return spmv_streamed(p, rx + p->base, x, y, st);
  if ((reinterpret_cast<uintptr_t>(rx) | reinterpret_cast<uintptr_t>(x)) & 15u)
    return fail(PDLP_ERR_ARG, "rx and x must be 16-byte aligned (bulk copies)");
  // launched as a programmatic dependent of the kernel before it in the
  // stream: its CTAs stage the plan's arrays while that kernel drains
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(p->nctas);
  cfg.blockDim = dim3(kPlanThreads);
  cfg.dynamicSmemBytes = kPlanStages * StageLayout<T>::bytes;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PDLP_CUDA(cudaLaunchKernelEx(&cfg, spmv_plan_kernel<T>, static_cast<const PlanTile*>(p->tiles),
                               static_cast<const int*>(p->cta_first),
                               static_cast<const int64_t*>(p->rp),
                               static_cast<const int*>(p->idx), rx, x, y,
                               static_cast<const int*>(p->long_rows),
                               static_cast<const int*>(p->halo_cols),
                               static_cast<const uint16_t*>(p->perm), (long long)p->base,
                               p->status));
  count_launches(1);
  return PDLP_OK;
}

}  // namespace
}  // namespace pdlp

extern "C" {

int pdlp_spmv_plan_create(int32_t m, int32_t n_cols, const int64_t* rp, const int32_t* ri,
                          void* stream, pdlp_spmv_plan** out) {
  return pdlp::plan_create(m, n_cols, rp, ri, static_cast<cudaStream_t>(stream), out);
}

int pdlp_spmv_plan_run_f64(pdlp_spmv_plan* plan, const double* rx, const double* x, double* y,
                           void* stream) {
  return pdlp::plan_run<double>(plan, rx, x, y, static_cast<cudaStream_t>(stream));
}

int pdlp_spmv_plan_run_f32(pdlp_spmv_plan* plan, const float* rx, const float* x, float* y,
                           void* stream) {
  return pdlp::plan_run<float>(plan, rx, x, y, static_cast<cudaStream_t>(stream));
}

int pdlp_spmv_plan_get_info(const pdlp_spmv_plan* plan, pdlp_spmv_plan_info* out) {
  if (!plan || !out) return pdlp::fail(PDLP_ERR_ARG, "NULL pointer");
  *out = plan->info;
  return PDLP_OK;
}

int pdlp_spmv_plan_status(pdlp_spmv_plan* plan, void* stream) {
  if (!plan) return pdlp::fail(PDLP_ERR_ARG, "plan is NULL");
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  int word = 0;
  PDLP_CUDA(cudaStreamSynchronize(st));
  PDLP_CUDA(cudaMemcpy(&word, plan->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (word == 0) return PDLP_OK;
  PDLP_CUDA(cudaMemset(plan->status, 0, sizeof(int)));
  return pdlp::fail(word, "a planned SpMV stopped: a wait on its copies ran out of time");
}

void pdlp_spmv_plan_destroy(pdlp_spmv_plan* plan) {
  if (!plan) return;
  int cur = 0;
  const bool switch_dev = cudaGetDevice(&cur) == cudaSuccess && cur != plan->device;
  if (switch_dev) cudaSetDevice(plan->device);
  pdlp::free_plan(plan);
  if (switch_dev) cudaSetDevice(cur);
}

}  // extern "C"
