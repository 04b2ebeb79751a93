// PDLP engine: kernels (persistent cooperative and per-pass) and the batch
// runtime behind the C ABI (admission, tile planning, launch, polling).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <thread>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "engine_passes.cuh"

namespace pdlp {

// ---- grid barrier (bounded) ----------------------------------------------------
//
// Barrier of one block team on a monotonic arrival counter: the k-th barrier
// of a launch is passed once the counter reaches k * (blocks of the team); the
// host zeroes the counters before each launch.  Arrival is an acquire-release
// add, the wait an acquire load, so one atomic and one poll separate the last
// arrival from the release of every block.  The wait is bounded in wall time:
// on timeout the block records PDLP_ERR_BARRIER_TIMEOUT and every block
// leaves the kernel.  A team of one block (`alone`) needs no counter.
//
// The next pass stages tiles and vectors with bulk asynchronous copies, which
// read global memory through the async proxy, while the data was written with
// ordinary stores (generic proxy), by this block or by others.  Neither the
// barrier's acquire nor a __threadfence orders generic writes before async-
// proxy reads, so the caller follows every barrier with a global proxy fence
// in each thread that issues copies (fence_proxy_async_global).
__device__ bool grid_barrier(Control* ctl, unsigned* counter, unsigned target,
                             long long timeout_ns, int* flag, bool alone, bool withhold) {
  __syncthreads();
  if (alone) {
    // A team of one block: no other block waits for it.  The __syncthreads
    // ordered every thread's writes before thread 0's fence, which makes them
    // visible at GPU scope (to the finishers of later passes, which read with
    // ld.global.cg) as the release of a multi-block barrier does.
    if (threadIdx.x == 0) {
      __threadfence();
      *flag = *(volatile int*)&ctl->error == 0;
    }
    __syncthreads();
    return *flag != 0;
  }
  // test hook: this block leaves without arriving; the rest of the team waits
  // until the bounded wait below runs out
  if (withhold) return false;
  if (threadIdx.x == 0) {
    volatile int* err = &ctl->error;
    int ok = 1;
    if (atom_add_acq_rel(counter, 1u) + 1u < target) {
      const long long t0 = global_ns();
      unsigned spins = 0;
      while (ld_acquire(counter) < target) {
        if ((++spins & 255u) == 0u) {
          if (*err != 0) { ok = 0; break; }
          if (global_ns() - t0 > timeout_ns) {
            atomicCAS((int*)&ctl->error, 0, PDLP_ERR_BARRIER_TIMEOUT);
            ok = 0;
            break;
          }
        }
      }
    }
    *flag = ok && (*err == 0);
  }
  __syncthreads();
  return *flag != 0;
}

// One launch runs up to max_steps engine steps; every warp owns a fixed range
// of row tiles and of column tiles for the whole launch.  The blocks form
// teams that do not wait for one another: each team's tiles are the tiles of
// its own instances, and its barriers count only its blocks.  A team stops
// when its instances are done, after max_steps, or when another team has
// stopped (the host then re-plans the teams for what is left).  The team's
// first block decides each next step between the step's two barriers, so
// that every block of the team sees the same decision.
extern __shared__ __align__(16) unsigned char g_smem[];
constexpr size_t kSmemBytes = sizeof(WarpSmem) * kWarps + 16;

__global__ void __launch_bounds__(kBlock, 4) engine_persistent(EngineArgs A) {
  WarpSmem* ws = reinterpret_cast<WarpSmem*>(g_smem);
  int& flag = *reinterpret_cast<int*>(g_smem + sizeof(WarpSmem) * kWarps);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& W = ws[warp];
  if (lane == 0) {
    W.inst_id = -1;
    mbar_init(&W.bar[0]);
    mbar_init(&W.bar[1]);
    mbar_init_fence();
  }
  __syncwarp();
  BulkPhase ph;
  const int gw = blockIdx.x * kWarps + warp;
  const int r0 = A.rwarp[gw], r1 = A.rwarp[gw + 1];
  const int c0 = A.cwarp[gw], c1 = A.cwarp[gw + 1];
  // the warp's first tile of each side stays in registers for the launch
  const Tile rfirst = r0 < r1 ? A.rtiles[r0] : Tile{};
  const Tile cfirst = c0 < c1 ? A.ctiles[c0] : Tile{};
  const int team = A.block_team[blockIdx.x];
  const bool leader = (int)blockIdx.x == A.team_first[team];
  unsigned* const bar = &A.ctl->team_bar[team];
  const unsigned nb = (unsigned)A.team_blocks[team];
  const bool withhold = (int)blockIdx.x == A.withhold_block;
  const long long budget = *(volatile int*)&A.ctl->team_budget[team];
  unsigned target = 0;
#ifdef PDLP_TRACE
  // phase timestamps of the first and the last block for the first steps
  long long* tr = nullptr;
  if (A.trace && threadIdx.x == 0 && (blockIdx.x == 0 || blockIdx.x == gridDim.x - 1))
    tr = A.trace + (blockIdx.x == 0 ? 0 : 64 * 5);
#define PDLP_STAMP(step, k) if (tr && (step) < 64) tr[(step) * 5 + (k)] = global_ns()
#else
#define PDLP_STAMP(step, k)
#endif
  long long step = 0;
  for (; step < budget; ++step) {
    if (threadIdx.x == 0)
      flag = *(volatile int*)&A.ctl->team_active[team] > 0 &&
             *(volatile int*)&A.ctl->team_go[team] != 0;
    __syncthreads();
    if (!flag) break;
    __syncthreads();
    PDLP_STAMP(step, 0);
    {
      Tile next = rfirst;
      PassCache pc;
      for (int t = r0; t < r1; ++t) {
        const Tile cur = next;
        if (t + 1 < r1) next = A.rtiles[t + 1];      // prefetch the next descriptor
        ph.flush = t + 1 >= r1 || next.group != cur.group;
        process_rtile(A, cur, t, W, lane, pc, ph);
      }
    }
    PDLP_STAMP(step, 1);
    target += nb;
    if (!grid_barrier(A.ctl, bar, target, A.barrier_timeout_ns, &flag, nb == 1u, withhold)) return;
    if (lane == 0) fence_proxy_async_global();
    PDLP_STAMP(step, 2);
    // the leader's decision for the next step, published by its arrival at
    // the next barrier
    if (leader && threadIdx.x == 0)
      A.ctl->team_go[team] = *(volatile int*)&A.ctl->stop == 0;
    {
      Tile next = cfirst;
      PassCache pc;
      for (int t = c0; t < c1; ++t) {
        const Tile cur = next;
        if (t + 1 < c1) next = A.ctiles[t + 1];
        ph.flush = t + 1 >= c1 || next.group != cur.group;
        process_ctile(A, cur, t, W, lane, pc, ph);
      }
    }
    PDLP_STAMP(step, 3);
    target += nb;
    if (!grid_barrier(A.ctl, bar, target, A.barrier_timeout_ns, &flag, nb == 1u, withhold)) return;
    if (lane == 0) fence_proxy_async_global();
    PDLP_STAMP(step, 4);
  }
  // This team is done for the launch; its leader reports the steps it ran.
  // After the launch's step cap the launch ends (the other teams leave at
  // their next step) and the host re-plans.  A team that spent the rest of
  // the call's budget of steps just leaves.  A team whose instance is done
  // ends the launch once an eighth of the blocks are idle, so that the host
  // can give them to what is left without re-planning at every finish.
  if (leader && threadIdx.x == 0) {
    A.ctl->team_steps[team] = (int)step;
    if (step == A.max_steps) {
      atomicExch(&A.ctl->stop, 1);
    } else if (step < budget && *(volatile int*)&A.ctl->team_active[team] <= 0) {
      const unsigned idle = atomicAdd(&A.ctl->idle, nb) + nb;
      if (idle * 8u >= gridDim.x) atomicExch(&A.ctl->stop, 1);
    }
  }
#undef PDLP_STAMP
}

// One pass over all tiles of one side; kernel boundaries are the barriers.
__global__ void __launch_bounds__(kBlock, 3) engine_pass(EngineArgs A, int side) {
  WarpSmem* ws = reinterpret_cast<WarpSmem*>(g_smem);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  WarpSmem& W = ws[warp];
  if (lane == 0) {
    W.inst_id = -1;
    mbar_init(&W.bar[0]);
    mbar_init(&W.bar[1]);
    mbar_init_fence();
  }
  __syncwarp();
  const int gw = blockIdx.x * kWarps + warp;
  const int nw = gridDim.x * kWarps;
  PassCache pc;
  BulkPhase ph;
  if (side == 0) {
    for (int t = gw; t < A.n_rtiles; t += nw) process_rtile(A, A.rtiles[t], t, W, lane, pc, ph);
  } else {
    for (int t = gw; t < A.n_ctiles; t += nw) process_ctile(A, A.ctiles[t], t, W, lane, pc, ph);
  }
}

// ---- infeasibility certificates (tested between launches) --------------------
//
// The candidates are the change of the scaled iterates since the previous
// test, e = x - x_prev and d = y - y_prev, with both signs s = +1, -1.
//
// Dual ray w = s d, with w_i set to 0 where its sign would need an infinite
// row bound.  For every feasible x, sum_i w_i (Ax)_i >= sum_i q(w_i), where
// q(w) = w rl if w > 0 and w ru if w < 0.  Also (A^T w)^T x <= sum_j u(g_j),
// where g = A^T w and u(g) = g hi if g > 0 and g lo if g < 0.  So
// sum q - sum u > 0 proves the LP infeasible, provided the u terms that would
// need an infinite bound vanish.  Their largest |g_j| is the violation.
//
// Primal ray v = s e, with v_j set to 0 where it would leave a finite column
// bound.  If c^T v < 0 and A v stays in the recession cone of the row bounds
// (h_i <= 0 where ru is finite, h_i >= 0 where rl is finite; the largest
// breach is the violation), the dual is infeasible.
//
// Each launch writes 8 partials per block; the host sums them in block order.
constexpr int kRayBlocks = 592;

__device__ __forceinline__ double ray_w(double d, double rl, double ru) {
  if (d > 0.0 && rl <= -kInf) return 0.0;
  if (d < 0.0 && ru >= kInf) return 0.0;
  return d;
}

__device__ __forceinline__ double ray_v(double e, double lo, double hi) {
  if (e > 0.0 && hi < kInf) return 0.0;
  if (e < 0.0 && lo > -kInf) return 0.0;
  return e;
}

// Fixed-order block reduction of 8 values (sums in 0, 1, 4, 5; maxima else).
__device__ void ray_block_reduce(double (&v)[8], double* out) {
  __shared__ double sh[8][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const bool is_sum = k == 0 || k == 1 || k == 4 || k == 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_xor_sync(0xffffffffu, v[k], off);
      v[k] = is_sum ? v[k] + o : fmax(v[k], o);
    }
    if (lane == 0) sh[w][k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    const int k = threadIdx.x;
    const bool is_sum = k == 0 || k == 1 || k == 4 || k == 5;
    double a = sh[0][k];
    for (int i = 1; i < 8; ++i) a = is_sum ? a + sh[i][k] : fmax(a, sh[i][k]);
    out[(size_t)blockIdx.x * 8 + k] = a;
  }
}

// Columns of A (CSR of A^T): for s = +/-1, sum -u(g_s) (0, 1), violation of
// g_s (2, 3), sum c_j v_s,j (4, 5) and max |v_s| (6, 7).
__global__ void __launch_bounds__(256) ray_cols_kernel(Inst I, const double* xprev,
                                                       const double* yprev, double* part) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < I.n; j += gridDim.x * blockDim.x) {
    double gp = 0.0, gm = 0.0;
    for (int p = I.cp[j]; p < I.cp[j + 1]; ++p) {
      const int i = I.ci[p];
      const double d = I.y[i] - yprev[i];
      const double a = I.cx[p];
      gp += a * ray_w(d, I.rl[i], I.ru[i]);
      gm += a * ray_w(-d, I.rl[i], I.ru[i]);
    }
    const double lo = I.lo[j], hi = I.hi[j];
    const double g2[2] = {gp, gm};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double g = g2[s];
      if (g > 0.0) { if (hi < kInf) v[s] -= g * hi; else v[2 + s] = fmax(v[2 + s], g); }
      else if (g < 0.0) { if (lo > -kInf) v[s] -= g * lo; else v[2 + s] = fmax(v[2 + s], -g); }
    }
    const double e = I.x[j] - xprev[j];
    const double vp = ray_v(e, lo, hi), vm = ray_v(-e, lo, hi);
    v[4] += I.c[j] * vp;
    v[5] += I.c[j] * vm;
    v[6] = fmax(v[6], fabs(vp));
    v[7] = fmax(v[7], fabs(vm));
  }
  ray_block_reduce(v, part);
}

// Rows of A (CSR of A): for s = +/-1, sum q(w_s) (0, 1), violation of
// h_s = A v_s (2, 3), unused (4, 5), max |w_s| (6, 7).
__global__ void __launch_bounds__(256) ray_rows_kernel(Inst I, const double* xprev,
                                                       const double* yprev, double* part) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < I.m; i += gridDim.x * blockDim.x) {
    double hp = 0.0, hm = 0.0;
    for (int p = I.rp[i]; p < I.rp[i + 1]; ++p) {
      const int j = I.ri[p];
      const double e = I.x[j] - xprev[j];
      const double a = I.rx[p];
      hp += a * ray_v(e, I.lo[j], I.hi[j]);
      hm += a * ray_v(-e, I.lo[j], I.hi[j]);
    }
    const double rl = I.rl[i], ru = I.ru[i];
    const double h2[2] = {hp, hm};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const double h = h2[s];
      if (h > 0.0 && ru < kInf) v[2 + s] = fmax(v[2 + s], h);
      if (h < 0.0 && rl > -kInf) v[2 + s] = fmax(v[2 + s], -h);
    }
    const double d = I.y[i] - yprev[i];
    const double wp = ray_w(d, rl, ru), wm = ray_w(-d, rl, ru);
    v[0] += wp > 0.0 ? wp * rl : (wp < 0.0 ? wp * ru : 0.0);
    v[1] += wm > 0.0 ? wm * rl : (wm < 0.0 ? wm * ru : 0.0);
    v[6] = fmax(v[6], fabs(wp));
    v[7] = fmax(v[7], fabs(wm));
  }
  ray_block_reduce(v, part);
}

// ---- admission kernels ----------------------------------------------------------

// All admission checks and the pointer conversions in one launch: task
// blockIdx.y walks one array with a grid-stride loop.
struct AdmitTasks {
  const long long* rp64; int* rp32; int m;
  const long long* cp64; int* cp32; int n;
  const int* ri; const int* ci; long long nnz;
  const double* rx0; const double* cx0;
  const double* c0; const double* lo0; const double* hi0;
  const double* rl0; const double* ru0;
  int* err;
};

// The checks of one admission: blockIdx.y picks the array (0, 1 pointers, 2, 3
// indices, 4..10 values, costs and bounds), x-blocks stride over it.
__device__ void admission_check_one(const AdmitTasks& T) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  switch (blockIdx.y) {
    case 0:
    case 1: {
      const long long* src = blockIdx.y == 0 ? T.rp64 : T.cp64;
      int* dst = blockIdx.y == 0 ? T.rp32 : T.cp32;
      const int len = blockIdx.y == 0 ? T.m : T.n;
      for (long long i = first; i <= len; i += stride) {
        const long long v = src[i];
        if (v < 0 || v > T.nnz || (i == 0 && v != 0) || (i == len && v != T.nnz) ||
            (i < len && src[i + 1] < v))
          atomicOr(T.err, 1);
        dst[i] = (int)v;
      }
      break;
    }
    case 2:
    case 3: {
      const int* idx = blockIdx.y == 2 ? T.ri : T.ci;
      const int bound = blockIdx.y == 2 ? T.n : T.m;
      for (long long p = first; p < T.nnz; p += stride) {
        const int v = idx[p];
        if (v < 0 || v >= bound) atomicOr(T.err, 1);
      }
      break;
    }
    default: {
      const int k = blockIdx.y - 4;
      const double* a = k == 0 ? T.rx0 : k == 1 ? T.cx0 : k == 2 ? T.c0 : k == 3 ? T.lo0
                      : k == 4 ? T.hi0 : k == 5 ? T.rl0 : T.ru0;
      const long long len = k <= 1 ? T.nnz : (k <= 4 ? T.n : T.m);
      const bool allow_inf = k >= 3;          // bounds may be +-inf; values and costs not
      for (long long i = first; i < len; i += stride) {
        const double v = a[i];
        if (isnan(v) || (!allow_inf && isinf(v))) atomicOr(T.err, 2);
      }
      break;
    }
  }
}

// Every admission of one admit call in one launch: blockIdx.z picks it.
__global__ void admission_check(const AdmitTasks* __restrict__ tasks) {
  admission_check_one(tasks[blockIdx.z]);
}

// A piece of an admission's input copies: bytes from src to dst, or, with
// src null, zeros.  The pieces of one admit call are copied by one launch
// (device-resident inputs) instead of a copy call per array.
struct CopyPiece {
  char* dst;
  const char* src;
  long long bytes;
};

__global__ void __launch_bounds__(256) gather_copy(const CopyPiece* __restrict__ pieces, int n) {
  for (int i = blockIdx.x; i < n; i += gridDim.x) {
    const CopyPiece pc = pieces[i];
    const unsigned long long a = (unsigned long long)pc.dst | (unsigned long long)pc.src |
                                 (unsigned long long)pc.bytes;
    if ((a & 15ull) == 0) {
      uint4* d = reinterpret_cast<uint4*>(pc.dst);
      const uint4* sv = reinterpret_cast<const uint4*>(pc.src);
      const long long w = pc.bytes / 16;
      for (long long k = threadIdx.x; k < w; k += blockDim.x) d[k] = pc.src ? sv[k] : make_uint4(0, 0, 0, 0);
    } else if ((a & 7ull) == 0) {
      unsigned long long* d = reinterpret_cast<unsigned long long*>(pc.dst);
      const unsigned long long* sv = reinterpret_cast<const unsigned long long*>(pc.src);
      const long long w = pc.bytes / 8;
      for (long long k = threadIdx.x; k < w; k += blockDim.x) d[k] = pc.src ? sv[k] : 0ull;
    } else {
      for (long long k = threadIdx.x; k < pc.bytes; k += blockDim.x)
        pc.dst[k] = pc.src ? pc.src[k] : (char)0;
    }
  }
}

}  // namespace pdlp

// ============================================================================
// host runtime
// ============================================================================

namespace {

using namespace pdlp;

thread_local std::string g_err;

constexpr size_t kAlign = 256;

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

int default_tile_rows() { return kWTileRows; }
int default_tile_nnz() { return kWTileNnz; }
int heavy_threshold() { return kWTileNnz; }  // longer rows: a warp-wide tile alone

// Lanes per row for the row sums of an LP side.  The products are already
// in shared memory, so a lane summing its row alone (in storage order) beats
// splitting the row across lanes, whose shuffle tree is a serial chain; only
// long rows get 2 or 4 lanes.
int lanes_for(long long nnz, long long rows) {
  if (rows <= 0) return 1;
  const double avg = (double)nnz / (double)rows;
  return avg <= 48.0 ? 1 : (avg <= 160.0 ? 2 : 4);
}

// Split the rows of one side into tiles of at most `rows_cap` rows and about
// `nnz_cap` entries; a row longer than the heavy threshold is a tile alone.
void plan_tiles(const int64_t* ptr, int nrows, int inst, int rows_cap, int nnz_cap,
                std::vector<Tile>& out, std::vector<double>& weight) {
  const size_t first = out.size();
  int b = 0;
  long long acc = 0;
  const int heavy = heavy_threshold();
  for (int r = 0; r < nrows; ++r) {
    long long len = ptr[r + 1] - ptr[r];
    if (len > heavy) {
      if (r > b) out.push_back({inst, b, r, 0, 0, (int)ptr[b], (int)(ptr[r] - ptr[b]), 0});
      out.push_back({inst, r, r + 1, 1, 0, (int)ptr[r], (int)len, 0});
      b = r + 1;
      acc = 0;
      continue;
    }
    if (r > b && (r - b >= rows_cap || acc + len > nnz_cap)) {
      out.push_back({inst, b, r, 0, 0, (int)ptr[b], (int)(ptr[r] - ptr[b]), 0});
      b = r;
      acc = 0;
    }
    acc += len;
  }
  if (nrows > b) out.push_back({inst, b, nrows, 0, 0, (int)ptr[b], (int)(ptr[nrows] - ptr[b]), 0});
  if (nrows == 0) out.push_back({inst, 0, 0, 0, 0, 0, 0, 0});   // the pass still finishes
  // work estimate per tile: entries (value + index + gather) and rows (vectors)
  for (size_t i = first; i < out.size(); ++i) {
    const Tile& t = out[i];
    weight.push_back((double)(ptr[t.end] - ptr[t.begin]) * 3.0 + (t.end - t.begin) * 10.0 + 200.0);
  }
}

struct Slot {
  bool used = false;
  bool reserved = false;      // taken by an admission in progress
  bool running = false;
  // infeasibility test (between launches): previous iterates, next check
  bool detect = false;
  double eps_inf = 1e-8;
  double* xprev = nullptr;
  double* yprev = nullptr;
  bool have_prev = false;
  long long next_check = 0;
  int hits = 0, hit_kind = 0;
  int m = 0, n = 0;
  long long nnz = 0;
  void* arena = nullptr;
  size_t bytes = 0;
  Inst inst{};
  std::vector<Tile> rt, ct;   // tiles with local ranges (inst field = slot)
  std::vector<double> rtw, ctw;   // work estimate per tile
  double bytes_per_iter = 0.0;
  double expected_iters = 0.0;    // the caller's scheduling hint (0: none)
};

}  // namespace

struct pdlp_batch {
  cudaStream_t stream = nullptr;
  pdlp_batch_config cfg{};
  std::vector<Slot> slots;
  int n_running = 0;
  size_t bytes_held = 0;
  // arenas of retired LPs, kept for later admissions: reusing one costs no
  // allocation and no device synchronisation (all use is stream-ordered)
  std::vector<std::pair<void*, size_t>> spare;
  size_t bytes_spare = 0;
  // device arrays
  Inst* d_inst = nullptr;
  State* d_state = nullptr;
  unsigned* d_counters = nullptr;
  Control* d_ctl = nullptr;
  Tile* d_rtiles = nullptr;
  Tile* d_ctiles = nullptr;
  int* d_rwarp = nullptr;
  int* d_cwarp = nullptr;
  int* d_teams = nullptr;          // block_team[grid], team_blocks[T], team_first[T]
  size_t cap_teams = 0;
  int n_teams = 1;
  std::vector<int> team_running;   // running instances per team, at the last rebuild
  int2* d_group_tiles = nullptr;
  double* d_partials = nullptr;
  double* d_gpartials = nullptr;
  unsigned* d_gcounters = nullptr;
  size_t cap_rtiles = 0, cap_ctiles = 0, cap_rwarp = 0, cap_cwarp = 0, cap_partials = 0;
  size_t cap_groups = 0, cap_gpartials = 0, cap_gcounters = 0;
  int n_rgroups = 0, n_groups = 0;
  int n_rtiles = 0, n_ctiles = 0, grid = 0;
  bool dirty = true;
  bool broken = false;
  // pinned host staging
  Control* h_ctl = nullptr;
  State* h_state = nullptr;
  int sms = 0, coop_blocks_per_sm = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // per-pass mode: `graph_chunk` steps (two launches each) captured once per
  // tile-list rebuild on a private stream and replayed on the batch's stream
  double* d_raypart = nullptr;     // infeasibility test partials (2 x kRayBlocks x 8)
  double* h_raypart = nullptr;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  int64_t graph_chunk = 0;
  bool graph_stale = true;
  double last_ms = 0.0, last_bytes = 0.0;
  long long last_iters = 0;
  std::vector<long long> iters_before;
  std::vector<long long> steps_left;   // per slot: steps it may still run in this call
  size_t bytes_pending = 0;            // arenas of admissions in progress
  int* h_errs = nullptr;               // pinned: admission verdicts, one per slot
  State* h_init = nullptr;             // pinned: initial states, one per slot
  int64_t* h_ptrs = nullptr;           // pinned: device pointer arrays read for admission
  size_t cap_hptrs = 0;
  CopyPiece* h_pieces = nullptr;       // pinned / device: an admit call's copy pieces
  CopyPiece* d_pieces = nullptr;
  size_t cap_pieces = 0;
  char* h_stage = nullptr;             // pinned: a re-plan's tile lists, packed for upload
  size_t cap_stage = 0;
  AdmitTasks* h_tasks = nullptr;       // pinned / device: an admit call's device checks
  AdmitTasks* d_tasks = nullptr;
  size_t cap_tasks = 0;
  bool force_set = false;              // tuning runs: every admission takes `force`
  pdlp_tuning force{};
  int force_blocks = 0;                // tuning runs: the one team's block count (0: free)
  int withhold_candidate = -1;         // last block of the first multi-block team
};

namespace pdlp {

void set_error(const std::string& msg) { g_err = msg; }
const std::string& get_error() { return g_err; }

static std::atomic<long long> g_launches{0};
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

}  // namespace pdlp

namespace {

int ensure_capacity(void** ptr, size_t* cap, size_t need, size_t elem) {
  if (need <= *cap && *ptr) return PDLP_OK;
  size_t n = std::max(need, (size_t)16);
  n = std::max(n, *cap * 2);
  if (*ptr) cudaFree(*ptr);
  *ptr = nullptr;
  cudaError_t e = cudaMalloc(ptr, n * elem);
  if (e != cudaSuccess) { *cap = 0; return cuda_fail(e, "cudaMalloc(engine tables)"); }
  *cap = n;
  return PDLP_OK;
}

// Arena layout of one slot.
struct Layout {
  size_t off = 0;
  size_t take(size_t bytes) { size_t o = off; off += align_up(bytes ? bytes : 1); return o; }
};

struct SlotLayout {
  size_t rp32, cp32, ri, ci, rx0, cx0, rx, cx, kind, v0, tmp64;
  size_t c0, rl0, ru0, lo0, hi0;
  size_t mvec[15];   // row-side vectors (the last: previous y of the infeasibility test)
  size_t nvec[16];
  size_t hist;
  size_t rx32, cx32, dx32, dy32;
  size_t total;
};

SlotLayout layout_for(int m, int n, long long nnz, bool kind, bool v0, int hist_cap, bool f32 = false) {
  Layout L;
  SlotLayout s{};
  s.rp32 = L.take(sizeof(int) * (size_t)(m + 1));
  s.cp32 = L.take(sizeof(int) * (size_t)(n + 1));
  s.ri = L.take(sizeof(int) * (size_t)nnz);
  s.ci = L.take(sizeof(int) * (size_t)nnz);
  s.rx0 = L.take(sizeof(double) * (size_t)nnz);
  s.cx0 = L.take(sizeof(double) * (size_t)nnz);
  s.rx = L.take(sizeof(double) * (size_t)nnz);
  s.cx = L.take(sizeof(double) * (size_t)nnz);
  s.kind = kind ? L.take((size_t)n) : 0;
  s.v0 = v0 ? L.take(sizeof(double) * (size_t)n) : 0;
  s.tmp64 = L.take(sizeof(long long) * (size_t)(m + 1 + n + 1));
  s.c0 = L.take(sizeof(double) * (size_t)n);
  s.lo0 = L.take(sizeof(double) * (size_t)n);
  s.hi0 = L.take(sizeof(double) * (size_t)n);
  s.rl0 = L.take(sizeof(double) * (size_t)m);
  s.ru0 = L.take(sizeof(double) * (size_t)m);
  for (int i = 0; i < 15; ++i) s.mvec[i] = L.take(sizeof(double) * (size_t)m);
  for (int i = 0; i < 16; ++i) s.nvec[i] = L.take(sizeof(double) * (size_t)n);
  s.hist = L.take(sizeof(double) * 5 * (size_t)std::max(hist_cap, 0));
  if (f32) {
    s.rx32 = L.take(sizeof(float) * (size_t)nnz);
    s.cx32 = L.take(sizeof(float) * (size_t)nnz);
    s.dx32 = L.take(sizeof(float) * (size_t)n);
    s.dy32 = L.take(sizeof(float) * (size_t)m);
  }
  L.take(256);     // 16-byte staging copies may read a few bytes past the last array
  s.total = L.off;
  return s;
}

// The device work of one admit call, gathered so that it takes two launches
// whatever the number of LPs: the copies of device-resident inputs and the
// zeroing of the slots' states (pieces of at most 256 KB, one gather_copy
// launch), and the validation of every LP's arrays (one admission_check).
struct AdmitBatch {
  std::vector<CopyPiece> pieces;
  std::vector<AdmitTasks> tasks;
  int gx = 1;
  void add(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPiece = (size_t)1 << 18;
    for (size_t o = 0; o < bytes; o += kPiece)
      pieces.push_back({(char*)dst + o, src ? (const char*)src + o : nullptr,
                        (long long)std::min(kPiece, bytes - o)});
  }
};

// Host inputs are copied at once (DMA from the caller's buffers); device
// inputs join the admit call's gathered copy, which a kernel reads: so an
// array declared as device memory must be device (or managed) memory, and
// anything else -- a host pointer passed with PDLP_MEM_DEVICE -- is refused
// here instead of being dereferenced on the device.
int copy_in(AdmitBatch& ab, void* dst, const void* src, size_t bytes, int memory, cudaStream_t st) {
  if (bytes == 0) return PDLP_OK;
  if (!src) return fail(PDLP_ERR_ARG, "a required input array is NULL");
  if (memory == PDLP_MEM_HOST) {
    PDLP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return PDLP_OK;
  }
  cudaPointerAttributes attr{};
  const cudaError_t e = cudaPointerGetAttributes(&attr, src);
  if (e != cudaSuccess) cudaGetLastError();        // an unknown pointer: not device memory
  if (e != cudaSuccess || (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged))
    return fail(PDLP_ERR_ARG, "an input array declared as device memory (PDLP_MEM_DEVICE) is not "
                              "device memory");
  ab.add(dst, src, bytes);
  return PDLP_OK;
}

// Contiguous chunks of the tile list with about equal work, one per block.
void block_ranges(const double* w, size_t T, int G, std::vector<int>& out) {
  double total = 0.0;
  for (size_t i = 0; i < T; ++i) total += w[i];
  out.assign(G + 1, (int)T);
  out[0] = 0;
  double acc = 0.0;
  int b = 1;
  for (size_t i = 0; i < T && b < G; ++i) {
    acc += w[i];
    while (b < G && acc >= total * b / G) { out[b] = (int)i + 1; ++b; }
  }
  for (; b < G; ++b) out[b] = (int)T;
  out[G] = (int)T;
}

}  // namespace

// Group the tiles of one instance-side into reduction groups of kGroupTiles
// consecutive tiles; appends (tile range) per group and stamps each tile.
// Iterations an instance is expected to need still, or a negative value when
// nothing is known.  From its own progress once its checks span at least
// kRateSpan iterations: the largest residual-to-tolerance ratio of the
// termination test fell from r0 to its best rb over that span, so at the same
// log-linear rate it needs log(rb) / rate more (an instance that has not
// improved is taken to need as many again as it has done).  Otherwise from
// the caller's estimate (pdlp_params.expected_iterations): an instance past
// it is taken to need half as many iterations again.  The state copy is the
// one read back after the last launch; it belongs to this instance once a
// launch has counted iterations for it.
static double expected_left(const pdlp_batch* b, int s) {
  constexpr long long kRateSpan = 256;
  const Slot& sl = b->slots[s];
  const double d = (double)b->iters_before[s];
  const State& hs = b->h_state[s];
  if (d > 0.0 && hs.kkt_k_first > 0 && hs.kkt_k - hs.kkt_k_first >= kRateSpan &&
      hs.kkt_best > 0.0) {
    if (hs.kkt_best <= 1.0) return 64.0;
    const double drop = std::log(hs.kkt_first / hs.kkt_best);
    if (!(drop > 0.0)) return std::max(d, 64.0);
    const double left = std::log(hs.kkt_best) * (double)(hs.kkt_k - hs.kkt_k_first) / drop;
    return std::min(std::max(left, 64.0), 1e7);
  }
  if (sl.expected_iters > 0.0) {
    const double e = sl.expected_iters;
    return std::max(d < e ? e - d : 0.5 * d, 0.1 * e);
  }
  return -1.0;
}

// The block teams of a persistent launch.  With many running instances one
// team of blocks steps them all.  With fewer (at most kTeamsFrom), each
// instance gets its own team, so that no instance waits at a barrier for
// another's tiles.  Teams get blocks in proportion to each instance's weight,
// but never more than one tile per warp can use: the blocks an instance
// cannot use go to the others (water-filling), and the blocks left by
// rounding go to the largest remainders.  The weight is the instance's work
// per iteration, times the square root of its expected remaining iterations
// when every running instance has an estimate (expected_left: from its own
// progress, else from pdlp_params.expected_iterations).  On the 256-LP batch
// the exponent of the remaining iterations set the median time to tolerance
// and left the throughput unchanged within noise: 0.5, 0.75 and 1 measured
// 487-491 solves/s with p50 0.225, 0.236 and 0.25 s; 1.5 and 2 lost 10-13
// solves/s (long runners given their blocks starve the rest for longer).
// On the 256-LP batch (engine time per batch, with the idle rule of the
// kernel), teams from 160, 200 and 256 running instances measured 585, 571
// and 541 ms.  Returns the blocks of each running instance's team, in `run`
// order, or nothing for one team.
static std::vector<int> plan_teams(const pdlp_batch* b, const std::vector<int>& run,
                                   int max_blocks) {
  constexpr int kTeamsFrom = 256;
  std::vector<int> tblocks;
  if (!b->cfg.persistent || run.size() < 2 ||
      (int)run.size() > std::min(kTeamsFrom, kMaxTeams) || (int)run.size() > max_blocks)
    return tblocks;
  const size_t T = run.size();
  bool hinted = true;
  std::vector<double> left(T);
  for (size_t k = 0; k < T; ++k) {
    left[k] = expected_left(b, run[k]);
    hinted = hinted && left[k] > 0.0;
  }
  std::vector<double> w(T);
  std::vector<int> want(T);
  for (size_t k = 0; k < T; ++k) {
    const Slot& sl = b->slots[run[k]];
    double per = 0.0;
    for (double v : sl.rtw) per += v;
    for (double v : sl.ctw) per += v;
    if (hinted) per *= std::sqrt(left[k]);
    w[k] = per;
    const int tiles = std::max(sl.inst.rt_end - sl.inst.rt_begin, sl.inst.ct_end - sl.inst.ct_begin);
    want[k] = std::max(1, (tiles + kWarps - 1) / kWarps);    // one tile per warp
  }
  tblocks.assign(T, 0);
  std::vector<char> full(T, 0);
  double wfree = 0.0;
  for (size_t k = 0; k < T; ++k) wfree += w[k];
  int free_blocks = max_blocks;
  size_t nfree = T;
  for (bool again = true; again && nfree > 0;) {
    again = false;
    const double wf = wfree;
    const int fb = free_blocks;
    const size_t nf = nfree;
    for (size_t k = 0; k < T; ++k) {
      if (full[k]) continue;
      const double share = wf > 0.0 ? fb * (w[k] / wf) : (double)fb / nf;
      if (share >= want[k]) {           // more than it can use: all it can use
        full[k] = 1;
        tblocks[k] = want[k];
        free_blocks -= want[k];
        wfree -= w[k];
        --nfree;
        again = true;
      }
    }
  }
  std::vector<std::pair<double, int>> frac;
  int used = 0;
  for (size_t k = 0; k < T; ++k) {
    if (!full[k]) {
      const double share = wfree > 0.0 ? free_blocks * (w[k] / wfree)
                                       : (double)free_blocks / (double)std::max<size_t>(nfree, 1);
      tblocks[k] = std::max(1, (int)share);
      frac.push_back({share - std::floor(share), (int)k});
    }
    used += tblocks[k];
  }
  std::sort(frac.begin(), frac.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b2) {
    return a.first != b2.first ? a.first > b2.first : a.second < b2.second;
  });
  for (const auto& f : frac) {
    if (used >= max_blocks) break;
    if (tblocks[f.second] < want[f.second]) { ++tblocks[f.second]; ++used; }
  }
  while (used > max_blocks) {                 // the one-block minimum left too many: trim the largest
    const size_t k = (size_t)(std::max_element(tblocks.begin(), tblocks.end()) - tblocks.begin());
    if (tblocks[k] <= 1) break;
    --tblocks[k];
    --used;
  }
  if (used > max_blocks) tblocks.clear();     // cannot give every instance a block
  return tblocks;
}

static int rebuild(pdlp_batch* b) {
  // where every running slot's tiles and reduction groups go in the launch's
  // lists: row-side groups first, then column-side groups (64 consecutive
  // tiles of a slot per group)
  std::vector<int> run;                       // running slots, in tile order
  for (size_t s = 0; s < b->slots.size(); ++s)
    if (b->slots[s].used && b->slots[s].running) run.push_back((int)s);
  auto ngroups = [](size_t tiles) { return (int)((tiles + kGroupTiles - 1) / kGroupTiles); };
  int nrt = 0, nct = 0, nrg = 0, ncg = 0;
  for (int s : run) {
    Slot& sl = b->slots[s];
    sl.inst.rt_begin = nrt;
    nrt += (int)sl.rt.size();
    sl.inst.rt_end = nrt;
    sl.inst.ct_begin = nct;
    nct += (int)sl.ct.size();
    sl.inst.ct_end = nct;
    sl.inst.rg_begin = nrg;
    nrg += ngroups(sl.rt.size());
    sl.inst.rg_end = nrg;
  }
  for (int s : run) {
    Slot& sl = b->slots[s];
    sl.inst.cg_begin = nrg + ncg;
    ncg += ngroups(sl.ct.size());
    sl.inst.cg_end = nrg + ncg;
  }
  b->n_rgroups = nrg;
  b->n_groups = nrg + ncg;
  b->n_rtiles = nrt;
  b->n_ctiles = nct;
  // persistent grid: enough warps for the larger tile list, at most what is
  // co-resident, in one team or in one team per instance (plan_teams)
  const int max_blocks = std::max(1, b->sms * b->coop_blocks_per_sm);
  const std::vector<int> tblocks = plan_teams(b, run, max_blocks);
  // per warp tile ranges, then the team arrays: block_team[G], team_blocks[T],
  // team_first[T]
  std::vector<int> rwr, cwr, teams;
  if (tblocks.empty()) {
    std::vector<double> rw, cw;                 // one team splits every running tile
    rw.reserve(nrt);
    cw.reserve(nct);
    for (int s : run) {
      const Slot& sl = b->slots[s];
      rw.insert(rw.end(), sl.rtw.begin(), sl.rtw.end());
      cw.insert(cw.end(), sl.ctw.begin(), sl.ctw.end());
    }
    const int want = (std::max(b->n_rtiles, b->n_ctiles) + kWarps - 1) / kWarps;
    int G = std::max(1, std::min(max_blocks, want));
    if (b->force_blocks > 0) G = std::min(G, b->force_blocks);
    b->grid = G;
    block_ranges(rw.data(), rw.size(), G * kWarps, rwr);
    block_ranges(cw.data(), cw.size(), G * kWarps, cwr);
    b->n_teams = 1;
    b->withhold_candidate = G >= 2 ? G - 1 : -1;
    teams.assign(G, 0);
    teams.push_back(G);
    teams.push_back(0);
    b->team_running.assign(1, (int)run.size());
    for (int s : run) b->slots[s].inst.team = 0;
  } else {
    const int T = (int)run.size();
    int G = 0;
    for (int k = 0; k < T; ++k) G += tblocks[k];
    b->grid = G;
    b->n_teams = T;
    b->withhold_candidate = -1;
    std::vector<int> first(T);
    std::vector<int> pr, pc;
    int fb = 0;
    for (int k = 0; k < T; ++k) {
      Slot& sl = b->slots[run[k]];
      sl.inst.team = k;
      first[k] = fb;
      fb += tblocks[k];
      if (b->withhold_candidate < 0 && tblocks[k] >= 2) b->withhold_candidate = fb - 1;
      for (int q = 0; q < tblocks[k]; ++q) teams.push_back(k);
      // the team's warps split its own tiles, as one team splits all of them
      const int r0 = sl.inst.rt_begin, c0 = sl.inst.ct_begin;
      block_ranges(sl.rtw.data(), sl.rtw.size(), tblocks[k] * kWarps, pr);
      block_ranges(sl.ctw.data(), sl.ctw.size(), tblocks[k] * kWarps, pc);
      for (int q = 0; q < tblocks[k] * kWarps; ++q) {
        rwr.push_back(r0 + pr[q]);
        cwr.push_back(c0 + pc[q]);
      }
    }
    rwr.push_back(b->n_rtiles);
    cwr.push_back(b->n_ctiles);
    for (int k = 0; k < T; ++k) teams.push_back(tblocks[k]);
    for (int k = 0; k < T; ++k) teams.push_back(first[k]);
    b->team_running.assign(T, 1);
  }
  const size_t ngr = (size_t)b->n_groups;
  int rc;
  if ((rc = ensure_capacity((void**)&b->d_rtiles, &b->cap_rtiles, nrt, sizeof(Tile)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_ctiles, &b->cap_ctiles, nct, sizeof(Tile)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_rwarp, &b->cap_rwarp, rwr.size(), sizeof(int)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_cwarp, &b->cap_cwarp, cwr.size(), sizeof(int)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_teams, &b->cap_teams, teams.size(), sizeof(int)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_partials, &b->cap_partials,
                            ((size_t)nrt + nct) * kNP, sizeof(double)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_group_tiles, &b->cap_groups, ngr, sizeof(int2)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_gpartials, &b->cap_gpartials, ngr * kNP,
                            sizeof(double)))) return rc;
  if ((rc = ensure_capacity((void**)&b->d_gcounters, &b->cap_gcounters, ngr,
                            sizeof(unsigned)))) return rc;
  // every list is written straight into one pinned staging area and uploaded
  // from there: the copies are asynchronous, and the staging area is next
  // written by the next re-plan, after the launch that follows this one has
  // been waited for
  cudaStream_t st = b->stream;
  auto up16 = [](size_t v) { return (v + 15) / 16 * 16; };
  const size_t b_rt = sizeof(Tile) * (size_t)nrt, b_ct = sizeof(Tile) * (size_t)nct;
  const size_t b_gr = sizeof(int2) * ngr, b_in = sizeof(Inst) * b->slots.size();
  const size_t total = up16(b_rt) + up16(b_ct) + up16(b_gr) + up16(b_in) +
                       up16(rwr.size() * sizeof(int)) + up16(cwr.size() * sizeof(int)) +
                       up16(teams.size() * sizeof(int));
  if (total > b->cap_stage) {
    if (b->h_stage) cudaFreeHost(b->h_stage);
    b->h_stage = nullptr;
    b->cap_stage = 0;
    PDLP_CUDA(cudaMallocHost((void**)&b->h_stage, total + total / 2));
    b->cap_stage = total + total / 2;
  }
  Tile* srt = reinterpret_cast<Tile*>(b->h_stage);
  Tile* sct = reinterpret_cast<Tile*>(b->h_stage + up16(b_rt));
  int2* sgr = reinterpret_cast<int2*>(b->h_stage + up16(b_rt) + up16(b_ct));
  Inst* sin = reinterpret_cast<Inst*>(b->h_stage + up16(b_rt) + up16(b_ct) + up16(b_gr));
  for (int s : run) {
    const Slot& sl = b->slots[s];
    const Inst& I = sl.inst;
    for (size_t k = 0; k < sl.rt.size(); ++k) {
      Tile t = sl.rt[k];
      t.group = I.rg_begin + (int)(k / kGroupTiles);
      srt[I.rt_begin + k] = t;
    }
    for (int g = I.rg_begin; g < I.rg_end; ++g) {
      const int g0 = I.rt_begin + (g - I.rg_begin) * kGroupTiles;
      sgr[g] = make_int2(g0, std::min(I.rt_end, g0 + kGroupTiles));
    }
    for (size_t k = 0; k < sl.ct.size(); ++k) {
      Tile t = sl.ct[k];
      t.group = I.cg_begin + (int)(k / kGroupTiles);
      sct[I.ct_begin + k] = t;
    }
    for (int g = I.cg_begin; g < I.cg_end; ++g) {
      const int g0 = I.ct_begin + (g - I.cg_begin) * kGroupTiles;
      sgr[g] = make_int2(g0, std::min(I.ct_end, g0 + kGroupTiles));
    }
  }
  for (size_t s = 0; s < b->slots.size(); ++s) sin[s] = b->slots[s].inst;
  size_t off = up16(b_rt) + up16(b_ct) + up16(b_gr) + up16(b_in);
  struct Part { void* dst; const void* src; size_t bytes; };
  const Part small[] = {{b->d_rwarp, rwr.data(), rwr.size() * sizeof(int)},
                        {b->d_cwarp, cwr.data(), cwr.size() * sizeof(int)},
                        {b->d_teams, teams.data(), teams.size() * sizeof(int)}};
  for (const Part& q : small) {
    std::memcpy(b->h_stage + off, q.src, q.bytes);
    PDLP_CUDA(cudaMemcpyAsync(q.dst, b->h_stage + off, q.bytes, cudaMemcpyHostToDevice, st));
    off += up16(q.bytes);
  }
  if (b_rt) PDLP_CUDA(cudaMemcpyAsync(b->d_rtiles, srt, b_rt, cudaMemcpyHostToDevice, st));
  if (b_ct) PDLP_CUDA(cudaMemcpyAsync(b->d_ctiles, sct, b_ct, cudaMemcpyHostToDevice, st));
  if (b_gr) PDLP_CUDA(cudaMemcpyAsync(b->d_group_tiles, sgr, b_gr, cudaMemcpyHostToDevice, st));
  PDLP_CUDA(cudaMemcpyAsync(b->d_inst, sin, b_in, cudaMemcpyHostToDevice, st));
  PDLP_CUDA(cudaMemsetAsync(b->d_gcounters, 0, ngr * sizeof(unsigned), st));
  PDLP_CUDA(cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned) * 2 * b->slots.size(), st));
  b->dirty = false;
  b->graph_stale = true;
  return PDLP_OK;
}

// The infeasibility test of one running slot, between launches.  The first
// call only records the iterates; later calls test the change since the
// previous call as a Farkas ray and, after two hits of the same kind in a
// row, return the status to end the solve with in *request (0: none).
static int infeasibility_test(pdlp_batch* b, Slot& sl, int* request) {
  *request = 0;
  const Inst& I = sl.inst;
  cudaStream_t st = b->stream;
  const size_t np = sizeof(double) * 8 * kRayBlocks;
  if (sl.have_prev) {
    ray_cols_kernel<<<kRayBlocks, 256, 0, st>>>(I, sl.xprev, sl.yprev, b->d_raypart);
    ray_rows_kernel<<<kRayBlocks, 256, 0, st>>>(I, sl.xprev, sl.yprev, b->d_raypart + 8 * kRayBlocks);
    count_launches(2);
    PDLP_CUDA(cudaGetLastError());
    PDLP_CUDA(cudaMemcpyAsync(b->h_raypart, b->d_raypart, 2 * np, cudaMemcpyDeviceToHost, st));
  }
  if (I.n) PDLP_CUDA(cudaMemcpyAsync(sl.xprev, I.x, sizeof(double) * I.n, cudaMemcpyDeviceToDevice, st));
  if (I.m) PDLP_CUDA(cudaMemcpyAsync(sl.yprev, I.y, sizeof(double) * I.m, cudaMemcpyDeviceToDevice, st));
  PDLP_CUDA(cudaStreamSynchronize(st));
  if (!sl.have_prev) { sl.have_prev = true; return PDLP_OK; }
  double col[8], row[8];
  for (int side = 0; side < 2; ++side) {
    double* out = side ? row : col;
    const double* part = b->h_raypart + (size_t)side * 8 * kRayBlocks;
    for (int k = 0; k < 8; ++k) {
      const bool is_sum = k == 0 || k == 1 || k == 4 || k == 5;
      double a = part[k];
      for (int g = 1; g < kRayBlocks; ++g) a = is_sum ? a + part[(size_t)g * 8 + k] : std::max(a, part[(size_t)g * 8 + k]);
      out[k] = a;
    }
  }
  int kind = 0;
  for (int s = 0; s < 2 && !kind; ++s) {
    const double dobj = row[s] + col[s], viol = col[2 + s], wmax = row[6 + s];
    if (wmax > 0.0 && dobj > 0.0 && viol <= sl.eps_inf * dobj) kind = PDLP_STATUS_INFEASIBLE;
  }
  for (int s = 0; s < 2 && !kind; ++s) {
    const double ctv = col[4 + s], viol = row[2 + s], vmax = col[6 + s];
    if (vmax > 0.0 && ctv < 0.0 && viol <= sl.eps_inf * -ctv) kind = PDLP_STATUS_INFEASIBLE_OR_UNBOUNDED;
  }
  if (kind && kind == sl.hit_kind) ++sl.hits;
  else { sl.hits = kind ? 1 : 0; sl.hit_kind = kind; }
  if (sl.hits >= 2) *request = kind;
  return PDLP_OK;
}

// ---- tuning cache ---------------------------------------------------------------
//
// Tuned choices by nnz profile (pdlp_tune_lp, pdlp_tune_cache_*), shared by
// every batch of the process; batches with cfg.autotune read it at admission.

namespace {

struct TuneKeyLess {
  bool operator()(const pdlp_tune_key& a, const pdlp_tune_key& b) const {
    if (a.rows_bucket != b.rows_bucket) return a.rows_bucket < b.rows_bucket;
    if (a.row_len_bucket != b.row_len_bucket) return a.row_len_bucket < b.row_len_bucket;
    return a.col_len_bucket < b.col_len_bucket;
  }
};

std::mutex g_tune_mu;
std::map<pdlp_tune_key, pdlp_tuning, TuneKeyLess> g_tune;

pdlp_tune_key tune_key(int m, int n, long long nnz) {
  pdlp_tune_key k;
  k.rows_bucket = (int)std::floor(std::log2((double)m + 1.0));
  k.row_len_bucket = m > 0 ? (int)std::floor(2.0 * std::log2((double)nnz / m + 1.0)) : 0;
  k.col_len_bucket = n > 0 ? (int)std::floor(2.0 * std::log2((double)nnz / n + 1.0)) : 0;
  return k;
}

bool tuning_valid(const pdlp_tuning& t) {
  auto pow2 = [](int v) { return v >= 1 && v <= 32 && (v & (v - 1)) == 0; };
  return pow2(t.lanes_rows) && pow2(t.lanes_cols) && t.tile_rows >= 1 &&
         t.tile_rows <= kWTileRows && t.tile_nnz >= 1 && t.tile_nnz <= kWTileNnz;
}

bool tune_lookup(int m, int n, long long nnz, pdlp_tuning* out) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(tune_key(m, n, nnz));
  if (it == g_tune.end()) return false;
  *out = it->second;
  return true;
}

}  // namespace

// ---- admission ---------------------------------------------------------------
//
// An admission runs in three phases so that many LPs can share the host's
// synchronisations: (1) admit_enqueue validates the arguments and the
// pointer arrays on the host, takes an arena and a slot, and enqueues the
// copies and the device check; (2) the caller reads every admission's
// verdict back with one synchronisation; (3) admit_complete fills the slot
// (descriptor, tiles, initial state) or gives the arena back.

struct Pending {
  bool ptrs_ok = false;            // pointer arrays checked (host, before the enqueue)
  int tile_rows = 0, tile_nnz = 0; // the tile shape admit_complete chose
  int slot = -1;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  SlotLayout L{};
  pdlp_params prm{};
  const pdlp_problem_desc* P = nullptr;
  const int64_t* rp = nullptr;     // host-readable pointer arrays
  const int64_t* cp = nullptr;
};

static int admit_args(pdlp_batch* b, const pdlp_problem_desc* P, const pdlp_params* params,
                      pdlp_params* prm) {
  if (!b || !P) return fail(PDLP_ERR_ARG, "NULL batch or problem");
  if (b->broken) return fail(PDLP_ERR_STATE, "batch is unusable after a device wait timed out");
  pdlp_params_default(prm);
  if (params) *prm = *params;
  const int m = P->m, n = P->n;
  const long long nnz = P->nnz;
  if (m < 0 || n < 0 || nnz < 0) return fail(PDLP_ERR_ARG, "negative dimension");
  if (nnz > 0x7fffffffLL) return fail(PDLP_ERR_ARG, "nnz must fit in int32");
  if (P->sense != 1 && P->sense != -1) return fail(PDLP_ERR_ARG, "sense must be 1 or -1");
  if (P->memory != PDLP_MEM_HOST && P->memory != PDLP_MEM_DEVICE)
    return fail(PDLP_ERR_ARG, "memory must be PDLP_MEM_HOST or PDLP_MEM_DEVICE");
  if (prm->check_every <= 0 || prm->stepsize_every <= 0)
    return fail(PDLP_ERR_ARG, "check_every and stepsize_every must be positive");
  if (prm->max_iter < 0) return fail(PDLP_ERR_ARG, "max_iter must be >= 0");
  if (prm->scaling < 0 || prm->scaling > 3) return fail(PDLP_ERR_ARG, "unknown scaling method");
  if (prm->precision != PDLP_PRECISION_FP64 && prm->precision != PDLP_PRECISION_FP32_SPMV)
    return fail(PDLP_ERR_ARG, "unknown precision");
  if (!std::isfinite(P->obj_offset)) return fail(PDLP_ERR_NUMERICAL, "obj_offset is not finite");
  if (!P->rp || !P->cp) return fail(PDLP_ERR_ARG, "rp/cp are NULL");
  return PDLP_OK;
}

// Phase 1.  pd.P, pd.prm, pd.rp and pd.cp are set by the caller (the pointer
// arrays already readable on the host).  On success the slot is reserved,
// the arena taken and the copies and the check enqueued on the stream.
// The compressed pointers start at 0, do not decrease and end at nnz.
static bool pointers_ok(const int64_t* p, int len, long long nnz) {
  if (p[0] != 0 || p[len] != nnz) return false;
  for (int i = 0; i < len; ++i) if (p[i + 1] < p[i]) return false;
  return true;
}

// Runs fn(i) for i in [0, n) on up to 16 host threads: the admission's
// per-LP host loops (pointer checks, tile planning) touch only that LP.
template <class F>
static void parallel_for(int n, F fn) {
  const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
  const int T = std::min({n, hw, 16});
  if (T <= 1) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(T);
  int started = 0;
  try {
    for (; started < T; ++started)
      pool.emplace_back([&fn, started, T, n] { for (int i = started; i < n; i += T) fn(i); });
  } catch (...) {                 // no thread could be started: this thread does the rest
    for (int t = started; t < T; ++t)
      for (int i = t; i < n; i += T) fn(i);
  }
  for (auto& th : pool) th.join();
}

static int admit_enqueue(pdlp_batch* b, Pending& pd, AdmitBatch& ab) {
  const pdlp_problem_desc* P = pd.P;
  const int m = P->m, n = P->n;
  const long long nnz = P->nnz;
  if (!pd.ptrs_ok)
    return fail(PDLP_ERR_ARG, "malformed compressed pointers (must start at 0, be non-decreasing and end at nnz)");
  int slot = -1;
  for (size_t s = 0; s < b->slots.size(); ++s)
    if (!b->slots[s].used && !b->slots[s].reserved) { slot = (int)s; break; }
  if (slot < 0) return fail(PDLP_ERR_STATE, "no free slot");
  cudaStream_t st = b->stream;
  const pdlp_params& prm = pd.prm;
  const int hist_cap = std::max(0, prm.history_capacity);
  const bool has_kind = P->kind != nullptr;
  const bool has_v0 = prm.power_start != nullptr;
  const bool f32 = prm.precision == PDLP_PRECISION_FP32_SPMV;
  pd.L = layout_for(m, n, nnz, has_kind, has_v0, hist_cap, f32);
  const SlotLayout& L = pd.L;
  // a retired arena that holds the layout without wasting more than half of itself
  int best = -1;
  for (size_t i = 0; i < b->spare.size(); ++i) {
    const size_t sz = b->spare[i].second;
    if (sz >= L.total && sz <= 2 * L.total + ((size_t)1 << 20) &&
        (best < 0 || sz < b->spare[(size_t)best].second))
      best = (int)i;
  }
  void* arena = nullptr;
  size_t arena_bytes = L.total;
  if (best >= 0) {
    arena = b->spare[(size_t)best].first;
    arena_bytes = b->spare[(size_t)best].second;
    b->spare.erase(b->spare.begin() + best);
    b->bytes_spare -= arena_bytes;
  } else {
    // a new arena: within the budget (spare arenas are released first if needed)
    auto fits = [&](bool* ok) -> int {
      if (b->cfg.memory_budget > 0) {
        *ok = b->bytes_held + b->bytes_pending + b->bytes_spare + L.total <=
              (size_t)b->cfg.memory_budget;
      } else {
        size_t fr = 0, tot = 0;
        PDLP_CUDA(cudaMemGetInfo(&fr, &tot));
        *ok = L.total <= (fr > ((size_t)1 << 30) ? fr - ((size_t)1 << 30) : 0);
      }
      return PDLP_OK;
    };
    bool ok = false;
    int frc = fits(&ok);
    if (frc) return frc;
    if (!ok && !b->spare.empty()) {
      PDLP_CUDA(cudaStreamSynchronize(st));
      for (auto& a : b->spare) cudaFree(a.first);
      b->spare.clear();
      b->bytes_spare = 0;
      if ((frc = fits(&ok))) return frc;
    }
    if (!ok) return fail(PDLP_ERR_OOM, "admission refused: the LP does not fit the memory budget");
    const cudaError_t e = cudaMalloc(&arena, L.total);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(PDLP_ERR_OOM, std::string("admission refused: cudaMalloc: ") + cudaGetErrorString(e));
    }
  }
  pd.slot = slot;
  pd.arena = arena;
  pd.arena_bytes = arena_bytes;
  b->slots[slot].reserved = true;
  b->bytes_pending += arena_bytes;
  char* base = (char*)arena;
  auto at = [&](size_t off) { return (void*)(base + off); };
  int rc = PDLP_OK;
  const int mem = P->memory;
  // the state's error word doubles as the validation flag
  int* err_flag = &b->d_state[slot].error;
  ab.add(&b->d_state[slot], nullptr, sizeof(State));
  long long* rp64 = (long long*)at(L.tmp64);
  long long* cp64 = rp64 + (m + 1);
  if ((rc = copy_in(ab, rp64, P->rp, sizeof(int64_t) * (m + 1), mem, st))) return rc;
  if ((rc = copy_in(ab, cp64, P->cp, sizeof(int64_t) * (n + 1), mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.ri), P->ri, sizeof(int) * nnz, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.ci), P->ci, sizeof(int) * nnz, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.rx0), P->rx, sizeof(double) * nnz, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.cx0), P->cx, sizeof(double) * nnz, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.c0), P->c, sizeof(double) * n, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.lo0), P->col_lb, sizeof(double) * n, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.hi0), P->col_ub, sizeof(double) * n, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.rl0), P->row_lb, sizeof(double) * m, mem, st))) return rc;
  if ((rc = copy_in(ab, at(L.ru0), P->row_ub, sizeof(double) * m, mem, st))) return rc;
  if (has_kind && (rc = copy_in(ab, at(L.kind), P->kind, (size_t)n, mem, st))) return rc;
  if (has_v0 && (rc = copy_in(ab, at(L.v0), prm.power_start, sizeof(double) * n, mem, st))) return rc;
  AdmitTasks T;
  T.rp64 = rp64; T.rp32 = (int*)at(L.rp32); T.m = m;
  T.cp64 = cp64; T.cp32 = (int*)at(L.cp32); T.n = n;
  T.ri = (const int*)at(L.ri); T.ci = (const int*)at(L.ci); T.nnz = nnz;
  T.rx0 = (const double*)at(L.rx0); T.cx0 = (const double*)at(L.cx0);
  T.c0 = (const double*)at(L.c0); T.lo0 = (const double*)at(L.lo0); T.hi0 = (const double*)at(L.hi0);
  T.rl0 = (const double*)at(L.rl0); T.ru0 = (const double*)at(L.ru0);
  T.err = err_flag;
  const long long most = std::max<long long>({nnz, (long long)m + 1, (long long)n + 1});
  ab.gx = std::max(ab.gx, (int)std::max(1LL, std::min(1024LL, (most + 255) / 256)));
  ab.tasks.push_back(T);
  return PDLP_OK;
}

// Grows a pinned staging array and its device twin to hold `need` elements
// (the previous contents are not kept; nothing is in flight on them between
// admit calls, each of which synchronises its stream).
template <typename E>
static int ensure_staging(E** h, E** d, size_t* cap, size_t need) {
  if (need <= *cap && *h && *d) return PDLP_OK;
  const size_t n = std::max(need, (size_t)64);
  if (*h) cudaFreeHost(*h);
  cudaFree(*d);
  *h = nullptr;
  *d = nullptr;
  *cap = 0;
  PDLP_CUDA(cudaMallocHost((void**)h, sizeof(E) * n));
  PDLP_CUDA(cudaMalloc((void**)d, sizeof(E) * n));
  *cap = n;
  return PDLP_OK;
}

// Launches the admit call's gathered copies, then its checks.
static int admit_flush(pdlp_batch* b, AdmitBatch& ab) {
  cudaStream_t st = b->stream;
  int rc;
  if (!ab.pieces.empty()) {
    const size_t n = ab.pieces.size();
    if ((rc = ensure_staging(&b->h_pieces, &b->d_pieces, &b->cap_pieces, n))) return rc;
    std::memcpy(b->h_pieces, ab.pieces.data(), sizeof(CopyPiece) * n);
    PDLP_CUDA(cudaMemcpyAsync(b->d_pieces, b->h_pieces, sizeof(CopyPiece) * n,
                              cudaMemcpyHostToDevice, st));
    const int g = (int)std::min<size_t>(n, (size_t)std::max(1, b->sms) * 8);
    gather_copy<<<g, 256, 0, st>>>(b->d_pieces, (int)n);
    PDLP_CUDA(cudaGetLastError());
    count_launches(1);
  }
  if (!ab.tasks.empty()) {
    const size_t n = ab.tasks.size();
    if ((rc = ensure_staging(&b->h_tasks, &b->d_tasks, &b->cap_tasks, n))) return rc;
    std::memcpy(b->h_tasks, ab.tasks.data(), sizeof(AdmitTasks) * n);
    PDLP_CUDA(cudaMemcpyAsync(b->d_tasks, b->h_tasks, sizeof(AdmitTasks) * n,
                              cudaMemcpyHostToDevice, st));
    for (size_t o = 0; o < n; o += 65535) {
      const unsigned z = (unsigned)std::min<size_t>(65535, n - o);
      admission_check<<<dim3(ab.gx, 11, z), 256, 0, st>>>(b->d_tasks + o);
      PDLP_CUDA(cudaGetLastError());
      count_launches(1);
    }
  }
  return PDLP_OK;
}

// Releases what a failed admission took (after its work on the stream is done).
static void admit_abandon(pdlp_batch* b, Pending& pd) {
  if (pd.slot >= 0) b->slots[pd.slot].reserved = false;
  if (pd.arena) {
    b->spare.push_back({pd.arena, pd.arena_bytes});
    b->bytes_spare += pd.arena_bytes;
    b->bytes_pending -= pd.arena_bytes;
  }
  pd.slot = -1;
  pd.arena = nullptr;
}

// Phase 3: herr is the device check's verdict for this admission.  The
// initial state is staged in b->h_init[slot] (pinned); the caller
// synchronises the stream before that buffer is reused.
static int admit_complete(pdlp_batch* b, Pending& pd, int herr) {
  if (herr & 1) { admit_abandon(b, pd); return fail(PDLP_ERR_ARG, "malformed sparse structure (pointer or index out of range)"); }
  if (herr & 2) { admit_abandon(b, pd); return fail(PDLP_ERR_NUMERICAL, "NaN in the data, or an infinite matrix entry or cost"); }
  const pdlp_problem_desc* P = pd.P;
  const pdlp_params& prm = pd.prm;
  const SlotLayout& L = pd.L;
  const int m = P->m, n = P->n;
  const long long nnz = P->nnz;
  const int slot = pd.slot;
  const int hist_cap = std::max(0, prm.history_capacity);
  const bool has_kind = P->kind != nullptr;
  const bool has_v0 = prm.power_start != nullptr;
  const bool f32 = prm.precision == PDLP_PRECISION_FP32_SPMV;
  char* base = (char*)pd.arena;
  auto at = [&](size_t off) { return (void*)(base + off); };
  Slot& S = b->slots[slot];
  S = Slot();
  S.used = true;
  S.running = true;
  S.m = m; S.n = n; S.nnz = nnz;
  S.arena = pd.arena;
  S.bytes = pd.arena_bytes;
  Inst& I = S.inst;
  std::memset(&I, 0, sizeof(I));
  I.m = m; I.n = n; I.nnz = nnz;
  // lanes per row and tile shape: forced (tuning runs), tuned (cache), or the
  // fixed rules
  pdlp_tuning tn{};
  const bool tuned = b->force_set ? (tn = b->force, true)
                                  : (b->cfg.autotune != 0 && tune_lookup(m, n, nnz, &tn));
  const int tile_rows = tuned ? tn.tile_rows : b->cfg.tile_rows;
  const int tile_nnz = tuned ? tn.tile_nnz : b->cfg.tile_nnz;
  I.lanes_r = b->cfg.lanes_override ? b->cfg.lanes_override
                                    : (tuned ? tn.lanes_rows : lanes_for(nnz, m));
  I.lanes_c = b->cfg.lanes_override ? b->cfg.lanes_override
                                    : (tuned ? tn.lanes_cols : lanes_for(nnz, n));
  I.sense = P->sense;
  I.ruiz_iters = prm.scaling == PDLP_SCALING_PDLP ? 10 : (prm.scaling == PDLP_SCALING_RUIZ ? 20 : 0);
  I.use_pc = prm.scaling == PDLP_SCALING_PDLP || prm.scaling == PDLP_SCALING_POCK_CHAMBOLLE;
  I.scale_none = prm.scaling == PDLP_SCALING_NONE;
  I.rp = (const int*)at(L.rp32); I.ri = (const int*)at(L.ri);
  I.cp = (const int*)at(L.cp32); I.ci = (const int*)at(L.ci);
  I.rx0 = (const double*)at(L.rx0); I.cx0 = (const double*)at(L.cx0);
  I.rx = (double*)at(L.rx); I.cx = (double*)at(L.cx);
  I.c0 = (const double*)at(L.c0); I.rl0 = (const double*)at(L.rl0); I.ru0 = (const double*)at(L.ru0);
  I.lo0 = (const double*)at(L.lo0); I.hi0 = (const double*)at(L.hi0);
  I.kind = has_kind ? (const unsigned char*)at(L.kind) : nullptr;
  I.offset0 = P->obj_offset;
  double** mv[14] = {&I.rl, &I.ru, &I.rs, &I.y, &I.ax, &I.dy, &I.ynew, &I.adx, &I.sumy,
                     &I.ybar, &I.axbar, &I.axf, &I.yrst, &I.yout};
  for (int i = 0; i < 14; ++i) *mv[i] = (double*)at(L.mvec[i]);
  double** nv[16] = {&I.c, &I.lo, &I.hi, &I.cs, &I.x, &I.aty, &I.dx, &I.xnew, &I.sumx,
                     &I.xbar, &I.atybar, &I.atyf, &I.xrst, &I.xout, &I.dout, nullptr};
  for (int i = 0; i < 15; ++i) *nv[i] = (double*)at(L.nvec[i]);
  S.xprev = (double*)at(L.nvec[15]);
  S.yprev = (double*)at(L.mvec[14]);
  S.detect = prm.detect_infeasibility != 0;
  S.expected_iters = std::isfinite(prm.expected_iterations) ? std::max(0.0, prm.expected_iterations) : 0.0;
  S.eps_inf = prm.eps_infeasible > 0.0 ? prm.eps_infeasible : 1e-8;
  I.v0 = has_v0 ? (const double*)at(L.v0) : nullptr;
  I.f32 = f32 ? 1 : 0;
  I.rx32 = f32 ? (float*)at(L.rx32) : nullptr;
  I.cx32 = f32 ? (float*)at(L.cx32) : nullptr;
  I.dx32 = f32 ? (float*)at(L.dx32) : nullptr;
  I.dy32 = f32 ? (float*)at(L.dy32) : nullptr;
  I.hist = hist_cap ? (double*)at(L.hist) : nullptr;
  I.hist_cap = hist_cap;
  I.eps_abs = prm.eps_abs; I.eps_rel = prm.eps_rel; I.feas_cap = prm.feas_cap;
  I.max_iter = prm.max_iter;
  I.time_limit_ns = prm.time_limit * 1e9;
  I.time_used_ns = prm.time_used * 1e9;
  I.check_every = prm.check_every; I.stepsize_every = prm.stepsize_every;
  I.beta_s = prm.beta_sufficient; I.beta_n = prm.beta_necessary; I.beta_a = prm.beta_artificial;
  I.theta = prm.primal_weight_smoothing;
  pd.tile_rows = tile_rows;          // the tiles are planned by admit_many, in parallel
  pd.tile_nnz = tile_nnz;
  // algorithmic bytes of one PDHG iteration: value + index per
  // entry and pointer per row on both passes, one gathered word per column /
  // row, the vectors each pass reads and writes
  S.bytes_per_iter = f32 ? 16.0 * (double)nnz + 4.0 * (m + 1) + 4.0 * (n + 1) +
                               4.0 * (m + n) + 8.0 * (9.0 * m + 10.0 * n) + 4.0 * (m + n)
                         : 24.0 * (double)nnz + 4.0 * (m + 1) + 4.0 * (n + 1) +
                               8.0 * (10.0 * m + 11.0 * n);
  State& init = b->h_init[slot];
  std::memset(&init, 0, sizeof(init));
  init.status = PDLP_STATUS_RUNNING;
  init.final_status = PDLP_STATUS_RUNNING;
  if (I.ruiz_iters > 0) { init.rmode = R_RUIZ; init.cmode = C_RUIZ; }
  else { init.rmode = R_PC; init.cmode = C_PC; }
  init.eta = 1.0; init.omega = 1.0; init.s_obj = 1.0;
  cudaStream_t st = b->stream;
  PDLP_CUDA(cudaMemcpyAsync(&b->d_state[slot], &init, sizeof(State), cudaMemcpyHostToDevice, st));
  PDLP_CUDA(cudaMemsetAsync(b->d_counters + 2 * slot, 0, 2 * sizeof(unsigned), st));
  b->bytes_pending -= pd.arena_bytes;
  b->bytes_held += pd.arena_bytes;
  b->n_running += 1;
  b->iters_before[slot] = 0;
  b->dirty = true;
  S.reserved = false;
  return PDLP_OK;
}

// Admits count LPs with one synchronisation for the device pointer arrays
// (when any are in device memory), one for the checks' verdicts and one at
// the end.  codes[i] receives each LP's code and slots[i] its slot (-1 when
// refused); the return value is the first failure's code (its message in
// pdlp_last_error) or PDLP_OK.
static int admit_many(pdlp_batch* b, int count, const pdlp_problem_desc* const* probs,
                      const pdlp_params* const* params, int32_t* slots, int32_t* codes) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (count < 0 || (count > 0 && !probs)) return fail(PDLP_ERR_ARG, "bad count or NULL problem list");
  if (count > (int)b->slots.size()) return fail(PDLP_ERR_STATE, "more LPs than slots");
  std::vector<Pending> pd(count);
  std::vector<int> code(count, PDLP_OK);
  std::string first_msg;
  int first = PDLP_OK;
  auto note = [&](int i, int c) {
    code[i] = c;
    if (c != PDLP_OK && first == PDLP_OK) { first = c; first_msg = get_error(); }
  };
  cudaStream_t st = b->stream;
  // device pointer arrays: one pinned staging area, one synchronisation
  size_t need = 0;
  for (int i = 0; i < count; ++i) {
    pd[i].P = probs[i];
    const int rc = admit_args(b, probs[i], params ? params[i] : nullptr, &pd[i].prm);
    note(i, rc);
    if (rc == PDLP_OK && probs[i]->memory == PDLP_MEM_DEVICE)
      need += (size_t)probs[i]->m + 1 + (size_t)probs[i]->n + 1;
  }
  if (need > b->cap_hptrs) {
    if (b->h_ptrs) cudaFreeHost(b->h_ptrs);
    b->h_ptrs = nullptr;
    b->cap_hptrs = 0;
    PDLP_CUDA(cudaMallocHost(&b->h_ptrs, sizeof(int64_t) * need));
    b->cap_hptrs = need;
  }
  size_t off = 0;
  for (int i = 0; i < count; ++i) {
    if (code[i] != PDLP_OK) continue;
    const pdlp_problem_desc* P = probs[i];
    if (P->memory == PDLP_MEM_DEVICE) {
      int64_t* hr = b->h_ptrs + off;
      int64_t* hc = hr + (P->m + 1);
      off += (size_t)P->m + 1 + (size_t)P->n + 1;
      PDLP_CUDA(cudaMemcpyAsync(hr, P->rp, sizeof(int64_t) * (P->m + 1), cudaMemcpyDeviceToHost, st));
      PDLP_CUDA(cudaMemcpyAsync(hc, P->cp, sizeof(int64_t) * (P->n + 1), cudaMemcpyDeviceToHost, st));
      pd[i].rp = hr;
      pd[i].cp = hc;
    } else {
      pd[i].rp = P->rp;
      pd[i].cp = P->cp;
    }
  }
  if (need) PDLP_CUDA(cudaStreamSynchronize(st));
  parallel_for(count, [&](int i) {
    if (code[i] == PDLP_OK)
      pd[i].ptrs_ok = pointers_ok(pd[i].rp, probs[i]->m, probs[i]->nnz) &&
                      pointers_ok(pd[i].cp, probs[i]->n, probs[i]->nnz);
  });
  AdmitBatch ab;
  for (int i = 0; i < count; ++i) {
    if (code[i] != PDLP_OK) continue;
    const size_t np = ab.pieces.size(), nt = ab.tasks.size();
    const int rc = admit_enqueue(b, pd[i], ab);
    if (rc != PDLP_OK) {
      ab.pieces.resize(np);             // nothing of a refused LP is copied or checked
      ab.tasks.resize(nt);
      cudaStreamSynchronize(st);        // its enqueued copies end before the arena is reused
      admit_abandon(b, pd[i]);
      note(i, rc);
    }
  }
  cudaError_t e = cudaSuccess;
  {
    const int frc = admit_flush(b, ab);
    if (frc != PDLP_OK) {
      cudaStreamSynchronize(st);
      for (int i = 0; i < count; ++i) if (code[i] == PDLP_OK) admit_abandon(b, pd[i]);
      return frc;
    }
  }
  // every verdict in one read-back (the states of all slots; nothing runs
  // between steps, so the running slots' copies are current too)
  e = cudaMemcpyAsync(b->h_state, b->d_state, sizeof(State) * b->slots.size(),
                      cudaMemcpyDeviceToHost, st);
  const cudaError_t e2 = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = e2;
  for (int i = 0; i < count; ++i)
    b->h_errs[i] = (code[i] == PDLP_OK && e == cudaSuccess) ? b->h_state[pd[i].slot].error : 0;
  if (e != cudaSuccess) {
    for (int i = 0; i < count; ++i) if (code[i] == PDLP_OK) admit_abandon(b, pd[i]);
    return cuda_fail(e, "admission copies");
  }
  for (int i = 0; i < count; ++i) {
    if (code[i] != PDLP_OK) continue;
    note(i, admit_complete(b, pd[i], b->h_errs[i]));
  }
  parallel_for(count, [&](int i) {
    if (code[i] != PDLP_OK) return;
    Slot& S = b->slots[pd[i].slot];
    plan_tiles(pd[i].rp, probs[i]->m, pd[i].slot, pd[i].tile_rows, pd[i].tile_nnz, S.rt, S.rtw);
    plan_tiles(pd[i].cp, probs[i]->n, pd[i].slot, pd[i].tile_rows, pd[i].tile_nnz, S.ct, S.ctw);
  });
  PDLP_CUDA(cudaStreamSynchronize(st));    // the initial states have left h_init
  for (int i = 0; i < count; ++i) {
    if (slots) slots[i] = code[i] == PDLP_OK ? pd[i].slot : -1;
    if (codes) codes[i] = code[i];
  }
  if (first != PDLP_OK) set_error(first_msg);
  return first;
}

extern "C" {

int pdlp_abi_version(void) { return PDLP_ABI_VERSION; }

int64_t pdlp_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

const char* pdlp_last_error(void) { return g_err.c_str(); }

void pdlp_params_default(pdlp_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->eps_abs = 1e-8;
  p->eps_rel = 1e-8;
  p->feas_cap = 1e-6;
  p->max_iter = 200000;
  p->time_limit = 600.0;
  p->check_every = 64;
  p->stepsize_every = 8;
  p->beta_sufficient = 0.2;
  p->beta_necessary = 0.8;
  p->beta_artificial = 0.36;
  p->primal_weight_smoothing = 0.5;
  p->scaling = PDLP_SCALING_PDLP;
  p->power_start = nullptr;
  p->time_used = 0.0;
  p->history_capacity = 0;
  p->detect_infeasibility = 0;
  p->eps_infeasible = 1e-8;
  p->expected_iterations = 0.0;
}

void pdlp_batch_config_default(pdlp_batch_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->max_slots = 1;
  c->persistent = 1;
  c->block_threads = kBlock;
  c->tile_rows = default_tile_rows();
  c->tile_nnz = default_tile_nnz();
  c->lanes_override = 0;
  c->memory_budget = 0;
  c->barrier_timeout_us = 0;
  c->autotune = 0;
  c->test_withhold_arrival = 0;
}

int64_t pdlp_slot_bytes(int32_t m, int32_t n, int64_t nnz) {
  return (int64_t)layout_for(m, n, nnz, true, true, 4096).total;
}

int pdlp_batch_create(const pdlp_batch_config* cfg, void* stream, pdlp_batch** out) {
  if (!out) return fail(PDLP_ERR_ARG, "out is NULL");
  *out = nullptr;
  pdlp_batch_config c;
  pdlp_batch_config_default(&c);
  if (cfg) c = *cfg;
  if (c.max_slots <= 0) return fail(PDLP_ERR_ARG, "max_slots must be positive");
  if (c.block_threads == 0) c.block_threads = kBlock;
  if (c.block_threads != kBlock) return fail(PDLP_ERR_ARG, "block_threads must be " + std::to_string(kBlock));
  if (c.tile_rows <= 0) c.tile_rows = default_tile_rows();
  if (c.tile_rows > kWTileRows) return fail(PDLP_ERR_ARG, "tile_rows exceeds " + std::to_string(kWTileRows));
  if (c.tile_nnz <= 0) c.tile_nnz = default_tile_nnz();
  if (c.tile_nnz > kWTileNnz) return fail(PDLP_ERR_ARG, "tile_nnz exceeds " + std::to_string(kWTileNnz));
  if (c.lanes_override && (c.lanes_override & (c.lanes_override - 1)))
    return fail(PDLP_ERR_ARG, "lanes_override must be a power of two");
  if (c.barrier_timeout_us < 0) return fail(PDLP_ERR_ARG, "barrier_timeout_us must be >= 0");
  pdlp_batch* b = new pdlp_batch();
  b->stream = (cudaStream_t)stream;
  b->cfg = c;
  b->slots.resize(c.max_slots);
  b->iters_before.assign(c.max_slots, 0);
  b->steps_left.assign(c.max_slots, 0);
  int dev = 0;
  cudaError_t e;
  auto bail = [&](cudaError_t err, const char* what) {
    pdlp_batch_destroy(b);
    return cuda_fail(err, what);
  };
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return bail(e, "cudaGetDevice");
  if ((e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
    return bail(e, "cudaDeviceGetAttribute");
  int coop = 0;
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if ((e = cudaFuncSetAttribute(engine_persistent, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSmemBytes)) != cudaSuccess)
    return bail(e, "cudaFuncSetAttribute");
  if ((e = cudaFuncSetAttribute(engine_pass, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kSmemBytes)) != cudaSuccess)
    return bail(e, "cudaFuncSetAttribute");
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->coop_blocks_per_sm, engine_persistent,
                                                          kBlock, kSmemBytes)) != cudaSuccess)
    return bail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
  if (!coop || b->coop_blocks_per_sm < 1) b->cfg.persistent = 0;
  if ((e = cudaMalloc(&b->d_inst, sizeof(Inst) * c.max_slots)) != cudaSuccess) return bail(e, "cudaMalloc");
  if ((e = cudaMalloc(&b->d_state, sizeof(State) * c.max_slots)) != cudaSuccess) return bail(e, "cudaMalloc");
  if ((e = cudaMalloc(&b->d_counters, sizeof(unsigned) * 2 * c.max_slots)) != cudaSuccess) return bail(e, "cudaMalloc");
  if ((e = cudaMalloc(&b->d_ctl, sizeof(Control))) != cudaSuccess) return bail(e, "cudaMalloc");
  if ((e = cudaMallocHost(&b->h_ctl, sizeof(Control))) != cudaSuccess) return bail(e, "cudaMallocHost");
  if ((e = cudaMalloc(&b->d_raypart, sizeof(double) * 16 * kRayBlocks)) != cudaSuccess)
    return bail(e, "cudaMalloc");
  if ((e = cudaMallocHost(&b->h_raypart, sizeof(double) * 16 * kRayBlocks)) != cudaSuccess)
    return bail(e, "cudaMallocHost");
  if ((e = cudaMallocHost(&b->h_state, sizeof(State) * c.max_slots)) != cudaSuccess) return bail(e, "cudaMallocHost");
  if ((e = cudaMallocHost(&b->h_init, sizeof(State) * c.max_slots)) != cudaSuccess) return bail(e, "cudaMallocHost");
  if ((e = cudaMallocHost(&b->h_errs, sizeof(int) * c.max_slots)) != cudaSuccess) return bail(e, "cudaMallocHost");
  cudaMemsetAsync(b->d_counters, 0, sizeof(unsigned) * 2 * c.max_slots, b->stream);
  cudaMemsetAsync(b->d_ctl, 0, sizeof(Control), b->stream);
  cudaMemsetAsync(b->d_state, 0, sizeof(State) * c.max_slots, b->stream);
  std::vector<Inst> zero(c.max_slots);
  std::memset(zero.data(), 0, sizeof(Inst) * zero.size());
  cudaMemcpyAsync(b->d_inst, zero.data(), sizeof(Inst) * zero.size(), cudaMemcpyHostToDevice, b->stream);
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  if (!b->cfg.persistent &&
      (e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(e, "cudaStreamCreateWithFlags");
  if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return bail(e, "cudaStreamSynchronize");
  *out = b;
  return PDLP_OK;
}

int pdlp_batch_destroy(pdlp_batch* b) {
  if (!b) return PDLP_OK;
  cudaStreamSynchronize(b->stream);
  for (auto& s : b->slots) if (s.arena) cudaFree(s.arena);
  for (auto& a : b->spare) cudaFree(a.first);
  cudaFree(b->d_inst); cudaFree(b->d_state); cudaFree(b->d_counters); cudaFree(b->d_ctl);
  cudaFree(b->d_rtiles); cudaFree(b->d_ctiles); cudaFree(b->d_rwarp); cudaFree(b->d_cwarp);
  cudaFree(b->d_teams);
  cudaFree(b->d_partials); cudaFree(b->d_group_tiles); cudaFree(b->d_gpartials);
  cudaFree(b->d_gcounters);
  cudaFree(b->d_raypart);
  if (b->h_raypart) cudaFreeHost(b->h_raypart);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  if (b->h_ctl) cudaFreeHost(b->h_ctl);
  if (b->h_state) cudaFreeHost(b->h_state);
  if (b->h_init) cudaFreeHost(b->h_init);
  if (b->h_errs) cudaFreeHost(b->h_errs);
  if (b->h_ptrs) cudaFreeHost(b->h_ptrs);
  if (b->h_pieces) cudaFreeHost(b->h_pieces);
  if (b->h_stage) cudaFreeHost(b->h_stage);
  if (b->h_tasks) cudaFreeHost(b->h_tasks);
  cudaFree(b->d_pieces);
  cudaFree(b->d_tasks);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  delete b;
  return PDLP_OK;
}

int pdlp_batch_admit(pdlp_batch* b, const pdlp_problem_desc* P, const pdlp_params* params,
                     int32_t* slot_out) {
  if (!b || !P) return fail(PDLP_ERR_ARG, "NULL batch or problem");
  int32_t slot = -1, code = PDLP_OK;
  const int rc = admit_many(b, 1, &P, &params, &slot, &code);
  if (rc == PDLP_OK && slot_out) *slot_out = slot;
  return rc;
}

int pdlp_batch_admit_many(pdlp_batch* b, int32_t count, const pdlp_problem_desc* probs,
                          const pdlp_params* params, int32_t* slots_out, int32_t* codes_out) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (count < 0 || (count > 0 && !probs)) return fail(PDLP_ERR_ARG, "bad count or NULL problem array");
  if (count > (int32_t)b->slots.size()) return fail(PDLP_ERR_STATE, "more LPs than slots");
  std::vector<const pdlp_problem_desc*> pp(count);
  std::vector<const pdlp_params*> qq(count);
  for (int i = 0; i < count; ++i) {
    pp[i] = probs + i;
    qq[i] = params ? params + i : nullptr;
  }
  return admit_many(b, count, pp.data(), qq.data(), slots_out, codes_out);
}

int pdlp_batch_step(pdlp_batch* b, int64_t max_steps, int32_t* active_out) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (b->broken) return fail(PDLP_ERR_STATE, "batch is unusable after a device wait timed out");
  b->last_ms = 0.0; b->last_bytes = 0.0; b->last_iters = 0;
  if (b->n_running == 0) { if (active_out) *active_out = 0; return PDLP_OK; }
  int rc;
  cudaStream_t st = b->stream;
  EngineArgs A{};
  A.trace = nullptr;
#ifdef PDLP_TRACE
  static long long* d_trace = nullptr;
  if (!d_trace) { cudaMalloc(&d_trace, sizeof(long long) * 1280); }
  cudaMemsetAsync(d_trace, 0, sizeof(long long) * 1280, b->stream);
  A.trace = d_trace;
#endif
  A.inst = b->d_inst; A.st = b->d_state;
  A.counters = b->d_counters; A.ctl = b->d_ctl;
  A.barrier_timeout_ns = b->cfg.barrier_timeout_us > 0 ? b->cfg.barrier_timeout_us * 1000LL
                                                       : 4000000000LL;
  A.n_inst = (int)b->slots.size();
  // Launches of at most kChunk steps: between launches the host drops
  // finished LPs from the tile lists and re-balances the blocks over what is
  // left.  Every running LP may advance max_steps steps in this call; each
  // team's budget for a launch is what its LP has left (one team: all its LPs
  // advance together and have the same budget left).
  const int64_t kChunk = 256;
  for (size_t s = 0; s < b->slots.size(); ++s)
    b->steps_left[s] = (b->slots[s].used && b->slots[s].running) ? std::max<int64_t>(max_steps, 0) : 0;
  double total_ms = 0.0;
  while (b->n_running > 0) {
    int64_t most = 0;                 // the largest budget left among running LPs
    for (size_t s = 0; s < b->slots.size(); ++s)
      if (b->slots[s].used && b->slots[s].running) most = std::max<int64_t>(most, b->steps_left[s]);
    if (most <= 0) break;
    if (b->dirty && (rc = rebuild(b))) return rc;
    A.rtiles = b->d_rtiles; A.n_rtiles = b->n_rtiles;
    A.ctiles = b->d_ctiles; A.n_ctiles = b->n_ctiles;
    A.rwarp = b->d_rwarp; A.cwarp = b->d_cwarp;
    A.block_team = b->d_teams;
    A.team_blocks = b->d_teams + b->grid;
    A.team_first = b->d_teams + b->grid + b->n_teams;
    A.group_tiles = b->d_group_tiles; A.n_rgroups = b->n_rgroups; A.n_groups = b->n_groups;
    A.partials = b->d_partials; A.gpartials = b->d_gpartials; A.gcounters = b->d_gcounters;
    const int64_t chunk = std::min(most, kChunk);
    A.max_steps = b->cfg.persistent ? kChunk : chunk;
    A.withhold_block = (b->cfg.persistent && b->cfg.test_withhold_arrival) ? b->withhold_candidate : -1;
    b->h_ctl->bar_count = 0; b->h_ctl->bar_gen = 0; b->h_ctl->active = b->n_running;
    b->h_ctl->error = 0; b->h_ctl->error_where = 0; b->h_ctl->stop = 0; b->h_ctl->idle = 0;
    for (int t = 0; t < kMaxTeams; ++t) {
      b->h_ctl->team_bar[t] = 0;
      b->h_ctl->team_go[t] = 1;
      b->h_ctl->team_active[t] = t < (int)b->team_running.size() ? b->team_running[t] : 0;
      b->h_ctl->team_budget[t] = 0;
      b->h_ctl->team_steps[t] = 0;
    }
    for (size_t s = 0; s < b->slots.size(); ++s) {
      const Slot& sl = b->slots[s];
      if (!sl.used || !sl.running) continue;
      const int t = b->n_teams > 1 ? sl.inst.team : 0;
      b->h_ctl->team_budget[t] = (int)std::min<int64_t>(b->steps_left[s], kChunk);
    }
    PDLP_CUDA(cudaMemcpyAsync(b->d_ctl, b->h_ctl, sizeof(Control), cudaMemcpyHostToDevice, st));
    PDLP_CUDA(cudaEventRecord(b->ev0, st));
    if (b->cfg.persistent) {
      void* args[] = {&A};
      PDLP_CUDA(cudaLaunchCooperativeKernel((void*)engine_persistent, dim3(b->grid), dim3(kBlock),
                                            args, kSmemBytes, st));
      count_launches(1);
    } else {
      if (b->graph_stale || !b->graph || b->graph_chunk != chunk) {
        if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
        const int cap = b->sms * b->coop_blocks_per_sm;
        const int g_r = std::max(1, std::min((b->n_rtiles + kWarps - 1) / kWarps, cap));
        const int g_c = std::max(1, std::min((b->n_ctiles + kWarps - 1) / kWarps, cap));
        cudaStream_t cs = b->cap_stream;
        PDLP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        for (int64_t s2 = 0; s2 < chunk; ++s2) {
          engine_pass<<<g_r, kBlock, kSmemBytes, cs>>>(A, 0);
          engine_pass<<<g_c, kBlock, kSmemBytes, cs>>>(A, 1);
        }
        cudaGraph_t g = nullptr;
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ce = cudaStreamEndCapture(cs, &g);
        if (le != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(le, "engine_pass capture"); }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
        const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) { b->graph = nullptr; return cuda_fail(ie, "cudaGraphInstantiate"); }
        b->graph_chunk = chunk;
        b->graph_stale = false;
      }
      PDLP_CUDA(cudaGraphLaunch(b->graph, st));
      count_launches(2 * chunk);
    }
    PDLP_CUDA(cudaEventRecord(b->ev1, st));
    PDLP_CUDA(cudaMemcpyAsync(b->h_ctl, b->d_ctl, sizeof(Control), cudaMemcpyDeviceToHost, st));
    PDLP_CUDA(cudaMemcpyAsync(b->h_state, b->d_state, sizeof(State) * b->slots.size(),
                              cudaMemcpyDeviceToHost, st));
    PDLP_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->ev0, b->ev1);
    total_ms += ms;
#ifdef PDLP_TRACE
    {
      long long h[1280];
      cudaMemcpy(h, A.trace, sizeof(h), cudaMemcpyDeviceToHost);
      {
        double acc[7] = {0};
        int cnt = 0;
        for (int q = 1; q < 63; ++q) {
          const long long* r = h + 640 + q * 8;
          if (!r[6] || !r[7]) continue;
          acc[0] += (r[0] - r[7]) * 1e-3;           // tile start -> hot path entry (state loads)
          for (int k = 1; k < 7; ++k) acc[k] += (r[k] - r[k - 1]) * 1e-3;
          ++cnt;
        }
        if (cnt) fprintf(stderr, "[trace] R hot tile (n=%d): pre=%.2f stage_issue=%.2f wait_matrix=%.2f gather=%.2f rowsum=%.2f wait_vec=%.2f epilogue=%.2f us\n",
                         cnt, acc[0] / cnt, acc[1] / cnt, acc[2] / cnt, acc[3] / cnt, acc[4] / cnt, acc[5] / cnt, acc[6] / cnt);
      }
      for (int blk = 0; blk < 2; ++blk) {
        double acc[4] = {0, 0, 0, 0};
        int cnt = 0;
        for (int st2 = 1; st2 < 64; ++st2) {
          const long long* r = h + blk * 320 + st2 * 5;
          if (!r[4]) break;
          for (int k = 0; k < 4; ++k) acc[k] += (r[k + 1] - r[k]) * 1e-3;
          ++cnt;
        }
        if (cnt) fprintf(stderr, "[trace] grid=%d block%s: steps=%d  Rtiles=%.2fus bar1=%.2fus Ctiles=%.2fus bar2=%.2fus\n",
                         b->grid, blk ? "last" : "0", cnt, acc[0] / cnt, acc[1] / cnt, acc[2] / cnt, acc[3] / cnt);
      }
      cudaMemsetAsync(A.trace, 0, sizeof(long long) * 1280, st);
    }
#endif
    if (b->h_ctl->error) {
      b->broken = true;
      if (b->h_ctl->error == PDLP_ERR_BOUNDS)
        return fail(PDLP_ERR_BOUNDS, "engine: an index check failed in the tile starting at row " +
                                         std::to_string(b->h_ctl->error_where) +
                                         "; the batch was stopped");
      return fail(b->h_ctl->error, "engine: a bounded device wait timed out; the batch was stopped");
    }
    int running = 0;
    for (size_t s = 0; s < b->slots.size(); ++s) {
      Slot& sl = b->slots[s];
      if (!sl.used || !sl.running) continue;
      b->steps_left[s] -= b->cfg.persistent ? b->h_ctl->team_steps[b->n_teams > 1 ? sl.inst.team : 0]
                                            : chunk;
      const State& hs = b->h_state[s];
      long long d = hs.iters_done - b->iters_before[s];
      b->iters_before[s] = hs.iters_done;
      b->last_iters += d;
      b->last_bytes += d * sl.bytes_per_iter;
      if (hs.status != PDLP_STATUS_RUNNING) { sl.running = false; b->dirty = true; }
      else {
        ++running;
        if (hs.rmode == R_NONE && hs.cmode == C_NONE) {
          b->broken = true;
          return fail(PDLP_ERR_STATE, "engine: a running LP has no pass scheduled (internal error)");
        }
        // iterating (past its first check) and due for the infeasibility test
        if (sl.detect && hs.cancel == 0 && hs.k >= 64 && hs.k >= sl.next_check) {
          int request = 0;
          if ((rc = infeasibility_test(b, sl, &request))) return rc;
          sl.next_check = hs.k + 256;
          if (request) {
            const int req = 100 + request;
            PDLP_CUDA(cudaMemcpyAsync(&b->d_state[s].cancel, &req, sizeof(int),
                                      cudaMemcpyHostToDevice, st));
            PDLP_CUDA(cudaStreamSynchronize(st));
          }
        }
      }
    }
    b->n_running = running;
  }
  b->last_ms = total_ms;
  if (active_out) *active_out = b->n_running;
  return PDLP_OK;
}

int pdlp_batch_last_timing(pdlp_batch* b, double* ms, double* iter_bytes, int64_t* iterations) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (ms) *ms = b->last_ms;
  if (iter_bytes) *iter_bytes = b->last_bytes;
  if (iterations) *iterations = b->last_iters;
  return PDLP_OK;
}

// The caller's view of one slot's state.
static void result_of(const State& hs, pdlp_result* r) {
  std::memset(r, 0, sizeof(*r));
  const double nan = std::nan("");
  r->status = hs.status;
  r->iterations = hs.k;
  r->restarts = hs.restarts;
  r->rejected_steps = hs.rejected;
  const bool opt = hs.status == PDLP_STATUS_OPTIMAL;
  r->primal_res = opt ? hs.fin[0] : nan;
  r->dual_res = opt ? hs.fin[1] : nan;
  r->gap = opt ? hs.fin[2] : nan;
  r->primal_obj = opt ? hs.fin[3] : nan;
  r->dual_obj = opt ? hs.fin[4] : nan;
  r->step_size = hs.eta;
  r->primal_weight = hs.omega;
  r->objective = hs.status == PDLP_STATUS_RUNNING ? nan : hs.objective;
  r->scale_obj = hs.s_obj;
  r->history_len = hs.hist_len;
  r->device_seconds = hs.t_end_ns > hs.t_start_ns ? (hs.t_end_ns - hs.t_start_ns) * 1e-9 : 0.0;
  r->device_start_ns = hs.t_start_ns;
  r->device_end_ns = hs.t_end_ns;
}

int pdlp_batch_poll(pdlp_batch* b, int32_t slot, pdlp_result* r) {
  if (!b || !r) return fail(PDLP_ERR_ARG, "NULL argument");
  if (slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return fail(PDLP_ERR_ARG, "no such slot");
  State hs;
  PDLP_CUDA(cudaMemcpyAsync(&hs, &b->d_state[slot], sizeof(State), cudaMemcpyDeviceToHost, b->stream));
  PDLP_CUDA(cudaStreamSynchronize(b->stream));
  result_of(hs, r);
  return PDLP_OK;
}

int pdlp_batch_collect_many(pdlp_batch* b, int32_t n, const int32_t* slots, pdlp_result* results,
                            double* const* x, double* const* y, double* const* d,
                            double* const* history, int32_t memory, int32_t retire) {
  if (!b || n < 0 || (n > 0 && !slots)) return fail(PDLP_ERR_ARG, "NULL argument");
  if (memory != PDLP_MEM_HOST && memory != PDLP_MEM_DEVICE)
    return fail(PDLP_ERR_ARG, "memory must be PDLP_MEM_HOST or PDLP_MEM_DEVICE");
  std::vector<char> seen(b->slots.size(), 0);
  for (int32_t i = 0; i < n; ++i) {
    const int32_t slot = slots[i];
    if (slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
      return fail(PDLP_ERR_ARG, "no such slot: " + std::to_string(slot));
    if (seen[slot]) return fail(PDLP_ERR_ARG, "slot listed twice: " + std::to_string(slot));
    seen[slot] = 1;
    if (b->slots[slot].running) return fail(PDLP_ERR_STATE, "slot is still running: " + std::to_string(slot));
  }
  if (n == 0) return PDLP_OK;
  const cudaMemcpyKind k = memory == PDLP_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  cudaStream_t st = b->stream;
  PDLP_CUDA(cudaMemcpyAsync(b->h_state, b->d_state, sizeof(State) * b->slots.size(),
                            cudaMemcpyDeviceToHost, st));
  for (int32_t i = 0; i < n; ++i) {
    const Slot& sl = b->slots[slots[i]];
    if (x && x[i] && sl.n) PDLP_CUDA(cudaMemcpyAsync(x[i], sl.inst.xout, sizeof(double) * sl.n, k, st));
    if (y && y[i] && sl.m) PDLP_CUDA(cudaMemcpyAsync(y[i], sl.inst.yout, sizeof(double) * sl.m, k, st));
    if (d && d[i] && sl.n) PDLP_CUDA(cudaMemcpyAsync(d[i], sl.inst.dout, sizeof(double) * sl.n, k, st));
  }
  PDLP_CUDA(cudaStreamSynchronize(st));
  if (history) {                    // each slot's check history, now that its length is known
    bool any = false;
    for (int32_t i = 0; i < n; ++i) {
      const Slot& sl = b->slots[slots[i]];
      const int len = std::min(b->h_state[slots[i]].hist_len, sl.inst.hist_cap);
      if (history[i] && len > 0) {
        PDLP_CUDA(cudaMemcpyAsync(history[i], sl.inst.hist, sizeof(double) * 5 * (size_t)len, k, st));
        any = true;
      }
    }
    if (any) PDLP_CUDA(cudaStreamSynchronize(st));
  }
  for (int32_t i = 0; i < n; ++i)
    if (results) result_of(b->h_state[slots[i]], results + i);
  if (retire) {
    for (int32_t i = 0; i < n; ++i) {
      Slot& sl = b->slots[slots[i]];
      b->spare.push_back({sl.arena, sl.bytes});
      b->bytes_spare += sl.bytes;
      b->bytes_held -= sl.bytes;
      sl = Slot();
    }
    b->dirty = true;
  }
  return PDLP_OK;
}

int pdlp_batch_fetch(pdlp_batch* b, int32_t slot, double* x, double* y, double* d,
                     double* history, int32_t memory) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return fail(PDLP_ERR_ARG, "no such slot");
  Slot& s = b->slots[slot];
  if (s.running) return fail(PDLP_ERR_STATE, "slot is still running");
  cudaMemcpyKind k = memory == PDLP_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  cudaStream_t st = b->stream;
  if (x && s.n) PDLP_CUDA(cudaMemcpyAsync(x, s.inst.xout, sizeof(double) * s.n, k, st));
  if (y && s.m) PDLP_CUDA(cudaMemcpyAsync(y, s.inst.yout, sizeof(double) * s.m, k, st));
  if (d && s.n) PDLP_CUDA(cudaMemcpyAsync(d, s.inst.dout, sizeof(double) * s.n, k, st));
  if (history && s.inst.hist_cap) {
    State hs;
    PDLP_CUDA(cudaMemcpyAsync(&hs, &b->d_state[slot], sizeof(State), cudaMemcpyDeviceToHost, st));
    PDLP_CUDA(cudaStreamSynchronize(st));
    if (hs.hist_len) PDLP_CUDA(cudaMemcpyAsync(history, s.inst.hist, sizeof(double) * 5 * hs.hist_len, k, st));
  }
  PDLP_CUDA(cudaStreamSynchronize(st));
  return PDLP_OK;
}

int pdlp_batch_statuses(pdlp_batch* b, int32_t* out, int32_t n) {
  if (!b || (!out && n > 0)) return fail(PDLP_ERR_ARG, "NULL argument");
  for (int32_t s = 0; s < n; ++s) {
    if (s >= (int)b->slots.size() || !b->slots[s].used) out[s] = PDLP_SLOT_FREE;
    else if (b->slots[s].running) out[s] = PDLP_STATUS_RUNNING;
    else out[s] = b->h_state[s].status;
  }
  return PDLP_OK;
}

int pdlp_batch_retire(pdlp_batch* b, int32_t slot) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return fail(PDLP_ERR_ARG, "no such slot");
  Slot& s = b->slots[slot];
  PDLP_CUDA(cudaStreamSynchronize(b->stream));
  if (s.running) { b->n_running -= 1; }
  b->spare.push_back({s.arena, s.bytes});
  b->bytes_spare += s.bytes;
  b->bytes_held -= s.bytes;
  s = Slot();
  b->dirty = true;
  return PDLP_OK;
}

int pdlp_batch_scaling(pdlp_batch* b, int32_t slot, double* row_scale, double* col_scale,
                       double* obj_scale, int32_t memory) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return fail(PDLP_ERR_ARG, "no such slot");
  if (memory != PDLP_MEM_HOST && memory != PDLP_MEM_DEVICE)
    return fail(PDLP_ERR_ARG, "memory must be PDLP_MEM_HOST or PDLP_MEM_DEVICE");
  Slot& s = b->slots[slot];
  cudaStream_t st = b->stream;
  State hs;
  PDLP_CUDA(cudaMemcpyAsync(&hs, &b->d_state[slot], sizeof(State), cudaMemcpyDeviceToHost, st));
  PDLP_CUDA(cudaStreamSynchronize(st));
  // the factors are final once the set-up pass that follows them has run
  const bool scaling = hs.rmode == R_RUIZ || hs.rmode == R_PC || hs.rmode == R_APPLY ||
                       hs.cmode == C_RUIZ || hs.cmode == C_PC || hs.cmode == C_APPLY;
  if (hs.status == PDLP_STATUS_RUNNING && (scaling || hs.rmode == R_SETUP0))
    return fail(PDLP_ERR_STATE, "the slot is still preconditioning");
  const cudaMemcpyKind k = memory == PDLP_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  if (row_scale && s.m) PDLP_CUDA(cudaMemcpyAsync(row_scale, s.inst.rs, sizeof(double) * s.m, k, st));
  if (col_scale && s.n) PDLP_CUDA(cudaMemcpyAsync(col_scale, s.inst.cs, sizeof(double) * s.n, k, st));
  if (obj_scale) {
    if (memory == PDLP_MEM_HOST) *obj_scale = hs.s_obj;
    else PDLP_CUDA(cudaMemcpyAsync(obj_scale, &b->d_state[slot].s_obj, sizeof(double), k, st));
  }
  PDLP_CUDA(cudaStreamSynchronize(st));
  return PDLP_OK;
}

int pdlp_batch_cancel(pdlp_batch* b, int32_t slot) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL batch");
  if (slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot].used)
    return fail(PDLP_ERR_ARG, "no such slot");
  int one = 1;
  PDLP_CUDA(cudaMemcpyAsync(&b->d_state[slot].cancel, &one, sizeof(int), cudaMemcpyHostToDevice, b->stream));
  PDLP_CUDA(cudaStreamSynchronize(b->stream));
  return PDLP_OK;
}

void pdlp_tune_key_of(int32_t m, int32_t n, int64_t nnz, pdlp_tune_key* key) {
  if (key) *key = tune_key(m, n, nnz);
}

int pdlp_tune_cache_size(void) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  return (int)g_tune.size();
}

int pdlp_tune_cache_get(int32_t i, pdlp_tune_key* key, pdlp_tuning* tuning) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  if (i < 0 || i >= (int)g_tune.size()) return fail(PDLP_ERR_ARG, "no such cache entry");
  auto it = g_tune.begin();
  std::advance(it, i);
  if (key) *key = it->first;
  if (tuning) *tuning = it->second;
  return PDLP_OK;
}

int pdlp_tune_cache_put(const pdlp_tune_key* key, const pdlp_tuning* tuning) {
  if (!key || !tuning) return fail(PDLP_ERR_ARG, "NULL key or tuning");
  if (!tuning_valid(*tuning))
    return fail(PDLP_ERR_ARG, "tuning out of range (lanes 1..32, a power of two; tile_rows 1..64; "
                              "tile_nnz 1..512)");
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[*key] = *tuning;
  return PDLP_OK;
}

void pdlp_tune_cache_clear(void) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune.clear();
}

int pdlp_tune_lp(const pdlp_problem_desc* prob, const pdlp_params* params, void* stream,
                 pdlp_tuning* out) {
  if (!prob) return fail(PDLP_ERR_ARG, "NULL problem");
  // the probe runs never converge: zero tolerances, no limits
  pdlp_params prm;
  pdlp_params_default(&prm);
  if (params) prm = *params;
  prm.eps_abs = 0.0; prm.eps_rel = 0.0; prm.feas_cap = 0.0;
  prm.max_iter = (int64_t)1 << 40;
  prm.time_limit = 1e9;
  prm.history_capacity = 0;
  prm.detect_infeasibility = 0;
  pdlp_batch_config cfg;
  pdlp_batch_config_default(&cfg);
  cfg.max_slots = 1;
  pdlp_batch* b = nullptr;
  int rc = pdlp_batch_create(&cfg, stream, &b);
  if (rc) return rc;
  constexpr int kSetupSteps = 48;     // scaling (<= 12 steps), set-up, 20 power rounds
  constexpr int kTimedSteps = 64;
  // Every candidate runs on the same number of blocks: about eight tiles of
  // the default shape per warp, the load a warp carries when a full batch
  // shares the GPU.  Timed alone on all the blocks it can use, an LP favours
  // small tiles (more warps on one LP), which lose in a loaded batch.
  {
    const long long by_nnz = (long long)prob->nnz / default_tile_nnz() + 1;
    const long long by_rows = (long long)std::max(prob->m, prob->n) / default_tile_rows() + 1;
    const long long tiles = std::max(by_nnz, by_rows);
    b->force_blocks = (int)std::max(1LL, (tiles + 8 * kWarps - 1) / (8 * kWarps));
  }
  auto probe = [&](const pdlp_tuning& cand, double* us) -> int {
    b->force_set = true;
    b->force = cand;
    int32_t slot = -1, active = 0;
    int r = pdlp_batch_admit(b, prob, &prm, &slot);
    if (r) return r;
    if ((r = pdlp_batch_step(b, kSetupSteps, &active))) return r;
    double best = INFINITY;
    for (int rep = 0; rep < 2 && active > 0; ++rep) {
      if ((r = pdlp_batch_step(b, kTimedSteps, &active))) return r;
      double ms = 0.0, by = 0.0;
      int64_t its = 0;
      pdlp_batch_last_timing(b, &ms, &by, &its);
      if (its > 0) best = std::min(best, 1000.0 * ms / (double)its);
    }
    *us = best;
    return pdlp_batch_retire(b, slot);
  };
  pdlp_tuning def{};
  def.lanes_rows = lanes_for(prob->nnz, prob->m);
  def.lanes_cols = lanes_for(prob->nnz, prob->n);
  def.tile_rows = default_tile_rows();
  def.tile_nnz = default_tile_nnz();
  pdlp_tuning best = def;
  double best_us = INFINITY, def_us = INFINITY;
  const int lanes[3] = {1, 2, 4};
  for (int a = 0; a < 3 && !rc; ++a) {
    for (int c = 0; c < 3 && !rc; ++c) {
      pdlp_tuning cand = def;
      cand.lanes_rows = lanes[a];
      cand.lanes_cols = lanes[c];
      double us = INFINITY;
      rc = probe(cand, &us);
      if (cand.lanes_rows == def.lanes_rows && cand.lanes_cols == def.lanes_cols) def_us = us;
      if (!rc && us < best_us) { best_us = us; best = cand; }
    }
  }
  const int shapes[3][2] = {{32, 512}, {64, 256}, {32, 256}};
  for (int k = 0; k < 3 && !rc; ++k) {
    pdlp_tuning cand = best;
    cand.tile_rows = shapes[k][0];
    cand.tile_nnz = shapes[k][1];
    double us = INFINITY;
    rc = probe(cand, &us);
    if (!rc && us < best_us) { best_us = us; best = cand; }
  }
  pdlp_batch_destroy(b);
  if (rc) return rc;
  if (!std::isfinite(best_us)) return fail(PDLP_ERR_STATE, "tuning: the LP finished inside its probe runs");
  best.us_per_iteration = best_us;
  best.default_us_per_iteration = def_us;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[tune_key(prob->m, prob->n, prob->nnz)] = best;
  }
  if (out) *out = best;
  return PDLP_OK;
}

int pdlp_solve(const pdlp_problem_desc* prob, const pdlp_params* params, void* stream,
               pdlp_result* result, double* x, double* y, double* d, double* history,
               int32_t out_memory) {
  pdlp_batch_config cfg;
  pdlp_batch_config_default(&cfg);
  cfg.max_slots = 1;
  pdlp_batch* b = nullptr;
  int rc = pdlp_batch_create(&cfg, stream, &b);
  if (rc) return rc;
  int slot = -1;
  if ((rc = pdlp_batch_admit(b, prob, params, &slot))) { pdlp_batch_destroy(b); return rc; }
  int active = 1;
  const double guard_s = (params ? params->time_limit : 600.0) + 120.0;
  const auto t0 = std::chrono::steady_clock::now();
  while (active > 0) {
    if ((rc = pdlp_batch_step(b, 1 << 16, &active))) { pdlp_batch_destroy(b); return rc; }
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (active > 0 && el > guard_s) {
      pdlp_batch_destroy(b);
      return fail(PDLP_ERR_STATE, "engine: the solve outran its time limit by two minutes");
    }
  }
  pdlp_result r;
  if ((rc = pdlp_batch_poll(b, slot, &r))) { pdlp_batch_destroy(b); return rc; }
  if (result) *result = r;
  if ((rc = pdlp_batch_fetch(b, slot, x, y, d, history, out_memory))) { pdlp_batch_destroy(b); return rc; }
  pdlp_batch_destroy(b);
  return PDLP_OK;
}

}  // extern "C"
