// Batched node relaxation (BNR): K node LPs that share one scaled problem
// (matrix, costs and row bounds) and differ only in their column bounds,
// advanced together by a fixed number of PDHG iterations with a step size per
// node, then bounded from below by the safe dual bound of each node.  The
// algorithm is the reference's BNREngine.solve_batch (src/sovopt/mip/bnr.py:
// 176-301) with safe_dual_bound_batch (src/sovopt/mip/safebound.py:194-235).
//
// Layout: every per-node block is (rows, K) with the node index fastest, so a
// sparse product reads A once for all K nodes (A X with X (n, K)).  One
// iteration is five launches:
//   primal step (+ sum dX dX)  ->  A dX  ->  dual step (+ sums dY AdX, dY dY)
//   ->  A^T dY  ->  per-node accept / step size.
// A taken trial is not stored but redone by the next step, which reads the
// same inputs anyway (see bnr_primal).
// The iterations of one call are captured once into a CUDA graph, keyed by
// (K, iterations, step exponents), and replayed.
//
// Products and sums keep the reference's operations in the same order
// (explicit round-to-nearest multiplies and adds: no fused multiply-add), so
// element-wise results equal the reference's CPU results.  The per-node sums
// are fixed-order trees, which differ from the reference's sequential sums
// only by rounding.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"

namespace pdlp {
namespace {

constexpr double kBnrInf = 1.0e30;               // core/tolerances.py:16
constexpr double kQuotientMax = 1.0715086071862673e301;   // 2^1000 (tolerances.py:23)
constexpr int kRowsPerBlock = 64;                // rows per block of the per-node sums

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
// numpy.minimum / numpy.maximum: a NaN operand gives NaN (fmin/fmax would drop it)
__device__ __forceinline__ double np_min(double a, double b) {
  return (isnan(a) || isnan(b)) ? a + b : fmin(a, b);
}
__device__ __forceinline__ double np_max(double a, double b) {
  return (isnan(a) || isnan(b)) ? a + b : fmax(a, b);
}
__device__ __forceinline__ double clipd(double v, double lo, double hi) {
  return np_min(np_max(v, lo), hi);     // numpy.clip: maximum, then minimum
}

// Y (rows, k) = A X with X (cols, k) node-fastest.  One thread per (row, V
// consecutive nodes): V = 2 when k is even (16-byte gathers and stores), else
// 1.  Each node's entries are added in storage order (the reference's CSR
// SpMM order).  The entries are taken two at a time, both gathers issued
// before the adds, with eight blocks resident per SM.  The products are bound
// by the latency of gathers that L2 serves; among one, two or four nodes per
// thread, two to eight entries per batch and one to eight blocks per SM, this
// form measured fastest on B200.
template <int V>
struct Lanes;
template <>
struct Lanes<1> {
  double v[1];
  __device__ static Lanes load(const double* p) { return Lanes{{*p}}; }
  __device__ void store(double* p) const { *p = v[0]; }
};
template <>
struct Lanes<2> {
  double v[2];
  __device__ static Lanes load(const double* p) {
    const double2 t = *reinterpret_cast<const double2*>(p);
    return Lanes{{t.x, t.y}};
  }
  __device__ void store(double* p) const { *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]); }
};

template <int V>
__global__ void __launch_bounds__(256, 8) bnr_spmm(int rows, int k, const int64_t* __restrict__ rp,
                                                const int* __restrict__ ri,
                                                const double* __restrict__ rx,
                                                const double* __restrict__ X,
                                                double* __restrict__ Y) {
  constexpr int kBatch = 2;
  const int groups = k / V;
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= (long long)rows * groups) return;
  const long long r = g / groups;
  const int col = (int)(g - r * groups) * V;
  const double* Xc = X + col;
  long long p = __ldg(rp + r);
  const long long end = __ldg(rp + r + 1);
  double acc[V];
#pragma unroll
  for (int u = 0; u < V; ++u) acc[u] = 0.0;
  for (; p + kBatch <= end; p += kBatch) {
    double v[kBatch];
    Lanes<V> x[kBatch];
#pragma unroll
    for (int u = 0; u < kBatch; ++u) {
      v[u] = __ldg(rx + p + u);
      x[u] = Lanes<V>::load(Xc + (long long)__ldg(ri + p + u) * k);
    }
#pragma unroll
    for (int u = 0; u < kBatch; ++u)
#pragma unroll
      for (int e = 0; e < V; ++e) acc[e] = add(acc[e], mul(v[u], x[u].v[e]));
  }
  for (; p < end; ++p) {
    const double v = __ldg(rx + p);
    const Lanes<V> x = Lanes<V>::load(Xc + (long long)__ldg(ri + p) * k);
#pragma unroll
    for (int e = 0; e < V; ++e) acc[e] = add(acc[e], mul(v, x.v[e]));
  }
  Lanes<V> out;
#pragma unroll
  for (int e = 0; e < V; ++e) out.v[e] = acc[e];
  out.store(Y + r * k + col);
}

// The per-node sums over rows run in a fixed order: blocks of kRowsPerBlock
// rows; in a block, phase y (threadIdx.y, 8 phases) adds rows r0 + y + 8 j
// for j ascending from 0.0; the phases are added in order; then
// warp_blocks_sum adds the blocks.  The element-wise kernels below walk their rows in that
// layout, block (32, 8) with threadIdx.x the node within a 32-node tile, and
// sum as they go.  Output pair of row block b and node j at
// part[2 (j pstride + b)], pstride = mblocks + nblocks + 1, so one node's
// partials are contiguous for the warp that adds them: m-side blocks
// [0, mblocks), n-side blocks [mblocks, mblocks + nblocks).
__device__ __forceinline__ void bnr_block_sums(double s0, double s1, int k, int node,
                                               int pstride, int part_block,
                                               double* __restrict__ part) {
  __shared__ double sh[2][8][32];
  sh[0][threadIdx.y][threadIdx.x] = s0;
  sh[1][threadIdx.y][threadIdx.x] = s1;
  __syncthreads();
  if (threadIdx.y == 0 && node < k) {
    double a = sh[0][0][threadIdx.x], c2 = sh[1][0][threadIdx.x];
    for (int y = 1; y < 8; ++y) {
      a = add(a, sh[0][y][threadIdx.x]);
      c2 = add(c2, sh[1][y][threadIdx.x]);
    }
    double* out = part + ((long long)node * pstride + part_block) * 2;
    out[0] = a;
    out[1] = c2;
  }
}

// A taken trial is not stored: the next step recomputes it.  pend[j] says
// that node j's last trial was taken, and eta_prev[j] is the step size that
// trial used.  The next primal and dual steps read X, AtY, Y and AX anyway;
// for a pending node they first redo the trial from them with the same
// operations, which gives the same bits, and store it as the current
// iterate together with the reference's other updates on acceptance,
// AtY += AtdY and AX += AdX (bnr.py:262-265).  Nothing is copied, and one
// buffer per iterate suffices.

// Xn = clip(X - tau (c + AtY), L, U), dX = Xn - X (bnr.py:233-236), and the
// node's sum of dX dX over the block's rows.
__global__ void __launch_bounds__(256) bnr_primal(int n, int k, int mblocks, int pstride,
                                                  const double* __restrict__ c,
                                                  const double* __restrict__ eta,
                                                  const double* __restrict__ eta_prev,
                                                  const double* __restrict__ omega,
                                                  const int* __restrict__ pend,
                                                  double* __restrict__ X,
                                                  double* __restrict__ AtY,
                                                  const double* __restrict__ AtdY,
                                                  const double* __restrict__ L,
                                                  const double* __restrict__ U,
                                                  double* __restrict__ dX,
                                                  double* __restrict__ part) {
  const int node = blockIdx.y * 32 + threadIdx.x;
  double s = 0.0;
  if (node < k) {
    const double tau = eta[node] / omega[node];
    const bool taken = pend[node] != 0;
    const double tau_prev = eta_prev[node] / omega[node];
    const int r0 = blockIdx.x * kRowsPerBlock, r1 = min(n, r0 + kRowsPerBlock);
    for (int r = r0 + threadIdx.y; r < r1; r += 8) {
      const long long g = (long long)r * k + node;
      const double cr = __ldg(c + r), lo = L[g], hi = U[g];
      double x = X[g], aty = AtY[g];
      if (taken) {
        x = clipd(sub(x, mul(tau_prev, add(cr, aty))), lo, hi);
        aty = add(aty, AtdY[g]);
        X[g] = x;
        AtY[g] = aty;
      }
      const double xn = clipd(sub(x, mul(tau, add(cr, aty))), lo, hi);
      const double d = sub(xn, x);
      dX[g] = d;
      s = add(s, mul(d, d));
    }
  }
  bnr_block_sums(s, 0.0, k, node, pstride, mblocks + blockIdx.x, part);
}

// The dual trial of a node with step sigma (bnr.py:238-242).
__device__ __forceinline__ double dual_trial(double y, double ax, double adx, double sigma,
                                             double lo, double hi) {
  const double w = add(y, mul(sigma, add(ax, mul(2.0, adx))));
  return sub(w, mul(sigma, clipd(w / sigma, lo, hi)));
}

// W = Y + sigma (AX + 2 AdX); Yn = W - sigma clip(W / sigma, rl, ru); dY = Yn - Y
// (bnr.py:238-242), and the node's sums of dY AdX and dY dY over the block's
// rows.  AdX_prev is the previous step's A dX, which the redone trial uses.
__global__ void __launch_bounds__(256) bnr_dual(int m, int k, int pstride,
                                                const double* __restrict__ rl,
                                                const double* __restrict__ ru,
                                                const double* __restrict__ eta,
                                                const double* __restrict__ eta_prev,
                                                const double* __restrict__ omega,
                                                const int* __restrict__ pend,
                                                double* __restrict__ Y, double* __restrict__ AX,
                                                const double* __restrict__ AdX_prev,
                                                const double* __restrict__ AdX,
                                                double* __restrict__ dY,
                                                double* __restrict__ part) {
  const int node = blockIdx.y * 32 + threadIdx.x;
  double s0 = 0.0, s1 = 0.0;
  if (node < k) {
    const double sigma = eta[node] * omega[node];
    const bool taken = pend[node] != 0;
    const double sigma_prev = eta_prev[node] * omega[node];
    const int r0 = blockIdx.x * kRowsPerBlock, r1 = min(m, r0 + kRowsPerBlock);
    for (int r = r0 + threadIdx.y; r < r1; r += 8) {
      const long long g = (long long)r * k + node;
      const double lo = __ldg(rl + r), hi = __ldg(ru + r), adx = AdX[g];
      double y = Y[g], ax = AX[g];
      if (taken) {
        const double adx_prev = AdX_prev[g];
        y = dual_trial(y, ax, adx_prev, sigma_prev, lo, hi);
        ax = add(ax, adx_prev);
        Y[g] = y;
        AX[g] = ax;
      }
      const double d = sub(dual_trial(y, ax, adx, sigma, lo, hi), y);
      dY[g] = d;
      s0 = add(s0, mul(d, adx));
      s1 = add(s1, mul(d, d));
    }
  }
  bnr_block_sums(s0, s1, k, node, pstride, blockIdx.x, part);
}

// The sum over nb row blocks (from block b0) of slot c of a node's partials,
// by one warp: lane l adds blocks l, l + 32, ... in order from 0.0, then the
// 32 lane sums are added in lane order.  Every lane returns the total.
__device__ __forceinline__ double lanes_total(double s) {
  double a = __shfl_sync(0xffffffffu, s, 0);
  for (int l = 1; l < 32; ++l) a = add(a, __shfl_sync(0xffffffffu, s, l));
  return a;
}

__device__ __forceinline__ double warp_blocks_sum(const double* __restrict__ part, int pstride,
                                                  int node, int b0, int nb, int c, int lane) {
  const double* p = part + ((long long)node * pstride + b0) * 2 + c;
  double s = 0.0;
#pragma unroll 8
  for (int b = lane; b < nb; b += 32) s = add(s, p[2 * b]);
  return lanes_total(s);
}

// Per node (one warp each): the step-size test's sums over the row blocks,
// then the test and the next step size (bnr.py:244-270).  A taken trial sets
// accept[node] (the next step's pend); eta_prev keeps the step it used.  fac holds the iteration's (1 - t^-growth,
// 1 + t^-damp), computed on the host with the C library's pow, as the
// reference computes them.
__global__ void __launch_bounds__(128) bnr_accept(int k, int mblocks, int nblocks,
                                                  const double* __restrict__ part,
                                                  double* __restrict__ eta,
                                                  double* __restrict__ eta_prev,
                                                  const double* __restrict__ omega,
                                                  int* __restrict__ accept,
                                                  const double* __restrict__ fac) {
  const int lane = threadIdx.x & 31;
  const int node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (node >= k) return;            // whole warps leave together
  const int pstride = mblocks + nblocks + 1;
  // the three sums, each in warp_blocks_sum's order, in one loop so that the
  // loads of both sides are in flight together; their lane totals interleaved
  // as three independent chains
  const double* base = part + (long long)node * pstride * 2;
  const double2* pm = reinterpret_cast<const double2*>(base);
  const double* pn = base + 2 * (long long)mblocks;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  const int nmax = max(mblocks, nblocks);
#pragma unroll 4
  for (int b = lane; b < nmax; b += 32) {
    if (b < mblocks) {
      const double2 v = pm[b];
      s0 = add(s0, v.x);
      s1 = add(s1, v.y);
    }
    if (b < nblocks) s2 = add(s2, pn[2 * b]);
  }
  double dyadx = __shfl_sync(0xffffffffu, s0, 0), dydy = __shfl_sync(0xffffffffu, s1, 0),
         dxdx = __shfl_sync(0xffffffffu, s2, 0);
  for (int l = 1; l < 32; ++l) {
    dyadx = add(dyadx, __shfl_sync(0xffffffffu, s0, l));
    dydy = add(dydy, __shfl_sync(0xffffffffu, s1, l));
    dxdx = add(dxdx, __shfl_sync(0xffffffffu, s2, l));
  }
  if (lane != 0) return;
  const double om = omega[node];
  const double interaction = fabs(dyadx);
  const double movement = mul(0.5, add(mul(om, dxdx), dydy / om));
  const double floor_ = np_max(movement, 1.0) / kQuotientMax;
  const double limit = interaction > 0.0 ? movement / np_max(interaction, floor_) : INFINITY;
  const double e = eta[node];
  accept[node] = (e <= limit) || (movement == 0.0);
  eta_prev[node] = e;
  double en = np_min(mul(fac[0], limit), mul(fac[1], e));
  en = fmax(isfinite(en) ? en : 1.0, 1e-14);
  eta[node] = en;
}

// Each node's final iterates: for a node whose last trial was taken, that
// trial, redone as in bnr_primal / bnr_dual; otherwise X and Y as they are.
__global__ void bnr_resolve_x(long long total, int k, const int* __restrict__ pend,
                              const double* __restrict__ eta_prev,
                              const double* __restrict__ omega, const double* __restrict__ c,
                              const double* __restrict__ X, const double* __restrict__ AtY,
                              const double* __restrict__ L, const double* __restrict__ U,
                              double* __restrict__ out) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int node = (int)(g % k);
  double x = X[g];
  if (pend[node]) {
    const double tau = eta_prev[node] / omega[node];
    x = clipd(sub(x, mul(tau, add(c[g / k], AtY[g]))), L[g], U[g]);
  }
  out[g] = x;
}

__global__ void bnr_resolve_y(long long total, int k, const int* __restrict__ pend,
                              const double* __restrict__ eta_prev,
                              const double* __restrict__ omega, const double* __restrict__ rl,
                              const double* __restrict__ ru, const double* __restrict__ Y,
                              const double* __restrict__ AX, const double* __restrict__ AdX,
                              double* __restrict__ out) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= total) return;
  const int node = (int)(g % k);
  double y = Y[g];
  if (pend[node]) {
    const long long i = g / k;
    y = dual_trial(y, AX[g], AdX[g], eta_prev[node] * omega[node], rl[i], ru[i]);
  }
  out[g] = y;
}

// X = clip(X, L, U) (bnr.py:211)
__global__ void bnr_clip(long long total, double* __restrict__ X, const double* __restrict__ L,
                         const double* __restrict__ U) {
  const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < total) X[g] = clipd(X[g], L[g], U[g]);
}

// Safe dual bound terms (safebound.py:212-230), per-node partial sums and
// flags over blocks of rows: the m side from Y, the n side from d = c - A^T Y.
// The pair of (node, block), laid out as for the step sums, is (sum, flags):
// flag 1 = a vacuous term, flag 2 = an empty column box L > U + 1e-12
// (bnr.py:203).
__global__ void __launch_bounds__(256) bnr_bound_terms(
    int m, int n, int k, int mblocks, int pstride, const double* __restrict__ Y,
    const double* __restrict__ rl, const double* __restrict__ ru,
    const double* __restrict__ c, const double* __restrict__ aty,
    const double* __restrict__ L, const double* __restrict__ U, double* __restrict__ part) {
  __shared__ double sh[8][32];
  __shared__ int bad_sh[8][32];
  const bool mside = (int)blockIdx.x < mblocks;
  const int b = mside ? blockIdx.x : blockIdx.x - mblocks;
  const int rows = mside ? m : n;
  const int node = blockIdx.y * 32 + threadIdx.x;
  double s = 0.0;
  int bad = 0;
  if (node < k) {
    const int r0 = b * kRowsPerBlock, r1 = min(rows, r0 + kRowsPerBlock);
    for (int r = r0 + threadIdx.y; r < r1; r += 8) {
      const long long g = (long long)r * k + node;
      if (mside) {
        const double y = Y[g];
        const bool pos = y > 0.0;
        const bool rbad = (pos ? rl[r] <= -kBnrInf : ru[r] >= kBnrInf) && y != 0.0;
        const double pick = pos ? rl[r] : ru[r];
        s = add(s, rbad ? 0.0 : mul(y, pick));
        bad |= rbad;
      } else {
        const double d = sub(c[r], aty[g]);
        const bool pos = d > 0.0;
        const bool cbad = (pos ? L[g] <= -kBnrInf : U[g] >= kBnrInf) && d != 0.0;
        const double pick = pos ? L[g] : U[g];
        s = add(s, cbad ? 0.0 : mul(d, pick));
        bad |= cbad;
        if (L[g] > U[g] + 1e-12) bad |= 2;
      }
    }
  }
  sh[threadIdx.y][threadIdx.x] = s;
  bad_sh[threadIdx.y][threadIdx.x] = bad;
  __syncthreads();
  if (threadIdx.y == 0 && node < k) {
    double a = sh[0][threadIdx.x];
    int f = bad_sh[0][threadIdx.x];
    for (int yy = 1; yy < 8; ++yy) {
      a = add(a, sh[yy][threadIdx.x]);
      f |= bad_sh[yy][threadIdx.x];
    }
    double* out = part + ((long long)node * pstride + blockIdx.x) * 2;
    out[0] = a;
    out[1] = (double)f;
  }
}

// Per node: bound = (row sum + column sum + offset) / obj_scale, -inf when
// vacuous, +inf for an empty box; also the infeasible flag (bnr.py:203, 283-290).
__global__ void __launch_bounds__(128) bnr_bound_final(int k, int mblocks, int nblocks,
                                                       const double* __restrict__ part,
                                                       double obj_offset, double obj_scale,
                                                       double* __restrict__ bounds,
                                                       unsigned char* __restrict__ empty) {
  const int lane = threadIdx.x & 31;
  const int node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (node >= k) return;            // whole warps leave together
  const int pstride = mblocks + nblocks + 1;
  const double rs = warp_blocks_sum(part, pstride, node, 0, mblocks, 0, lane);
  const double cs = warp_blocks_sum(part, pstride, node, mblocks, nblocks, 0, lane);
  int flags = 0;
  for (int b = lane; b < mblocks + nblocks; b += 32)
    flags |= (int)part[((long long)node * pstride + b) * 2 + 1];
  flags = __reduce_or_sync(0xffffffffu, flags);
  if (lane != 0) return;
  const bool vac = flags & 1, emp = flags & 2;
  const double bound = vac ? -INFINITY : add(rs, cs);
  bounds[node] = emp ? INFINITY : (bound + obj_offset) / obj_scale;
  empty[node] = emp ? 1 : 0;
}

int blocks_for(long long total) { return (int)std::max(1LL, (total + 255) / 256); }

// Y (rows, k) = A X on stream s, two nodes per thread when k is even.
void launch_spmm(int rows, int k, const int64_t* rp, const int* ri, const double* rx,
                 const double* X, double* Y, cudaStream_t s) {
  if (k % 2 == 0)
    bnr_spmm<2><<<blocks_for((long long)rows * (k / 2)), 256, 0, s>>>(rows, k, rp, ri, rx, X, Y);
  else
    bnr_spmm<1><<<blocks_for((long long)rows * k), 256, 0, s>>>(rows, k, rp, ri, rx, X, Y);
}

}  // namespace
}  // namespace pdlp

using namespace pdlp;

struct pdlp_bnr {
  cudaStream_t stream = nullptr;
  int m = 0, n = 0;
  long long nnz = 0;
  double obj_scale = 1.0, obj_offset = 0.0;
  // shared problem (device)
  int64_t *rp = nullptr, *cp = nullptr;
  int *ri = nullptr, *ci = nullptr;
  double *rx = nullptr, *cx = nullptr, *c = nullptr, *rl = nullptr, *ru = nullptr;
  // per-node blocks, sized for cap nodes
  int cap = 0;
  // A dX in two buffers, alternating by iteration (a step redoes the
  // previous trial with the previous A dX)
  double *L = nullptr, *U = nullptr, *X = nullptr, *dX = nullptr, *AtY = nullptr,
         *AtdY = nullptr;
  double *Y = nullptr, *dY = nullptr, *AX = nullptr, *AdX0 = nullptr, *AdX1 = nullptr;
  double *eta = nullptr, *eta_prev = nullptr, *omega = nullptr, *part = nullptr,
         *bounds = nullptr;
  int* accept = nullptr;
  unsigned char* empty = nullptr;
  std::vector<double> h_eta, h_omega;   // persistent step sizes (bnr.py:168-171)
  // the captured iterations
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  double* fac = nullptr;          // per iteration (1 - t^-growth, 1 + t^-damp)
  int g_k = -1, g_iters = -1;
  long long g_launches = 0;
  double g_growth = 0.0, g_damp = 0.0;
};

namespace {

void bnr_free_blocks(pdlp_bnr* b) {
  double** ds[] = {&b->L, &b->U, &b->X, &b->dX, &b->AtY, &b->AtdY, &b->Y, &b->dY, &b->AX,
                   &b->AdX0, &b->AdX1, &b->eta, &b->eta_prev, &b->omega, &b->part, &b->bounds};
  for (double** d : ds) { cudaFree(*d); *d = nullptr; }
  cudaFree(b->accept); b->accept = nullptr;
  cudaFree(b->empty); b->empty = nullptr;
  if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
}

// Capacity for K nodes (the reference doubles its buffers: bnr.py:166-171).
int bnr_ensure(pdlp_bnr* b, int K) {
  if (K <= b->cap) return PDLP_OK;
  const int cap = std::max(K, b->cap * 2);
  PDLP_CUDA(cudaStreamSynchronize(b->stream));
  bnr_free_blocks(b);
  const size_t nk = (size_t)b->n * cap, mk = (size_t)b->m * cap;
  const int mblocks = (b->m + kRowsPerBlock - 1) / kRowsPerBlock;
  const int nblocks = (b->n + kRowsPerBlock - 1) / kRowsPerBlock;
  struct { double** p; size_t n; } want[] = {
      {&b->L, nk}, {&b->U, nk}, {&b->X, nk}, {&b->dX, nk}, {&b->AtY, nk}, {&b->AtdY, nk},
      {&b->Y, mk}, {&b->dY, mk}, {&b->AX, mk}, {&b->AdX0, mk}, {&b->AdX1, mk},
      {&b->eta, (size_t)cap}, {&b->eta_prev, (size_t)cap}, {&b->omega, (size_t)cap},
      {&b->part, (size_t)(mblocks + nblocks + 1) * cap * 2}, {&b->bounds, (size_t)cap}};
  for (auto& w : want) {
    const cudaError_t e = cudaMalloc(w.p, sizeof(double) * std::max<size_t>(w.n, 1));
    if (e != cudaSuccess) { bnr_free_blocks(b); b->cap = 0; return fail(PDLP_ERR_OOM, "bnr: cudaMalloc"); }
  }
  if (cudaMalloc(&b->accept, sizeof(int) * cap) != cudaSuccess ||
      cudaMalloc(&b->empty, (size_t)cap) != cudaSuccess) {
    bnr_free_blocks(b);
    b->cap = 0;
    return fail(PDLP_ERR_OOM, "bnr: cudaMalloc");
  }
  // growing restarts every node's step sizes at 1, as the reference's
  // buffer growth does (bnr.py:149-171); otherwise they persist across calls
  b->h_eta.assign(cap, 1.0);
  b->h_omega.assign(cap, 1.0);
  b->cap = cap;
  return PDLP_OK;
}

template <typename T>
int bnr_upload(T** dst, const T* src, size_t count, int memory, cudaStream_t st) {
  PDLP_CUDA(cudaMalloc(dst, sizeof(T) * std::max<size_t>(count, 1)));
  if (count == 0) return PDLP_OK;
  if (!src) return fail(PDLP_ERR_ARG, "bnr: a required array is NULL");
  PDLP_CUDA(cudaMemcpyAsync(*dst, src, sizeof(T) * count,
                            memory == PDLP_MEM_HOST ? cudaMemcpyHostToDevice
                                                    : cudaMemcpyDeviceToDevice, st));
  return PDLP_OK;
}

// The launches of `iters` iterations for K nodes, on stream s; returns how
// many kernels it launched.
long long bnr_enqueue_iterations(pdlp_bnr* b, int K, int iters, cudaStream_t s) {
  const int mblocks = (b->m + kRowsPerBlock - 1) / kRowsPerBlock;
  const int nblocks = (b->n + kRowsPerBlock - 1) / kRowsPerBlock;
  const dim3 tb(32, 8);
  const dim3 ngrid(std::max(1, nblocks), (K + 31) / 32), mgrid(std::max(1, mblocks), (K + 31) / 32);
  long long launches = 0;
  for (int it = 0; it < iters; ++it) {
    double* adx = (it & 1) ? b->AdX1 : b->AdX0;        // this step's A dX
    double* adx_prev = (it & 1) ? b->AdX0 : b->AdX1;   // the previous step's
    // an empty side has no rows to step and no sums to write
    if (nblocks > 0)
      bnr_primal<<<ngrid, tb, 0, s>>>(b->n, K, mblocks, mblocks + nblocks + 1, b->c, b->eta,
                                      b->eta_prev, b->omega, b->accept, b->X, b->AtY, b->AtdY,
                                      b->L, b->U, b->dX, b->part);
    launch_spmm(b->m, K, b->rp, b->ri, b->rx, b->dX, adx, s);
    if (mblocks > 0)
      bnr_dual<<<mgrid, tb, 0, s>>>(b->m, K, mblocks + nblocks + 1, b->rl, b->ru, b->eta,
                                    b->eta_prev, b->omega, b->accept, b->Y, b->AX, adx_prev, adx,
                                    b->dY, b->part);
    launch_spmm(b->n, K, b->cp, b->ci, b->cx, b->dY, b->AtdY, s);
    bnr_accept<<<(K + 3) / 4, 128, 0, s>>>(K, mblocks, nblocks, b->part, b->eta, b->eta_prev,
                                           b->omega, b->accept, b->fac + 2 * it);
    launches += 3 + (nblocks > 0) + (mblocks > 0);
  }
  return launches;
}

}  // namespace

extern "C" {

int pdlp_bnr_create(const pdlp_problem_desc* P, double obj_scale, int32_t max_batch,
                    void* stream, pdlp_bnr** out) {
  if (!P || !out) return fail(PDLP_ERR_ARG, "NULL problem or output");
  *out = nullptr;
  if (P->m < 0 || P->n < 0 || P->nnz < 0) return fail(PDLP_ERR_ARG, "negative dimension");
  if (P->nnz > 0x7fffffffLL) return fail(PDLP_ERR_ARG, "nnz must fit in int32");
  if (P->memory != PDLP_MEM_HOST && P->memory != PDLP_MEM_DEVICE)
    return fail(PDLP_ERR_ARG, "memory must be PDLP_MEM_HOST or PDLP_MEM_DEVICE");
  if (!(obj_scale > 0.0) || !std::isfinite(obj_scale)) return fail(PDLP_ERR_ARG, "obj_scale must be positive");
  pdlp_bnr* b = new pdlp_bnr();
  b->stream = (cudaStream_t)stream;
  b->m = P->m; b->n = P->n; b->nnz = P->nnz;
  b->obj_scale = obj_scale;
  b->obj_offset = P->obj_offset;
  cudaStream_t st = b->stream;
  int rc = PDLP_OK;
  const int mem = P->memory;
  if ((rc = bnr_upload(&b->rp, P->rp, (size_t)P->m + 1, mem, st)) ||
      (rc = bnr_upload(&b->ri, P->ri, (size_t)P->nnz, mem, st)) ||
      (rc = bnr_upload(&b->rx, P->rx, (size_t)P->nnz, mem, st)) ||
      (rc = bnr_upload(&b->cp, P->cp, (size_t)P->n + 1, mem, st)) ||
      (rc = bnr_upload(&b->ci, P->ci, (size_t)P->nnz, mem, st)) ||
      (rc = bnr_upload(&b->cx, P->cx, (size_t)P->nnz, mem, st)) ||
      (rc = bnr_upload(&b->c, P->c, (size_t)P->n, mem, st)) ||
      (rc = bnr_upload(&b->rl, P->row_lb, (size_t)P->m, mem, st)) ||
      (rc = bnr_upload(&b->ru, P->row_ub, (size_t)P->m, mem, st)) ||
      (rc = bnr_ensure(b, std::max(1, (int)max_batch)))) {
    pdlp_bnr_destroy(b);
    return rc;
  }
  cudaError_t e = cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) { pdlp_bnr_destroy(b); return cuda_fail(e, "bnr create"); }
  *out = b;
  return PDLP_OK;
}

int pdlp_bnr_destroy(pdlp_bnr* b) {
  if (!b) return PDLP_OK;
  cudaStreamSynchronize(b->stream);
  bnr_free_blocks(b);
  void* arrays[] = {b->rp, b->ri, b->rx, b->cp, b->ci, b->cx, b->c, b->rl, b->ru};
  for (void* a : arrays) cudaFree(a);
  cudaFree(b->fac);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  delete b;
  return PDLP_OK;
}

int pdlp_bnr_solve_batch(pdlp_bnr* b, int32_t K, const double* col_lb, const double* col_ub,
                         const double* warm_x, const double* warm_y, int32_t iters,
                         double step_growth, double step_damp, double* bounds, double* x,
                         double* y, uint8_t* infeasible, int32_t memory) {
  if (!b) return fail(PDLP_ERR_ARG, "NULL handle");
  if (K <= 0 || iters < 0) return fail(PDLP_ERR_ARG, "K must be positive and iters >= 0");
  if (!col_lb || !col_ub) return fail(PDLP_ERR_ARG, "col_lb / col_ub are NULL");
  if (memory != PDLP_MEM_HOST && memory != PDLP_MEM_DEVICE)
    return fail(PDLP_ERR_ARG, "memory must be PDLP_MEM_HOST or PDLP_MEM_DEVICE");
  if ((warm_x == nullptr) != (warm_y == nullptr)) return fail(PDLP_ERR_ARG, "warm_x and warm_y go together");
  int rc = bnr_ensure(b, K);
  if (rc) return rc;
  cudaStream_t st = b->stream;
  const cudaMemcpyKind in = memory == PDLP_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  const cudaMemcpyKind outk = memory == PDLP_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const size_t nk = (size_t)b->n * K, mk = (size_t)b->m * K;
  if (nk) {
    PDLP_CUDA(cudaMemcpyAsync(b->L, col_lb, sizeof(double) * nk, in, st));
    PDLP_CUDA(cudaMemcpyAsync(b->U, col_ub, sizeof(double) * nk, in, st));
  }
  if (warm_x) {
    if (nk) PDLP_CUDA(cudaMemcpyAsync(b->X, warm_x, sizeof(double) * nk, in, st));
    if (mk) PDLP_CUDA(cudaMemcpyAsync(b->Y, warm_y, sizeof(double) * mk, in, st));
  } else {
    if (nk) PDLP_CUDA(cudaMemsetAsync(b->X, 0, sizeof(double) * nk, st));
    if (mk) PDLP_CUDA(cudaMemsetAsync(b->Y, 0, sizeof(double) * mk, st));
  }
  // no trial pending at the start
  PDLP_CUDA(cudaMemsetAsync(b->accept, 0, sizeof(int) * K, st));
  PDLP_CUDA(cudaMemcpyAsync(b->eta, b->h_eta.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  PDLP_CUDA(cudaMemcpyAsync(b->omega, b->h_omega.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  PDLP_CUDA(cudaMemcpyAsync(b->eta_prev, b->h_eta.data(), sizeof(double) * K, cudaMemcpyHostToDevice, st));
  // X = clip(X, L, U); AX = A X; AtY = A^T Y
  bnr_clip<<<blocks_for((long long)nk), 256, 0, st>>>((long long)nk, b->X, b->L, b->U);
  launch_spmm(b->m, K, b->rp, b->ri, b->rx, b->X, b->AX, st);
  launch_spmm(b->n, K, b->cp, b->ci, b->cx, b->Y, b->AtY, st);
  count_launches(3);
  PDLP_CUDA(cudaGetLastError());
  // the iterations, from a graph captured once per (K, iters, exponents)
  if (iters > 0) {
    if (!b->graph || b->g_k != K || b->g_iters != iters || b->g_growth != step_growth ||
        b->g_damp != step_damp) {
      if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
      // the step-size factors of iteration i use t = i + 2 (attempts + 1,
      // bnr.py:267), with the host's pow as in the reference
      std::vector<double> fac(2 * (size_t)iters);
      for (int it = 0; it < iters; ++it) {
        const double t = (double)(it + 2);
        fac[2 * it] = 1.0 - std::pow(t, -step_growth);
        fac[2 * it + 1] = 1.0 + std::pow(t, -step_damp);
      }
      PDLP_CUDA(cudaStreamSynchronize(st));
      cudaFree(b->fac);
      b->fac = nullptr;
      PDLP_CUDA(cudaMalloc(&b->fac, sizeof(double) * fac.size()));
      PDLP_CUDA(cudaMemcpy(b->fac, fac.data(), sizeof(double) * fac.size(), cudaMemcpyHostToDevice));
      PDLP_CUDA(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
      b->g_launches = bnr_enqueue_iterations(b, K, iters, b->cap_stream);
      cudaGraph_t g = nullptr;
      const cudaError_t le = cudaGetLastError();
      const cudaError_t ce = cudaStreamEndCapture(b->cap_stream, &g);
      if (le != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(le, "bnr capture"); }
      if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture");
      const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) { b->graph = nullptr; return cuda_fail(ie, "cudaGraphInstantiate"); }
      b->g_k = K; b->g_iters = iters; b->g_growth = step_growth; b->g_damp = step_damp;
    }
    PDLP_CUDA(cudaGraphLaunch(b->graph, st));
    count_launches(b->g_launches);
  }
  // each node's final iterates, into dX (x) and dY (y); the last step's
  // A dX is in AdX[(iters - 1) % 2]
  bnr_resolve_x<<<blocks_for((long long)nk), 256, 0, st>>>(
      (long long)nk, K, b->accept, b->eta_prev, b->omega, b->c, b->X, b->AtY, b->L, b->U, b->dX);
  bnr_resolve_y<<<blocks_for((long long)mk), 256, 0, st>>>(
      (long long)mk, K, b->accept, b->eta_prev, b->omega, b->rl, b->ru, b->Y, b->AX,
      ((iters - 1) & 1) ? b->AdX1 : b->AdX0, b->dY);
  // the bound: A^T Y, its terms, then per node (safebound.py:194-235)
  const int mblocks = (b->m + kRowsPerBlock - 1) / kRowsPerBlock;
  const int nblocks = (b->n + kRowsPerBlock - 1) / kRowsPerBlock;
  launch_spmm(b->n, K, b->cp, b->ci, b->cx, b->dY, b->AtdY, st);
  bnr_bound_terms<<<dim3(std::max(1, mblocks + nblocks), (K + 31) / 32), dim3(32, 8), 0, st>>>(
      b->m, b->n, K, mblocks, mblocks + nblocks + 1, b->dY, b->rl, b->ru, b->c, b->AtdY, b->L,
      b->U, b->part);
  bnr_bound_final<<<(K + 3) / 4, 128, 0, st>>>(K, mblocks, nblocks, b->part, b->obj_offset,
                                               b->obj_scale, b->bounds, b->empty);
  count_launches(5);
  PDLP_CUDA(cudaGetLastError());
  // outputs; the step sizes stay with the engine for the next call
  if (bounds) PDLP_CUDA(cudaMemcpyAsync(bounds, b->bounds, sizeof(double) * K, outk, st));
  if (x && nk) PDLP_CUDA(cudaMemcpyAsync(x, b->dX, sizeof(double) * nk, outk, st));
  if (y && mk) PDLP_CUDA(cudaMemcpyAsync(y, b->dY, sizeof(double) * mk, outk, st));
  if (infeasible) PDLP_CUDA(cudaMemcpyAsync(infeasible, b->empty, (size_t)K, outk, st));
  PDLP_CUDA(cudaMemcpyAsync(b->h_eta.data(), b->eta, sizeof(double) * K, cudaMemcpyDeviceToHost, st));
  PDLP_CUDA(cudaStreamSynchronize(st));
  return PDLP_OK;
}

int pdlp_bnr_step_sizes(pdlp_bnr* b, int32_t K, double* eta, double* omega) {
  if (!b || K < 0) return fail(PDLP_ERR_ARG, "NULL handle or negative K");
  if (K > b->cap) return fail(PDLP_ERR_ARG, "K beyond the engine's capacity");
  for (int i = 0; i < K; ++i) {
    if (eta) eta[i] = b->h_eta[i];
    if (omega) omega[i] = b->h_omega[i];
  }
  return PDLP_OK;
}

}  // extern "C"
