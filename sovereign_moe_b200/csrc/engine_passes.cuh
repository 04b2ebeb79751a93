// The A pass (row tiles) and the A^T pass (column tiles) of one engine step,
// and the finishers that advance each LP's state machine.
//
// Reference for every formula: src/sovopt/lp/pdlp.py (loop 313-463, KKT
// 162-230, unscaled KKT 497-530), src/sovopt/core/backend.py (the step kernels
// 204-291), src/sovopt/numerics/scaling.py (Ruiz 149-170, Pock-Chambolle
// 274-295, pdlp 298-309, pow2 119-131, scale_problem 374-478).
#pragma once

#include "engine_device.cuh"

namespace pdlp {

// ---- state-machine helpers (run by one thread of a finisher) ----------------

__device__ __forceinline__ int plan_primal(const Inst& I, long long k) {
  // primal half-step to compute for iteration k right after iteration k-1
  if (k % I.check_every == 0) return P_NONE;        // a check comes first
  if (k >= I.max_iter) return P_NONE;
  return (k % I.stepsize_every == 0) ? P_TRIAL : P_NORMAL;
}

__device__ __forceinline__ void schedule_final(State* S, int status, int src) {
  S->final_src = src;
  S->final_status = status;    // published when C_FINAL completes
  S->rmode = R_FINAL;
  S->cmode = C_NONE;           // the R_FINAL finisher schedules C_FINAL
}

// Top of iteration k of the reference loop (pdlp.py:313-317), reached after a
// check (with or without a restart) or after the set-up.
__device__ void begin_iteration(const Inst& I, State* S, bool restart) {
  const long long k = S->k;
  const int src = restart ? S->restart_src : 0;
  if (k >= I.max_iter) { schedule_final(S, PDLP_STATUS_ITERATION_LIMIT, src); return; }
  if (k % I.check_every == 0) {
    if ((double)(global_ns() - S->t_start_ns) + I.time_used_ns > I.time_limit_ns) {
      schedule_final(S, PDLP_STATUS_TIME_LIMIT, src);
      return;
    }
    // a host request to stop: 1 = cancelled (INTERRUPTED), 100 + s = end with status s
    const int req = *(volatile int*)&S->cancel;
    if (req) { schedule_final(S, req >= 100 ? req - 100 : PDLP_STATUS_INTERRUPTED, src); return; }
  }
  const int kind = (k % I.stepsize_every == 0) ? P_TRIAL : P_NORMAL;
  S->cprimal = kind;
  if (restart) { S->rmode = R_RESTART; S->cmode = C_RESTART; }
  else { S->rmode = R_NONE; S->cmode = C_PRIMAL; }
}

__device__ __forceinline__ double merit(double omega, double p, double d, double g) {
  return sqrt((omega * p) * (omega * p) + (d / omega) * (d / omega) + g * g);
}

// ---- finisher protocol ------------------------------------------------------
//
// Two-level, fixed-order reduction of an instance's tile partials: the warp
// that completes the last tile of a group (64 consecutive tiles of the
// instance) sums the group's tile partials in tile order; the warp that
// completes the instance's last group sums the group partials in group order
// and advances the state machine.  Returns true in that warp, with the
// instance's reduced values in res (every lane).  A warp that goes on with
// another tile of the same group only counts this one (ph.pend) and returns
// false; its atomic, when it leaves the group, counts them all and releases
// their partials together (every partial is written by lane 0, the lane that
// issues the atomic).  Which warp completes a group changes nothing in the
// sums, whose order is the tile order.  A pass with nothing to reduce (a
// normal iteration's A^T pass only advances the state machine) skips the
// group level: warps count their tiles straight into the instance's counter
// (n_tiles on this side), which takes one atomic round trip off the pass's
// last warp.  Every tile of an instance in one pass has the same mode, so a
// pass uses the counter one way only.
__device__ __forceinline__ bool warp_finish(const EngineArgs& A, const Tile& t, int side,
                                            int g_first, int g_last, int n_tiles, bool need_red,
                                            Ops ops, double* res, int lane, BulkPhase& ph) {
  ph.pend += 1;
  if (!ph.flush) return false;
  const unsigned done = ph.pend;
  ph.pend = 0;
  if (!need_red) {
    unsigned fin = 0;
    __syncwarp();
    if (lane == 0)
      fin = atom_add_acq_rel(A.counters + 2 * t.inst + side, done) + done == (unsigned)n_tiles;
    fin = __shfl_sync(kFull, fin, 0);
    if (!fin) return false;
    if (lane == 0) A.counters[2 * t.inst + side] = 0;
    __syncwarp();
    return true;
  }
  const int g = t.group;
  const int2 gt = A.group_tiles[g];
  const double* tp = A.partials + (side ? (size_t)A.n_rtiles * kNP : 0);
  unsigned last = 0;
  __syncwarp();
  if (lane == 0)   // release these tiles' partials; acquire the group's if last
    last = atom_add_acq_rel(A.gcounters + g, done) + done == (unsigned)(gt.y - gt.x);
  last = __shfl_sync(kFull, last, 0);
  if (!last) return false;
  __syncwarp();                            // order the lanes' reads after lane 0's acquire
  double v[kNP];
  if (need_red) {
#pragma unroll
    for (int s = 0; s < kNP; ++s) v[s] = identity_of(ops.op(s));
    for (int tt = gt.x + lane; tt < gt.y; tt += 32) {
#pragma unroll
      for (int s = 0; s < kNP; ++s) v[s] = combine(v[s], ld_mut(tp + (size_t)tt * kNP + s), ops.op(s));
    }
    warp_reduce(v, ops);
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < kNP; ++s) A.gpartials[(size_t)g * kNP + s] = v[s];
    }
  }
  __syncwarp();
  if (lane == 0) {
    A.gcounters[g] = 0;
    last = atom_add_acq_rel(A.counters + 2 * t.inst + side, 1u) == (unsigned)(g_last - g_first - 1);
  }
  last = __shfl_sync(kFull, last, 0);
  if (!last) return false;
  __syncwarp();
  if (need_red) {
#pragma unroll
    for (int s = 0; s < kNP; ++s) v[s] = identity_of(ops.op(s));
    for (int gg = g_first + lane; gg < g_last; gg += 32) {
#pragma unroll
      for (int s = 0; s < kNP; ++s) v[s] = combine(v[s], ld_mut(A.gpartials + (size_t)gg * kNP + s), ops.op(s));
    }
    warp_reduce(v, ops);
#pragma unroll
    for (int s = 0; s < kNP; ++s) res[s] = v[s];
  }
  if (lane == 0) A.counters[2 * t.inst + side] = 0;
  return true;
}

// Copy the tile's instance descriptor into the warp's shared memory (once per
// run of tiles of the same instance).
__device__ __forceinline__ const Inst& warp_inst(const EngineArgs& A, int inst, WarpSmem& W,
                                                 int lane) {
  if (W.inst_id != inst) {
    const int* src = reinterpret_cast<const int*>(A.inst + inst);
    int* dst = reinterpret_cast<int*>(&W.inst);
    for (int i = lane; i < (int)(sizeof(Inst) / sizeof(int)); i += 32) dst[i] = src[i];
    __syncwarp();
    if (lane == 0) W.inst_id = inst;
    __syncwarp();
  }
  return W.inst;
}

// The scheduling fields of one LP's state as one warp saw them in the current
// pass.  They cannot change while a tile of that LP is still unprocessed in
// the pass: only the LP's finisher writes them, and it runs after the LP's
// last tile of the pass has completed.  So a warp reads them once per LP per
// pass instead of once per tile (a cache is declared per pass and starts
// empty).
struct PassCache {
  int inst = -1;
  int mode = 0, aux = 0, commit = 0;
  double eta = 0.0, omega = 0.0;
  __device__ void load_r(const State* S, int id) {
    inst = id;
    mode = ld_mut(&S->rmode);
    commit = ld_mut(&S->ycommit);
    eta = ld_mut(&S->eta);
    omega = ld_mut(&S->omega);
  }
  __device__ void load_c(const State* S, int id) {
    inst = id;
    mode = ld_mut(&S->cmode);
    aux = ld_mut(&S->cprimal);
    commit = ld_mut(&S->xcommit);
    eta = ld_mut(&S->eta);
    omega = ld_mut(&S->omega);
  }
};

// ---- A pass ---------------------------------------------------------------

__device__ void r_finish(const EngineArgs& A, const Inst& I, State* S, int rmode, const double* red) {
  if (S->t_start_ns == 0) S->t_start_ns = global_ns();   // first pass of this LP
  S->ycommit = 0;               // every non-idle R pass applies a pending commit
  switch (rmode) {
    case R_RUIZ: S->ruiz_dev_r = red[0]; break;
    case R_APPLY: S->rhs_orig = red[0]; S->bn2 = red[1]; break;
    case R_POWER: if (S->power_round == 1) S->p0 = red[0]; break;
    case R_TRIAL: {
      // adaptive step (pdlp.py:340-381)
      S->attempts += 1;
      S->trials += 1;
      const double eta = S->eta, omega = S->omega;
      const double interaction = fabs(red[0]);
      const double movement = 0.5 * (omega * S->dxdx + red[1] / omega);
      bool accepted = false;
      double eta_new = eta;
      if (movement == 0.0) {
        accepted = true;
      } else {
        const double eta_limit = interaction > 0.0 ? movement / interaction : INFINITY;
        const double t = (double)(S->attempts + 1);
        const double eta_next = fmax(fmin((1.0 - pow(t, -0.3)) * eta_limit,
                                          (1.0 + pow(t, -0.6)) * eta), 1e-14);
        if (eta <= eta_limit) accepted = true;
        else S->rejected += 1;
        eta_new = eta_next;
      }
      S->eta = eta_new;
      if (accepted) {
        S->trials = 0;
        S->ycommit = 1;
        S->xcommit = 1;
        S->cprimal = plan_primal(I, S->k + 1);
        S->cmode = C_ITER;
      } else if (S->trials >= kMaxLineSearch) {
        S->cmode = C_NONE;
        schedule_final(S, PDLP_STATUS_NUMERICAL, 0);
      } else {
        S->cprimal = P_TRIAL;
        S->cmode = C_PRIMAL;
      }
      break;
    }
    case R_CHECK_A: for (int s = 0; s < 5; ++s) S->ra[s] = red[s]; break;
    case R_CHECK_B: for (int s = 0; s < 3; ++s) S->rb[s] = red[s]; break;
    case R_FINAL: S->cmode = C_FINAL; break;
    default: break;
  }
}

__device__ void c_finish(const EngineArgs& A, const Inst& I, State* S, int cmode, const double* red);

// ---- hot modes: staged tile passes ------------------------------------------
//
// The iteration (R_ITER, C_ITER), line-search trial (R_TRIAL) and primal step
// (C_PRIMAL) passes run from shared memory.  The caller has issued the bulk
// copies of the tile's matrix arrays; here one lane issues those of the
// epilogue vectors, which land while the gathers are in flight, so a pass
// waits for about two global round trips.  The arithmetic is exactly the
// generic passes' (same operands, same order).

// Bounds-checked builds (-DPDLP_BOUNDS_CHECK) test every gathered index
// against the source vector's length and every staged row pointer against the
// tile: a failure records PDLP_ERR_BOUNDS (the launch ends at its next grid
// barrier) and the access is skipped.  Product builds compile none of it.
#ifdef PDLP_BOUNDS_CHECK
__device__ __forceinline__ bool index_ok(const EngineArgs& A, int i, int n, int where) {
  if ((unsigned)i < (unsigned)n) return true;
  if (atomicCAS(&A.ctl->error, 0, PDLP_ERR_BOUNDS) == 0) A.ctl->error_where = where;
  return false;
}
// The staged row pointers of a normal tile: start at the tile's first entry,
// never decrease, and end at its last.
__device__ __forceinline__ bool tile_ptrs_ok(const EngineArgs& A, const Tile& t, const int* tptr,
                                             int lane) {
  const int rows = t.end - t.begin;
  bool ok = true;
  for (int i = lane; i < rows; i += 32) ok &= tptr[i] <= tptr[i + 1];
  if (lane == 0) ok &= tptr[0] == t.p0 && tptr[rows] == t.p0 + t.cnt;
  ok = __all_sync(0xffffffffu, ok);
  if (!ok && lane == 0 && atomicCAS(&A.ctl->error, 0, PDLP_ERR_BOUNDS) == 0)
    A.ctl->error_where = t.begin;
  return ok;
}
#else
__device__ __forceinline__ bool index_ok(const EngineArgs&, int, int, int) { return true; }
__device__ __forceinline__ bool tile_ptrs_ok(const EngineArgs&, const Tile&, const int*, int) {
  return true;
}
#endif

__device__ __forceinline__ void gather_products(const EngineArgs& A, const Tile& t,
                                                const double* src, int len, WarpSmem& W,
                                                int offi, int offv, int lane) {
  double* prod = W.sval + offv;
  const int* idx = W.sidx + offi;
  const int cnt = t.cnt;
  double g[kWTileNnz / 32];
#pragma unroll
  for (int u = 0; u < kWTileNnz / 32; ++u) {
    const int q = lane + 32 * u;
    g[u] = (q < cnt && index_ok(A, idx[q], len, t.begin)) ? ld_gather(src + idx[q]) : 0.0;
  }
#pragma unroll
  for (int u = 0; u < kWTileNnz / 32; ++u) {
    const int q = lane + 32 * u;
    if (q < cnt) prod[q] *= g[u];
  }
  __syncwarp();
}

__device__ __forceinline__ void gather_products_f32(const EngineArgs& A, const Tile& t,
                                                    const float* src, int len, WarpSmem& W,
                                                    int offi, int offv, int lane) {
  float* prod = reinterpret_cast<float*>(W.sval) + offv;
  const int* idx = W.sidx + offi;
  const int cnt = t.cnt;
  float g[kWTileNnz / 32];
#pragma unroll
  for (int u = 0; u < kWTileNnz / 32; ++u) {
    const int q = lane + 32 * u;
    g[u] = (q < cnt && index_ok(A, idx[q], len, t.begin)) ? ld_gather(src + idx[q]) : 0.0f;
  }
#pragma unroll
  for (int u = 0; u < kWTileNnz / 32; ++u) {
    const int q = lane + 32 * u;
    if (q < cnt) prod[q] *= g[u];
  }
  __syncwarp();
}

// Waits for the current phase of one of the warp's copy barriers, then
// advances the phase bit.  Bounded: after barrier_timeout_ns of wall time it
// records PDLP_ERR_BARRIER_TIMEOUT (the launch then ends at its next grid
// barrier) and returns false, and the caller skips the tile's work.
__device__ bool bulk_wait(const EngineArgs& A, unsigned long long* bar, unsigned& parity) {
  bool ok = mbar_try_wait(bar, parity);
  if (!ok) {
    const long long t0 = global_ns();
    for (unsigned spins = 1; !ok; ++spins) {
      ok = mbar_try_wait(bar, parity);
      if (!ok && (spins & 63u) == 0u && global_ns() - t0 > A.barrier_timeout_ns) {
        atomicCAS(&A.ctl->error, 0, PDLP_ERR_BARRIER_TIMEOUT);
        break;
      }
    }
  }
  parity ^= 1u;
  return ok;
}

__device__ void hot_rtile(const EngineArgs& A, const Tile& t, int ti, const Inst& I, State* S,
                          WarpSmem& W, int lane, int rmode, bool commit, double eta,
                          double omega, int offp, int offi, int offv, BulkPhase& ph) {
#ifdef PDLP_TRACE
  // stage timestamps of the first warp of block 0 (slots after the step trace)
  // counter in trace[1279], records at trace[640 + 8 k], k < 63
  long long* tq = (A.trace && blockIdx.x == 0 && threadIdx.x == 0) ? A.trace + 640 : nullptr;
  long long tk = 0;
  if (tq) { tk = A.trace[1279]; if (tk < 0 || tk >= 63) tq = nullptr; else tq += tk * 8; }
#define HOT_STAMP(k) if (tq) tq[k] = global_ns()
#else
#define HOT_STAMP(k)
#endif
  HOT_STAMP(0);
  const int rows = t.end - t.begin;
  const double sigma = eta * omega;
  // vectors: 0 ax, 1 y, 2 rl, 3 ru, 4 sum_y, 5 y_new, 6 adx
  const bool with_sum = rmode == R_ITER || commit;
  if (lane == 0) {
    const unsigned b = bulk_bytes<8>(t.begin, rows);
    mbar_arrive_tx(&W.bar[1], b * (4u + (with_sum ? 1u : 0u) + (commit ? 2u : 0u)));
    bulk_stage<8>(W.vec[0], I.ax, t.begin, rows, &W.bar[1]);
    bulk_stage<8>(W.vec[1], I.y, t.begin, rows, &W.bar[1]);
    bulk_stage<8>(W.vec[2], I.rl, t.begin, rows, &W.bar[1]);
    bulk_stage<8>(W.vec[3], I.ru, t.begin, rows, &W.bar[1]);
    if (with_sum) bulk_stage<8>(W.vec[4], I.sumy, t.begin, rows, &W.bar[1]);
    if (commit) {
      bulk_stage<8>(W.vec[5], I.ynew, t.begin, rows, &W.bar[1]);
      bulk_stage<8>(W.vec[6], I.adx, t.begin, rows, &W.bar[1]);
    }
  }
  const int off = bulk_offset<8>(t.begin);
  HOT_STAMP(1);
  if (!bulk_wait(A, &W.bar[0], ph.m)) { bulk_wait(A, &W.bar[1], ph.v); return; }
  if (!tile_ptrs_ok(A, t, W.sptr + offp, lane)) { bulk_wait(A, &W.bar[1], ph.v); return; }
  HOT_STAMP(2);
  if (I.f32) {
    gather_products_f32(A, t, I.dx32, I.n, W, offi, offv, lane);
    HOT_STAMP(3);
    staged_row_sums_f32(W.sptr + offp, reinterpret_cast<const float*>(W.sval) + offv, rows,
                        I.lanes_r, W.s0, lane);
  } else {
    gather_products(A, t, I.dx, I.n, W, offi, offv, lane);
    HOT_STAMP(3);
    staged_row_sums(W.sptr + offp, W.sval + offv, rows, I.lanes_r, W.s0, lane);
  }
  HOT_STAMP(4);
  if (!bulk_wait(A, &W.bar[1], ph.v)) return;
  HOT_STAMP(5);
  double acc[kNP];
#pragma unroll
  for (int s = 0; s < kNP; ++s) acc[s] = 0.0;
  for (int li = lane; li < rows; li += 32) {
    const int r = t.begin + li;
    const int v = off + li;
    double ax = W.vec[0][v], y = W.vec[1][v], sumy = W.vec[4][v];
    const double rl = W.vec[2][v], ru = W.vec[3][v];
    if (commit) {                     // pdlp.py:385-389
      const double yn = W.vec[5][v];
      y = yn;
      ax = ax + W.vec[6][v];
      sumy = sumy + eta * yn;
      I.y[r] = y;
      I.ax[r] = ax;
      I.sumy[r] = sumy;
    }
    const double a = W.s0[li];
    if (rmode == R_ITER) {            // backend.py:260-279
      const double axn = ax + a;
      I.ax[r] = axn;
      const double w = y + sigma * (axn + a);
      const double yn = prox(w, sigma, rl, ru);
      I.dy[r] = yn - y;
      if (I.f32) I.dy32[r] = (float)(yn - y);
      I.y[r] = yn;
      I.sumy[r] = sumy + eta * yn;
    } else {                          // pdlp.py:347-356
      I.adx[r] = a;
      const double axb = ax + 2.0 * a;
      const double w = y + sigma * axb;
      const double yn = prox(w, sigma, rl, ru);
      I.ynew[r] = yn;
      const double d = yn - y;
      I.dy[r] = d;
      if (I.f32) I.dy32[r] = (float)d;
      acc[0] += d * a;
      acc[1] += d * d;
    }
  }
  HOT_STAMP(6);
#ifdef PDLP_TRACE
  if (tq) A.trace[1279] = tk + 1;
#endif
#undef HOT_STAMP
  const bool need_red = rmode == R_TRIAL;
  const bool need_fin = need_red || commit;
  Ops ops;
  if (need_red) {
    warp_reduce(acc, ops);
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < kNP; ++s) A.partials[(size_t)ti * kNP + s] = acc[s];
    }
  }
  if (!need_fin) return;
  double res[kNP];
  if (warp_finish(A, t, 0, I.rg_begin, I.rg_end, I.rt_end - I.rt_begin, need_red, ops, res,
                  lane, ph)) {
    if (lane == 0) r_finish(A, I, S, rmode, res);
    __syncwarp();
  }
}

__device__ void hot_ctile(const EngineArgs& A, const Tile& t, int ti, const Inst& I, State* S,
                          WarpSmem& W, int lane, int cmode, int cprimal, bool xcommit,
                          double eta, double omega, int offp, int offi, int offv,
                          BulkPhase& ph) {
  const int rows = t.end - t.begin;
  const double tau = eta / omega;
  const bool iter = cmode == C_ITER;
  const bool xc = iter && xcommit;
  // vectors: 0 aty, 1 x (x_new on a commit), 2 c, 3 lo, 4 hi, 5 sum_x
  if (lane == 0) {
    const unsigned b = bulk_bytes<8>(t.begin, rows);
    mbar_arrive_tx(&W.bar[1], b * (iter ? 6u : 5u));
    bulk_stage<8>(W.vec[0], I.aty, t.begin, rows, &W.bar[1]);
    bulk_stage<8>(W.vec[1], xc ? I.xnew : I.x, t.begin, rows, &W.bar[1]);
    bulk_stage<8>(W.vec[2], I.c, t.begin, rows, &W.bar[1]);
    bulk_stage<8>(W.vec[3], I.lo, t.begin, rows, &W.bar[1]);
    bulk_stage<8>(W.vec[4], I.hi, t.begin, rows, &W.bar[1]);
    if (iter) bulk_stage<8>(W.vec[5], I.sumx, t.begin, rows, &W.bar[1]);
  }
  const int off = bulk_offset<8>(t.begin);
  if (iter) {     // only the iteration staged the matrix (the primal step needs none)
    if (!bulk_wait(A, &W.bar[0], ph.m)) { bulk_wait(A, &W.bar[1], ph.v); return; }
    if (!tile_ptrs_ok(A, t, W.sptr + offp, lane)) { bulk_wait(A, &W.bar[1], ph.v); return; }
    if (I.f32) {
      gather_products_f32(A, t, I.dy32, I.m, W, offi, offv, lane);
      staged_row_sums_f32(W.sptr + offp, reinterpret_cast<const float*>(W.sval) + offv, rows,
                          I.lanes_c, W.s0, lane);
    } else {
      gather_products(A, t, I.dy, I.m, W, offi, offv, lane);
      staged_row_sums(W.sptr + offp, W.sval + offv, rows, I.lanes_c, W.s0, lane);
    }
  }
  if (!bulk_wait(A, &W.bar[1], ph.v)) return;
  double acc[kNP];
#pragma unroll
  for (int s = 0; s < kNP; ++s) acc[s] = 0.0;
  for (int li = lane; li < rows; li += 32) {
    const int j = t.begin + li;
    const int v = off + li;
    const double xv = W.vec[1][v];
    double atyv = W.vec[0][v];
    if (iter) {                       // backend.py:282-291
      atyv = atyv + W.s0[li];
      I.aty[j] = atyv;
      I.sumx[j] = W.vec[5][v] + eta * xv;
    }
    if (cprimal == P_NONE) {
      if (xc) I.x[j] = xv;
    } else {                          // backend.py:204-215 / 241-255
      const double xn = clip(xv - tau * (W.vec[2][v] + atyv), W.vec[3][v], W.vec[4][v]);
      const double d = xn - xv;
      I.dx[j] = d;
      if (I.f32) I.dx32[j] = (float)d;
      if (cprimal == P_TRIAL) {
        I.xnew[j] = xn;
        if (xc) I.x[j] = xv;
        acc[0] += d * d;
      } else {
        I.x[j] = xn;
      }
    }
  }
  const bool need_red = cprimal == P_TRIAL;
  Ops ops;
  if (need_red) {
    warp_reduce(acc, ops);
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < kNP; ++s) A.partials[(size_t)(A.n_rtiles + ti) * kNP + s] = acc[s];
    }
  }
  double res[kNP];
  if (warp_finish(A, t, 1, I.cg_begin, I.cg_end, I.ct_end - I.ct_begin, need_red, ops, res,
                  lane, ph)) {
    if (lane == 0) c_finish(A, I, S, cmode, res);
    __syncwarp();
  }
}

__device__ void process_rtile(const EngineArgs& A, const Tile t, int ti, WarpSmem& W, int lane,
                              PassCache& pc, BulkPhase& ph) {
#ifdef PDLP_TRACE
  if (A.trace && blockIdx.x == 0 && threadIdx.x == 0) {
    const long long k = A.trace[1279];
    if (k >= 0 && k < 63) A.trace[640 + k * 8 + 7] = global_ns();
  }
#endif
  State* S = A.st + t.inst;
  const Inst& I = warp_inst(A, t.inst, W, lane);
  if (pc.inst != t.inst) pc.load_r(S, t.inst);
  const int rmode = pc.mode;
  const bool commit = pc.commit != 0;
  const double eta = pc.eta, omega = pc.omega;
  if (rmode == R_NONE) return;
  // the tile's row pointers, indices and values, one bulk copy each
  int offp = 0, offi = 0, offv = 0;
  if (!t.heavy) {
    const int rows1 = t.end - t.begin + 1;
    __syncwarp();                   // every lane is done with the previous tile's buffers
    if (lane == 0) {
      fence_proxy_async();
      const unsigned bv = I.f32 ? bulk_bytes<4>(t.p0, t.cnt) : bulk_bytes<8>(t.p0, t.cnt);
      mbar_arrive_tx(&W.bar[0], bulk_bytes<4>(t.begin, rows1) + bulk_bytes<4>(t.p0, t.cnt) + bv);
      bulk_stage<4>(W.sptr, I.rp, t.begin, rows1, &W.bar[0]);
      bulk_stage<4>(W.sidx, I.ri, t.p0, t.cnt, &W.bar[0]);
      if (I.f32) bulk_stage<4>(W.sval, I.rx32, t.p0, t.cnt, &W.bar[0]);
      else bulk_stage<8>(W.sval, I.rx, t.p0, t.cnt, &W.bar[0]);
    }
    offp = bulk_offset<4>(t.begin);
    offi = bulk_offset<4>(t.p0);
    offv = I.f32 ? bulk_offset<4>(t.p0) : bulk_offset<8>(t.p0);
  }
  if ((rmode == R_ITER || rmode == R_TRIAL) && !t.heavy) {
    hot_rtile(A, t, ti, I, S, W, lane, rmode, commit, eta, omega, offp, offi, offv, ph);
    return;
  }
  if (!t.heavy && !bulk_wait(A, &W.bar[0], ph.m)) return;
  __syncwarp();
  const int* tptr = W.sptr + offp;
  if (!t.heavy && !tile_ptrs_ok(A, t, tptr, lane)) return;

  const int L = I.lanes_r;
  const int* __restrict__ rp = I.rp;
  const int* __restrict__ ri = I.ri;
  double acc[kNP];
#pragma unroll
  for (int s = 0; s < kNP; ++s) acc[s] = 0.0;
  Ops ops;
  const int rend = row_loop_end(t, lane);
  const double sigma = eta * omega;

  // pending commit of an accepted line-search trial (pdlp.py:385-389):
  // y <- y_new, ax += adx, sum_y += eta y
  auto do_commit = [&](int r) {
    if (commit) {
      const double yn = ld_mut(I.ynew + r);
      I.y[r] = yn;
      I.ax[r] = ld_mut(I.ax + r) + ld_mut(I.adx + r);
      I.sumy[r] = ld_mut(I.sumy + r) + eta * yn;
    }
  };

  switch (rmode) {
    case R_RUIZ: {
      const int it = ld_mut(&S->ruiz_it);
      const bool last = ld_mut(&S->ruiz_last) != 0;
      const double* src = it <= 1 ? I.rx0 : I.rx;
      const double* dr_old = (it - 1) & 1 ? I.ynew : I.dy;     // factors of iteration it-1
      const double* dc_old = (it - 1) & 1 ? I.xnew : I.dx;
      double* dr_new = it & 1 ? I.ynew : I.dy;
      double* rr = I.yrst;                                      // running Ruiz row factor
      warp_rowmax(t, rp, L, [&](int r, int p) {
        double v = it <= 1 ? ld_ro(src + p) : ld_mut(src + p);
        if (it >= 1) {
          v = v * (ld_mut(dr_old + r) * ld_mut(dc_old + ld_ro(ri + p)));
          I.rx[p] = v;
        }
        return fabs(v);
      }, W, lane);
      ops.maxmask = 1u;
      for (int r = t.begin + lane; r < rend; r += 32) {
        const int li = r - t.begin;
        rr[r] = it == 0 ? 1.0 : ld_mut(rr + r) * ld_mut(dr_old + r);
        if (!last) {
          double rmax = W.s0[li];
          if (rmax <= 0.0) rmax = 1.0;
          acc[0] = fmax(acc[0], fabs(1.0 - rmax));
          dr_new[r] = 1.0 / sqrt(rmax);
        }
      }
      break;
    }
    case R_PC: {
      // Pock-Chambolle row sums over |A_ij (r_i c_j)| in storage order
      // (scaling.py:274-295 through sparse.py:50-58), one thread per row.
      const double* rr = I.yrst;
      const double* cr = I.xrst;
      const bool have_ruiz = I.ruiz_iters > 0;
      for (int r = t.begin + lane; r < rend; r += 32) {
        const double ri_r = have_ruiz ? ld_mut(rr + r) : 1.0;
        double f;
        if (I.scale_none) {
          f = 1.0;
        } else if (I.use_pc) {
          double s = 0.0;
          const int p0 = ld_ro(rp + r), p1 = ld_ro(rp + r + 1);
          for (int p = p0; p < p1; ++p) {
            const double cj = have_ruiz ? ld_mut(cr + ld_ro(ri + p)) : 1.0;
            s += fabs(ld_ro(I.rx0 + p) * (ri_r * cj));
          }
          if (s <= 0.0) s = 1.0;
          f = pow2_round(ri_r * (1.0 / sqrt(s)));
        } else {
          f = pow2_round(ri_r);
        }
        I.rs[r] = f;
      }
      break;
    }
    case R_APPLY: {
      warp_entries(t, rp, [&](int r, int p) {
        const double v = ld_ro(I.rx0 + p) * (ld_mut(I.rs + r) * ld_mut(I.cs + ld_ro(ri + p)));
        I.rx[p] = v;
        if (I.f32) I.rx32[p] = (float)v;
      }, lane);
      ops.maxmask = 1u;
      for (int r = t.begin + lane; r < rend; r += 32) {
        const double s = ld_mut(I.rs + r);
        const double l0 = ld_ro(I.rl0 + r), u0 = ld_ro(I.ru0 + r);
        const double l = row_bound(l0, s), u = row_bound(u0, s);
        I.rl[r] = l;
        I.ru[r] = u;
        acc[0] = fmax(acc[0], fmax(l0 > -kInf ? fabs(l0) : 0.0, u0 < kInf ? fabs(u0) : 0.0));
        const double bc = (l > -kInf ? l : 0.0) + (u < kInf ? u : 0.0);
        acc[1] += bc * bc;
      }
      break;
    }
    case R_SETUP0: {
      for (int r = t.begin + lane; r < rend; r += 32) {
        I.y[r] = 0.0; I.sumy[r] = 0.0; I.yrst[r] = 0.0; I.dy[r] = 0.0;
        if (I.f32) I.dy32[r] = 0.0f;
      }
      break;
    }
    case R_POWER: {
      const int round = ld_mut(&S->power_round);
      const double scale = ld_mut(&S->power_scale);
      const double* v = I.xbar;                    // A^T A power vector
      const double* rx = I.rx;
      auto term = [&](int p, int rhs) {
        const int j = ld_ro(ri + p);
        const double a = ld_mut(rx + p);
        if (rhs == 0) return a * (scale != 0.0 ? ld_mut(v + j) / scale : 0.0);
        return a * ld_mut(I.x + j);
      };
      if (round == 1) warp_spmv<2>(t, rp, tptr, L, term, W, lane);
      else warp_spmv<1>(t, rp, tptr, L, term, W, lane);
      ops.maxmask = 1u;
      for (int r = t.begin + lane; r < rend; r += 32) {
        const int li = r - t.begin;
        I.ybar[r] = W.s0[li];
        if (round == 1) {
          const double axv = W.s1[li];
          I.ax[r] = axv;
          acc[0] = fmax(acc[0], pviol(axv, ld_mut(I.rl + r), ld_mut(I.ru + r)));
        }
      }
      break;
    }
    case R_ITER: {
      // backend.py:260-279: ax += adx; w = y + sigma (ax + adx); prox; dy
      const double* rx = I.rx;
      const double* dxv = I.dx;
      warp_spmv<1>(t, rp, tptr, L, [&](int p, int) {
        return ld_mut(rx + p) * ld_mut(dxv + ld_ro(ri + p));
      }, W, lane);
      for (int r = t.begin + lane; r < rend; r += 32) {
        do_commit(r);
        const double a = W.s0[r - t.begin];
        const double axn = ld_mut(I.ax + r) + a;
        I.ax[r] = axn;
        const double yo = ld_mut(I.y + r);
        const double w = yo + sigma * (axn + a);
        const double yn = prox(w, sigma, ld_mut(I.rl + r), ld_mut(I.ru + r));
        I.dy[r] = yn - yo;
        if (I.f32) I.dy32[r] = (float)(yn - yo);
        I.y[r] = yn;
        I.sumy[r] = ld_mut(I.sumy + r) + eta * yn;
      }
      break;
    }
    case R_TRIAL: {
      // pdlp.py:347-356: adx = A dx; ax_bar = ax + 2 adx; dual_step; dy; dots
      const double* rx = I.rx;
      const double* dxv = I.dx;
      warp_spmv<1>(t, rp, tptr, L, [&](int p, int) {
        return ld_mut(rx + p) * ld_mut(dxv + ld_ro(ri + p));
      }, W, lane);
      for (int r = t.begin + lane; r < rend; r += 32) {
        do_commit(r);
        const double a = W.s0[r - t.begin];
        I.adx[r] = a;
        const double axb = ld_mut(I.ax + r) + 2.0 * a;
        const double yo = ld_mut(I.y + r);
        const double w = yo + sigma * axb;
        const double yn = prox(w, sigma, ld_mut(I.rl + r), ld_mut(I.ru + r));
        I.ynew[r] = yn;
        const double d = yn - yo;
        I.dy[r] = d;
        if (I.f32) I.dy32[r] = (float)d;
        acc[0] += d * a;
        acc[1] += d * d;
      }
      break;
    }
    case R_CHECK_A: {
      const double se = ld_mut(&S->sum_eta);
      ops.maxmask = 1u;
      for (int r = t.begin + lane; r < rend; r += 32) {
        do_commit(r);
        const double yv = ld_mut(I.y + r);
        const double yb = se > 0.0 ? ld_mut(I.sumy + r) / se : yv;
        I.ybar[r] = yb;
        const double l = ld_mut(I.rl + r), u = ld_mut(I.ru + r);
        const double yr = ld_mut(I.yrst + r);
        acc[0] = fmax(acc[0], pviol(ld_mut(I.ax + r), l, u));
        acc[1] += supp(yv, l, u);
        acc[2] += (yv - yr) * (yv - yr);
        acc[3] += (yb - yr) * (yb - yr);
        acc[4] += supp(yb, l, u);
      }
      break;
    }
    case R_CHECK_B: {
      const double* rx = I.rx;
      const double* xb = I.xbar;
      const double* xc = I.x;
      warp_spmv<2>(t, rp, tptr, L, [&](int p, int rhs) {
        const int j = ld_ro(ri + p);
        return ld_mut(rx + p) * ld_mut((rhs == 0 ? xb : xc) + j);
      }, W, lane);
      ops.maxmask = 7u;
      for (int r = t.begin + lane; r < rend; r += 32) {
        const int li = r - t.begin;
        const double axb = W.s0[li], axf = W.s1[li];
        I.axbar[r] = axb;
        I.axf[r] = axf;
        const double l = ld_mut(I.rl + r), u = ld_mut(I.ru + r), s = ld_mut(I.rs + r);
        const double pa = pviol(axb, l, u), pf = pviol(axf, l, u);
        acc[0] = fmax(acc[0], pa);
        acc[1] = fmax(acc[1], pa / s);
        acc[2] = fmax(acc[2], pf / s);
      }
      break;
    }
    case R_RESTART: {
      const bool avg = ld_mut(&S->restart_src) != 0;
      for (int r = t.begin + lane; r < rend; r += 32) {
        double yv;
        if (avg) { yv = ld_mut(I.ybar + r); I.y[r] = yv; I.ax[r] = ld_mut(I.axbar + r); }
        else { yv = ld_mut(I.y + r); I.ax[r] = ld_mut(I.axf + r); }
        I.yrst[r] = yv;
        I.sumy[r] = 0.0;
      }
      break;
    }
    case R_FINAL: {
      const bool avg = ld_mut(&S->final_src) != 0;
      const double s = ld_mut(&S->s_obj);
      const double ysign = I.sense == 1 ? -1.0 : 1.0;
      for (int r = t.begin + lane; r < rend; r += 32) {
        do_commit(r);
        const double yv = avg ? ld_mut(I.ybar + r) : ld_mut(I.y + r);
        I.yout[r] = ysign * ((yv * ld_mut(I.rs + r)) / s);
      }
      break;
    }
    default: break;
  }

  // R_ITER carries no reduction, and needs its finisher only to retire a
  // pending commit; the other modes reduce and/or advance the state machine.
  const bool need_red = rmode == R_RUIZ || rmode == R_APPLY || rmode == R_POWER ||
                        rmode == R_TRIAL || rmode == R_CHECK_A || rmode == R_CHECK_B;
  const bool need_fin = !(rmode == R_ITER && !commit);
  if (need_red) {
    warp_reduce(acc, ops);
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < kNP; ++s) A.partials[(size_t)ti * kNP + s] = acc[s];
    }
  }
  if (!need_fin) return;
  double res[kNP];
  if (warp_finish(A, t, 0, I.rg_begin, I.rg_end, I.rt_end - I.rt_begin, need_red, ops, res,
                  lane, ph)) {
    if (lane == 0) r_finish(A, I, S, rmode, res);
    __syncwarp();
  }
}

// ---- A^T pass ----------------------------------------------------------------

// Primal half-step for iteration k (backend.py:204-215 trial / 241-255 in place).
// Returns dx^2 for a trial.
__device__ __forceinline__ double primal_half(const Inst& I, int j, double xv, double atyv,
                                              double tau, int kind, bool wrote_x) {
  const double l = ld_mut(I.lo + j), h = ld_mut(I.hi + j);
  const double xn = clip(xv - tau * (ld_mut(I.c + j) + atyv), l, h);
  const double d = xn - xv;
  I.dx[j] = d;
  if (I.f32) I.dx32[j] = (float)d;
  if (kind == P_TRIAL) {
    I.xnew[j] = xn;
    if (wrote_x) I.x[j] = xv;
    return d * d;
  }
  I.x[j] = xn;
  return 0.0;
}

__device__ void c_finish(const EngineArgs& A, const Inst& I, State* S, int cmode, const double* red) {
  switch (cmode) {
    case C_RUIZ: {
      if (S->ruiz_last) {
        S->rmode = R_PC; S->cmode = C_PC;
      } else {
        const double dev = fmax(S->ruiz_dev_r, red[0]);
        if (dev < kRuizTol || S->ruiz_it + 1 >= I.ruiz_iters) S->ruiz_last = 1;
        S->ruiz_it += 1;
        S->rmode = R_RUIZ; S->cmode = C_RUIZ;
      }
      break;
    }
    case C_PC: S->rmode = R_APPLY; S->cmode = C_APPLY; break;
    case C_APPLY: {
      // objective scale (scaling.py:435-444)
      double s = 1.0;
      const double mx = red[0], mn = red[1];
      if (mn < INFINITY) {
        const double g = pow2_round(sqrt(mx * mn));
        const double gg = isfinite(sqrt(mx * mn)) ? g : INFINITY;
        if (gg > 0.0 && isfinite(gg)) s = 1.0 / gg;
      }
      S->s_obj = s;
      S->cn_orig = red[2];
      S->offset = (I.sense == 1 ? I.offset0 : -I.offset0) * s;
      S->rmode = R_SETUP0; S->cmode = C_SETUP0;
      break;
    }
    case C_SETUP0: {
      // primal weight (pdlp.py:292-296)
      const double cn = sqrt(red[0]);
      const double bn = sqrt(S->bn2);
      double om = bn > 0.0 ? exp(log(fmax(cn, 1e-12)) - log(fmax(bn, 1e-12))) : 1.0;
      S->omega = fmin(fmax(om, 1e-4), 1e4);
      const double nv = sqrt(red[1]);
      S->power_scale = nv;
      S->power_dead = nv == 0.0;
      S->d0 = red[2];
      S->pobj0 = red[3] + S->offset;
      S->dobj0 = red[4] + S->offset;
      S->power_round = 1;
      S->est = 1.0;
      S->rmode = R_POWER; S->cmode = C_POWER;
      break;
    }
    case C_POWER: {
      // power iteration (pdlp.py:140-159); first round also the initial merit (304)
      if (S->power_round == 1)
        S->mu_restart = merit(S->omega, S->p0, S->d0, fabs(S->pobj0 - S->dobj0));
      const double nrm = sqrt(red[0]);
      double anorm = -1.0;
      if (S->power_dead || nrm <= 0.0) {
        anorm = 1.0;
      } else {
        S->est = sqrt(nrm);
        S->power_scale = nrm;
        if (S->power_round >= kPowerIters) anorm = fmax(S->est, 1e-12);
      }
      if (anorm > 0.0) {
        S->eta = 1.0 / anorm;
        S->k = 0; S->epoch = 0; S->sum_eta = 0.0; S->mu_last = INFINITY;
        begin_iteration(I, S, false);
      } else {
        S->power_round += 1;
        S->rmode = R_POWER; S->cmode = C_POWER;
      }
      break;
    }
    case C_ITER: {
      S->xcommit = 0;
      S->sum_eta += S->eta;
      S->k += 1;
      S->epoch += 1;
      S->iters_done += 1;
      const int kind = S->cprimal;
      if (kind == P_TRIAL) {
        S->dxdx = red[0];
        S->rmode = R_TRIAL; S->cmode = C_NONE;
      } else if (kind == P_NORMAL) {
        S->cprimal = plan_primal(I, S->k + 1);
        S->rmode = R_ITER; S->cmode = C_ITER;
      } else if (S->k % I.check_every == 0) {
        S->rmode = R_CHECK_A; S->cmode = C_CHECK_A;
      } else {
        schedule_final(S, PDLP_STATUS_ITERATION_LIMIT, 0);
      }
      break;
    }
    case C_PRIMAL:
    case C_RESTART: {
      if (S->cprimal == P_TRIAL) {
        S->dxdx = red[0];
        S->rmode = R_TRIAL; S->cmode = C_NONE;
      } else {
        S->cprimal = plan_primal(I, S->k + 1);
        S->rmode = R_ITER; S->cmode = C_ITER;
      }
      break;
    }
    case C_CHECK_A: {
      for (int s = 0; s < 6; ++s) S->ca[s] = red[s];
      S->rmode = R_CHECK_B; S->cmode = C_CHECK_B;
      break;
    }
    case C_CHECK_B: {
      // restart / termination check (pdlp.py:406-463)
      const double omega = S->omega, off = S->offset, s = S->s_obj;
      const double pobj_c = S->ca[1] + off;
      const double dobj_c = -S->ra[1] + S->ca[2] + off;
      const double mu_c = merit(omega, S->ra[0], S->ca[0], fabs(pobj_c - dobj_c));
      const bool have_avg = S->sum_eta > 0.0;
      double mu_a = INFINITY, pobj_a = 0.0, dobj_a = 0.0;
      if (have_avg) {
        pobj_a = S->ca[5] + off;
        dobj_a = -S->ra[4] + red[1] + off;
        mu_a = merit(omega, S->rb[0], red[0], fabs(pobj_a - dobj_a));
      }
      const bool use_avg = mu_a < mu_c;
      const double mu_cand = use_avg ? mu_a : mu_c;
      double pu, du, pou, dou;
      if (use_avg) {
        pu = fmax(S->rb[1], red[3]); du = red[2];
        pou = pobj_a / s; dou = dobj_a / s;
      } else {
        pu = fmax(S->rb[2], red[6]); du = red[4];
        pou = pobj_c / s; dou = (-S->ra[1] + red[5] + off) / s;
      }
      const double gu = fabs(pou - dou);
      const double ptol = fmin(I.eps_abs + I.eps_rel * S->rhs_orig, I.feas_cap);
      const double dtol = fmin(I.eps_abs + I.eps_rel * S->cn_orig, I.feas_cap);
      const bool conv = pu <= ptol && du <= dtol &&
                        gu <= I.eps_abs + I.eps_rel * (fabs(pou) + fabs(dou));
      if (conv) {
        S->fin[0] = pu; S->fin[1] = du; S->fin[2] = gu; S->fin[3] = pou; S->fin[4] = dou;
        schedule_final(S, PDLP_STATUS_OPTIMAL, use_avg ? 1 : 0);
        break;
      }
      {   // how far from the test, for the host's team planning (no effect on the solve)
        const double gtol = I.eps_abs + I.eps_rel * (fabs(pou) + fabs(dou));
        const double r = fmax(pu / fmax(ptol, 1e-300), fmax(du / fmax(dtol, 1e-300), gu / fmax(gtol, 1e-300)));
        if (isfinite(r) && r > 0.0) {
          if (S->kkt_k_first == 0) { S->kkt_first = r; S->kkt_k_first = S->k; S->kkt_best = r; }
          else if (r < S->kkt_best) S->kkt_best = r;
          S->kkt_k = S->k;
        }
      }
      if (S->hist_len < I.hist_cap) {
        double* h = I.hist + 5 * (size_t)S->hist_len;
        h[0] = (double)S->k; h[1] = pu; h[2] = du; h[3] = gu; h[4] = pou;
        S->hist_len += 1;
      }
      const bool restart =
          mu_cand <= I.beta_s * S->mu_restart ||
          (mu_cand <= I.beta_n * S->mu_restart && mu_cand > S->mu_last) ||
          (double)S->epoch >= I.beta_a * (double)(S->k > 1 ? S->k : 1);
      S->mu_last = mu_cand;
      if (restart) {
        const double ddx = sqrt(use_avg ? S->ca[4] : S->ca[3]);
        const double ddy = sqrt(use_avg ? S->ra[3] : S->ra[2]);
        if (ddx > 1e-12 && ddy > 1e-12) {
          const double th = I.theta;
          const double om = exp(th * log(ddy / ddx) + (1.0 - th) * log(omega));
          S->omega = fmin(fmax(om, 1e-6), 1e6);
        }
        S->mu_restart = mu_cand;
        S->sum_eta = 0.0;
        S->epoch = 0;
        S->restarts += 1;
        S->restart_src = use_avg ? 1 : 0;
      }
      begin_iteration(I, S, restart);
      break;
    }
    case C_FINAL: {
      S->objective = red[0] + I.offset0;
      S->t_end_ns = global_ns();
      S->rmode = R_NONE; S->cmode = C_NONE;
      __threadfence();
      S->status = S->final_status;
      atomicSub(&A.ctl->active, 1);
      atomicSub(&A.ctl->team_active[I.team], 1);
      break;
    }
    default: break;
  }
}

__device__ void process_ctile(const EngineArgs& A, const Tile t, int ti, WarpSmem& W, int lane,
                              PassCache& pc, BulkPhase& ph) {
  State* S = A.st + t.inst;
  const Inst& I = warp_inst(A, t.inst, W, lane);
  if (pc.inst != t.inst) pc.load_c(S, t.inst);
  const int cmode = pc.mode;
  const int cprimal = pc.aux;
  const bool xcommit = pc.commit != 0;
  const double eta = pc.eta, omega = pc.omega;
  if (cmode == C_NONE) return;
  const bool hot = (cmode == C_ITER || cmode == C_PRIMAL) && !t.heavy;
  // the tile's column pointers, row indices and values (not needed by the
  // staged primal step, which reads only vectors)
  int offp = 0, offi = 0, offv = 0;
  __syncwarp();                     // every lane is done with the previous tile's buffers
  if (lane == 0) fence_proxy_async();
  if (!t.heavy && !(hot && cmode == C_PRIMAL)) {
    const int rows1 = t.end - t.begin + 1;
    if (lane == 0) {
      const unsigned bv = I.f32 ? bulk_bytes<4>(t.p0, t.cnt) : bulk_bytes<8>(t.p0, t.cnt);
      mbar_arrive_tx(&W.bar[0], bulk_bytes<4>(t.begin, rows1) + bulk_bytes<4>(t.p0, t.cnt) + bv);
      bulk_stage<4>(W.sptr, I.cp, t.begin, rows1, &W.bar[0]);
      bulk_stage<4>(W.sidx, I.ci, t.p0, t.cnt, &W.bar[0]);
      if (I.f32) bulk_stage<4>(W.sval, I.cx32, t.p0, t.cnt, &W.bar[0]);
      else bulk_stage<8>(W.sval, I.cx, t.p0, t.cnt, &W.bar[0]);
    }
    offp = bulk_offset<4>(t.begin);
    offi = bulk_offset<4>(t.p0);
    offv = I.f32 ? bulk_offset<4>(t.p0) : bulk_offset<8>(t.p0);
  }
  if (hot) {
    hot_ctile(A, t, ti, I, S, W, lane, cmode, cprimal, xcommit, eta, omega, offp, offi, offv, ph);
    return;
  }
  if (!t.heavy && !bulk_wait(A, &W.bar[0], ph.m)) return;
  __syncwarp();
  const int* tptr = W.sptr + offp;
  if (!t.heavy && !tile_ptrs_ok(A, t, tptr, lane)) return;

  const int L = I.lanes_c;
  const int* __restrict__ cp = I.cp;
  const int* __restrict__ ci = I.ci;
  double acc[kNP];
#pragma unroll
  for (int s = 0; s < kNP; ++s) acc[s] = 0.0;
  Ops ops;
  const int rend = row_loop_end(t, lane);
  const double tau = eta / omega;

  switch (cmode) {
    case C_RUIZ: {
      const int it = ld_mut(&S->ruiz_it);
      const bool last = ld_mut(&S->ruiz_last) != 0;
      const double* src = it <= 1 ? I.cx0 : I.cx;
      const double* dr_old = (it - 1) & 1 ? I.ynew : I.dy;
      const double* dc_old = (it - 1) & 1 ? I.xnew : I.dx;
      double* dc_new = it & 1 ? I.xnew : I.dx;
      double* cr = I.xrst;
      warp_rowmax(t, cp, L, [&](int j, int p) {
        double v = it <= 1 ? ld_ro(src + p) : ld_mut(src + p);
        if (it >= 1) {
          v = v * (ld_mut(dr_old + ld_ro(ci + p)) * ld_mut(dc_old + j));
          I.cx[p] = v;
        }
        return fabs(v);
      }, W, lane);
      ops.maxmask = 1u;
      for (int j = t.begin + lane; j < rend; j += 32) {
        const int li = j - t.begin;
        cr[j] = it == 0 ? 1.0 : ld_mut(cr + j) * ld_mut(dc_old + j);
        if (!last) {
          double cmax = W.s0[li];
          if (cmax <= 0.0) cmax = 1.0;
          acc[0] = fmax(acc[0], fabs(1.0 - cmax));
          dc_new[j] = 1.0 / sqrt(cmax);
        }
      }
      break;
    }
    case C_PC: {
      const double* rr = I.yrst;
      const double* cr = I.xrst;
      const bool have_ruiz = I.ruiz_iters > 0;
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double cj = have_ruiz ? ld_mut(cr + j) : 1.0;
        double f;
        if (I.scale_none) {
          f = 1.0;
        } else if (I.use_pc) {
          double s = 0.0;
          const int p0 = ld_ro(cp + j), p1 = ld_ro(cp + j + 1);
          for (int p = p0; p < p1; ++p) {
            const double ri_ = have_ruiz ? ld_mut(rr + ld_ro(ci + p)) : 1.0;
            s += fabs(ld_ro(I.cx0 + p) * (ri_ * cj));
          }
          if (s <= 0.0) s = 1.0;
          f = pow2_round(cj * (1.0 / sqrt(s)));
        } else {
          f = pow2_round(cj);
        }
        if (I.kind != nullptr && I.kind[j] != 0) f = 1.0;
        I.cs[j] = f;
      }
      break;
    }
    case C_APPLY: {
      warp_entries(t, cp, [&](int j, int p) {
        const double v = ld_ro(I.cx0 + p) * (ld_mut(I.rs + ld_ro(ci + p)) * ld_mut(I.cs + j));
        I.cx[p] = v;
        if (I.f32) I.cx32[p] = (float)v;
      }, lane);
      ops.maxmask = 5u;       // slots 0 and 2
      ops.minmask = 2u;       // slot 1
      acc[1] = INFINITY;
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double s = ld_mut(I.cs + j);
        const double c0 = ld_ro(I.c0 + j);
        const double cw = I.sense == 1 ? c0 : -c0;
        const double cc = cw * s;
        I.c[j] = cc;
        I.lo[j] = col_bound(ld_ro(I.lo0 + j), s);
        I.hi[j] = col_bound(ld_ro(I.hi0 + j), s);
        if (cc != 0.0) {
          acc[0] = fmax(acc[0], fabs(cc));
          acc[1] = fmin(acc[1], fabs(cc));
        }
        acc[2] = fmax(acc[2], fabs(c0));
      }
      break;
    }
    case C_SETUP0: {
      const double s = ld_mut(&S->s_obj);
      ops.maxmask = 4u;       // slot 2
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double c = ld_mut(I.c + j) * s;
        I.c[j] = c;
        const double l = ld_mut(I.lo + j), h = ld_mut(I.hi + j);
        const double x0 = clip(0.0, l, h);
        I.x[j] = x0; I.xrst[j] = x0; I.aty[j] = 0.0; I.sumx[j] = 0.0; I.dx[j] = 0.0;
        if (I.f32) I.dx32[j] = 0.0f;
        const double v0 = I.v0 != nullptr ? ld_ro(I.v0 + j)
                                          : gen_normal((unsigned long long)j);
        I.xbar[j] = v0;
        acc[0] += c * c;
        acc[1] += v0 * v0;
        acc[2] = fmax(acc[2], dres(c, l, h));
        acc[3] += c * x0;
        acc[4] += bndterm(c, l, h);
      }
      break;
    }
    case C_POWER: {
      const double* cx = I.cx;
      const double* av = I.ybar;
      warp_spmv<1>(t, cp, tptr, L, [&](int p, int) {
        return ld_mut(cx + p) * ld_mut(av + ld_ro(ci + p));
      }, W, lane);
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double v = W.s0[j - t.begin];
        I.xbar[j] = v;
        acc[0] += v * v;
      }
      break;
    }
    case C_ITER: {
      // backend.py:282-291 (aty += ady; sum_x += eta x) then the next primal step
      const double* cx = I.cx;
      const bool xc = xcommit;
      const int kind = cprimal;
      const double* dyv = I.dy;
      warp_spmv<1>(t, cp, tptr, L, [&](int p, int) {
        return ld_mut(cx + p) * ld_mut(dyv + ld_ro(ci + p));
      }, W, lane);
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double xv = xc ? ld_mut(I.xnew + j) : ld_mut(I.x + j);
        const double atyv = ld_mut(I.aty + j) + W.s0[j - t.begin];
        I.aty[j] = atyv;
        I.sumx[j] = ld_mut(I.sumx + j) + eta * xv;
        if (kind == P_NONE) {
          if (xc) I.x[j] = xv;
        } else {
          acc[0] += primal_half(I, j, xv, atyv, tau, kind, xc);
        }
      }
      break;
    }
    case C_PRIMAL: {
      const int kind = cprimal;
      for (int j = t.begin + lane; j < rend; j += 32)
        acc[0] += primal_half(I, j, ld_mut(I.x + j), ld_mut(I.aty + j), tau, kind, false);
      break;
    }
    case C_CHECK_A: {
      const double se = ld_mut(&S->sum_eta);
      ops.maxmask = 1u;
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double xv = ld_mut(I.x + j);
        const double xb = se > 0.0 ? ld_mut(I.sumx + j) / se : xv;
        I.xbar[j] = xb;
        const double c = ld_mut(I.c + j), l = ld_mut(I.lo + j), h = ld_mut(I.hi + j);
        const double d = c + ld_mut(I.aty + j);
        const double xr = ld_mut(I.xrst + j);
        acc[0] = fmax(acc[0], dres(d, l, h));
        acc[1] += c * xv;
        acc[2] += bndterm(d, l, h);
        acc[3] += (xv - xr) * (xv - xr);
        acc[4] += (xb - xr) * (xb - xr);
        acc[5] += c * xb;
      }
      break;
    }
    case C_CHECK_B: {
      const double* cx = I.cx;
      const double* yb = I.ybar;
      const double* yc = I.y;
      warp_spmv<2>(t, cp, tptr, L, [&](int p, int rhs) {
        const int i = ld_ro(ci + p);
        return ld_mut(cx + p) * ld_mut((rhs == 0 ? yb : yc) + i);
      }, W, lane);
      const double s = ld_mut(&S->s_obj);
      ops.maxmask = (1u << 0) | (1u << 2) | (1u << 3) | (1u << 4) | (1u << 6);
      for (int j = t.begin + lane; j < rend; j += 32) {
        const int li = j - t.begin;
        const double atb = W.s0[li], atf = W.s1[li];
        I.atybar[j] = atb;
        I.atyf[j] = atf;
        const double c = ld_mut(I.c + j), l = ld_mut(I.lo + j), h = ld_mut(I.hi + j);
        const double cs = ld_mut(I.cs + j);
        const double da = c + atb, df = c + atf;
        const double ra = dres(da, l, h);
        acc[0] = fmax(acc[0], ra);
        acc[1] += bndterm(da, l, h);
        acc[2] = fmax(acc[2], ra / (s * cs));
        acc[3] = fmax(acc[3], bviol(ld_mut(I.xbar + j), l, h) * cs);
        acc[4] = fmax(acc[4], dres(df, l, h) / (s * cs));
        acc[5] += bndterm(df, l, h);
        acc[6] = fmax(acc[6], bviol(ld_mut(I.x + j), l, h) * cs);
      }
      break;
    }
    case C_RESTART: {
      const bool avg = ld_mut(&S->restart_src) != 0;
      const int kind = cprimal;
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double xv = avg ? ld_mut(I.xbar + j) : ld_mut(I.x + j);
        const double atyv = avg ? ld_mut(I.atybar + j) : ld_mut(I.atyf + j);
        I.x[j] = xv;
        I.aty[j] = atyv;
        I.xrst[j] = xv;
        I.sumx[j] = 0.0;
        acc[0] += primal_half(I, j, xv, atyv, tau, kind, false);
      }
      break;
    }
    case C_FINAL: {
      // x clipped to its original bounds, d = c - A^T y in original units
      // (pdlp.py:466-484), objective c'x + offset
      const bool avg = ld_mut(&S->final_src) != 0;
      const double* ysrc = avg ? I.ybar : I.y;
      const double* cx = I.cx;
      warp_spmv<1>(t, cp, tptr, L, [&](int p, int) {
        return ld_mut(cx + p) * ld_mut(ysrc + ld_ro(ci + p));
      }, W, lane);
      const double s = ld_mut(&S->s_obj);
      const double dsign = I.sense == 1 ? 1.0 : -1.0;
      for (int j = t.begin + lane; j < rend; j += 32) {
        const double cs = ld_mut(I.cs + j);
        const double xv = avg ? ld_mut(I.xbar + j) : ld_mut(I.x + j);
        const double xo = clip(xv * cs, ld_ro(I.lo0 + j), ld_ro(I.hi0 + j));
        I.xout[j] = xo;
        I.dout[j] = dsign * ((ld_mut(I.c + j) + W.s0[j - t.begin]) / (s * cs));
        acc[0] += ld_ro(I.c0 + j) * xo;
      }
      break;
    }
    default: break;
  }

  const bool trial = (cmode == C_ITER || cmode == C_PRIMAL || cmode == C_RESTART) &&
                     cprimal == P_TRIAL;
  const bool need_red = trial || cmode == C_RUIZ || cmode == C_APPLY || cmode == C_SETUP0 ||
                        cmode == C_POWER || cmode == C_CHECK_A || cmode == C_CHECK_B ||
                        cmode == C_FINAL;
  if (need_red) {
    warp_reduce(acc, ops);
    if (lane == 0) {
#pragma unroll
      for (int s = 0; s < kNP; ++s)
        A.partials[(size_t)(A.n_rtiles + ti) * kNP + s] = acc[s];
    }
  }
  double res[kNP];
  if (warp_finish(A, t, 1, I.cg_begin, I.cg_end, I.ct_end - I.ct_begin, need_red, ops, res,
                  lane, ph)) {
    if (lane == 0) c_finish(A, I, S, cmode, res);
    __syncwarp();
  }
}

}  // namespace pdlp
