// Device-side data structures of the PDLP engine.
//
// One engine advances a set of LPs ("instances") together.  Each instance owns
// its arrays (allocated at admission); the engine sees the set as one
// block-diagonal problem through two tile lists: row tiles (ranges of rows of
// A, the A pass) and column tiles (ranges of rows of A^T, the A^T pass).  A
// tile never spans two instances, so every per-instance reduction is a sum
// over that instance's own tiles in a fixed order, and its result does not
// depend on which other LPs share the launch.
//
// Every engine step runs the A pass over all row tiles, a grid-wide barrier,
// the A^T pass over all column tiles and another barrier.  A tile is the work
// of one warp (a few hundred entries); warps never wait for one another
// inside a pass.  What a tile does is set by its instance's state machine
// (RMode / CMode below).  Per-instance reductions go through a fixed two-level
// tree: tile partials -> group partials (64 consecutive tiles) -> instance;
// the warp that completes a group reduces it, and the warp that completes the
// instance's last group advances the state machine (the "finisher").
#pragma once

#include <cstdint>

namespace pdlp {

constexpr double kInf = 1.0e30;          // infinite-bound sentinel (tolerances.py:16)
constexpr int kNP = 8;                   // partial slots per tile
constexpr int kMaxLineSearch = 60;       // pdlp.py:340
constexpr int kPowerIters = 20;          // pdlp.py:140

// What a row tile does in the A pass.
enum RMode : int {
  R_NONE = 0,
  R_RUIZ,      // apply the previous Ruiz factors to the CSR copy, new row maxima
  R_PC,        // Pock-Chambolle row sums, final pow2 row factors
  R_APPLY,     // scaled CSR values, scaled row bounds
  R_SETUP0,    // y = 0, running sums zeroed
  R_POWER,     // power iteration: av = A v (first round also ax = A x)
  R_ITER,      // fused PDHG dual half-step
  R_TRIAL,     // line-search trial dual step (out of place)
  R_CHECK_A,   // averages and KKT partials of the current point (row side)
  R_CHECK_B,   // A xbar and A x (fresh), KKT partials of the average
  R_RESTART,   // restart copy (row side)
  R_FINAL,     // unscaled y
};

// What a column tile does in the A^T pass.
enum CMode : int {
  C_NONE = 0,
  C_RUIZ,
  C_PC,
  C_APPLY,
  C_SETUP0,
  C_POWER,
  C_ITER,      // A^T dy, aty update, sum_x, then the next primal half-step
  C_PRIMAL,    // primal half-step only (trial or normal)
  C_CHECK_A,
  C_CHECK_B,
  C_RESTART,
  C_FINAL,
};

enum PrimalKind : int { P_NONE = 0, P_NORMAL = 1, P_TRIAL = 2 };

enum ScalingKind : int { SC_PDLP = 0, SC_NONE = 1, SC_RUIZ = 2, SC_PC = 3 };

// Immutable for the duration of a launch.
struct Inst {
  int m, n;
  long long nnz;
  int lanes_r, lanes_c;     // lanes per row of the A / A^T pass (power of two)
  int sense;                // 1 minimise, -1 maximise
  int ruiz_iters;           // 0 = no Ruiz
  int use_pc;
  int scale_none;
  int team;                 // the block team that runs this instance (persistent launches)
  // matrix: CSR of A (row tiles) and CSR of A^T (column tiles), int32 pointers
  const int* rp; const int* ri;
  const int* cp; const int* ci;
  const double* rx0; const double* cx0;     // original values
  double* rx; double* cx;                   // Ruiz working copy, then scaled A
  const double* c0; const double* rl0; const double* ru0;
  const double* lo0; const double* hi0;
  const unsigned char* kind;
  double offset0;
  double *c, *rl, *ru, *lo, *hi;            // scaled data
  double *rs, *cs;                          // pow2 row / column factors
  // row-side vectors (length m)
  double *y, *ax, *dy, *ynew, *adx, *sumy, *ybar, *axbar, *axf, *yrst, *yout;
  // column-side vectors (length n)
  double *x, *aty, *dx, *xnew, *sumx, *xbar, *atybar, *atyf, *xrst, *xout, *dout;
  const double* v0;                         // power-iteration start, or null
  int f32;                                  // 1: iteration SpMVs in float32
  float* rx32; float* cx32;                 // float32 scaled values (f32 only)
  float* dx32; float* dy32;                 // float32 copies of dx, dy (f32 only)
  double* hist;
  int hist_cap;
  // parameters (pdlp.py:79-116)
  double eps_abs, eps_rel, feas_cap;
  long long max_iter;
  double time_limit_ns, time_used_ns;
  int check_every, stepsize_every;
  double beta_s, beta_n, beta_a, theta;
  // tile and group ranges in the launch's lists
  int rt_begin, rt_end, ct_begin, ct_end;
  int rg_begin, rg_end, cg_begin, cg_end;
};

// Mutable; written only by the instance's finishers (and by the host between
// launches).
struct State {
  int rmode, cmode;
  int status;               // -1 running, else a PDLP_STATUS_* code
  int cprimal;              // primal kind the current C pass computes at its end
  int xcommit;              // C pass: x <- xnew before the update
  int ycommit;              // R pass: y <- ynew, ax += adx, sum_y += eta y first
  int final_src;            // 0 current point, 1 average
  int restart_src;          // 0 current point (fresh products), 1 average
  int ruiz_it, ruiz_last;
  int power_round, power_dead;
  int trials;
  int hist_len;
  int cancel;               // set by the host
  int error;                // admission: malformed input found on the device
  int final_status;         // status the scheduled final pass will publish
  long long k, attempts, rejected, restarts, epoch, iters_done;
  double eta, omega, sum_eta, mu_restart, mu_last;
  double power_scale, est;
  double s_obj, offset;
  double rhs_orig, cn_orig, bn2;
  double ruiz_dev_r;
  double p0, d0, pobj0, dobj0;
  double dxdx;
  double ra[5];             // R_CHECK_A reductions
  double rb[3];             // R_CHECK_B reductions
  double ca[6];             // C_CHECK_A reductions
  double fin[5];            // (pu, du, gu, pobj, dobj) at OPTIMAL
  double objective;
  long long t_start_ns, t_end_ns;
  // scheduling only: the largest residual-to-tolerance ratio of the
  // termination test at the first check and the smallest since, with the
  // iterations they were seen at (0: no check yet)
  double kkt_first, kkt_best;
  long long kkt_k_first, kkt_k;
};

struct Tile {
  int inst;
  int begin, end;           // local row range
  int heavy;                // 1: a single long row, reduced by the whole warp
  int group;                // global index of the tile's reduction group
  int p0, cnt;              // first entry and entry count of the row range
  int pad;
};

constexpr int kGroupTiles = 64;          // tiles per reduction group

constexpr int kMaxTeams = 256;           // block teams of one launch

// Engine-wide control block in device memory.  The blocks of a launch form
// teams (one team normally; one per instance when few instances are left):
// each team steps at its own pace behind its own barrier.
struct Control {
  unsigned int bar_count;
  unsigned int bar_gen;
  int active;               // instances still running
  int error;                // nonzero: a bounded wait gave up (code)
  int error_where;
  int stop;                 // set to end the launch: every team leaves at its next step
  unsigned int idle;        // blocks of teams whose instances are all done
  unsigned int pad;
  unsigned int team_bar[kMaxTeams];   // each team's barrier arrival counter
  int team_active[kMaxTeams];         // each team's instances still running
  int team_go[kMaxTeams];             // the team leader's decision for the next step
  int team_budget[kMaxTeams];         // steps each team may run in this launch (host)
  int team_steps[kMaxTeams];          // steps each team completed (its leader, at exit)
};

struct EngineArgs {
  Inst* inst;
  State* st;
  const Tile* rtiles; int n_rtiles;
  const Tile* ctiles; int n_ctiles;
  const int* rwarp;         // persistent: warp w owns row tiles [rwarp[w], rwarp[w+1])
  const int* cwarp;
  const int* block_team;    // persistent: team of each block
  const int* team_blocks;   // [n_teams] blocks per team
  const int* team_first;    // [n_teams] first block of each team (its leader)
  const int2* group_tiles;  // [n_groups]: tile range of each group (row groups first)
  int n_rgroups, n_groups;
  double* partials;         // [(n_rtiles + n_ctiles) * kNP] tile partials
  double* gpartials;        // [n_groups * kNP] group partials
  unsigned int* gcounters;  // [n_groups] tiles done per group
  unsigned int* counters;   // [2 * n_inst] groups done per instance and side
  Control* ctl;
  long long max_steps;       // the launch's step cap; reaching it ends the launch
  long long barrier_timeout_ns;
  int withhold_block;       // test hook: this block leaves at its first barrier
                            // without arriving (-1: none)
  int n_inst;
  long long* trace;         // tracing builds only: phase timestamps, else null
};

}  // namespace pdlp
