// Crossover from a PDLP point to an optimal basis, on the host cores.
//
// Two entry points (declared in pdlp_b200.h):
//
//   pdlp_basis_from_point  -- basis identification from a primal(-dual)
//       point: the ranking of Bixby & Saltzman (distance of each variable of
//       [x ; s] to its nearest bound, relative to its range) followed by a
//       rank-tested push of the candidates into the all-logical basis, one
//       FTRAN each, pivoting on the largest entry in a row that still holds
//       its logical.  This is the algorithm of sovopt's
//       src/sovopt/lp/crossover.py:80-187, with the same scores, order,
//       pivot rule, tolerances and status assignment, so the status vector
//       it returns is the reference's.
//   pdlp_simplex_solve     -- a bounded primal simplex (composite phase 1,
//       then phase 2) started from a status vector; it finishes the
//       crossover, the role src/sovopt/lp/simplex.py:1181-1374 plays in
//       crossover.py:190-222.  It terminates only at a basis that is primal
//       and dual feasible within the tolerances, so a poor identification
//       costs pivots and never correctness.
//
// Pivoting is sequential: every pivot depends on the previous one, and a
// basis solve is a chain of sparse triangular substitutions.  So this file is
// host code; the point it starts from is the engine's result, read back once.
//
// Basis representation (own design).  M = [A | -I], z = [x ; s], M z = 0;
// the logical of row i is variable n+i with column -e_i and the row's bounds.
// The basis matrix B = M[:, basic] is factored as a sparse LU by a
// left-looking factorisation with partial pivoting (Gilbert & Peierls,
// "Sparse partial pivoting in time proportional to arithmetic operations",
// SIAM J. Sci. Stat. Comput. 9 (1988) 862-874): columns in order of
// increasing length, each column's pattern found by a depth-first search of
// L's graph, its largest remaining entry taken as the pivot.  Between
// refactorisations each pivot appends an eta vector (product form of the
// inverse, Dantzig & Orchard-Hays 1954).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "common.cuh"

namespace pdlp {
namespace xo {

constexpr double kBound = 1.0e30;   // |bound| >= 1e30 is no bound (sovopt INF)
constexpr double kHuge = std::numeric_limits<double>::infinity();

enum : uint8_t { kBasic = 0, kAtLower = 1, kAtUpper = 2, kFree = 3, kFixed = 4 };

struct Lp {
  int m, n;
  const int64_t* rp; const int32_t* ri; const double* rx;   // CSR (may be null)
  const int64_t* cp; const int32_t* ci; const double* cx;   // CSC
};

// ---- sparse LU of the basis matrix ---------------------------------------

class LuFactor {
 public:
  // Factor B = M[:, basic].  Returns -1, or the basis position of a column
  // that is dependent (to abs_tol relative to its largest entry) on the
  // columns factored before it.
  int factor(const Lp& A, const int* basic) {
    const int m = A.m;
    m_ = m;
    std::vector<int> order(m);
    std::iota(order.begin(), order.end(), 0);
    auto len = [&](int p) -> int64_t {
      const int j = basic[p];
      return j < A.n ? A.cp[j + 1] - A.cp[j] : 1;
    };
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return len(a) < len(b); });
    lp_.assign(1, 0); up_.assign(1, 0);
    li_.clear(); lx_.clear(); ui_.clear(); ux_.clear();
    ud_.assign(m, 0.0); prow_.assign(m, -1); pos_.assign(m, -1); pinv_.assign(m, -1);
    x_.assign(m, 0.0); mark_.assign(m, -1); stack_.resize(m); head_.resize(m); topo_.resize(m);
    w_.assign(m, 0.0);
    // entries of B per row, the sparsity preference of the pivot choice
    rowcnt_.assign(m, 0);
    for (int p = 0; p < m; ++p) {
      const int j = basic[p];
      if (j < A.n) {
        for (int64_t e = A.cp[j]; e < A.cp[j + 1]; ++e) ++rowcnt_[A.ci[e]];
      } else {
        ++rowcnt_[j - A.n];
      }
    }
    for (int k = 0; k < m; ++k) {
      const int p = order[k], j = basic[p];
      int top = m;
      double colmax = 0.0;
      if (j < A.n) {
        for (int64_t e = A.cp[j]; e < A.cp[j + 1]; ++e) {
          const int r = A.ci[e];
          x_[r] = A.cx[e];
          colmax = std::max(colmax, std::fabs(A.cx[e]));
          if (mark_[r] != k) reach(r, k, top);
        }
      } else {
        const int r = j - A.n;
        x_[r] = -1.0;
        colmax = 1.0;
        reach(r, k, top);
      }
      // x = L \ b over the reached rows, in topological order
      for (int t = top; t < m; ++t) {
        const int r = topo_[t], s = pinv_[r];
        if (s < 0) continue;
        const double xr = x_[r];
        if (xr == 0.0) continue;
        for (int64_t e = lp_[s]; e < lp_[s + 1]; ++e) x_[li_[e]] -= lx_[e] * xr;
      }
      // threshold partial pivoting: of the entries within a factor 10 of the
      // column's largest, the one in the row with the fewest entries of B
      double bmax = 0.0;
      for (int t = top; t < m; ++t) {
        const int r = topo_[t];
        if (pinv_[r] < 0) bmax = std::max(bmax, std::fabs(x_[r]));
      }
      if (!(bmax > 1e-11 * std::max(1.0, colmax))) {
        for (int t = top; t < m; ++t) x_[topo_[t]] = 0.0;
        return p;
      }
      int best = -1, bcnt = 0;
      double bval = 0.0;
      for (int t = top; t < m; ++t) {
        const int r = topo_[t];
        const double a = std::fabs(x_[r]);
        if (pinv_[r] >= 0 || a < 0.1 * bmax) continue;
        if (best < 0 || rowcnt_[r] < bcnt || (rowcnt_[r] == bcnt && a > bval)) {
          best = r; bcnt = rowcnt_[r]; bval = a;
        }
      }
      for (int t = top; t < m; ++t) {
        const int r = topo_[t];
        if (pinv_[r] >= 0 && x_[r] != 0.0) { ui_.push_back(pinv_[r]); ux_.push_back(x_[r]); }
      }
      up_.push_back((int64_t)ui_.size());
      const double piv = x_[best];
      ud_[k] = piv; prow_[k] = best; pinv_[best] = k; pos_[k] = p;
      for (int t = top; t < m; ++t) {
        const int r = topo_[t];
        if (pinv_[r] < 0 && x_[r] != 0.0) { li_.push_back(r); lx_.push_back(x_[r] / piv); }
        x_[r] = 0.0;
      }
      lp_.push_back((int64_t)li_.size());
    }
    return -1;
  }

  bool pivoted(int row) const { return pinv_[row] >= 0; }
  int64_t nnz() const { return (int64_t)li_.size() + (int64_t)ui_.size() + m_; }

  // v <- B^-1 v: v holds a row-indexed right-hand side and returns the
  // solution indexed by basis position.
  void ftran(double* v) const {
    for (int k = 0; k < m_; ++k) {
      const double t = v[prow_[k]];
      w_[k] = t;
      if (t == 0.0) continue;
      for (int64_t e = lp_[k]; e < lp_[k + 1]; ++e) v[li_[e]] -= lx_[e] * t;
    }
    for (int k = m_ - 1; k >= 0; --k) {
      const double u = w_[k] / ud_[k];
      w_[k] = u;
      if (u == 0.0) continue;
      for (int64_t e = up_[k]; e < up_[k + 1]; ++e) w_[ui_[e]] -= ux_[e] * u;
    }
    for (int k = 0; k < m_; ++k) v[pos_[k]] = w_[k];
  }

  // v <- B^-T v: v holds a position-indexed right-hand side and returns the
  // solution indexed by row.
  void btran(double* v) const {
    for (int k = 0; k < m_; ++k) {
      double s = v[pos_[k]];
      for (int64_t e = up_[k]; e < up_[k + 1]; ++e) s -= ux_[e] * w_[ui_[e]];
      w_[k] = s / ud_[k];
    }
    for (int k = m_ - 1; k >= 0; --k) {
      double s = w_[k];
      for (int64_t e = lp_[k]; e < lp_[k + 1]; ++e) s -= lx_[e] * v[li_[e]];
      v[prow_[k]] = s;
    }
  }

 private:
  // Depth-first search from row r0 over L's graph (a pivotal row leads to the
  // rows of its L column); finished rows are pushed onto topo_ from the top,
  // so topo_[top..m) is a topological order of the reached rows.
  void reach(int r0, int k, int& top) {
    int depth = 0;
    stack_[0] = r0;
    while (depth >= 0) {
      const int r = stack_[depth];
      const int s = pinv_[r];
      if (mark_[r] != k) {
        mark_[r] = k;
        head_[depth] = s >= 0 ? lp_[s] : 0;
      }
      bool done = true;
      if (s >= 0) {
        for (int64_t e = head_[depth]; e < lp_[s + 1]; ++e) {
          const int c = li_[e];
          if (mark_[c] == k) continue;
          head_[depth] = e + 1;
          stack_[++depth] = c;
          done = false;
          break;
        }
      }
      if (done) {
        --depth;
        topo_[--top] = r;
      }
    }
  }

  int m_ = 0;
  std::vector<int64_t> lp_, up_;
  std::vector<int> li_, ui_;
  std::vector<double> lx_, ux_, ud_;
  std::vector<int> prow_, pos_, pinv_;
  std::vector<double> x_;
  std::vector<int> mark_, stack_, topo_, rowcnt_;
  std::vector<int64_t> head_;
  mutable std::vector<double> w_;
};

// ---- basis: LU plus product-form etas -----------------------------------

class Basis {
 public:
  Basis(const Lp& A, const double* lower, const double* upper, int refactor_freq)
      : A_(A), lower_(lower), upper_(upper), freq_(std::max(1, refactor_freq)) {
    basic.resize(A.m);
    pos.assign((size_t)A.n + A.m, -1);
  }

  std::vector<int> basic;    // position -> variable
  std::vector<int> pos;      // variable -> position or -1
  int factorizations = 0, repairs = 0;

  uint8_t nonbasic_status(int j) const {
    const double lo = lower_[j], up = upper_[j];
    if (lo <= -kBound && up >= kBound) return kFree;
    if (up - lo <= 0.0) return kFixed;
    if (lo > -kBound) return kAtLower;
    return kAtUpper;
  }

  void set_logical(uint8_t* status) {
    for (int i = 0; i < A_.m; ++i) basic[i] = A_.n + i;
    for (int j = 0; j < A_.n; ++j) status[j] = nonbasic_status(j);
    for (int i = 0; i < A_.m; ++i) status[A_.n + i] = kBasic;
    refactor(status);
  }

  // Factor the current basis.  A dependent column is replaced by the logical
  // of a row that the failed factorisation left without a pivot and whose
  // logical is nonbasic; that always terminates (the all-logical basis is -I).
  void refactor(uint8_t* status) {
    for (int attempt = 0; attempt <= A_.m + 1; ++attempt) {
      const int bad = lu_.factor(A_, basic.data());
      if (bad < 0) {
        ++factorizations;
        clear_etas();
        std::fill(pos.begin(), pos.end(), -1);
        for (int p = 0; p < A_.m; ++p) pos[basic[p]] = p;
        return;
      }
      std::vector<char> held(A_.m, 0);
      for (int p = 0; p < A_.m; ++p)
        if (basic[p] >= A_.n) held[basic[p] - A_.n] = 1;
      int row = -1;
      for (int i = 0; i < A_.m && row < 0; ++i)
        if (!held[i] && !lu_.pivoted(i)) row = i;
      for (int i = 0; i < A_.m && row < 0; ++i)
        if (!held[i]) row = i;
      const int leaving = basic[bad];
      status[leaving] = nonbasic_status(leaving);
      basic[bad] = A_.n + row;
      status[A_.n + row] = kBasic;
      ++repairs;
    }
  }

  // out (zeroed, length m) += M[:, j]
  void column(int j, double* out) const {
    if (j < A_.n) {
      for (int64_t e = A_.cp[j]; e < A_.cp[j + 1]; ++e) out[A_.ci[e]] = A_.cx[e];
    } else {
      out[j - A_.n] = -1.0;
    }
  }

  void ftran(double* v) const {
    lu_.ftran(v);
    for (size_t e = 0; e + 1 < es_.size(); ++e) {
      const int r = er_[e];
      double zr = v[r];
      if (zr == 0.0) continue;
      zr /= ep_[e];
      v[r] = zr;
      for (int64_t k = es_[e]; k < es_[e + 1]; ++k) v[ei_[k]] -= ex_[k] * zr;
    }
  }

  void btran(double* v) const {
    for (size_t e = es_.size() - 1; e-- > 0;) {
      const int r = er_[e];
      double s = v[r];
      for (int64_t k = es_[e]; k < es_[e + 1]; ++k) s -= ex_[k] * v[ei_[k]];
      v[r] = s / ep_[e];
    }
    lu_.btran(v);
  }

  // Variable q replaces basic[r]; alpha = B^-1 M[:, q] (by position).
  // Returns the leaving variable.
  int update(int r, int q, const double* alpha) {
    for (int i = 0; i < A_.m; ++i)
      if (i != r && alpha[i] != 0.0) { ei_.push_back(i); ex_.push_back(alpha[i]); }
    er_.push_back(r);
    ep_.push_back(alpha[r]);
    es_.push_back((int64_t)ei_.size());
    const int leaving = basic[r];
    basic[r] = q;
    pos[leaving] = -1;
    pos[q] = r;
    return leaving;
  }

  bool needs_refactor() const { return (int)er_.size() >= freq_; }
  int64_t lu_nnz() const { return lu_.nnz(); }

 private:
  void clear_etas() {
    es_.assign(1, 0); ei_.clear(); ex_.clear(); er_.clear(); ep_.clear();
  }

  const Lp& A_;
  const double* lower_;
  const double* upper_;
  int freq_;
  LuFactor lu_;
  std::vector<int64_t> es_{0};
  std::vector<int> ei_, er_;
  std::vector<double> ex_, ep_;
};

// ---- basis identification ----------------------------------------------

struct Bounds {
  std::vector<double> lower, upper;
  Bounds(const pdlp_problem_desc& d) : lower((size_t)d.n + d.m), upper((size_t)d.n + d.m) {
    for (int j = 0; j < d.n; ++j) { lower[j] = d.col_lb[j]; upper[j] = d.col_ub[j]; }
    for (int i = 0; i < d.m; ++i) { lower[d.n + i] = d.row_lb[i]; upper[d.n + i] = d.row_ub[i]; }
  }
};

// crossover.py:80-187.  Sums (A x by CSR rows, A^T y by CSC columns) run in
// storage order from zero, the order of sovopt's matvec / rmatvec kernels.
int identify(const Lp& A, const pdlp_problem_desc& d, const double* x, const double* y,
             double tol_fixed, double pivot_tol, uint8_t* status, pdlp_crossover_info* info) {
  const int m = A.m, n = A.n, N = n + m;
  Bounds bd(d);
  const double* lower = bd.lower.data();
  const double* upper = bd.upper.data();

  std::vector<double> z(N), dd(N, 0.0);
  for (int j = 0; j < n; ++j) z[j] = x[j];
  for (int i = 0; i < m; ++i) {
    double acc = 0.0;
    for (int64_t e = A.rp[i]; e < A.rp[i + 1]; ++e) acc += A.rx[e] * x[A.ri[e]];
    z[n + i] = acc;
  }
  if (y) {
    for (int j = 0; j < n; ++j) {
      double acc = 0.0;
      for (int64_t e = A.cp[j]; e < A.cp[j + 1]; ++e) acc += A.cx[e] * y[A.ci[e]];
      dd[j] = d.c[j] - acc;
    }
    for (int i = 0; i < m; ++i) dd[n + i] = y[i];
  }

  std::vector<char> fixed(N), free_(N), has_lo(N), has_hi(N);
  std::vector<double> score(N);
  for (int j = 0; j < N; ++j) {
    const double lo = lower[j], up = upper[j], zj = z[j];
    has_lo[j] = lo > -kBound;
    has_hi[j] = up < kBound;
    fixed[j] = has_lo[j] && has_hi[j] && (up - lo <= tol_fixed * std::max(1.0, std::fabs(lo)));
    free_[j] = !has_lo[j] && !has_hi[j];
    const double span = (has_lo[j] && has_hi[j]) ? up - lo : 0.0;
    const double scale = std::max(1.0, span > 0 ? span : std::fabs(zj));
    const double dlo = has_lo[j] ? zj - lo : kHuge;
    const double dhi = has_hi[j] ? up - zj : kHuge;
    double interior = std::min(dlo, dhi) / scale;
    if (!std::isfinite(interior)) interior = kHuge;
    double s = interior - 1e-9 * std::fabs(dd[j]);
    if (fixed[j]) s = -kHuge;
    if (free_[j]) s = kHuge;
    score[j] = s;
  }

  // candidates: free structurals first (index order), then the structurals
  // measurably off their bounds by decreasing score, ties by index
  std::vector<int> order;
  for (int j = 0; j < n; ++j)
    if (free_[j]) order.push_back(j);
  std::vector<int> live;
  for (int j = 0; j < n; ++j)
    if (score[j] > 1e-9 && std::isfinite(score[j])) live.push_back(j);
  std::stable_sort(live.begin(), live.end(),
                   [&](int a, int b) { return score[a] > score[b]; });
  for (int j : live)
    if (!free_[j]) order.push_back(j);

  // push into the all-logical basis (Basis' default of 60 etas between
  // refactorisations, lp/basis.py:137)
  std::vector<uint8_t> bstat(N);
  Basis B(A, lower, upper, 60);
  B.set_logical(bstat.data());
  std::vector<char> taken(m, 0);
  std::vector<double> alpha(m);
  int placed = 0, rejected = 0;
  for (int j : order) {
    if (placed == m) break;
    std::fill(alpha.begin(), alpha.end(), 0.0);
    B.column(j, alpha.data());
    B.ftran(alpha.data());
    int r = 0;
    double best = -1.0;
    for (int i = 0; i < m; ++i) {
      const double v = taken[i] ? 0.0 : std::fabs(alpha[i]);
      if (v > best) { best = v; r = i; }
    }
    if (m == 0 || best <= pivot_tol) { ++rejected; continue; }
    const int leaving = B.update(r, j, alpha.data());
    bstat[leaving] = B.nonbasic_status(leaving);
    bstat[j] = kBasic;
    taken[r] = 1;
    ++placed;
    if (B.needs_refactor()) B.refactor(bstat.data());
  }

  for (int j = 0; j < N; ++j) {
    const bool at_lower = (std::fabs(z[j] - lower[j]) <= std::fabs(upper[j] - z[j])) || !has_hi[j];
    status[j] = (at_lower && has_lo[j]) ? kAtLower : (has_hi[j] ? kAtUpper : kFree);
    if (fixed[j]) status[j] = kFixed;
  }
  for (int p = 0; p < m; ++p) status[B.basic[p]] = kBasic;
  if (info) {
    info->placed = placed;
    info->candidates = (int32_t)order.size();
    info->rejected = rejected;
    info->factorizations = B.factorizations;
    info->repairs = B.repairs;
  }
  return PDLP_OK;
}

// ---- the simplex that finishes a crossover --------------------------------
//
// Works on a scaled copy of the LP (row and column factors that are powers
// of two, so scaling and unscaling are exact): a few passes of geometric-mean
// scaling (each row, then each column, divided by the square root of its
// smallest and largest magnitude).  Tolerances apply to the scaled model, as
// in the reference's simplex (simplex.py:1207).

struct Model {
  Lp A;                       // scaled matrix, CSR and CSC
  std::vector<double> cx, rx; // scaled values behind A.cx and A.rx
  std::vector<double> cost;   // n + m: scaled c, 0 on logicals
  std::vector<double> lower, upper;   // n + m, scaled
  std::vector<double> R, C;   // row and column factors
};

inline double pow2_near(double v) {
  if (!(v > 0) || !std::isfinite(v)) return 1.0;
  return std::ldexp(1.0, (int)std::lround(std::log2(v)));
}

void build_model(const pdlp_problem_desc& d, Model& M) {
  const int m = d.m, n = d.n;
  M.cx.assign(d.cx, d.cx + d.nnz);
  M.R.assign(m, 1.0);
  M.C.assign(n, 1.0);
  std::vector<double> lo(m), hi(n > m ? n : m);
  for (int pass = 0; pass < 6; ++pass) {
    std::vector<double> rmin(m, kHuge), rmax(m, 0.0);
    for (int j = 0; j < n; ++j)
      for (int64_t e = d.cp[j]; e < d.cp[j + 1]; ++e) {
        const double a = std::fabs(M.cx[e]);
        if (a == 0.0) continue;
        const int i = d.ci[e];
        rmin[i] = std::min(rmin[i], a);
        rmax[i] = std::max(rmax[i], a);
      }
    for (int i = 0; i < m; ++i) {
      const double f = rmax[i] > 0 ? pow2_near(1.0 / std::sqrt(rmin[i] * rmax[i])) : 1.0;
      M.R[i] *= f;
      rmin[i] = f;   // this pass's factor
    }
    for (int j = 0; j < n; ++j) {
      double cmin = kHuge, cmax = 0.0;
      for (int64_t e = d.cp[j]; e < d.cp[j + 1]; ++e) {
        M.cx[e] *= rmin[d.ci[e]];
        const double a = std::fabs(M.cx[e]);
        if (a == 0.0) continue;
        cmin = std::min(cmin, a);
        cmax = std::max(cmax, a);
      }
      const double f = cmax > 0 ? pow2_near(1.0 / std::sqrt(cmin * cmax)) : 1.0;
      M.C[j] *= f;
      for (int64_t e = d.cp[j]; e < d.cp[j + 1]; ++e) M.cx[e] *= f;
    }
  }
  M.rx.resize(d.nnz);
  for (int i = 0; i < m; ++i)
    for (int64_t e = d.rp[i]; e < d.rp[i + 1]; ++e) M.rx[e] = d.rx[e] * M.R[i] * M.C[d.ri[e]];
  M.A = Lp{m, n, d.rp, d.ri, M.rx.data(), d.cp, d.ci, M.cx.data()};
  M.cost.assign((size_t)n + m, 0.0);
  M.lower.resize((size_t)n + m);
  M.upper.resize((size_t)n + m);
  auto sc = [](double b, double f) { return std::fabs(b) >= kBound ? b : b * f; };
  for (int j = 0; j < n; ++j) {
    M.cost[j] = d.c[j] * M.C[j];
    M.lower[j] = sc(d.col_lb[j], 1.0 / M.C[j]);
    M.upper[j] = sc(d.col_ub[j], 1.0 / M.C[j]);
  }
  for (int i = 0; i < m; ++i) {
    M.lower[n + i] = sc(d.row_lb[i], M.R[i]);
    M.upper[n + i] = sc(d.row_ub[i], M.R[i]);
  }
}

class Simplex {
 public:
  Simplex(const Model& M, const pdlp_simplex_params& p)
      : M_(M), A_(M.A), p_(p), m_(M.A.m), n_(M.A.n), N_(M.A.n + M.A.m),
        lower_(M.lower.data()), upper_(M.upper.data()),
        B_(M.A, M.lower.data(), M.upper.data(), p.refactor_freq) {
    cost_ = M.cost;
    st_.resize(N_);
    zB_.assign(m_, 0.0); pi_.assign(m_, 0.0); rho_.assign(m_, 0.0); tau_.assign(m_, 0.0);
    alpha_.assign(m_, 0.0); dj_.assign(N_, 0.0); arow_.assign(N_, 0.0);
    t0_ = std::chrono::steady_clock::now();
  }

  // Start from a status vector with exactly m BASIC entries, else from the
  // all-logical basis with every nonbasic at the bound its cost prefers
  // (simplex.py:1214-1225).
  void start(const uint8_t* warm) {
    int nb = 0;
    if (warm)
      for (int j = 0; j < N_; ++j) nb += warm[j] == kBasic;
    if (warm && nb == m_) {
      int p = 0;
      for (int j = 0; j < N_; ++j) {
        if (warm[j] == kBasic) { st_[j] = kBasic; B_.basic[p++] = j; }
        else st_[j] = sane_status(j, warm[j]);
      }
      B_.refactor(st_.data());
    } else {
      B_.set_logical(st_.data());
      for (int j = 0; j < n_; ++j) st_[j] = cost_status(j);
    }
    basic_values();
  }

  int run(pdlp_simplex_info* info) {
    int status = PDLP_STATUS_ITERATION_LIMIT;
    for (int round = 0; round < 8; ++round) {
      basic_values();
      if (primal_infeasibility() > p_.feas_tol) {
        // make the basis dual feasible (boxed nonbasics to the bound their
        // reduced cost wants, cost shifts on the rest), then the dual simplex
        duals();
        int shifted = 0;
        for (int j = 0; j < N_; ++j) {
          if (st_[j] == kBasic || dual_violation(j) <= p_.opt_tol) continue;
          if (lower_[j] > -kBound && upper_[j] < kBound && st_[j] != kFixed) {
            st_[j] = dj_[j] < 0 ? kAtUpper : kAtLower;
          } else {
            cost_[j] -= dj_[j];
            ++shifted;
          }
        }
        shifts_ += shifted;
        basic_values();
        int s = dual_loop();
        cost_ = M_.cost;
        if (s == PDLP_STATUS_INFEASIBLE || s == PDLP_STATUS_NUMERICAL) {
          // confirm (or recover) with the composite primal phase 1
          s = primal_loop(1);
          if (s != PDLP_STATUS_OPTIMAL) { status = s; break; }
          B_.refactor(st_.data());
          basic_values();
          if (primal_infeasibility() > 10 * std::max(p_.feas_tol, 1e-6)) {
            status = PDLP_STATUS_INFEASIBLE;
            break;
          }
        } else if (s != PDLP_STATUS_OPTIMAL) {
          status = s;
          break;
        }
      }
      status = primal_loop(2);
      if (status != PDLP_STATUS_OPTIMAL) break;
      B_.refactor(st_.data());
      basic_values();
      duals();
      if (primal_infeasibility() <= p_.feas_tol && dual_infeasibility() <= p_.opt_tol) break;
      status = PDLP_STATUS_ITERATION_LIMIT;
    }
    cost_ = M_.cost;
    B_.refactor(st_.data());
    basic_values();
    duals();
    if (info) {
      info->status = status;
      info->phase = phase1_ ? 1 : 2;
      info->iterations = iters_;
      info->phase1_iterations = phase1_iters_;
      info->bound_flips = flips_;
      info->degenerate_pivots = degenerate_;
      info->factorizations = B_.factorizations;
      info->repairs = B_.repairs;
      info->primal_infeasibility = primal_infeasibility();
      info->dual_infeasibility = dual_infeasibility();
      info->lu_nnz = B_.lu_nnz();
      info->dual_iterations = dual_iters_;
      info->cost_shifts = shifts_;
    }
    return status;
  }

  // Unscaled x (n), y (m), d (n) and the statuses.
  void write(double* x, double* y, double* dcost, uint8_t* status) const {
    for (int j = 0; j < n_; ++j) x[j] = value(j) * M_.C[j];
    for (int i = 0; i < m_; ++i) y[i] = pi_[i] * M_.R[i];
    for (int j = 0; j < n_; ++j) dcost[j] = st_[j] == kBasic ? 0.0 : dj_[j] / M_.C[j];
    std::memcpy(status, st_.data(), (size_t)N_);
  }

 private:
  uint8_t sane_status(int j, uint8_t s) const {
    const bool lo = lower_[j] > -kBound, hi = upper_[j] < kBound;
    if (!lo && !hi) return kFree;
    if (hi && lo && upper_[j] - lower_[j] <= 0.0) return kFixed;
    if (s == kAtUpper && hi) return kAtUpper;
    if (s == kAtLower && lo) return kAtLower;
    return lo ? kAtLower : kAtUpper;
  }

  uint8_t cost_status(int j) const {
    const bool lo = lower_[j] > -kBound, hi = upper_[j] < kBound;
    if (!lo && !hi) return kFree;
    if (hi && lo && upper_[j] - lower_[j] <= 0.0) return kFixed;
    if (cost_[j] >= 0.0) return lo ? kAtLower : kAtUpper;
    return hi ? kAtUpper : kAtLower;
  }

  double value(int j) const { return st_[j] == kBasic ? zB_[B_.pos[j]] : nb_value(j); }

  double nb_value(int j) const {
    switch (st_[j]) {
      case kAtLower: case kFixed: return lower_[j];
      case kAtUpper: return upper_[j];
      default: return 0.0;
    }
  }

  // rows += M[:, j] * v
  void add_column(int j, double v, double* rows) const {
    if (j < n_) {
      for (int64_t e = A_.cp[j]; e < A_.cp[j + 1]; ++e) rows[A_.ci[e]] += A_.cx[e] * v;
    } else {
      rows[j - n_] -= v;
    }
  }

  double column_dot(int j, const double* rows) const {
    if (j >= n_) return -rows[j - n_];
    double acc = 0.0;
    for (int64_t e = A_.cp[j]; e < A_.cp[j + 1]; ++e) acc += A_.cx[e] * rows[A_.ci[e]];
    return acc;
  }

  // z_B = B^-1 (-M_N z_N), with one step of iterative refinement
  void basic_values() {
    std::vector<double> rhs(m_, 0.0), res(m_);
    for (int j = 0; j < N_; ++j) {
      if (st_[j] == kBasic) continue;
      const double v = nb_value(j);
      if (v != 0.0) add_column(j, -v, rhs.data());
    }
    std::copy(rhs.begin(), rhs.end(), zB_.begin());
    B_.ftran(zB_.data());
    std::copy(rhs.begin(), rhs.end(), res.begin());
    for (int p = 0; p < m_; ++p)
      if (zB_[p] != 0.0) add_column(B_.basic[p], -zB_[p], res.data());
    B_.ftran(res.data());
    for (int p = 0; p < m_; ++p) zB_[p] += res[p];
  }

  double violation(int p) const {
    const int j = B_.basic[p];
    const double z = zB_[p];
    if (z < lower_[j]) return lower_[j] - z;
    if (z > upper_[j]) return z - upper_[j];
    return 0.0;
  }

  double primal_infeasibility() const {
    double worst = 0.0;
    for (int p = 0; p < m_; ++p) worst = std::max(worst, violation(p));
    return worst;
  }

  // pi = B^-T c_B and d_j = c_j - M_j' pi for every nonbasic j, with the
  // working costs (phase 2, possibly shifted) or the composite phase-1
  // costs (-1 below a bound, +1 above, on the basics only)
  void duals(bool phase1 = false) {
    for (int p = 0; p < m_; ++p) {
      const int j = B_.basic[p];
      if (!phase1) {
        pi_[p] = cost_[j];
      } else {
        const double z = zB_[p];
        pi_[p] = z < lower_[j] - p_.feas_tol ? -1.0 : (z > upper_[j] + p_.feas_tol ? 1.0 : 0.0);
      }
    }
    B_.btran(pi_.data());
    for (int j = 0; j < N_; ++j)
      dj_[j] = st_[j] == kBasic ? 0.0 : (phase1 ? 0.0 : cost_[j]) - column_dot(j, pi_.data());
  }

  // How far d_j has the wrong sign for variable j's status (0 when none).
  double dual_violation(int j) const {
    const double d = dj_[j];
    switch (st_[j]) {
      case kAtLower: return d < 0.0 ? -d : 0.0;
      case kAtUpper: return d > 0.0 ? d : 0.0;
      case kFree: return std::fabs(d);
      default: return 0.0;
    }
  }

  double dual_infeasibility() const {
    double worst = 0.0;
    for (int j = 0; j < N_; ++j) worst = std::max(worst, dual_violation(j));
    return worst;
  }

  bool out_of_time() const {
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
    return s > p_.time_limit;
  }

  // q enters at position r (its value moved by step_q); returns true when
  // the basis was refactorised (and the basic values recomputed)
  bool pivot(int r, int q, double step_q, uint8_t leaving_status) {
    const double enter = nb_value(q) + step_q;
    const int leaving = B_.basic[r];
    zB_[r] = enter;
    B_.update(r, q, alpha_.data());
    st_[q] = kBasic;
    const bool fixed = lower_[leaving] > -kBound && upper_[leaving] < kBound &&
                       upper_[leaving] - lower_[leaving] <= 0.0;
    st_[leaving] = fixed ? kFixed : leaving_status;
    ++iters_;
    if (B_.needs_refactor()) {
      B_.refactor(st_.data());
      basic_values();
      return true;
    }
    return false;
  }

  // Bounded dual simplex from a dual feasible basis: the most infeasible
  // basic leaves, to the bound it violates; the entering column comes from a
  // Harris two-pass dual ratio test on the pivot row rho' M.  Returns
  // OPTIMAL when the basis is primal feasible, INFEASIBLE when a row admits
  // no entering column (a dual ray), NUMERICAL when the pivot read from the
  // row and from the column keep disagreeing.
  int dual_loop() {
    int disagree = 0;
    dse_.assign(m_, 1.0);
    duals();
    for (;;) {
      if (iters_ >= p_.max_iter) return PDLP_STATUS_ITERATION_LIMIT;
      if ((iters_ & 63) == 0 && out_of_time()) return PDLP_STATUS_TIME_LIMIT;
      // leaving: the largest infeasibility^2 / steepest-edge weight
      int r = -1;
      double best = 0.0;
      for (int p = 0; p < m_; ++p) {
        const double v = violation(p);
        if (v <= p_.feas_tol) continue;
        const double sc = v * v / dse_[p];
        if (sc > best) { best = sc; r = p; }
      }
      if (r < 0) return PDLP_STATUS_OPTIMAL;
      const int jr = B_.basic[r];
      const bool to_lower = zB_[r] < lower_[jr];
      const double target = to_lower ? lower_[jr] : upper_[jr];
      // rho = B^-T e_r and the pivot row rho' M, row by row over rho's support
      std::fill(rho_.begin(), rho_.end(), 0.0);
      rho_[r] = 1.0;
      B_.btran(rho_.data());
      std::fill(arow_.begin(), arow_.end(), 0.0);
      double wr = 0.0;
      for (int i = 0; i < m_; ++i) {
        const double v = rho_[i];
        if (v == 0.0) continue;
        wr += v * v;
        for (int64_t e = A_.rp[i]; e < A_.rp[i + 1]; ++e) arow_[A_.ri[e]] += A_.rx[e] * v;
        arow_[n_ + i] = -v;
      }
      const double sg = to_lower ? -1.0 : 1.0;
      double bound = kHuge;
      for (int j = 0; j < N_; ++j) {
        double dd;
        const double a = arow_[j];
        if (a == 0.0 || st_[j] == kBasic || !dual_candidate(j, a, sg, dd)) continue;
        bound = std::min(bound, (dd + p_.opt_tol) / std::fabs(a));
      }
      if (bound == kHuge) return PDLP_STATUS_INFEASIBLE;
      int q = -1;
      double qa = 0.0;
      for (int j = 0; j < N_; ++j) {
        double dd;
        const double a = arow_[j];
        if (a == 0.0 || st_[j] == kBasic || !dual_candidate(j, a, sg, dd)) continue;
        if (dd / std::fabs(a) <= bound && std::fabs(a) > qa) { qa = std::fabs(a); q = j; }
      }
      if (q < 0) return PDLP_STATUS_NUMERICAL;
      std::fill(alpha_.begin(), alpha_.end(), 0.0);
      B_.column(q, alpha_.data());
      B_.ftran(alpha_.data());
      if (std::fabs(alpha_[r] - arow_[q]) > 1e-6 * (1.0 + std::fabs(alpha_[r]))) {
        if (++disagree > 3) return PDLP_STATUS_NUMERICAL;
        B_.refactor(st_.data());
        basic_values();
        duals();
        continue;
      }
      disagree = 0;
      // steepest-edge weights ||e_p' B^-1||^2 after the pivot (tau = B^-1 rho)
      std::copy(rho_.begin(), rho_.end(), tau_.begin());
      B_.ftran(tau_.data());
      const double ar = alpha_[r];
      for (int p = 0; p < m_; ++p) {
        if (p == r || alpha_[p] == 0.0) continue;
        const double k = alpha_[p] / ar;
        dse_[p] = std::max(dse_[p] - 2.0 * k * tau_[p] + k * k * wr, 1e-6);
      }
      dse_[r] = std::max(wr / (ar * ar), 1e-6);
      // reduced costs: d_j -= theta * (rho' M_j); the leaving one becomes
      // -theta.  An entering d_q of the wrong sign (within the Harris
      // tolerance) is shifted to zero first, so theta never has the wrong
      // sign; a d_j the step pushes past opt_tol is shifted back to zero.
      // Shifts leave the true costs at the end (the primal simplex cleans up).
      if (dual_violation(q) > 0.0) {
        cost_[q] -= dj_[q];
        dj_[q] = 0.0;
        ++shifts_;
      }
      const double theta = dj_[q] / arow_[q];
      for (int j = 0; j < N_; ++j) {
        if (arow_[j] == 0.0 || st_[j] == kBasic) continue;
        dj_[j] -= theta * arow_[j];
        if (j != q && dual_violation(j) > p_.opt_tol) {
          cost_[j] -= dj_[j];
          dj_[j] = 0.0;
          ++shifts_;
        }
      }
      dj_[q] = 0.0;
      dj_[jr] = -theta;
      const double step = (zB_[r] - target) / ar;   // change of z_q
      for (int p = 0; p < m_; ++p) zB_[p] -= alpha_[p] * step;
      if (step == 0.0) ++degenerate_;
      ++dual_iters_;
      if (pivot(r, q, step, to_lower ? kAtLower : kAtUpper)) duals();
    }
  }

  // Is nonbasic j, with pivot-row entry a, a dual ratio-test candidate when
  // the leaving variable must move by sign -sg?  dd is its reduced cost's
  // distance from changing sign (0 when slightly infeasible).
  bool dual_candidate(int j, double a, double sg, double& dd) const {
    if (std::fabs(a) <= p_.pivot_tol) return false;
    const double d = dj_[j];
    switch (st_[j]) {
      case kAtLower: if (sg * a <= 0) return false; dd = std::max(d, 0.0); return true;
      case kAtUpper: if (sg * a >= 0) return false; dd = std::max(-d, 0.0); return true;
      case kFree: dd = std::fabs(d); return true;
      default: return false;
    }
  }

  // Bounded primal simplex (phase 1: composite costs; phase 2: the working
  // costs).  Devex pricing (reference weights, Forrest & Goldfarb 1992;
  // Bland's rule after 50 degenerate pivots in a row), Harris two-pass ratio
  // test with bound flips.  In phase 2 the reduced costs are updated from
  // the pivot row; phase 1 recomputes them, since its costs change as basics
  // reach their bounds.
  int primal_loop(int phase) {
    int degenerate_run = 0;
    bool bland = false;
    if (phase == 1) phase1_ = true;
    std::vector<double> w(N_, 1.0);
    duals(phase == 1);
    for (;;) {
      if (iters_ >= p_.max_iter) return PDLP_STATUS_ITERATION_LIMIT;
      if ((iters_ & 63) == 0 && out_of_time()) return PDLP_STATUS_TIME_LIMIT;
      if (phase == 1) duals(true);
      int q = -1;
      double best = 0.0;
      for (int j = 0; j < N_; ++j) {
        const double v = dual_violation(j);
        if (v <= p_.opt_tol) continue;
        if (bland) { q = j; break; }
        const double sc = v * v / w[j];
        if (sc > best) { best = sc; q = j; }
      }
      if (q < 0) {
        if (phase == 1) return PDLP_STATUS_OPTIMAL;
        // confirm with freshly computed reduced costs
        duals();
        bool clean = true;
        for (int j = 0; j < N_ && clean; ++j) clean = dual_violation(j) <= p_.opt_tol;
        if (clean) return PDLP_STATUS_OPTIMAL;
        continue;
      }
      const double dir = st_[q] == kAtUpper ? -1.0 : (st_[q] == kAtLower ? 1.0 : (dj_[q] > 0 ? -1.0 : 1.0));
      std::fill(alpha_.begin(), alpha_.end(), 0.0);
      B_.column(q, alpha_.data());
      B_.ftran(alpha_.data());

      double theta = kHuge;
      for (int p = 0; p < m_; ++p) {
        double tgt, dist, rate;
        if (!blocking(p, dir, tgt, dist, rate)) continue;
        theta = std::min(theta, (dist + p_.feas_tol) / std::fabs(rate));
      }
      const double range = (lower_[q] > -kBound && upper_[q] < kBound) ? upper_[q] - lower_[q] : kHuge;
      if (range <= theta && range < kHuge) {
        for (int p = 0; p < m_; ++p) zB_[p] -= dir * alpha_[p] * range;
        st_[q] = st_[q] == kAtLower ? kAtUpper : kAtLower;
        ++iters_; ++flips_;
        if (phase == 1) ++phase1_iters_;
        degenerate_run = 0;
        continue;
      }
      if (theta == kHuge) return phase == 2 ? PDLP_STATUS_UNBOUNDED : PDLP_STATUS_NUMERICAL;
      int r = -1;
      double rbest = 0.0, step = 0.0, rtgt = 0.0;
      int rvar = std::numeric_limits<int>::max();
      for (int p = 0; p < m_; ++p) {
        double tgt, dist, rate;
        if (!blocking(p, dir, tgt, dist, rate)) continue;
        const double t = dist / std::fabs(rate);
        if (t > theta) continue;
        const double a = std::fabs(alpha_[p]);
        const bool better = bland ? B_.basic[p] < rvar : a > rbest;
        if (better) { r = p; rbest = a; step = t; rtgt = tgt; rvar = B_.basic[p]; }
      }
      if (r < 0) return PDLP_STATUS_NUMERICAL;
      // pivot row rho' M (rho = B^-T e_r) for the weights and reduced costs
      std::fill(rho_.begin(), rho_.end(), 0.0);
      rho_[r] = 1.0;
      B_.btran(rho_.data());
      std::fill(arow_.begin(), arow_.end(), 0.0);
      for (int i = 0; i < m_; ++i) {
        const double v = rho_[i];
        if (v == 0.0) continue;
        for (int64_t e = A_.rp[i]; e < A_.rp[i + 1]; ++e) arow_[A_.ri[e]] += A_.rx[e] * v;
        arow_[n_ + i] = -v;
      }
      const double ar = alpha_[r];
      const double wq = w[q];
      const int leaving = B_.basic[r];
      for (int j = 0; j < N_; ++j) {
        if (arow_[j] == 0.0 || st_[j] == kBasic) continue;
        const double k = arow_[j] / ar;
        w[j] = std::max(w[j], k * k * wq);
      }
      w[leaving] = std::max(wq / (ar * ar), 1.0);
      if (phase == 2) {
        const double th = dj_[q] / ar;
        for (int j = 0; j < N_; ++j)
          if (arow_[j] != 0.0 && st_[j] != kBasic) dj_[j] -= th * arow_[j];
        dj_[q] = 0.0;
        dj_[leaving] = -th;
      }
      for (int p = 0; p < m_; ++p) zB_[p] -= dir * alpha_[p] * step;
      if (phase == 1) ++phase1_iters_;
      if (step == 0.0) {
        ++degenerate_;
        if (++degenerate_run > 50) bland = true;
      } else {
        degenerate_run = 0;
        bland = false;
      }
      if (pivot(r, q, dir * step, rtgt == lower_[leaving] ? kAtLower : kAtUpper) && phase == 2) duals();
    }
  }

  // Does basic position p block a step in direction dir?  Returns the bound
  // it stops at, its distance (>= 0) and its rate of change.
  bool blocking(int p, double dir, double& tgt, double& dist, double& rate) const {
    const double a = alpha_[p];
    if (std::fabs(a) <= p_.pivot_tol) return false;
    rate = -dir * a;
    const int j = B_.basic[p];
    const double z = zB_[p], lo = lower_[j], up = upper_[j];
    if (rate < 0.0) {
      if (z > up + p_.feas_tol) tgt = up;              // infeasible above: stops at up
      else if (z >= lo - p_.feas_tol && lo > -kBound) tgt = lo;
      else return false;
      dist = std::max(0.0, z - tgt);
    } else {
      if (z < lo - p_.feas_tol) tgt = lo;              // infeasible below: stops at lo
      else if (z <= up + p_.feas_tol && up < kBound) tgt = up;
      else return false;
      dist = std::max(0.0, tgt - z);
    }
    return true;
  }

  const Model& M_;
  const Lp& A_;
  pdlp_simplex_params p_;
  int m_, n_, N_;
  const double* lower_;
  const double* upper_;
  Basis B_;
  std::vector<double> cost_;
  std::vector<uint8_t> st_;
  std::vector<double> zB_, pi_, rho_, tau_, alpha_, dj_, arow_, dse_;
  int64_t iters_ = 0, phase1_iters_ = 0, dual_iters_ = 0, flips_ = 0, degenerate_ = 0, shifts_ = 0;
  bool phase1_ = false;
  std::chrono::steady_clock::time_point t0_;
};

int check_host_problem(const pdlp_problem_desc* d, bool need_csr) {
  if (!d) return fail(PDLP_ERR_ARG, "problem is NULL");
  if (d->memory != PDLP_MEM_HOST) return fail(PDLP_ERR_ARG, "crossover needs host arrays");
  if (d->m < 0 || d->n < 0) return fail(PDLP_ERR_ARG, "negative dimension");
  if (!d->cp || (d->nnz > 0 && (!d->ci || !d->cx)))
    return fail(PDLP_ERR_ARG, "CSC arrays of A are required");
  if (need_csr && (!d->rp || (d->nnz > 0 && (!d->ri || !d->rx))))
    return fail(PDLP_ERR_ARG, "CSR arrays of A are required");
  if ((d->n > 0 && (!d->c || !d->col_lb || !d->col_ub)) ||
      (d->m > 0 && (!d->row_lb || !d->row_ub)))
    return fail(PDLP_ERR_ARG, "cost or bound arrays missing");
  if (d->cp[0] != 0 || d->cp[d->n] != d->nnz) return fail(PDLP_ERR_ARG, "CSC pointers malformed");
  for (int j = 0; j < d->n; ++j)
    if (d->cp[j + 1] < d->cp[j]) return fail(PDLP_ERR_ARG, "CSC pointers decrease");
  for (int64_t e = 0; e < d->nnz; ++e)
    if (d->ci[e] < 0 || d->ci[e] >= d->m) return fail(PDLP_ERR_ARG, "CSC row index out of range");
  if (need_csr) {
    if (d->rp[0] != 0 || d->rp[d->m] != d->nnz) return fail(PDLP_ERR_ARG, "CSR pointers malformed");
    for (int i = 0; i < d->m; ++i)
      if (d->rp[i + 1] < d->rp[i]) return fail(PDLP_ERR_ARG, "CSR pointers decrease");
    for (int64_t e = 0; e < d->nnz; ++e)
      if (d->ri[e] < 0 || d->ri[e] >= d->n) return fail(PDLP_ERR_ARG, "CSR column index out of range");
  }
  return PDLP_OK;
}

}  // namespace xo
}  // namespace pdlp

using namespace pdlp::xo;

extern "C" {

int pdlp_simplex_default_params(pdlp_simplex_params* p) {
  if (!p) return pdlp::fail(PDLP_ERR_ARG, "params is NULL");
  p->feas_tol = 1e-7;
  p->opt_tol = 1e-7;
  p->pivot_tol = 1e-7;
  p->max_iter = 1000000;
  p->time_limit = 300.0;
  p->refactor_freq = 150;
  p->reserved = 0;
  return PDLP_OK;
}

int pdlp_basis_from_point(const pdlp_problem_desc* prob, const double* x, const double* y,
                          double tol_fixed, double pivot_tol, uint8_t* status_out,
                          pdlp_crossover_info* info) {
  const int rc = check_host_problem(prob, true);
  if (rc != PDLP_OK) return rc;
  if ((prob->n > 0 && !x) || !status_out) return pdlp::fail(PDLP_ERR_ARG, "x or status_out is NULL");
  for (int j = 0; j < prob->n; ++j)
    if (!std::isfinite(x[j])) return pdlp::fail(PDLP_ERR_NUMERICAL, "x is not finite");
  const auto t0 = std::chrono::steady_clock::now();
  Lp A{prob->m, prob->n, prob->rp, prob->ri, prob->rx, prob->cp, prob->ci, prob->cx};
  if (info) std::memset(info, 0, sizeof(*info));
  const int r = identify(A, *prob, x, y, tol_fixed, pivot_tol, status_out, info);
  if (info) info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

int pdlp_simplex_solve(const pdlp_problem_desc* prob, const pdlp_simplex_params* params,
                       const uint8_t* warm_status, double* x, double* y, double* d,
                       uint8_t* basis_status, pdlp_simplex_info* info) {
  const int rc = check_host_problem(prob, true);
  if (rc != PDLP_OK) return rc;
  if ((prob->n > 0 && (!x || !d)) || (prob->m > 0 && !y) || !basis_status)
    return pdlp::fail(PDLP_ERR_ARG, "output array is NULL");
  pdlp_simplex_params p;
  pdlp_simplex_default_params(&p);
  if (params) p = *params;
  if (!(p.feas_tol > 0) || !(p.opt_tol > 0) || !(p.pivot_tol > 0) || p.refactor_freq < 1)
    return pdlp::fail(PDLP_ERR_ARG, "tolerances must be positive and refactor_freq >= 1");
  if (warm_status)
    for (int64_t j = 0; j < (int64_t)prob->n + prob->m; ++j)
      if (warm_status[j] > kFixed) return pdlp::fail(PDLP_ERR_ARG, "unknown basis status");
  const auto t0 = std::chrono::steady_clock::now();
  if (info) std::memset(info, 0, sizeof(*info));
  Model M;
  build_model(*prob, M);
  Simplex S(M, p);
  S.start(warm_status);
  S.run(info);
  S.write(x, y, d, basis_status);
  if (info) {
    double obj = 0.0;
    for (int j = 0; j < prob->n; ++j) obj += prob->c[j] * x[j];
    info->objective = obj;
  }
  if (info) info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return PDLP_OK;
}

}  // extern "C"
