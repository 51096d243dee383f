// engine.cpp -- host orchestration of the batched Newton-Raphson engine.
//
// The NR loop follows NewtonSolver::run_iteration_stages
// (cuPF/cpp/src/newton_solver/core/newton_solver.cpp:497-558): evaluate the
// mismatch and its norm, stop when the batch maximum is within tolerance
// (checked before the Jacobian, so the converged state is not perturbed),
// otherwise Jacobian -> factorize -> solve -> voltage update.  The iteration
// count is shared by the batch and reported per scenario; per-scenario
// convergence is final_mismatch <= tol (newton_solver.cpp:321-341).
#include "engine.hpp"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>

#include "kernels.hpp"
#include "static_scratch.hpp"

namespace cupf_b200 {

#define CUPF_CUDA(expr)                                                                                   \
  do {                                                                                                    \
    cudaError_t _e = (expr);                                                                              \
    if (_e != cudaSuccess)                                                                                \
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(_e) + " at " #expr);      \
  } while (0)

namespace {

// CUPF_DEBUG_SYNC=1: synchronize and check for an error after every launch
// (diagnostics; off by default, never inside a graph capture).
bool debug_sync() {
  static const bool on = [] {
    const char* v = std::getenv("CUPF_DEBUG_SYNC");
    return v && v[0] == '1';
  }();
  return on;
}

void debug_check(cudaStream_t s, const char* what) {
  if (!debug_sync()) return;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cs);
  if (cs != cudaStreamCaptureStatusNone) return;
  cudaError_t e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string("CUDA error after ") + what + ": " + cudaGetErrorString(e));
}

struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void reserve(size_t nbytes) {
    if (nbytes <= bytes && p) return;
    release();
    if (nbytes == 0) nbytes = 16;
    CUPF_CUDA(cudaMalloc(&p, nbytes));
    bytes = nbytes;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(p);
  }
  template <typename T>
  void upload(const std::vector<T>& v) {
    reserve(std::max<size_t>(v.size(), 1) * sizeof(T));
    if (!v.empty()) CUPF_CUDA(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  }
};

template <typename T>
std::vector<long long> to_ll(const std::vector<T>& v) {
  return std::vector<long long>(v.begin(), v.end());
}

}  // namespace

struct Engine::Impl {
  // grid
  DBuf y_ptr, y_col, y_row, y_diag, y_re, y_im, map11, map21, map12, map22, bus_fa, bus_fm, bus_fa_p, bus_fm_p, pv, pq,
      jt_ptr, jt_row, jt_q;
  // factor program
  DBuf fsz, nc, first, front_ptr, front_rows, u_off, l_off, cb_off, tv_off, arow_ptr, arow_q, arow_col, crow_ptr,
      crow_child, crow_r, crow_src, crow_dst, asm_ptr, asm_local, perm, iperm, row_iperm, col_perm, level_fronts, fe_split, fe_dst, fe_src, front_meta;
  std::vector<LevelLaunch> levels;
  // backward sweep: the narrow top levels (launch-list entries from bw_first
  // on) run as one launch over bw_bounds (descending level boundaries)
  int bw_first = 0, bw_nlev = 0;
  LevelLaunch bw_top;
  DBuf bw_bounds;
  // the front tree of the single-system factorization launch (SingleTree)
  DBuf tree_parent, tree_nchild, tree_e0, tree_leaves, tree_done;
  int tree_max_fsz = 0, tree_list_cap = 0, tree_leaf_count = 0;
  int64_t tv_total = 0;
  DevGrid g;
  DevPlan pl;
  // workspace
  int Bp_cap = 0, B = 0, Bp = 0;
  DBuf v_re, v_im, va, vm, s_re, s_im, i_re, i_im, F, Fp, norm, sing;
  bool state_f32 = false;  // ComputePolicy::FP32: the arrays above up to F hold float (reserved at 8 bytes)
  bool fp_double = false;
  DBuf J, U, L, CB, Y, X, front_scratch;
  size_t front_scratch_elems = 0;
  DBuf stage_in, stage_out, fin;
  DBuf G, R, lam, dlam, TV, W, Z, Jd, red;
  DBuf yb_re, yb_im;           // per-scenario Ybus values [nnz_y][Bp]
  bool yb_active = false;      // the current batch uses them
  const void* graph_yb = nullptr;  // yb pointer baked into the captured iteration
  unsigned long long* h_norm = nullptr;
  double* h_final = nullptr;
  int h_cap = 0;
  cudaStream_t own = nullptr;
  // stage timers
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pairs;
  cudaEvent_t ev_open[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  double stage_ms[5] = {0, 0, 0, 0, 0};
  int64_t stage_launches[5] = {0, 0, 0, 0, 0};
  cudaEvent_t next_event() {
    if (ev_used == ev_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev_pool.push_back(e);
    }
    return ev_pool[ev_used++];
  }
  // graph of a whole solve: the first mismatch and its test, then a WHILE
  // node around (update, mismatch, test); per batch size, precision and Ybus
  cudaGraphExec_t exec = nullptr;
  int graph_Bp = -1;
  bool graph_double = false;
  int64_t graph_body_launches = 0;
  DBuf ctl, fin_dev;           // LoopCtl, final norms [Bp]
  LoopCtl* h_ctl = nullptr;    // pinned
  // batch size and precision the factor and backward launches were tuned for
  int tuned_Bp = -1, tuned_bw_Bp = -1;
  bool tuned_double = false, tuned_bw_double = false, tuned_single = false;
  bool graph_single = false;  // the graph's factor launches use the single-system schedule
  void invalidate_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    graph_Bp = -1;
  }

  ~Impl() {
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    if (exec) cudaGraphExecDestroy(exec);
    if (h_norm) cudaFreeHost(h_norm);
    if (h_final) cudaFreeHost(h_final);
    if (h_ctl) cudaFreeHost(h_ctl);
    if (own) cudaStreamDestroy(own);
  }

  DevState state() const {
    DevState st;
    st.B = B;
    st.Bp = Bp;
    st.state_f32 = state_f32 ? 1 : 0;
    st.v_re = v_re.as<double>();
    st.v_im = v_im.as<double>();
    st.va = va.as<double>();
    st.vm = vm.as<double>();
    st.s_re = s_re.as<double>();
    st.s_im = s_im.as<double>();
    st.i_re = i_re.as<double>();
    st.i_im = i_im.as<double>();
    // the mismatch in Jacobian-row order is written only for evaluate_host();
    // the Newton loop reads F in pivot order (Fp) and its norm
    st.F = nullptr;
    st.Fp = Fp.p;
    st.fp_double = fp_double ? 1 : 0;
    st.norm_bits = norm.as<unsigned long long>();
    st.sing = sing.as<int>();
    st.yb_re = yb_active ? yb_re.as<double>() : nullptr;
    st.yb_im = yb_active ? yb_im.as<double>() : nullptr;
    return st;
  }
};

Engine::Engine(const EngineConfig& cfg) : d_(new Impl()), cfg_(cfg) {
  if (cfg_.max_panel_width < 1 || cfg_.max_panel_width > 8)
    throw std::invalid_argument("max_panel_width must be in [1, 8] for this engine");
  d_->state_f32 = cfg_.compute == kComputeFP32;
}

Engine::~Engine() = default;

// FP32 state cannot carry FP64 factors: under ComputePolicy::FP32 an FP64
// factor precision falls back to FP32, as the reference's custom solver does
// (cuda_custom_solver.cpp:71-72); TF32 stays available.
bool Engine::factor_is_double() const {
  return cfg_.compute == kComputeFP64 || (cfg_.compute != kComputeFP32 && cfg_.factor_precision == kFactorFP64);
}

bool Engine::tf32_factors() const { return cfg_.factor_precision == kFactorTF32 && !factor_is_double(); }

bool Engine::single_system() const { return cfg_.batch1_schedule == 0 && d_->B == 1; }

// The single-system factorization as one tree launch: batch 1, no
// tensor-core launch among the levels, every front and list in shared memory.
bool Engine::single_tree(size_t elem_bytes) const {
  if (!single_system()) return false;
  for (const auto& lv : d_->levels)
    if (lv.tier == 2) return false;
  return single_smem_bytes(d_->tree_max_fsz, d_->tree_list_cap, elem_bytes) <= kSmemLimit;
}

void Engine::assign_tiers(int tc_min) {
  const int wide_min = std::min(cfg_.wide_min_front > 0 ? cfg_.wide_min_front : kWideFrontRows, kWideFrontRows);
  tc_min_ = tf32_factors() ? tc_min : 0;
  for (auto& lv : d_->levels) {
    lv.tier = lv.max_fsz >= wide_min ? 1 : 0;
    if (tc_min_ > 0 && lv.max_fsz >= tc_min_) lv.tier = 2;
  }
}

std::vector<int32_t> Engine::factor_level_tiers() const {
  std::vector<int32_t> t;
  for (const auto& lv : d_->levels) t.push_back(lv.tier);
  return t;
}

void Engine::initialize(int32_t n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                        const int32_t* pv, int32_t n_pv, const int32_t* pq, int32_t n_pq) {
  if (!indptr || !indices || !ydata) throw std::invalid_argument("initialize: Ybus arrays must not be null");
  analyze_host(n_bus, indptr, indices, pv, n_pv, pq, n_pq);

  auto& d = *d_;
  const int32_t nnz_y = indptr[n_bus];
  std::vector<int32_t> yptr(indptr, indptr + n_bus + 1), ycol(indices, indices + nnz_y), yrow(nnz_y),
      ydiag(n_bus, -1);
  std::vector<double> yre(nnz_y), yim(nnz_y);
  for (int32_t r = 0; r < n_bus; ++r)
    for (int32_t k = indptr[r]; k < indptr[r + 1]; ++k) {
      yrow[k] = r;
      if (indices[k] == r) ydiag[r] = k;
    }
  for (int32_t k = 0; k < nnz_y; ++k) {
    yre[k] = ydata[2 * k];
    yim[k] = ydata[2 * k + 1];
  }
  d.y_ptr.upload(yptr);
  d.y_col.upload(ycol);
  d.y_row.upload(yrow);
  d.y_diag.upload(ydiag);
  d.y_re.upload(yre);
  d.y_im.upload(yim);
  d.map11.upload(ja_.map11);
  d.map21.upload(ja_.map21);
  d.map12.upload(ja_.map12);
  d.map22.upload(ja_.map22);
  d.bus_fa.upload(ja_.row_pvpq);
  d.bus_fm.upload(ja_.row_pq);
  {
    std::vector<int32_t> fa_p(n_bus, -1), fm_p(n_bus, -1);
    for (int32_t i = 0; i < n_bus; ++i) {
      // equation rows go where the row ordering puts them
      if (ja_.row_pvpq[i] >= 0) fa_p[i] = fp_.row_iperm[ja_.row_pvpq[i]];
      if (ja_.row_pq[i] >= 0) fm_p[i] = fp_.row_iperm[ja_.row_pq[i]];
    }
    d.bus_fa_p.upload(fa_p);
    d.bus_fm_p.upload(fm_p);
  }
  d.pv.upload(std::vector<int32_t>(pv, pv + n_pv));
  d.pq.upload(std::vector<int32_t>(pq, pq + n_pq));
  // J^T as CSR over J's positions (csr_transpose.cpp:257-289, own layout)
  {
    std::vector<int32_t> tp(ja_.dim + 1, 0), trow(ja_.nnz), tq(ja_.nnz);
    for (int32_t q = 0; q < ja_.nnz; ++q) tp[ja_.col_idx[q] + 1]++;
    for (int32_t c = 0; c < ja_.dim; ++c) tp[c + 1] += tp[c];
    std::vector<int32_t> cur(tp.begin(), tp.end() - 1);
    for (int32_t r = 0; r < ja_.dim; ++r)
      for (int32_t q = ja_.row_ptr[r]; q < ja_.row_ptr[r + 1]; ++q) {
        const int32_t dst = cur[ja_.col_idx[q]]++;
        trow[dst] = r;
        tq[dst] = q;
      }
    d.jt_ptr.upload(tp);
    d.jt_row.upload(trow);
    d.jt_q.upload(tq);
  }
  upload_plan();

  DevGrid& g = d.g;
  g.n_bus = n_bus;
  g.nnz_y = nnz_y;
  g.dim = ja_.dim;
  g.nnz_j = ja_.nnz;
  g.n_pv = n_pv;
  g.n_pq = n_pq;
  g.y_ptr = d.y_ptr.as<int>();
  g.y_col = d.y_col.as<int>();
  g.y_row = d.y_row.as<int>();
  g.y_diag = d.y_diag.as<int>();
  g.jac_kind = cfg_.jacobian_kind;
  g.y_re = d.y_re.as<double>();
  g.y_im = d.y_im.as<double>();
  g.map11 = d.map11.as<int>();
  g.map21 = d.map21.as<int>();
  g.map12 = d.map12.as<int>();
  g.map22 = d.map22.as<int>();
  g.bus_fa = d.bus_fa.as<int>();
  g.bus_fm = d.bus_fm.as<int>();
  g.bus_fa_p = d.bus_fa_p.as<int>();
  g.bus_fm_p = d.bus_fm_p.as<int>();
  g.pv = d.pv.as<int>();
  g.pq = d.pq.as<int>();
  g.jt_ptr = d.jt_ptr.as<int>();
  g.jt_row = d.jt_row.as<int>();
  g.jt_q = d.jt_q.as<int>();
  if (!d.own) CUPF_CUDA(cudaStreamCreateWithFlags(&d.own, cudaStreamNonBlocking));
  if (d.exec) {
    cudaGraphExecDestroy(d.exec);
    d.exec = nullptr;
    d.graph_Bp = -1;
  }
  initialized_ = true;
  adjoint_ready_ = false;
}

void Engine::update_ybus_values(const double* ydata) {
  auto& d = *d_;
  const size_t nnz = ja_.map11.size();
  std::vector<double> yre(nnz), yim(nnz);
  for (size_t k = 0; k < nnz; ++k) {
    yre[k] = ydata[2 * k];
    yim[k] = ydata[2 * k + 1];
  }
  d.y_re.upload(yre);
  d.y_im.upload(yim);
  adjoint_ready_ = false;
}

void Engine::upload_plan() {
  auto& d = *d_;
  d.fsz.upload(fp_.fsz);
  d.nc.upload(fp_.nc);
  d.first.upload(fp_.first);
  d.front_ptr.upload(fp_.front_ptr);
  d.front_rows.upload(fp_.front_rows);
  d.u_off.upload(to_ll(fp_.u_off));
  d.l_off.upload(to_ll(fp_.l_off));
  d.cb_off.upload(to_ll(fp_.cb_off));
  {
    std::vector<long long> tv(fp_.P + 1, 0);
    for (int32_t p = 0; p < fp_.P; ++p) tv[p + 1] = tv[p] + (fp_.fsz[p] - fp_.nc[p]);
    d.tv_total = tv[fp_.P];
    d.tv_off.upload(tv);
    // the sweeps' gather list: each child entry's update-vector element and
    // its row in the parent front (entries are grouped by front row)
    const size_t ne = fp_.crow_child.size();
    std::vector<long long> src(std::max<size_t>(ne, 1), 0);
    std::vector<int32_t> dst(std::max<size_t>(ne, 1), 0);
    for (int32_t p = 0; p < fp_.P; ++p)
      for (int32_t i = 0; i < fp_.fsz[p]; ++i) {
        const int32_t fr = fp_.front_ptr[p] + i;
        for (int32_t e = fp_.crow_ptr[fr]; e < fp_.crow_ptr[fr + 1]; ++e) {
          src[e] = tv[fp_.crow_child[e]] + fp_.crow_r[e];
          dst[e] = i;
        }
      }
    d.crow_src.upload(src);
    d.crow_dst.upload(dst);
  }
  d.arow_ptr.upload(fp_.arow_ptr);
  d.arow_q.upload(fp_.arow_q);
  d.arow_col.upload(fp_.arow_col);
  d.crow_ptr.upload(fp_.crow_ptr);
  d.crow_child.upload(fp_.crow_child);
  d.crow_r.upload(fp_.crow_r);
  d.asm_ptr.upload(fp_.asm_ptr);
  d.asm_local.upload(fp_.asm_local);
  d.perm.upload(fp_.perm);
  d.iperm.upload(fp_.iperm);
  d.row_iperm.upload(fp_.row_iperm);
  d.col_perm.upload(fp_.col_perm);
  d.level_fronts.upload(fp_.level_fronts);
  d.fe_split.upload(to_ll(fp_.fe_split));

  d.front_meta.upload(fp_.front_meta);
  // Launch list: each level of the front tree, cut into runs of similar front
  // size (fronts are size-sorted inside a level) when both sides of a cut
  // hold enough fronts to fill the GPU, so that the shared memory of a launch
  // is sized for its own fronts rather than the level's largest.
  d.levels.clear();
  auto bucket = [](int32_t f) {
    for (int32_t c : {6, 8, 10, 12, 16, 20, 24, 32, 48, 64})
      if (f <= c) return c;
    return 1 << 30;
  };
  constexpr int32_t kMinRun = 64;
  for (int32_t L = 0; L < fp_.num_levels; ++L) {
    const int32_t b0 = fp_.level_ptr[L], b1 = fp_.level_ptr[L + 1];
    std::vector<int32_t> cuts{b0};
    for (int32_t q = b0 + 1; q < b1; ++q) {
      if (bucket(fp_.fsz[fp_.level_fronts[q]]) == bucket(fp_.fsz[fp_.level_fronts[q - 1]])) continue;
      if (q - cuts.back() >= kMinRun && b1 - q >= kMinRun) cuts.push_back(q);
    }
    cuts.push_back(b1);
    for (size_t c = 0; c + 1 < cuts.size(); ++c) {
      LevelLaunch lv;
      lv.begin = cuts[c];
      lv.count = cuts[c + 1] - cuts[c];
      for (int32_t q = lv.begin; q < lv.begin + lv.count; ++q) {
        const int32_t f = fp_.level_fronts[q];
        lv.max_fsz = std::max(lv.max_fsz, fp_.fsz[f]);
        lv.max_nc = std::max(lv.max_nc, fp_.nc[f]);
        lv.max_src = std::max<int>(lv.max_src, (int)(fp_.fe_ptr[f + 1] - fp_.fe_ptr[f]));
      }
      d.levels.push_back(lv);
    }
  }
  assign_tiers(cfg_.tc_min_front > 0 ? cfg_.tc_min_front : kTcDefaultMinFront);
  // The top of the tree for the backward sweep: the trailing levels of at
  // most kBackwardTopFronts fronts.
  d.bw_first = (int)d.levels.size();
  d.bw_nlev = 0;
  d.bw_top = LevelLaunch{};
  {
    constexpr int32_t kBackwardTopFronts = 8;
    int32_t Ls = fp_.num_levels;
    while (Ls > 0 && fp_.level_ptr[Ls] - fp_.level_ptr[Ls - 1] <= kBackwardTopFronts) --Ls;
    if (fp_.num_levels - Ls >= 2) {
      std::vector<int32_t> bounds;
      for (int32_t L = fp_.num_levels; L >= Ls; --L) bounds.push_back(fp_.level_ptr[L]);
      d.bw_bounds.upload(bounds);
      d.bw_nlev = fp_.num_levels - Ls;
      LevelLaunch& t = d.bw_top;
      t.begin = fp_.level_ptr[Ls];
      t.count = fp_.P - t.begin;
      for (int32_t q = t.begin; q < fp_.P; ++q) {
        const int32_t f = fp_.level_fronts[q];
        t.max_fsz = std::max(t.max_fsz, fp_.fsz[f]);
        t.max_nc = std::max(t.max_nc, fp_.nc[f]);
      }
      d.bw_first = 0;
      while (d.bw_first < (int)d.levels.size() && d.levels[d.bw_first].begin < t.begin) ++d.bw_first;
    }
  }
  // source lists in launch order, each padded to its launch's longest
  {
    std::vector<long long> psrc;
    std::vector<int32_t> pdst;
    for (auto& lv : d.levels) {
      lv.max_src = std::max(lv.max_src, 1);
      lv.fe_base = (long long)psrc.size();
      for (int32_t q = lv.begin; q < lv.begin + lv.count; ++q) {
        const int32_t f = fp_.level_fronts[q];
        const int64_t a = fp_.fe_ptr[f], z = fp_.fe_ptr[f + 1];
        for (int64_t e = a; e < z; ++e) {
          psrc.push_back(fp_.fe_src[e]);
          pdst.push_back(fp_.fe_dst[e]);
        }
        for (int64_t e = z - a; e < lv.max_src; ++e) {
          psrc.push_back(0);
          pdst.push_back(-1);
        }
      }
    }
    d.fe_src.upload(psrc);
    d.fe_dst.upload(pdst);
  }
  // the front tree in level order for the single-system launch: each front's
  // parent and child count (the assembly's children are the tree's), and
  // where its list starts in the padded lists
  {
    const int32_t P = fp_.P;
    std::vector<int32_t> qof(P, -1), parent(P, -1), nchild(P, 0);
    std::vector<long long> e0(P, 0);
    for (int32_t q = 0; q < P; ++q) qof[fp_.level_fronts[q]] = q;
    for (int32_t q = 0; q < P; ++q) {
      const int32_t pf = sp_.panel_parent[fp_.level_fronts[q]];
      if (pf >= 0) {
        parent[q] = qof[pf];
        ++nchild[qof[pf]];
      }
    }
    d.tree_max_fsz = 0;
    d.tree_list_cap = 1;
    for (const auto& lv : d.levels) {
      for (int32_t q = lv.begin; q < lv.begin + lv.count; ++q)
        e0[q] = lv.fe_base + (long long)(q - lv.begin) * lv.max_src;
      d.tree_max_fsz = std::max(d.tree_max_fsz, lv.max_fsz);
      d.tree_list_cap = std::max(d.tree_list_cap, lv.max_src);
    }
    std::vector<int32_t> leaves;
    for (int32_t q = 0; q < P; ++q)
      if (nchild[q] == 0) leaves.push_back(q);
    d.tree_leaf_count = (int)leaves.size();
    d.tree_parent.upload(parent);
    d.tree_nchild.upload(nchild);
    d.tree_e0.upload(e0);
    d.tree_leaves.upload(leaves);
    d.tree_done.reserve(((size_t)P + 1) * sizeof(int));
  }

  DevPlan& pl = d.pl;
  pl.P = fp_.P;
  pl.dim = fp_.dim;
  pl.nnz = fp_.nnz;
  pl.fsz = d.fsz.as<int>();
  pl.nc = d.nc.as<int>();
  pl.first = d.first.as<int>();
  pl.front_ptr = d.front_ptr.as<int>();
  pl.front_rows = d.front_rows.as<int>();
  pl.u_off = d.u_off.as<long long>();
  pl.l_off = d.l_off.as<long long>();
  pl.cb_off = d.cb_off.as<long long>();
  pl.tv_off = d.tv_off.as<long long>();
  pl.arow_ptr = d.arow_ptr.as<int>();
  pl.arow_q = d.arow_q.as<int>();
  pl.arow_col = d.arow_col.as<int>();
  pl.crow_ptr = d.crow_ptr.as<int>();
  pl.crow_child = d.crow_child.as<int>();
  pl.crow_r = d.crow_r.as<int>();
  pl.crow_src = d.crow_src.as<long long>();
  pl.crow_dst = d.crow_dst.as<int>();
  pl.asm_ptr = d.asm_ptr.as<int>();
  pl.asm_local = d.asm_local.as<int>();
  pl.perm = d.perm.as<int>();
  pl.iperm = d.iperm.as<int>();
  pl.row_iperm = d.row_iperm.as<int>();
  pl.col_perm = d.col_perm.as<int>();
  pl.level_fronts = d.level_fronts.as<int>();
  pl.fe_split = d.fe_split.as<long long>();
  pl.fe_dst = d.fe_dst.as<int>();
  pl.fe_src = d.fe_src.as<long long>();
  pl.front_meta = d.front_meta.as<int>();
  if (!d.own) CUPF_CUDA(cudaStreamCreateWithFlags(&d.own, cudaStreamNonBlocking));
  if (d.exec) {
    cudaGraphExecDestroy(d.exec);
    d.exec = nullptr;
    d.graph_Bp = -1;
  }
  d.Bp_cap = 0;
}

void Engine::analyze_host(int32_t n_bus, const int32_t* indptr, const int32_t* indices, const int32_t* pv,
                          int32_t n_pv, const int32_t* pq, int32_t n_pq) {
  initialized_ = false;
  adjoint_ready_ = false;
  ja_ = analyze_jacobian(n_bus, indptr, indices, pv, n_pv, pq, n_pq);
  SymbolicOptions so;
  so.max_panel_width = cfg_.max_panel_width;
  so.serial_nd = cfg_.serial_nd != 0;
  so.use_matching = cfg_.use_matching != 0;
  so.par_nd_depth = cfg_.par_nd_depth;
  so.par_nd_base_small = cfg_.par_nd_base_small;
  so.par_nd_base_large = cfg_.par_nd_base_large;
  sp_ = analyze_symbolic(ja_.dim, ja_.row_ptr.data(), ja_.col_idx.data(), so);
  fp_ = build_factor_program(sp_);
}

void Engine::analyze_matrix_host(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx) {
  if (n <= 0 || nnz < 0 || !row_ptr || !col_idx) throw std::invalid_argument("SetData: invalid CSR pattern");
  if (row_ptr[n] != nnz) throw std::invalid_argument("SetData: row_ptr[n] != nnz");
  initialized_ = false;
  adjoint_ready_ = false;
  ja_ = JacobianAnalysis();
  ja_.dim = n;
  ja_.nnz = nnz;
  ja_.row_ptr.assign(row_ptr, row_ptr + n + 1);
  ja_.col_idx.assign(col_idx, col_idx + nnz);
  SymbolicOptions so;
  so.max_panel_width = cfg_.max_panel_width;
  so.serial_nd = cfg_.serial_nd != 0;
  so.use_matching = cfg_.use_matching != 0;
  so.par_nd_depth = cfg_.par_nd_depth;
  so.par_nd_base_small = cfg_.par_nd_base_small;
  so.par_nd_base_large = cfg_.par_nd_base_large;
  sp_ = analyze_symbolic(n, row_ptr, col_idx, so);
  fp_ = build_factor_program(sp_);
}

void Engine::initialize_matrix(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx) {
  if (n <= 0 || nnz < 0 || !row_ptr || !col_idx) throw std::invalid_argument("SetData: invalid CSR pattern");
  if (row_ptr[n] != nnz) throw std::invalid_argument("SetData: row_ptr[n] != nnz");
  ja_ = JacobianAnalysis();
  ja_.dim = n;
  ja_.nnz = nnz;
  ja_.row_ptr.assign(row_ptr, row_ptr + n + 1);
  ja_.col_idx.assign(col_idx, col_idx + nnz);
  SymbolicOptions so;
  so.max_panel_width = cfg_.max_panel_width;
  so.serial_nd = cfg_.serial_nd != 0;
  so.use_matching = cfg_.use_matching != 0;
  so.par_nd_depth = cfg_.par_nd_depth;
  so.par_nd_base_small = cfg_.par_nd_base_small;
  so.par_nd_base_large = cfg_.par_nd_base_large;
  sp_ = analyze_symbolic(n, row_ptr, col_idx, so);
  fp_ = build_factor_program(sp_);
  upload_plan();
  initialized_ = true;
  adjoint_ready_ = false;
}

void Engine::ensure_workspace(int32_t B) {
  if (!initialized_) throw std::runtime_error("NewtonSolver::solve_batch(): initialize() must be called first");
  if (B <= 0) throw std::invalid_argument("NewtonSolver::solve_batch(): batch_size must be positive");
  auto& d = *d_;
  const int Bp = (B + kWarp - 1) / kWarp * kWarp;
  d.B = B;
  d.Bp = Bp;
  if (Bp > d.Bp_cap) {
    const size_t n = ja_.n_bus, dim = ja_.dim;
    const size_t es = factor_is_double() ? sizeof(double) : sizeof(float);
    for (DBuf* b : {&d.v_re, &d.v_im, &d.va, &d.vm, &d.s_re, &d.s_im, &d.i_re, &d.i_im}) b->reserve(n * Bp * 8);
    d.F.reserve(dim * Bp * 8);
    d.Fp.reserve(dim * Bp * es);
    d.fp_double = factor_is_double();
    if (d.fp_double)
      configure_front_kernels<double, double>();
    else
      configure_front_kernels<float, float>();
    d.norm.reserve(Bp * 8);
    d.sing.reserve(Bp * 4);
    d.J.reserve((size_t)ja_.nnz * Bp * es);
    d.U.reserve((size_t)fp_.u_total * Bp * es);
    d.L.reserve((size_t)std::max<int64_t>(fp_.l_total, 1) * Bp * es);
    d.CB.reserve((size_t)std::max<int64_t>(fp_.cb_total, 1) * Bp * es);
    d.Y.reserve(dim * Bp * es);
    d.X.reserve(dim * Bp * es);
    // dense fronts of levels too large for shared memory (and every wide-tier
    // front) live in global scratch; one launch at a time uses it
    size_t scratch = 0;
    for (const auto& lv : d.levels) {
      LevelLaunch widest = lv;  // the tier with the largest scratch this launch may be given
      if (tf32_factors() && lv.max_fsz >= std::min(tc_min_ > 0 ? tc_min_ : kTcSmallestMinFront, kTcSmallestMinFront))
        widest.tier = 2;
      scratch = std::max({scratch, level_scratch_capacity(lv, es, Bp / kWarp),
                          level_scratch_capacity(widest, es, Bp / kWarp)});
    }
    d.front_scratch_elems = scratch;
    if (scratch) d.front_scratch.reserve(scratch * kWarp * es);
    // The allocation-free entry point's static area: the runtime loads the
    // module that holds it (and reserves its memory) at the first lookup of
    // its address, so that lookup happens here, in a call that allocates,
    // and never in the first allocation-free factorization.
    static_front_scratch();
    d.Bp_cap = Bp;
    if (d.exec) {
      cudaGraphExecDestroy(d.exec);
      d.exec = nullptr;
      d.graph_Bp = -1;
    }
    adjoint_ready_ = false;
  }
  if (Bp > d.h_cap) {
    if (d.h_norm) cudaFreeHost(d.h_norm);
    if (d.h_final) cudaFreeHost(d.h_final);
    CUPF_CUDA(cudaMallocHost(&d.h_norm, Bp * sizeof(unsigned long long)));
    CUPF_CUDA(cudaMallocHost(&d.h_final, Bp * sizeof(double)));
    d.h_cap = Bp;
  }
  if (d.graph_Bp != Bp && d.exec) {
    cudaGraphExecDestroy(d.exec);
    d.exec = nullptr;
    d.graph_Bp = -1;
  }
}

namespace {
// NVTX ranges with the reference's stage labels (newton_solver.cpp:521-553,
// StageScope :42-50).  The v3 headers are header-only and do nothing unless a
// profiler is attached.
const char* const kStageNames[5] = {"NR.iteration.mismatch", "NR.iteration.jacobian", "NR.iteration.factorize",
                                    "NR.iteration.solve", "NR.iteration.voltage_update"};
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};
}  // namespace

void Engine::stage_begin(int stage, cudaStream_t s) {
  nvtxRangePushA(kStageNames[stage]);
  if (!profiling_) return;
  auto& d = *d_;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(s, &cs);
  if (cs != cudaStreamCaptureStatusNone) return;
  d.ev_open[stage] = d.next_event();
  cudaEventRecord(d.ev_open[stage], s);
}

void Engine::stage_end(int stage, cudaStream_t s) {
  nvtxRangePop();
  if (!profiling_) return;
  auto& d = *d_;
  if (!d.ev_open[stage]) return;
  cudaEvent_t e = d.next_event();
  cudaEventRecord(e, s);
  d.ev_pairs.push_back({stage, {d.ev_open[stage], e}});
  d.ev_open[stage] = nullptr;
}

void Engine::collect_stage_times() {
  auto& d = *d_;
  for (auto& pr : d.ev_pairs) {
    float ms = 0.f;
    cudaEventSynchronize(pr.second.second);
    cudaEventElapsedTime(&ms, pr.second.first, pr.second.second);
    d.stage_ms[pr.first] += ms;
  }
  d.ev_pairs.clear();
  d.ev_used = 0;
}

void Engine::stage_times_ms(double* out5, int64_t* launches5) const {
  for (int i = 0; i < 5; ++i) {
    if (out5) out5[i] = d_->stage_ms[i];
    if (launches5) launches5[i] = d_->stage_launches[i];
  }
}

template <typename T>
FactorArgs<T, T> Engine::factor_args(int store_l, const void* J) const {
  const auto& d = *d_;
  FactorArgs<T, T> a;
  a.plan = d.pl;
  a.groups = d.Bp / kWarp;
  a.Bp = d.Bp;
  a.J = static_cast<const T*>(J);
  a.Fp = d.Fp.as<T>();
  a.U = d.U.as<T>();
  a.L = d.L.as<T>();
  a.CB = d.CB.as<T>();
  a.Y = d.Y.as<T>();
  a.store_l = store_l;
  a.eps = cfg_.shift_epsilon;
  a.static_pivot = (cfg_.static_pivot && cfg_.shift_epsilon > 0.0) ? 1 : 0;
  a.sing = d.sing.as<int>();
  a.front_scratch = d.front_scratch_elems ? d.front_scratch.as<T>() : nullptr;
  a.front_scratch_elems = d.front_scratch_elems;
  a.single = single_system() ? 1 : 0;
  return a;
}

namespace {

// Chooses a launch shape for each of n launches that run in sequence on
// stream s.  Candidate shapes are opaque codes (cand, none of them 0);
// set(i, code) gives launch i the shape code (0: its built-in rule);
// launch(i) issues it.  Every candidate and the rule each run the whole
// sequence three times with an event after every launch; a launch keeps the
// fastest candidate if it beats the rule by 3 % and by 0.5 us, else the rule.
// Then the whole sequence is timed as a solve runs it (chained launches, no
// events in between), three times with the choice and three with the rule;
// the choice stays only if it is at least 1 % faster.  Leaves the chosen
// shapes set; returns whether they were kept.
template <typename Set, typename Launch>
bool choose_block_shapes(size_t n, const std::vector<int>& cand, Set set, Launch launch, cudaStream_t s,
                         const char* what) {
  const size_t nc = cand.size();
  std::vector<double> t((nc + 1) * n, 1e30);  // [candidate 0..nc-1, rule = nc][launch]
  std::vector<cudaEvent_t> ev(n + 1, nullptr);
  auto cleanup = [&] {
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
  };
  std::vector<int> choice(n, 0);
  double whole[2] = {1e30, 1e30};  // [rule, choice]
  try {
    for (auto& e : ev) CUPF_CUDA(cudaEventCreate(&e));
    for (int rep = 0; rep < 3; ++rep)
      for (size_t c = 0; c <= nc; ++c) {
        for (size_t i = 0; i < n; ++i) set(i, c < nc ? cand[c] : 0);
        CUPF_CUDA(cudaEventRecord(ev[0], s));
        for (size_t i = 0; i < n; ++i) {
          launch(i);
          CUPF_CUDA(cudaEventRecord(ev[i + 1], s));
        }
        CUPF_CUDA(cudaEventSynchronize(ev[n]));
        for (size_t i = 0; i < n; ++i) {
          float ms = 0.f;
          CUPF_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
          double& cell = t[c * n + i];
          cell = std::min(cell, (double)ms);
        }
      }
    for (size_t i = 0; i < n; ++i) {
      const double rule = t[nc * n + i];
      int best = -1;
      double bt = std::min(rule * 0.97, rule - 0.5e-3);
      for (size_t c = 0; c < nc; ++c)
        if (t[c * n + i] < bt) {
          bt = t[c * n + i];
          best = (int)c;
        }
      choice[i] = best >= 0 ? cand[best] : 0;
    }
    for (int rep = 0; rep < 3; ++rep)
      for (int v = 0; v < 2; ++v) {
        for (size_t i = 0; i < n; ++i) set(i, v ? choice[i] : 0);
        CUPF_CUDA(cudaEventRecord(ev[0], s));
        for (size_t i = 0; i < n; ++i) launch(i);
        CUPF_CUDA(cudaEventRecord(ev[1], s));
        CUPF_CUDA(cudaEventSynchronize(ev[1]));
        float ms = 0.f;
        CUPF_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        whole[v] = std::min(whole[v], (double)ms);
      }
  } catch (...) {
    for (size_t i = 0; i < n; ++i) set(i, 0);
    cleanup();
    throw;
  }
  cleanup();
  const bool keep = whole[1] < 0.99 * whole[0];
  for (size_t i = 0; i < n; ++i) set(i, keep ? choice[i] : 0);
  if (debug_sync()) {
    std::fprintf(stderr, "[cupf] %s autotune: rule %.3f ms, choice %.3f ms, %s\n", what, whole[0], whole[1],
                 keep ? "kept" : "rule kept");
    for (size_t i = 0; i < n; ++i) {
      std::fprintf(stderr, "[cupf] %s launch %zu: rule %.2f us, chosen %d;", what, i, 1e3 * t[nc * n + i], choice[i]);
      for (size_t c = 0; c < nc; ++c) std::fprintf(stderr, " %d: %.2f", cand[c], 1e3 * t[c * n + i]);
      std::fprintf(stderr, "\n");
    }
  }
  return keep;
}

}  // namespace

// The autotuner of the factor launches: each block factors one front for 32
// scenarios and its warps split the staging, the assembly and the non-pivot
// rows, so every element sees the same operations in the same order whatever
// the split.  Tunes once per batch size and precision, on the values J.
template <typename T>
void Engine::autotune_factor(cudaStream_t s, const void* J) {
  auto& d = *d_;
  const bool dbl = std::is_same<T, double>::value;
  if (d.tuned_Bp == d.Bp && d.tuned_double == dbl && d.tuned_single == single_system()) return;
  if (single_system()) {
    // batch 1: the single-system kernel has no launch shapes to choose (the
    // tensor-core threshold of TF32 factors stays at its default)
    d.tuned_Bp = d.Bp;
    d.tuned_double = dbl;
    d.tuned_single = true;
    d.invalidate_graph();
    return;
  }
  const FactorArgs<T, T> a = factor_args<T>(1, J);
  if (tf32_factors() && cfg_.tc_min_front == 0) {
    // the small/large-front split of TF32 factors: the tensor-core threshold
    // whose whole factorization is fastest (three timings each, built-in
    // block shapes); a larger threshold must win by 1 %
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CUPF_CUDA(cudaEventCreate(&e0));
    CUPF_CUDA(cudaEventCreate(&e1));
    int best = kTcSmallestMinFront;
    double best_ms = 1e30;
    try {
      for (int t : {kTcSmallestMinFront, 49, 65}) {
        assign_tiers(t);
        double ms_t = 1e30;
        for (int rep = 0; rep < 3; ++rep) {
          CUPF_CUDA(cudaEventRecord(e0, s));
          for (const auto& lv : d.levels) launch_factor_level<T, T>(lv, a, s);
          CUPF_CUDA(cudaEventRecord(e1, s));
          CUPF_CUDA(cudaEventSynchronize(e1));
          float ms = 0.f;
          CUPF_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          ms_t = std::min(ms_t, (double)ms);
        }
        if (debug_sync()) std::fprintf(stderr, "[cupf] tensor-core threshold %d: %.3f ms\n", t, ms_t);
        if (ms_t < 0.99 * best_ms) {
          best = t;
          best_ms = ms_t;
        }
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      assign_tiers(kTcDefaultMinFront);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    assign_tiers(best);
  }
  // shapes: warps per block (1, 2, 4, 8), and for the register tier where
  // the dense fronts live (code = warps + 256 x placement: shared memory 1,
  // global scratch 2); and the wide tier with 8, 16 or 32 warps (placement
  // 3) for the launches of large fronts (the wide tier's own launches take
  // its 16 and 32 warps as their warp counts; other launches run their
  // built-in rule under these codes)
  std::vector<int> cand;
  for (int p : {1, 2})
    for (int w : {1, 2, 4, 8}) cand.push_back(w + 256 * p);
  for (int w : {8, 16, 32}) cand.push_back(w + 256 * 3);
  choose_block_shapes(
      d.levels.size(), cand,
      [&](size_t i, int code) {
        LevelLaunch& lv = d.levels[i];
        int w = code & 0xff, p = code >> 8;
        if (p == 3 && !(lv.tier == 1 || wide_option(lv))) w = p = 0;
        lv.warps = w;
        lv.placement = lv.tier == 0 ? p : 0;
      },
      [&](size_t i) { launch_factor_level<T, T>(d.levels[i], a, s); }, s, "factor");
  d.tuned_Bp = d.Bp;
  d.tuned_double = dbl;
  d.tuned_single = false;
  d.invalidate_graph();  // a captured solve holds the old launch shapes
}

// The same for the backward sweep (the tree-top launch, then the levels):
// each warp back-substitutes one front for 32 scenarios on its own, so the
// block shape only groups independent warps.  Reads the factors the last
// factorization left (U, Y) and rewrites X, as every sweep does.
template <typename T>
void Engine::autotune_backward(cudaStream_t s) {
  auto& d = *d_;
  const bool dbl = std::is_same<T, double>::value;
  if (d.tuned_bw_Bp == d.Bp && d.tuned_bw_double == dbl) return;
  const SweepArgs<T> a = sweep_args<T>();
  std::vector<LevelLaunch*> seq;
  if (d.bw_nlev > 0) seq.push_back(&d.bw_top);
  for (int l = d.bw_first - 1; l >= 0; --l) seq.push_back(&d.levels[l]);
  const bool has_top = d.bw_nlev > 0;
  choose_block_shapes(
      seq.size(), std::vector<int>{1, 2, 4, 8}, [&](size_t i, int w) { seq[i]->bw_wpb = w; },
      [&](size_t i) {
        if (i == 0 && has_top)
          launch_backward_top<T>(d.bw_top, d.bw_bounds.as<int>(), d.bw_nlev, a, s);
        else
          launch_backward_level<T>(*seq[i], a, s);
      },
      s, "backward");
  d.tuned_bw_Bp = d.Bp;
  d.tuned_bw_double = dbl;
  d.invalidate_graph();
}

template <typename T>
SweepArgs<T> Engine::sweep_args() const {
  const auto& d = *d_;
  SweepArgs<T> a;
  a.plan = d.pl;
  a.groups = d.Bp / kWarp;
  a.Bp = d.Bp;
  a.U = d.U.as<T>();
  a.Y = d.Y.as<T>();
  a.X = d.X.as<T>();
  return a;
}

std::vector<int32_t> Engine::factor_level_warps() const {
  std::vector<int32_t> w;
  for (const auto& lv : d_->levels) w.push_back(lv.warps);
  return w;
}

std::vector<int32_t> Engine::factor_level_placements() const {
  std::vector<int32_t> p;
  const size_t es = factor_is_double() ? sizeof(double) : sizeof(float);
  for (const auto& lv : d_->levels)
    p.push_back(lv.tier > 0 ? 2 : runs_wide(lv, es) ? 3 : (front_in_shared_memory(lv, es) ? 1 : 2));
  return p;
}

std::vector<int32_t> Engine::backward_launch_warps() const {
  std::vector<int32_t> w;
  if (d_->bw_nlev > 0) w.push_back(d_->bw_top.bw_wpb);
  for (int l = d_->bw_first - 1; l >= 0; --l) w.push_back(d_->levels[l].bw_wpb);
  return w;
}

template <typename T>
void Engine::factor_tree(const FactorArgs<T, T>& a, cudaStream_t s) {
  auto& d = *d_;
  SingleTree t;
  t.parent = d.tree_parent.as<int>();
  t.nchild = d.tree_nchild.as<int>();
  t.q_e0 = d.tree_e0.as<long long>();
  t.leaves = d.tree_leaves.as<int>();
  t.done = d.tree_done.as<int>();
  t.P = fp_.P;
  t.n_leaves = d.tree_leaf_count;
  t.max_fsz = d.tree_max_fsz;
  t.list_cap = d.tree_list_cap;
  CUPF_CUDA(cudaMemsetAsync(t.done, 0, ((size_t)t.P + 1) * sizeof(int), s));
  launch_factor_single_tree<T, T>(a, t, s);
}

template <typename T>
void Engine::factor_all(cudaStream_t s, int store_l, const void* J) {
  auto& d = *d_;
  const FactorArgs<T, T> a = factor_args<T>(store_l, J);
  stage_begin(2, s);
  if (single_tree(sizeof(T))) {
    factor_tree<T>(a, s);
    debug_check(s, "factor tree");
    ++launches_;
    ++d.stage_launches[2];
  } else {
    for (const auto& lv : d.levels) {
      launch_factor_level<T, T>(lv, a, s);
      debug_check(s, "factor level");
      ++launches_;
      ++d.stage_launches[2];
    }
  }
  stage_end(2, s);
}

template <typename T>
void Engine::backward_all(cudaStream_t s) {
  auto& d = *d_;
  const SweepArgs<T> a = sweep_args<T>();
  stage_begin(3, s);
  const int64_t n = backward_levels<T>(a, s);
  launches_ += n;
  d.stage_launches[3] += n;
  stage_end(3, s);
}

// Backward substitution over the whole tree, root first: the narrow top in
// one launch, then level by level.  Returns the launches made.
template <typename T>
int64_t Engine::backward_levels(const SweepArgs<T>& a, cudaStream_t s) {
  auto& d = *d_;
  int64_t n = 0;
  if (d.bw_nlev > 0) {
    launch_backward_top<T>(d.bw_top, d.bw_bounds.as<int>(), d.bw_nlev, a, s);
    debug_check(s, "backward tree top");
    ++n;
  }
  for (int L = d.bw_first - 1; L >= 0; --L) {
    launch_backward_level<T>(d.levels[L], a, s);
    debug_check(s, "backward level");
    ++n;
  }
  return n;
}

template <typename T>
void Engine::iteration_tail(cudaStream_t s, int store_l) {
  auto& d = *d_;
  const DevState st = d.state();
  stage_begin(1, s);
  launch_jacobian<T>(d.g, st, d.J.as<T>(), s);
  stage_end(1, s);
  debug_check(s, "jacobian");
  ++launches_;
  ++d.stage_launches[1];
  factor_all<T>(s, store_l, d.J.p);
  backward_all<T>(s);
  stage_begin(4, s);
  launch_voltage_update<T>(d.g, d.pl, st, d.X.as<T>(), s);
  stage_end(4, s);
  debug_check(s, "voltage update");
  ++launches_;
  ++d.stage_launches[4];
}

// Builds the graph of a whole solve for this batch size, precision and Ybus
// source: [mismatch, test] -> WHILE(test says "update") { Jacobian, factor,
// backward sweep, voltage update, mismatch, test }.  The test kernel sets the
// WHILE node's condition (a CUDA graph conditional node), so the iterations
// run back to back on the device and the host synchronises once per solve.
template <typename T>
void Engine::ensure_loop_graph(const DevState& st) {
  auto& d = *d_;
  const bool dbl = std::is_same<T, double>::value;
  if (d.exec && d.graph_Bp == d.Bp && d.graph_double == dbl && d.graph_yb == static_cast<const void*>(st.yb_re) &&
      d.graph_single == single_system())
    return;
  if (d.exec) cudaGraphExecDestroy(d.exec);
  d.exec = nullptr;
  d.graph_Bp = -1;
  d.ctl.reserve(sizeof(LoopCtl));
  d.fin_dev.reserve((size_t)d.Bp * sizeof(double));
  if (!d.h_ctl) CUPF_CUDA(cudaMallocHost(&d.h_ctl, sizeof(LoopCtl)));
  LoopCtl* ctl = d.ctl.as<LoopCtl>();
  auto* norm = d.norm.as<unsigned long long>();
  double* fin = d.fin_dev.as<double>();
  cudaStream_t cs = d.own;
  const int64_t before = launches_;
  cudaGraph_t graph = nullptr;
  CUPF_CUDA(cudaGraphCreate(&graph, 0));
  bool capturing = false;
  try {
    cudaGraphConditionalHandle h;
    CUPF_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
    CUPF_CUDA(cudaStreamBeginCaptureToGraph(cs, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    launch_ibus_mismatch(d.g, st, cs);
    launch_loop_check(h, ctl, norm, fin, cs);
    cudaStreamCaptureStatus cst;
    cudaGraph_t cap = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    CUPF_CUDA(cudaStreamGetCaptureInfo(cs, &cst, nullptr, &cap, &deps, &ndeps));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t wn;
    CUPF_CUDA(cudaGraphAddNode(&wn, cap, deps, ndeps, &p));
    CUPF_CUDA(cudaStreamUpdateCaptureDependencies(cs, &wn, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t done = nullptr;
    capturing = false;
    CUPF_CUDA(cudaStreamEndCapture(cs, &done));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    CUPF_CUDA(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    const int64_t b0 = launches_;
    iteration_tail<T>(cs, 0);
    d.graph_body_launches = (launches_ - b0) + 2;
    launch_ibus_mismatch(d.g, st, cs);
    launch_loop_check(h, ctl, norm, fin, cs);
    capturing = false;
    CUPF_CUDA(cudaStreamEndCapture(cs, &done));
    CUPF_CUDA(cudaGraphInstantiate(&d.exec, graph, 0));
  } catch (...) {
    if (capturing) {
      cudaGraph_t g2 = nullptr;
      cudaStreamEndCapture(cs, &g2);
    }
    cudaGraphDestroy(graph);
    launches_ = before;
    throw;
  }
  cudaGraphDestroy(graph);
  d.graph_Bp = d.Bp;
  d.graph_double = dbl;
  d.graph_single = single_system();
  d.graph_yb = st.yb_re;
  launches_ = before;
}

template <typename T>
SolveStats Engine::run_loop(double tol, int32_t max_iter, int32_t prepare_adjoint, cudaStream_t s, double* d_final,
                            double* d_v_out) {
  const NvtxRange range("NR.solve_batch");
  auto& d = *d_;
  const DevState st = d.state();
  SolveStats stats;
  launches_ = 0;
  adjoint_ready_ = false;
  if (cfg_.autotune && max_iter > 0 &&
      (d.tuned_Bp != d.Bp || d.tuned_double != std::is_same<T, double>::value || d.tuned_bw_Bp != d.Bp ||
       d.tuned_bw_double != std::is_same<T, double>::value || d.tuned_single != single_system())) {
    // tune on the Jacobian of the starting state (the loop recomputes it)
    launch_ibus_mismatch(d.g, st, s);
    launch_jacobian<T>(d.g, st, d.J.as<T>(), s);
    autotune_factor<T>(s, d.J.p);
    autotune_backward<T>(s);  // on the factors the factor tuning left
  }
  CUPF_CUDA(cudaMemsetAsync(d.norm.p, 0, d.Bp * sizeof(unsigned long long), s));
  CUPF_CUDA(cudaMemsetAsync(d.sing.p, 0, d.Bp * sizeof(int), s));
  for (int b = 0; b < d.B; ++b) d.h_final[b] = 0.0;
  int completed = 0;
  double gmax = 0.0;
  bool nonfinite = false;  // a tolerated scenario whose norm went non-finite
  for (int i = 0; i < 5; ++i) {
    d.stage_ms[i] = 0.0;
    d.stage_launches[i] = 0;
  }
  d.ev_pairs.clear();
  d.ev_used = 0;
  const bool use_graph = cfg_.use_cuda_graph != 0 && max_iter > 0;
  if (use_graph) {
    // the whole solve is one graph launch: no host round trip per iteration
    ensure_loop_graph<T>(st);
    LoopCtl* hc = d.h_ctl;
    *hc = LoopCtl{};
    hc->tol = tol;
    hc->max_iter = max_iter;
    hc->B = d.B;
    hc->tolerate = tolerate_nonfinite_ ? 1 : 0;
    // control in and results out by kernels on pinned memory (no copy-engine
    // transfers that could queue behind a caller's batch copies)
    launch_ctl_load(hc, d.ctl.as<LoopCtl>(), s);
    CUPF_CUDA(cudaGraphLaunch(d.exec, s));
    launch_ctl_store(d.ctl.as<LoopCtl>(), hc, d.fin_dev.as<double>(), d.h_final, d_final, d.B, s);
    if (d_v_out && !prepare_adjoint) {
      // the voltages do not depend on what the host reads back: queue them
      // before the synchronisation, so the device does not idle through the
      // host's round trip
      launch_pack_voltage(d.g, st, d_v_out, s);
      ++launches_;
      d_v_out = nullptr;
    }
    CUPF_CUDA(cudaStreamSynchronize(s));
    completed = hc->completed;
    gmax = hc->gmax;
    nonfinite = hc->nonfinite != 0;
    // control load and store, the first mismatch + test, then per update:
    // the body, plus the closing mismatch and test when the cap stopped the loop
    const int64_t updates = (gmax <= tol || hc->status) ? completed - 1 : completed;
    launches_ += 4 + updates * d.graph_body_launches;
    if (debug_sync()) std::fprintf(stderr, "[cupf] %d norm evaluations, max ||F||inf = %.3e\n", completed, gmax);
    if (hc->status) throw std::runtime_error("NewtonSolver: mismatch norm is not finite");
  } else if (max_iter > 0) {
    stage_begin(0, s);
    launch_ibus_mismatch(d.g, st, s);
    stage_end(0, s);
    ++launches_;
    ++d.stage_launches[0];
  }
  for (int it = 0; it < (use_graph ? 0 : max_iter); ++it) {
    completed = it + 1;
    CUPF_CUDA(cudaMemcpyAsync(d.h_norm, d.norm.p, d.Bp * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CUPF_CUDA(cudaStreamSynchronize(s));
    gmax = 0.0;
    nonfinite = false;
    bool finite = true;
    for (int b = 0; b < d.B; ++b) {
      double v;
      std::memcpy(&v, &d.h_norm[b], sizeof(double));
      d.h_final[b] = v;
      if (!std::isfinite(v)) {
        if (tolerate_nonfinite_) {  // warm-started solves: the scenario failed, its fallback solves it
          d.h_final[b] = std::numeric_limits<double>::infinity();
          nonfinite = true;
          continue;
        }
        finite = false;
      }
      gmax = std::max(gmax, v);
    }
    if (debug_sync()) std::fprintf(stderr, "[cupf] iteration %d max ||F||inf = %.3e\n", it, gmax);
    if (!finite) throw std::runtime_error("NewtonSolver: mismatch norm is not finite");
    if (gmax <= tol) break;
    iteration_tail<T>(s, 0);
    if (it + 1 < max_iter) {
      stage_begin(0, s);
      launch_ibus_mismatch(d.g, st, s);
      stage_end(0, s);
      ++launches_;
      ++d.stage_launches[0];
    }
  }
  CUPF_CUDA(cudaGetLastError());
  stats.iterations = completed;
  stats.max_final_mismatch = gmax;
  stats.all_converged = (gmax <= tol && !nonfinite) ? 1 : 0;
  if (prepare_adjoint) {
    // final-state factorization with L kept (newton_solver.cpp:388-491)
    CUPF_CUDA(cudaMemsetAsync(d.norm.p, 0, d.Bp * sizeof(unsigned long long), s));
    launch_ibus_mismatch(d.g, st, s);
    launch_jacobian<T>(d.g, st, d.J.as<T>(), s);
    factor_all<T>(s, 1, d.J.p);
    launches_ += 2;
    B_ = d.B;
    adjoint_ready_ = true;
  }
  // (graph mode: the store kernel already wrote d_final)
  if (d_final && !use_graph)
    CUPF_CUDA(cudaMemcpyAsync(d_final, d.h_final, d.B * sizeof(double), cudaMemcpyHostToDevice, s));
  if (d_v_out) {
    launch_pack_voltage(d.g, st, d_v_out, s);
    ++launches_;
  }
  CUPF_CUDA(cudaStreamSynchronize(s));
  CUPF_CUDA(cudaGetLastError());
  if (profiling_) collect_stage_times();
  return stats;
}

SolveStats Engine::solve_batch_host(const double* sbus, int64_t sbus_stride, const double* v0, int64_t v0_stride,
                                    int32_t B, double tol, int32_t max_iter, int32_t prepare_adjoint, double* v_out,
                                    int32_t* iterations, double* final_mismatch, uint8_t* converged,
                                    const double* ybus, int64_t ybus_stride) {
  if (!sbus || !v0) throw std::invalid_argument("NewtonSolver::solve_batch(): sbus/V0 must not be null");
  if (sbus_stride < ja_.n_bus) throw std::invalid_argument("NewtonSolver::solve_batch(): sbus stride must be at least n_bus");
  if (v0_stride < ja_.n_bus) throw std::invalid_argument("NewtonSolver::solve_batch(): V0 stride must be at least n_bus");
  ensure_workspace(B);
  auto& d = *d_;
  const size_t n = ja_.n_bus;
  const size_t y_elems = ybus ? 2 * (size_t)B * ybus_stride : 0;
  const size_t in_elems = 2 * ((size_t)B * sbus_stride + (size_t)B * v0_stride) + y_elems;
  d.stage_in.reserve(in_elems * sizeof(double));
  d.stage_out.reserve(2 * (size_t)B * n * sizeof(double));
  d.fin.reserve(std::max<size_t>(B, 1) * sizeof(double));
  double* din = d.stage_in.as<double>();
  double* dv0 = din + 2 * (size_t)B * sbus_stride;
  cudaStream_t s = d.own;
  CUPF_CUDA(cudaMemcpyAsync(din, sbus, 2 * (size_t)B * sbus_stride * sizeof(double), cudaMemcpyHostToDevice, s));
  CUPF_CUDA(cudaMemcpyAsync(dv0, v0, 2 * (size_t)B * v0_stride * sizeof(double), cudaMemcpyHostToDevice, s));
  double* dyb = ybus ? dv0 + 2 * (size_t)B * v0_stride : nullptr;
  if (ybus) CUPF_CUDA(cudaMemcpyAsync(dyb, ybus, y_elems * sizeof(double), cudaMemcpyHostToDevice, s));
  SolveStats st = solve_batch_device(din, sbus_stride, dv0, v0_stride, B, tol, max_iter, prepare_adjoint,
                                     d.stage_out.as<double>(), nullptr, s, dyb, ybus_stride);
  if (v_out)
    CUPF_CUDA(cudaMemcpyAsync(v_out, d.stage_out.p, 2 * (size_t)B * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CUPF_CUDA(cudaStreamSynchronize(s));
  for (int b = 0; b < B; ++b) {
    if (iterations) iterations[b] = st.iterations;
    if (final_mismatch) final_mismatch[b] = max_iter > 0 ? d.h_final[b] : 0.0;
    if (converged) converged[b] = (max_iter > 0 ? d.h_final[b] : 0.0) <= tol ? 1 : 0;
  }
  return st;
}

void Engine::use_scenario_ybus(const double* d_ybus, int64_t ybus_stride, int32_t B, cudaStream_t s) {
  auto& d = *d_;
  if (!d_ybus) {
    d.yb_active = false;
    return;
  }
  const int nnz = (int)ja_.map11.size();
  if (ybus_stride < nnz) throw std::invalid_argument("solve_batch: per-scenario Ybus stride must be at least nnz");
  d.yb_re.reserve((size_t)nnz * d.Bp * sizeof(double));
  d.yb_im.reserve((size_t)nnz * d.Bp * sizeof(double));
  launch_ybus_to_rows(d_ybus, ybus_stride, nnz, B, d.Bp, d.yb_re.as<double>(), d.yb_im.as<double>(), s);
  d.yb_active = true;
}

SolveStats Engine::solve_batch_device(const double* d_sbus, int64_t sbus_stride, const double* d_v0, int64_t v0_stride,
                                      int32_t B, double tol, int32_t max_iter, int32_t prepare_adjoint,
                                      double* d_v_out, double* d_final_mismatch, cudaStream_t stream,
                                      const double* d_ybus, int64_t ybus_stride) {
  ensure_workspace(B);
  auto& d = *d_;
  cudaStream_t s = stream ? stream : d.own;
  use_scenario_ybus(d_ybus, ybus_stride, B, s);
  const DevState st = d.state();
  launch_seed_state(d.g, st, d_sbus, sbus_stride, d_v0, v0_stride, s);
  SolveStats out = factor_is_double()
                       ? run_loop<double>(tol, max_iter, prepare_adjoint, s, d_final_mismatch, d_v_out)
                       : run_loop<float>(tol, max_iter, prepare_adjoint, s, d_final_mismatch, d_v_out);
  launches_ += 1;
  return out;
}

SolveStats Engine::solve_batch_warm_device(const double* d_sbus, int64_t sbus_stride, const double* d_v0,
                                           int64_t v0_stride, const float* d_pred, int64_t pred_ld,
                                           const float* d_scale, const float* d_shift, int32_t B,
                                           double tol, int32_t max_iter, int32_t prepare_adjoint, double* d_v_out,
                                           double* d_final_mismatch, cudaStream_t stream) {
  if (!d_pred) throw std::invalid_argument("solve_batch_warm: prediction must not be null");
  if (pred_ld < ja_.dim) throw std::invalid_argument("solve_batch_warm: prediction row stride must be >= dim_f");
  ensure_workspace(B);
  auto& d = *d_;
  cudaStream_t s = stream ? stream : d.own;
  use_scenario_ybus(nullptr, 0, B, s);
  const DevState st = d.state();
  launch_seed_warm(d.g, st, d_sbus, sbus_stride, d_v0, v0_stride, d_pred, pred_ld, d_scale, d_shift, s);
  // a poor prediction may send a scenario to infinity: it is reported as not
  // converged (final mismatch = inf) instead of failing the whole batch
  struct Tolerate {
    bool& f;
    explicit Tolerate(bool& x) : f(x) { f = true; }
    ~Tolerate() { f = false; }
  } tolerate(tolerate_nonfinite_);
  SolveStats out = factor_is_double()
                       ? run_loop<double>(tol, max_iter, prepare_adjoint, s, d_final_mismatch, d_v_out)
                       : run_loop<float>(tol, max_iter, prepare_adjoint, s, d_final_mismatch, d_v_out);
  launches_ += 1;
  return out;
}

SolveStats Engine::solve_from_load(const void* base_re, const void* base_im, const void* load_p, const void* load_q,
                                   const void* va0, const void* vm0, int32_t batched_v0, void* va_out, void* vm_out,
                                   int32_t B, int32_t is_double, double tol, int32_t max_iter,
                                   int32_t prepare_adjoint, cudaStream_t stream, double* d_final_mismatch) {
  if (!base_re || !base_im || !load_p || !load_q || !va0 || !vm0 || !va_out || !vm_out)
    throw std::invalid_argument("cupf::torch_api::solve_forward(): null device pointer");
  ensure_workspace(B);
  auto& d = *d_;
  cudaStream_t s = stream ? stream : d.own;
  use_scenario_ybus(nullptr, 0, B, s);
  const DevState st = d.state();
  if (batched_v0)
    launch_set_inputs_batched(d.g, st, base_re, base_im, load_p, load_q, va0, vm0, is_double, s);
  else
    launch_set_inputs_from_load(d.g, st, base_re, base_im, load_p, load_q, va0, vm0, is_double, s);
  SolveStats out = factor_is_double() ? run_loop<double>(tol, max_iter, prepare_adjoint, s, d_final_mismatch)
                                      : run_loop<float>(tol, max_iter, prepare_adjoint, s, d_final_mismatch);
  launch_copy_voltage_outputs(d.g, st, va_out, vm_out, is_double, s);
  launches_ += 2;
  CUPF_CUDA(cudaStreamSynchronize(s));
  return out;
}

template <typename T>
void Engine::transpose_solve(const double* d_G, double* d_lam, cudaStream_t s) {
  auto& d = *d_;
  AdjointSweepArgs<T> a;
  a.plan = d.pl;
  a.groups = d.Bp / kWarp;
  a.Bp = d.Bp;
  a.U = d.U.as<T>();
  a.L = d.L.as<T>();
  a.G = d_G;
  a.TV = d.TV.as<T>();
  a.W = d.W.as<T>();
  a.Z = d.Z.as<T>();
  for (const auto& lv : d.levels) launch_ut_forward_level<T>(lv, a, s);
  for (int L = (int)d.levels.size() - 1; L >= 0; --L) launch_lt_backward_level<T>(d.levels[L], a, s);
  // lambda is indexed by equation rows: undo the row ordering
  launch_permuted_to_rows<T>(d.pl.row_iperm, ja_.dim, d.Bp, d.Z.as<T>(), d_lam, s);
}

double Engine::solve_adjoint_device(const void* grad_va, const void* grad_vm, void* grad_p, void* grad_q,
                                    double* d_lambda, int32_t B, int32_t is_double, cudaStream_t stream,
                                    bool residual) {
  if (d_->state_f32)
    throw std::runtime_error(
        "NewtonSolver::solve_adjoint(): the adjoint's FP64 residual refinement needs the FP64 state of "
        "ComputePolicy::FP64 or Mixed; ComputePolicy::FP32 keeps the state in FP32");
  if (!adjoint_ready_)
    throw std::runtime_error("NewtonSolver::solve_adjoint(): missing exact final-state adjoint cache");
  if (B != B_) throw std::invalid_argument("NewtonSolver::solve_adjoint(): batch_size does not match the last forward solve");
  if (!grad_va || !grad_vm) throw std::invalid_argument("NewtonSolver::solve_adjoint(): grad_va/grad_vm must not be null");
  auto& d = *d_;
  cudaStream_t s = stream ? stream : d.own;
  const size_t dim = ja_.dim, Bp = d.Bp;
  const size_t es = factor_is_double() ? sizeof(double) : sizeof(float);
  for (DBuf* b : {&d.G, &d.R, &d.lam, &d.dlam}) b->reserve(dim * Bp * 8);
  d.TV.reserve((size_t)std::max<int64_t>(d.tv_total, 1) * Bp * es);
  d.W.reserve(dim * Bp * es);
  d.Z.reserve(dim * Bp * es);
  const DevState st = d.state();
  launch_gather_adjoint_rhs(d.g, st, grad_va, grad_vm, is_double, d.G.as<double>(), s);
  const bool dbl = factor_is_double();
  if (dbl) transpose_solve<double>(d.G.as<double>(), d.lam.as<double>(), s);
  else transpose_solve<float>(d.G.as<double>(), d.lam.as<double>(), s);
  // FP64 residual refinement: r = g - J^T lambda with the FP64 Jacobian at the
  // final state, lambda += (J^T)^-1 r on the cached factors.
  d.Jd.reserve((size_t)ja_.nnz * Bp * 8);
  launch_jacobian<double>(d.g, st, d.Jd.as<double>(), s);
  const int steps = std::max(0, cfg_.adjoint_refine_steps);
  for (int k = 0; k < steps; ++k) {
    launch_jt_residual(d.g, d.Bp, d.Jd.as<double>(), d.lam.as<double>(), d.G.as<double>(), d.R.as<double>(), s);
    if (dbl) transpose_solve<double>(d.R.as<double>(), d.dlam.as<double>(), s);
    else transpose_solve<float>(d.R.as<double>(), d.dlam.as<double>(), s);
    launch_axpy(d.lam.as<double>(), d.dlam.as<double>(), (long long)(dim * Bp), s);
  }
  launch_project_load_gradients(d.g, st, d.lam.as<double>(), grad_p, grad_q, is_double, s);
  if (d_lambda) launch_rows_to_batch<double, double>(d.lam.as<double>(), d_lambda, (int)dim, B, d.Bp, s);
  double res = 0.0;
  if (residual) {
    // relative residual ||J^T lambda - g|| / ||g|| over the real scenarios,
    // reduced on the device; two doubles come back
    launch_jt_residual(d.g, d.Bp, d.Jd.as<double>(), d.lam.as<double>(), d.G.as<double>(), d.R.as<double>(), s);
    d.red.reserve((2 + 2 * 296) * sizeof(double));
    launch_sumsq2(d.R.as<double>(), d.G.as<double>(), (int)dim, B, d.Bp, d.red.as<double>(), s);
    CUPF_CUDA(cudaMemcpyAsync(d.h_norm, d.red.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  CUPF_CUDA(cudaGetLastError());
  if (residual) {
    // without the norm the call stays stream-ordered and returns at once
    CUPF_CUDA(cudaStreamSynchronize(s));
    double sums[2];
    std::memcpy(sums, d.h_norm, sizeof(sums));
    res = std::sqrt(sums[0]) / std::max(std::sqrt(std::max(sums[1], 1e-60)), 1e-30);
  }
  return res;
}

void Engine::factorize_values(const void* d_values, int32_t values_is_double, int32_t B, cudaStream_t stream) {
  ensure_workspace(B);
  auto& d = *d_;
  cudaStream_t s = stream ? stream : d.own;
  const bool dbl = factor_is_double();
  // [B][nnz] (batch-strided, solver.hpp:76-79) -> [nnz][Bp]
  if (dbl) {
    if (values_is_double)
      launch_batch_to_rows<double, double>(static_cast<const double*>(d_values), d.J.as<double>(), ja_.nnz, B, d.Bp, s);
    else
      launch_batch_to_rows<float, double>(static_cast<const float*>(d_values), d.J.as<double>(), ja_.nnz, B, d.Bp, s);
  } else {
    if (values_is_double)
      launch_batch_to_rows<double, float>(static_cast<const double*>(d_values), d.J.as<float>(), ja_.nnz, B, d.Bp, s);
    else
      launch_batch_to_rows<float, float>(static_cast<const float*>(d_values), d.J.as<float>(), ja_.nnz, B, d.Bp, s);
  }
  CUPF_CUDA(cudaMemsetAsync(d.F.p, 0, (size_t)ja_.dim * d.Bp * 8, s));
  CUPF_CUDA(cudaMemsetAsync(d.Fp.p, 0, (size_t)ja_.dim * d.Bp * (dbl ? 8 : 4), s));
  if (cfg_.autotune) {
    if (dbl) autotune_factor<double>(s, d.J.p);
    else autotune_factor<float>(s, d.J.p);
  }
  CUPF_CUDA(cudaMemsetAsync(d.sing.p, 0, d.Bp * sizeof(int), s));
  if (dbl) factor_all<double>(s, 1, d.J.p);
  else factor_all<float>(s, 1, d.J.p);
  B_ = B;
  adjoint_ready_ = false;
  CUPF_CUDA(cudaStreamSynchronize(s));
  CUPF_CUDA(cudaGetLastError());
}

// Factorization whose global front scratch is a caller-supplied fixed area
// (the static scratch of cls_factorize_static_scratch).  Allocates nothing:
// the handle's workspace must already hold this batch size, and the levels'
// scratch need must fit the area.  No stage timers (their events are created
// on demand).
template <typename T>
void Engine::factor_all_external(cudaStream_t s, const void* J, T* scratch, size_t scratch_elems) {
  auto& d = *d_;
  FactorArgs<T, T> a;
  a.plan = d.pl;
  a.groups = d.Bp / kWarp;
  a.Bp = d.Bp;
  a.J = static_cast<const T*>(J);
  a.Fp = d.Fp.as<T>();
  a.U = d.U.as<T>();
  a.L = d.L.as<T>();
  a.CB = d.CB.as<T>();
  a.Y = d.Y.as<T>();
  a.store_l = 1;
  a.eps = cfg_.shift_epsilon;
  a.static_pivot = (cfg_.static_pivot && cfg_.shift_epsilon > 0.0) ? 1 : 0;
  a.sing = d.sing.as<int>();
  a.front_scratch = scratch;
  a.front_scratch_elems = scratch_elems;
  a.single = single_system() ? 1 : 0;
  if (single_tree(sizeof(T))) {  // (no scratch: every front is in shared memory)
    factor_tree<T>(a, s);
    ++launches_;
    return;
  }
  for (LevelLaunch lv : d.levels) {
    lv.placement = 0;  // the built-in placement: the static area is sized for it
    if (lv.tier == 0 && lv.warps > 8) lv.warps = 0;  // (a wide-tier shape of the autotuner)
    launch_factor_level<T, T>(lv, a, s);
    ++launches_;
  }
}

void Engine::factorize_values_static_scratch(const void* d_values, int32_t values_is_double, int32_t B,
                                             void* scratch, size_t scratch_bytes, cudaStream_t stream) {
  if (!initialized_) throw std::runtime_error("Factorize: Analyze() must be called first");
  if (B <= 0) throw std::invalid_argument("Factorize: batch size must be positive");
  auto& d = *d_;
  const int Bp = (B + kWarp - 1) / kWarp * kWarp;
  if (Bp > d.Bp_cap)
    throw std::runtime_error(
        "Factorize (static scratch): the handle has no workspace for this batch size; this entry point allocates "
        "nothing, so run one regular cls_factorize at this batch size (or larger) first");
  const bool dbl = factor_is_double();
  const size_t es = dbl ? sizeof(double) : sizeof(float);
  size_t need = 0;  // elements x 32 lanes, with the built-in front placement
  for (LevelLaunch lv : d.levels) {
    lv.placement = 0;
    need = std::max(need, level_scratch_elems(lv, es, Bp / kWarp));
  }
  if (need * kWarp * es > scratch_bytes)
    throw std::invalid_argument("Factorize (static scratch): this batch needs " + std::to_string(need * kWarp * es) +
                                " bytes of front scratch, the static area holds " + std::to_string(scratch_bytes));
  d.B = B;
  d.Bp = Bp;
  cudaStream_t s = stream ? stream : d.own;
  if (dbl) {
    if (values_is_double)
      launch_batch_to_rows<double, double>(static_cast<const double*>(d_values), d.J.as<double>(), ja_.nnz, B, d.Bp, s);
    else
      launch_batch_to_rows<float, double>(static_cast<const float*>(d_values), d.J.as<double>(), ja_.nnz, B, d.Bp, s);
  } else {
    if (values_is_double)
      launch_batch_to_rows<double, float>(static_cast<const double*>(d_values), d.J.as<float>(), ja_.nnz, B, d.Bp, s);
    else
      launch_batch_to_rows<float, float>(static_cast<const float*>(d_values), d.J.as<float>(), ja_.nnz, B, d.Bp, s);
  }
  CUPF_CUDA(cudaMemsetAsync(d.F.p, 0, (size_t)ja_.dim * d.Bp * 8, s));
  CUPF_CUDA(cudaMemsetAsync(d.Fp.p, 0, (size_t)ja_.dim * d.Bp * es, s));
  CUPF_CUDA(cudaMemsetAsync(d.sing.p, 0, d.Bp * sizeof(int), s));
  const size_t elems = scratch_bytes / (kWarp * es);
  if (dbl) factor_all_external<double>(s, d.J.p, static_cast<double*>(scratch), elems);
  else factor_all_external<float>(s, d.J.p, static_cast<float*>(scratch), elems);
  B_ = B;
  adjoint_ready_ = false;
  CUPF_CUDA(cudaStreamSynchronize(s));
  CUPF_CUDA(cudaGetLastError());
}

void Engine::solve_values(const void* d_rhs, int32_t rhs_is_double, void* d_x, int32_t x_is_double, int32_t B,
                          bool transpose, cudaStream_t stream) {
  if (B != B_) throw std::invalid_argument("Solve: batch size differs from the factorization");
  auto& d = *d_;
  cudaStream_t s = stream ? stream : d.own;
  const size_t dim = ja_.dim, Bp = d.Bp;
  const bool dbl = factor_is_double();
  const size_t es = dbl ? sizeof(double) : sizeof(float);
  d.G.reserve(dim * Bp * 8);
  d.lam.reserve(dim * Bp * 8);
  d.TV.reserve((size_t)std::max<int64_t>(d.tv_total, 1) * Bp * es);
  d.W.reserve(dim * Bp * es);
  d.Z.reserve(dim * Bp * es);
  if (rhs_is_double)
    launch_batch_to_rows<double, double>(static_cast<const double*>(d_rhs), d.G.as<double>(), (int)dim, B, (int)Bp, s);
  else
    launch_batch_to_rows<float, double>(static_cast<const float*>(d_rhs), d.G.as<double>(), (int)dim, B, (int)Bp, s);
  auto run = [&](auto tag) {
    using T = decltype(tag);
    if (transpose) {
      transpose_solve<T>(d.G.as<double>(), d.lam.as<double>(), s);
      return;
    }
    AdjointSweepArgs<T> a;
    a.plan = d.pl;
    a.groups = (int)Bp / kWarp;
    a.Bp = (int)Bp;
    a.U = d.U.as<T>();
    a.L = d.L.as<T>();
    a.G = d.G.as<double>();
    a.TV = d.TV.as<T>();
    a.W = d.W.as<T>();
    for (const auto& lv : d.levels) launch_l_forward_level<T>(lv, a, s);
    SweepArgs<T> bk;
    bk.plan = d.pl;
    bk.groups = (int)Bp / kWarp;
    bk.Bp = (int)Bp;
    bk.U = d.U.as<T>();
    bk.Y = d.W.as<T>();
    bk.X = d.X.as<T>();
    backward_levels<T>(bk, s);
    // x is indexed by columns: undo the column ordering
    launch_permuted_to_rows<T>(d.pl.iperm, (int)dim, (int)Bp, d.X.as<T>(), d.lam.as<double>(), s);
  };
  if (dbl) run(double{});
  else run(float{});
  if (x_is_double)
    launch_rows_to_batch<double, double>(d.lam.as<double>(), static_cast<double*>(d_x), (int)dim, B, (int)Bp, s);
  else
    launch_rows_to_batch<double, float>(d.lam.as<double>(), static_cast<float*>(d_x), (int)dim, B, (int)Bp, s);
  CUPF_CUDA(cudaStreamSynchronize(s));
  CUPF_CUDA(cudaGetLastError());
}

void Engine::evaluate_host(const double* V, const double* sbus, int32_t B, double* F_out, double* J_out) {
  ensure_workspace(B);
  auto& d = *d_;
  cudaStream_t s = d.own;
  const size_t n = ja_.n_bus, dim = ja_.dim;
  d.stage_in.reserve(4 * (size_t)B * n * sizeof(double));
  double* ds = d.stage_in.as<double>();
  double* dv = ds + 2 * (size_t)B * n;
  CUPF_CUDA(cudaMemcpyAsync(ds, sbus, 2 * (size_t)B * n * sizeof(double), cudaMemcpyHostToDevice, s));
  CUPF_CUDA(cudaMemcpyAsync(dv, V, 2 * (size_t)B * n * sizeof(double), cudaMemcpyHostToDevice, s));
  use_scenario_ybus(nullptr, 0, B, s);
  DevState st = d.state();
  st.F = d.F.as<double>();
  launch_seed_state(d.g, st, ds, (long long)n, dv, (long long)n, s);
  CUPF_CUDA(cudaMemsetAsync(d.norm.p, 0, d.Bp * sizeof(unsigned long long), s));
  launch_ibus_mismatch(d.g, st, s);
  d.Jd.reserve((size_t)ja_.nnz * d.Bp * 8);
  launch_jacobian<double>(d.g, st, d.Jd.as<double>(), s);
  d.G.reserve(std::max<size_t>(dim, (size_t)ja_.nnz) * B * 8);
  if (d.state_f32)
    launch_rows_to_batch<float, double>(d.F.as<float>(), d.G.as<double>(), (int)dim, B, d.Bp, s);
  else
    launch_rows_to_batch<double, double>(d.F.as<double>(), d.G.as<double>(), (int)dim, B, d.Bp, s);
  CUPF_CUDA(cudaMemcpyAsync(F_out, d.G.p, dim * B * 8, cudaMemcpyDeviceToHost, s));
  CUPF_CUDA(cudaStreamSynchronize(s));
  launch_rows_to_batch<double, double>(d.Jd.as<double>(), d.G.as<double>(), ja_.nnz, B, d.Bp, s);
  CUPF_CUDA(cudaMemcpyAsync(J_out, d.G.p, (size_t)ja_.nnz * B * 8, cudaMemcpyDeviceToHost, s));
  CUPF_CUDA(cudaStreamSynchronize(s));
  CUPF_CUDA(cudaGetLastError());
}

std::vector<int32_t> Engine::singular_flags() const {
  std::vector<int32_t> out;
  if (!d_->sing.p || d_->B == 0) return out;
  std::vector<int32_t> tmp(d_->Bp);
  cudaMemcpy(tmp.data(), d_->sing.p, d_->Bp * sizeof(int32_t), cudaMemcpyDeviceToHost);
  out.assign(tmp.begin(), tmp.begin() + d_->B);
  return out;
}

template SolveStats Engine::run_loop<float>(double, int32_t, int32_t, cudaStream_t, double*, double*);
template SolveStats Engine::run_loop<double>(double, int32_t, int32_t, cudaStream_t, double*, double*);

}  // namespace cupf_b200
