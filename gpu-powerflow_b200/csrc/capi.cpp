// capi.cpp -- the C ABI of include/cupf_b200.h over cupf_b200::Engine.
//
// Exceptions never cross the boundary: std::invalid_argument becomes
// PF_INVALID_ARGUMENT / CLS_INVALID_VALUE, anything else PF_RUNTIME_ERROR or
// the phase's failure status, with the message kept on the handle.
#include "../../include/cupf_b200.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "engine.hpp"
#include "static_scratch.hpp"

using cupf_b200::Engine;
using cupf_b200::EngineConfig;

struct cls_solver_s {
  cls_config cfg{};
  std::unique_ptr<Engine> eng;
  std::vector<int32_t> row_ptr, col_idx;
  int32_t n = 0, nnz = 0;
  bool has_data = false, analyzed = false;
  int32_t batch = 0;
  cudaStream_t stream = nullptr;
  std::string err;
};

struct pf_solver_s {
  pf_options opt{};
  std::unique_ptr<Engine> eng;
  std::string err;
  std::vector<int32_t> ind_ptr, ind, pv, pq;
  std::vector<double> ydata;
  int32_t n_bus = 0;
};

namespace {

EngineConfig engine_config(const cls_config& c, int32_t compute, int32_t use_graph) {
  EngineConfig e;
  e.compute = compute;
  e.factor_precision = c.precision;
  e.max_panel_width = c.max_panel_width;
  e.serial_nd = c.serial_nd;
  e.use_matching = c.matching;
  e.static_pivot = c.pivot_strategy == CLS_PIVOT_STATIC_DIAGONAL_SHIFT ? 1 : 0;
  e.shift_epsilon = c.shift_retry_epsilon;
  e.autotune = c.autotune;
  e.par_nd_depth = c.parallel_nd_depth > 0 ? c.parallel_nd_depth : 4;
  e.par_nd_base_small = c.parallel_nd_base_small > 0 ? c.parallel_nd_base_small : 4000;
  e.par_nd_base_large = c.parallel_nd_base_large > 0 ? c.parallel_nd_base_large : 20000;
  e.wide_min_front = c.wide_min_front > 0 ? c.wide_min_front : 65;
  e.tc_min_front = c.tc_min_front;
  e.batch1_schedule = c.batch1_schedule;
  e.use_cuda_graph = use_graph;
  return e;
}

bool copy_plan_array(const Engine& e, const char* name, int32_t* out, int64_t cap, int64_t* len) {
  const auto& sp = e.symbolic();
  const auto& ja = e.jacobian();
  const std::vector<int32_t>* v = nullptr;
  const std::string n(name ? name : "");
#define CUPF_ARR(key, vec) \
  if (n == key) v = &(vec);
  CUPF_ARR("perm", sp.perm)
  CUPF_ARR("iperm", sp.iperm)
  CUPF_ARR("row_iperm", sp.row_iperm)
  CUPF_ARR("col_perm", sp.col_perm)
  CUPF_ARR("row_to_col", sp.row_to_col)
  CUPF_ARR("parent", sp.parent)
  CUPF_ARR("Lp", sp.Lp)
  CUPF_ARR("Li", sp.Li)
  CUPF_ARR("panel_first", sp.panel_first)
  CUPF_ARR("panel_ncols", sp.panel_ncols)
  CUPF_ARR("panel_width", sp.panel_width)
  CUPF_ARR("panel_of", sp.panel_of)
  CUPF_ARR("front_ptr", sp.front_ptr)
  CUPF_ARR("front_rows", sp.front_rows)
  CUPF_ARR("panel_parent", sp.panel_parent)
  CUPF_ARR("asm_ptr", sp.asm_ptr)
  CUPF_ARR("asm_idx", sp.asm_idx)
  CUPF_ARR("asm_local", sp.asm_local)
  CUPF_ARR("plevel", sp.plevel)
  CUPF_ARR("level_ptr", sp.level_ptr)
  CUPF_ARR("plcols_level", sp.plcols_level)
  CUPF_ARR("front_off", sp.front_off)
  CUPF_ARR("a_pos_csr", sp.a_pos_csr)
  CUPF_ARR("graph_xadj", sp.graph_xadj)
  CUPF_ARR("graph_adjncy", sp.graph_adjncy)
  CUPF_ARR("sym_col_ptr", sp.sym_col_ptr)
  CUPF_ARR("sym_row_idx", sp.sym_row_idx)
  const auto& fp = e.program();
  CUPF_ARR("fp_fsz", fp.fsz)
  CUPF_ARR("fp_nc", fp.nc)
  CUPF_ARR("fp_arow_ptr", fp.arow_ptr)
  CUPF_ARR("fp_arow_q", fp.arow_q)
  CUPF_ARR("fp_arow_col", fp.arow_col)
  CUPF_ARR("fp_crow_ptr", fp.crow_ptr)
  CUPF_ARR("fp_crow_child", fp.crow_child)
  CUPF_ARR("fp_crow_r", fp.crow_r)
  CUPF_ARR("fp_level_ptr", fp.level_ptr)
  CUPF_ARR("fp_level_fronts", fp.level_fronts)
  CUPF_ARR("fe_dst", fp.fe_dst)
  CUPF_ARR("front_meta", fp.front_meta)
  CUPF_ARR("jac_row_ptr", ja.row_ptr)
  CUPF_ARR("jac_col_idx", ja.col_idx)
  CUPF_ARR("map11", ja.map11)
  CUPF_ARR("map21", ja.map21)
  CUPF_ARR("map12", ja.map12)
  CUPF_ARR("map22", ja.map22)
  CUPF_ARR("diag11", ja.diag11)
  CUPF_ARR("diag21", ja.diag21)
  CUPF_ARR("diag12", ja.diag12)
  CUPF_ARR("diag22", ja.diag22)
#undef CUPF_ARR
  if (n == "factor_level_warps" || n == "backward_launch_warps" || n == "factor_level_tiers" ||
      n == "tc_threshold" || n == "factor_level_placement") {  // the autotuner's choices, each launch's kernel
    const std::vector<int32_t> w = n == "factor_level_warps"       ? e.factor_level_warps()
                                   : n == "factor_level_tiers"     ? e.factor_level_tiers()
                                   : n == "factor_level_placement" ? e.factor_level_placements()
                                   : n == "tc_threshold"           ? std::vector<int32_t>{e.tc_threshold()}
                                                                   : e.backward_launch_warps();
    if (len) *len = (int64_t)w.size();
    if (out) {
      if (cap < (int64_t)w.size()) return false;
      std::copy(w.begin(), w.end(), out);
    }
    return true;
  }
  if (!v) return false;
  if (len) *len = (int64_t)v->size();
  if (out) {
    if (cap < (int64_t)v->size()) return false;
    if (!v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(int32_t));
  }
  return true;
}

bool write_text_file(const char* path, const std::string& text) {
  FILE* f = std::fopen(path, "w");
  if (!f) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return std::fclose(f) == 0 && ok;
}

// Stream of a device-pointer entry point: the caller's stream, where NULL is
// the legacy default stream (torch's default stream reports handle 0), so
// the engine's kernels stay ordered with the caller's earlier work on it.
cudaStream_t caller_stream(void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
}

const char* dtype_expected(const pf_options& o) { return o.compute == PF_COMPUTE_FP64 ? "float64" : "float32"; }

}  // namespace

// ===========================================================================
// cls_*
// ===========================================================================
extern "C" {

const char* cls_status_string(cls_status s) {
  switch (s) {
    case CLS_SUCCESS: return "success";
    case CLS_INVALID_VALUE: return "invalid value";
    case CLS_INVALID_STATE: return "invalid state";
    case CLS_ALLOCATION_FAILED: return "allocation failed";
    case CLS_ANALYSIS_FAILED: return "analysis failed";
    case CLS_FACTORIZATION_FAILED: return "factorization failed";
    case CLS_SOLVE_FAILED: return "Solve failed";
  }
  return "unknown";
}

cls_status cls_create(const cls_config* config, cls_handle* out) {
  if (!out) return CLS_INVALID_VALUE;
  *out = nullptr;
  cls_config c{CLS_PRECISION_FP64, 0, CLS_PIVOT_STATIC_DIAGONAL_SHIFT, 1, 8, 1e-8};
  if (config) c = *config;
  if ((c.matching != 0 && c.matching != 1) || c.max_panel_width < 1 || c.max_panel_width > 8 ||
      (c.autotune != 0 && c.autotune != 1) || c.parallel_nd_depth < 0 || c.parallel_nd_base_small < 0 ||
      c.parallel_nd_base_large < 0 || c.wide_min_front < 0 || c.wide_min_front > 65 || c.tc_min_front < 0 ||
      (c.batch1_schedule != 0 && c.batch1_schedule != 1) || c.precision < CLS_PRECISION_FP64 ||
      c.precision > CLS_PRECISION_TF32)
    return CLS_INVALID_VALUE;
  auto* h = new (std::nothrow) cls_solver_s();
  if (!h) return CLS_ALLOCATION_FAILED;
  h->cfg = c;
  *out = h;
  return CLS_SUCCESS;
}

cls_status cls_destroy(cls_handle h) {
  delete h;
  return CLS_SUCCESS;
}

const char* cls_last_error(cls_handle h) { return h ? h->err.c_str() : "null handle"; }

cls_status cls_set_data(cls_handle h, int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx,
                        int32_t location) {
  if (!h) return CLS_INVALID_STATE;
  if (n <= 0 || nnz < 0 || !row_ptr || !col_idx) return CLS_INVALID_VALUE;
  h->row_ptr.resize(n + 1);
  h->col_idx.resize(nnz);
  if (location == CLS_LOCATION_DEVICE) {
    if (cudaMemcpy(h->row_ptr.data(), row_ptr, (n + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
        (nnz && cudaMemcpy(h->col_idx.data(), col_idx, nnz * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess))
      return CLS_INVALID_VALUE;
  } else if (location == CLS_LOCATION_HOST) {
    std::memcpy(h->row_ptr.data(), row_ptr, (n + 1) * sizeof(int32_t));
    if (nnz) std::memcpy(h->col_idx.data(), col_idx, nnz * sizeof(int32_t));
  } else {
    return CLS_INVALID_VALUE;
  }
  if (h->row_ptr[n] != nnz) return CLS_INVALID_VALUE;
  h->n = n;
  h->nnz = nnz;
  h->has_data = true;
  h->analyzed = false;
  return CLS_SUCCESS;
}

cls_status cls_analyze(cls_handle h) {
  if (!h || !h->has_data) return CLS_INVALID_STATE;
  try {
    const int32_t compute = h->cfg.precision == CLS_PRECISION_FP64 ? cupf_b200::kComputeFP64 : cupf_b200::kComputeMixed;
    h->eng.reset(new Engine(engine_config(h->cfg, compute, 0)));
    h->eng->initialize_matrix(h->n, h->nnz, h->row_ptr.data(), h->col_idx.data());
    h->analyzed = true;
    return CLS_SUCCESS;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CLS_ANALYSIS_FAILED;
  }
}

cls_status cls_analyze_host(cls_handle h) {
  if (!h || !h->has_data) return CLS_INVALID_STATE;
  try {
    const int32_t compute = h->cfg.precision == CLS_PRECISION_FP64 ? cupf_b200::kComputeFP64 : cupf_b200::kComputeMixed;
    h->eng.reset(new Engine(engine_config(h->cfg, compute, 0)));
    h->eng->analyze_matrix_host(h->n, h->nnz, h->row_ptr.data(), h->col_idx.data());
    h->analyzed = false;
    return CLS_SUCCESS;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CLS_ANALYSIS_FAILED;
  }
}

cls_status cls_setup(cls_handle h, int32_t batch_size) {
  if (!h || !h->analyzed) return CLS_INVALID_STATE;
  if (batch_size <= 0) return CLS_INVALID_VALUE;
  h->batch = batch_size;
  return CLS_SUCCESS;
}

cls_status cls_set_stream(cls_handle h, void* stream) {
  if (!h || !h->analyzed || h->batch == 0) return CLS_INVALID_STATE;
  h->stream = caller_stream(stream);
  return CLS_SUCCESS;
}

cls_status cls_factorize(cls_handle h, const void* values, int32_t value_type) {
  if (!h || !h->analyzed) return CLS_INVALID_STATE;
  if (!values) return CLS_INVALID_STATE;
  if (value_type != CLS_VALUE_FLOAT64 && value_type != CLS_VALUE_FLOAT32) return CLS_INVALID_VALUE;
  if (h->batch == 0) h->batch = 1;  // auto Setup(1), solver.cpp:281-284
  try {
    h->eng->factorize_values(values, value_type == CLS_VALUE_FLOAT64, h->batch, h->stream);
    return CLS_SUCCESS;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CLS_FACTORIZATION_FAILED;
  }
}

cls_status cls_factorize_static_scratch(cls_handle h, const void* values, int32_t value_type) {
  if (!h || !h->analyzed) return CLS_INVALID_STATE;
  if (!values) return CLS_INVALID_STATE;
  if (value_type != CLS_VALUE_FLOAT64 && value_type != CLS_VALUE_FLOAT32) return CLS_INVALID_VALUE;
  if (h->batch == 0) h->batch = 1;
  try {
    void* scratch = cupf_b200::static_front_scratch();
    h->eng->factorize_values_static_scratch(values, value_type == CLS_VALUE_FLOAT64, h->batch, scratch,
                                            cupf_b200::kStaticFrontScratchBytes, h->stream);
    return CLS_SUCCESS;
  } catch (const std::invalid_argument& e) {
    h->err = e.what();
    return CLS_INVALID_VALUE;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CLS_FACTORIZATION_FAILED;
  }
}

static cls_status cls_solve_impl(cls_handle h, const void* rhs, int32_t rt, void* sol, int32_t st, bool transpose) {
  if (!h || !h->analyzed || h->batch == 0) return CLS_INVALID_STATE;
  if (!rhs || !sol) return CLS_INVALID_VALUE;
  const bool ok_pair = (rt == CLS_VALUE_FLOAT64 && st == CLS_VALUE_FLOAT64) ||
                       (rt == CLS_VALUE_FLOAT64 && st == CLS_VALUE_FLOAT32) ||
                       (rt == CLS_VALUE_FLOAT32 && st == CLS_VALUE_FLOAT32);
  if (!ok_pair) return CLS_INVALID_VALUE;
  try {
    h->eng->solve_values(rhs, rt == CLS_VALUE_FLOAT64, sol, st == CLS_VALUE_FLOAT64, h->batch, transpose, h->stream);
    return CLS_SUCCESS;
  } catch (const std::exception& e) {
    h->err = e.what();
    return CLS_SOLVE_FAILED;
  }
}

cls_status cls_solve(cls_handle h, const void* rhs, int32_t rhs_type, void* solution, int32_t solution_type) {
  return cls_solve_impl(h, rhs, rhs_type, solution, solution_type, false);
}

cls_status cls_solve_transpose(cls_handle h, const void* rhs, int32_t rhs_type, void* solution,
                               int32_t solution_type) {
  return cls_solve_impl(h, rhs, rhs_type, solution, solution_type, true);
}

cls_status cls_singular_flags(cls_handle h, int32_t* out_host, int32_t batch) {
  if (!h || !h->analyzed) return CLS_INVALID_STATE;
  if (!out_host || batch != h->batch) return CLS_INVALID_VALUE;
  const std::vector<int32_t> f = h->eng->singular_flags();
  for (int32_t b = 0; b < batch; ++b) out_host[b] = b < (int32_t)f.size() ? f[b] : 0;
  return CLS_SUCCESS;
}

cls_status cls_plan_array(cls_handle h, const char* name, int32_t* out, int64_t capacity, int64_t* len) {
  if (!h || !h->eng) return CLS_INVALID_STATE;
  return copy_plan_array(*h->eng, name, out, capacity, len) ? CLS_SUCCESS : CLS_INVALID_VALUE;
}

cls_status cls_dump_fronts_csv(cls_handle h, const char* path) {
  if (!h || !h->eng || h->eng->symbolic().level_ptr.empty()) return CLS_INVALID_STATE;
  if (!path) return CLS_INVALID_VALUE;
  return write_text_file(path, fronts_csv(h->eng->symbolic())) ? CLS_SUCCESS : CLS_INVALID_VALUE;
}

// ===========================================================================
// pf_*
// ===========================================================================

#define PF_TRY(h, ...)                                    \
  try {                                                   \
    __VA_ARGS__;                                          \
    return PF_OK;                                         \
  } catch (const std::invalid_argument& e) {              \
    (h)->err = e.what();                                  \
    return PF_INVALID_ARGUMENT;                           \
  } catch (const std::exception& e) {                     \
    (h)->err = e.what();                                  \
    return PF_RUNTIME_ERROR;                              \
  }

pf_status pf_create(const pf_options* options, pf_handle* out) {
  if (!out) return PF_INVALID_ARGUMENT;
  *out = nullptr;
  pf_options o{};
  o.backend = PF_BACKEND_CUDA;
  o.compute = PF_COMPUTE_MIXED;
  o.cuda_linear_solver = PF_CUDA_SOLVER_CUSTOM;
  o.cuda_jacobian = PF_JACOBIAN_EDGE;
  o.custom = cls_config{CLS_PRECISION_FP32, 0, CLS_PIVOT_STATIC_DIAGONAL_SHIFT, 1, 8, 1e-8};
  o.use_cuda_graph = 0;
  if (options) o = *options;
  auto* h = new (std::nothrow) pf_solver_s();
  if (!h) return PF_RUNTIME_ERROR;
  h->opt = o;
  try {
    if (o.backend != PF_BACKEND_CUDA)
      throw std::invalid_argument("NewtonSolver: this engine provides the CUDA backend only");
    if (o.cuda_linear_solver != PF_CUDA_SOLVER_CUSTOM)
      throw std::invalid_argument("NewtonSolver: this engine provides the custom CUDA linear solver only");
    if (o.compute != PF_COMPUTE_FP64 && o.compute != PF_COMPUTE_FP32 && o.compute != PF_COMPUTE_MIXED)
      throw std::invalid_argument("NewtonSolver: unsupported compute policy");
    if (o.custom.matching != 0 && o.custom.matching != 1)
      throw std::invalid_argument("NewtonSolver: matching must be None or Structural");
    if (o.custom.autotune != 0 && o.custom.autotune != 1)
      throw std::invalid_argument("NewtonSolver: autotune must be 0 or 1");
    if (o.custom.parallel_nd_depth < 0 || o.custom.parallel_nd_base_small < 0 || o.custom.parallel_nd_base_large < 0)
      throw std::invalid_argument("NewtonSolver: the parallel nested-dissection parameters must not be negative");
    if (o.custom.wide_min_front < 0 || o.custom.wide_min_front > 65 || o.custom.tc_min_front < 0)
      throw std::invalid_argument("NewtonSolver: wide_min_front must be in [0, 65] and tc_min_front non-negative");
    if (o.custom.batch1_schedule != 0 && o.custom.batch1_schedule != 1)
      throw std::invalid_argument("NewtonSolver: batch1_schedule must be 0 (single-system kernel) or 1 (lane kernels)");
    if (o.custom.precision < CLS_PRECISION_FP64 || o.custom.precision > CLS_PRECISION_TF32)
      throw std::invalid_argument("NewtonSolver: unknown custom solver precision");
    if (o.cuda_jacobian < PF_JACOBIAN_EDGE || o.cuda_jacobian > PF_JACOBIAN_VERTEX_WARP)
      throw std::invalid_argument("NewtonSolver: cuda_jacobian must be Edge, EdgeAtomic or VertexWarp");
    cls_config c = o.custom;
    if (o.compute == PF_COMPUTE_FP64) c.precision = CLS_PRECISION_FP64;
    // FP32 state factors in FP32 (or TF32), never FP64 (cuda_custom_solver.cpp:71-72)
    if (o.compute == PF_COMPUTE_FP32 && c.precision == CLS_PRECISION_FP64) c.precision = CLS_PRECISION_FP32;
    EngineConfig ec = engine_config(c, o.compute, o.use_cuda_graph);
    ec.jacobian_kind = o.cuda_jacobian;
    h->eng.reset(new Engine(ec));
  } catch (const std::exception& e) {
    // keep the handle so the caller can read the message, then report failure
    h->err = e.what();
    *out = h;
    return dynamic_cast<const std::invalid_argument*>(&e) ? PF_INVALID_ARGUMENT : PF_RUNTIME_ERROR;
  }
  *out = h;
  return PF_OK;
}

pf_status pf_destroy(pf_handle h) {
  delete h;
  return PF_OK;
}

const char* pf_last_error(pf_handle h) { return h ? h->err.c_str() : "null handle"; }

pf_status pf_initialize(pf_handle h, const int32_t* indptr, const int32_t* indices, const double* data, int32_t rows,
                        int32_t cols, int32_t nnz, const int32_t* pv, int32_t n_pv, const int32_t* pq,
                        int32_t n_pq) {
  if (!h) return PF_INVALID_ARGUMENT;
  if (!h->eng) {
    h->err = "NewtonSolver: construction failed";
    return PF_RUNTIME_ERROR;
  }
  PF_TRY(h, {
    if (rows <= 0 || cols <= 0 || rows != cols) throw std::invalid_argument("Ybus rows/cols must be positive and equal");
    if (!indptr || !indices || !data) throw std::invalid_argument("Ybus arrays must not be null");
    if (indptr[rows] != nnz) throw std::invalid_argument("Ybus indptr[rows] must equal nnz");
    h->eng->initialize(rows, indptr, indices, data, pv, n_pv, pq, n_pq);
    h->n_bus = rows;
    h->ind_ptr.assign(indptr, indptr + rows + 1);
    h->ind.assign(indices, indices + nnz);
    h->ydata.assign(data, data + 2 * (size_t)nnz);
    h->pv.assign(pv, pv + n_pv);
    h->pq.assign(pq, pq + n_pq);
  })
}

pf_status pf_analyze_host(pf_handle h, const int32_t* indptr, const int32_t* indices, int32_t rows, int32_t nnz,
                          const int32_t* pv, int32_t n_pv, const int32_t* pq, int32_t n_pq) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (rows <= 0 || !indptr || !indices) throw std::invalid_argument("Ybus pattern must not be empty");
    if (indptr[rows] != nnz) throw std::invalid_argument("Ybus indptr[rows] must equal nnz");
    h->eng->analyze_host(rows, indptr, indices, pv, n_pv, pq, n_pq);
  })
}

static void check_same_case(pf_handle h, const int32_t* indptr, const int32_t* indices, const double* data,
                            int32_t rows, int32_t nnz, const int32_t* pv, int32_t n_pv, const int32_t* pq,
                            int32_t n_pq) {
  if (!h->eng->initialized()) throw std::runtime_error("NewtonSolver::solve_batch(): initialize()를 먼저 호출해야 합니다.");
  if (rows != h->n_bus || nnz != (int32_t)h->ind.size())
    throw std::runtime_error("Ybus dimensions do not match initialize()");
  if (std::memcmp(indptr, h->ind_ptr.data(), (rows + 1) * sizeof(int32_t)) ||
      (nnz && std::memcmp(indices, h->ind.data(), nnz * sizeof(int32_t))))
    throw std::runtime_error("Ybus sparsity pattern changed after initialize()");
  if (data && std::memcmp(data, h->ydata.data(), 2 * (size_t)nnz * sizeof(double))) {
    // new branch values on the same pattern (the reference re-uploads them
    // every solve, cpu_fp64_storage.cpp:355-360)
    h->eng->update_ybus_values(data);
    h->ydata.assign(data, data + 2 * (size_t)nnz);
  }
  if (n_pv != (int32_t)h->pv.size() || n_pq != (int32_t)h->pq.size() ||
      (n_pv && std::memcmp(pv, h->pv.data(), n_pv * sizeof(int32_t))) ||
      (n_pq && std::memcmp(pq, h->pq.data(), n_pq * sizeof(int32_t))))
    throw std::invalid_argument("pv/pq must match initialize()");
}

pf_status pf_solve_batch(pf_handle h, const int32_t* indptr, const int32_t* indices, const double* data,
                         int32_t rows, int32_t cols, int32_t nnz, const double* sbus, int64_t sbus_stride,
                         const double* V0, int64_t V0_stride, int32_t batch, const int32_t* pv, int32_t n_pv,
                         const int32_t* pq, int32_t n_pq, const pf_nr_config* config,
                         const pf_solve_options* solve_options, double* V_out, int32_t* iterations,
                         double* final_mismatch, uint8_t* converged) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    (void)cols;
    if (batch <= 0) throw std::invalid_argument("NewtonSolver::solve_batch(): batch_size must be positive");
    check_same_case(h, indptr, indices, data, rows, nnz, pv, n_pv, pq, n_pq);
    const pf_nr_config cfg = config ? *config : pf_nr_config{1e-8, 50};
    const int prep = solve_options ? solve_options->prepare_adjoint_cache : 0;
    h->eng->solve_batch_host(sbus, sbus_stride, V0, V0_stride, batch, cfg.tolerance, cfg.max_iter, prep, V_out,
                             iterations, final_mismatch, converged);
  })
}

pf_status pf_solve_batch_device(pf_handle h, const double* sbus, int64_t sbus_stride, const double* V0,
                                int64_t V0_stride, int32_t batch, const pf_nr_config* config,
                                const pf_solve_options* solve_options, double* V_out, double* final_mismatch,
                                void* stream, pf_adjoint_result* result) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (!sbus || !V0) throw std::invalid_argument("sbus/V0 must not be null");
    if (sbus_stride < h->n_bus || V0_stride < h->n_bus) throw std::invalid_argument("stride must be at least n_bus");
    const pf_nr_config cfg = config ? *config : pf_nr_config{1e-8, 50};
    const int prep = solve_options ? solve_options->prepare_adjoint_cache : 0;
    const auto st = h->eng->solve_batch_device(sbus, sbus_stride, V0, V0_stride, batch, cfg.tolerance, cfg.max_iter,
                                               prep, V_out, final_mismatch, caller_stream(stream));
    if (result) {
      std::memset(result, 0, sizeof(*result));
      result->n_bus = h->n_bus;
      result->batch_size = batch;
      result->dim_f = h->eng->dim();
      result->success = 1;
      result->iterations = st.iterations;
      result->max_final_mismatch = st.max_final_mismatch;
      result->all_converged = st.all_converged;
    }
  })
}

pf_status pf_solve_batch_ybus(pf_handle h, const double* ybus_data, int64_t ybus_stride, const double* sbus,
                              int64_t sbus_stride, const double* V0, int64_t V0_stride, int32_t batch,
                              const pf_nr_config* config, const pf_solve_options* solve_options, double* V_out,
                              int32_t* iterations, double* final_mismatch, uint8_t* converged) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (!h->eng->initialized()) throw std::runtime_error("NewtonSolver::solve_batch(): initialize() must be called first");
    if (batch <= 0) throw std::invalid_argument("NewtonSolver::solve_batch(): batch_size must be positive");
    if (!ybus_data) throw std::invalid_argument("per-scenario Ybus values must not be null");
    if (ybus_stride < (int64_t)h->ind.size())
      throw std::invalid_argument("per-scenario Ybus stride must be at least the Ybus nnz");
    const pf_nr_config cfg = config ? *config : pf_nr_config{1e-8, 50};
    const int prep = solve_options ? solve_options->prepare_adjoint_cache : 0;
    h->eng->solve_batch_host(sbus, sbus_stride, V0, V0_stride, batch, cfg.tolerance, cfg.max_iter, prep, V_out,
                             iterations, final_mismatch, converged, ybus_data, ybus_stride);
  })
}

pf_status pf_solve_batch_ybus_device(pf_handle h, const double* ybus_data, int64_t ybus_stride, const double* sbus,
                                     int64_t sbus_stride, const double* V0, int64_t V0_stride, int32_t batch,
                                     const pf_nr_config* config, const pf_solve_options* solve_options,
                                     double* V_out, double* final_mismatch, void* stream, pf_adjoint_result* result) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (!sbus || !V0 || !ybus_data) throw std::invalid_argument("sbus/V0/ybus must not be null");
    if (sbus_stride < h->n_bus || V0_stride < h->n_bus) throw std::invalid_argument("stride must be at least n_bus");
    if (ybus_stride < (int64_t)h->ind.size())
      throw std::invalid_argument("per-scenario Ybus stride must be at least the Ybus nnz");
    const pf_nr_config cfg = config ? *config : pf_nr_config{1e-8, 50};
    const int prep = solve_options ? solve_options->prepare_adjoint_cache : 0;
    const auto st = h->eng->solve_batch_device(sbus, sbus_stride, V0, V0_stride, batch, cfg.tolerance, cfg.max_iter,
                                               prep, V_out, final_mismatch, caller_stream(stream), ybus_data,
                                               ybus_stride);
    if (result) {
      std::memset(result, 0, sizeof(*result));
      result->n_bus = h->n_bus;
      result->batch_size = batch;
      result->dim_f = h->eng->dim();
      result->success = 1;
      result->iterations = st.iterations;
      result->max_final_mismatch = st.max_final_mismatch;
      result->all_converged = st.all_converged;
    }
  })
}

pf_status pf_solve_batch_warm_device(pf_handle h, const double* sbus, int64_t sbus_stride, const double* V0,
                                     int64_t V0_stride, const float* pred, int64_t pred_ld, const float* pred_scale,
                                     const float* pred_shift, int32_t batch,
                                     const pf_nr_config* config, const pf_solve_options* solve_options,
                                     double* V_out, double* final_mismatch, void* stream, pf_adjoint_result* result) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (!sbus || !V0 || !pred) throw std::invalid_argument("sbus/V0/pred must not be null");
    if (sbus_stride < h->n_bus || (V0_stride != 0 && V0_stride < h->n_bus))
      throw std::invalid_argument("stride must be at least n_bus (V0_stride 0 = one V0 row for every scenario)");
    const pf_nr_config cfg = config ? *config : pf_nr_config{1e-8, 50};
    const int prep = solve_options ? solve_options->prepare_adjoint_cache : 0;
    if ((pred_scale == nullptr) != (pred_shift == nullptr))
      throw std::invalid_argument("pred_scale and pred_shift must be given together");
    const auto st = h->eng->solve_batch_warm_device(sbus, sbus_stride, V0, V0_stride, pred, pred_ld, pred_scale,
                                                    pred_shift, batch,
                                                    cfg.tolerance, cfg.max_iter, prep, V_out, final_mismatch,
                                                    caller_stream(stream));
    if (result) {
      std::memset(result, 0, sizeof(*result));
      result->n_bus = h->n_bus;
      result->batch_size = batch;
      result->dim_f = h->eng->dim();
      result->success = 1;
      result->iterations = st.iterations;
      result->max_final_mismatch = st.max_final_mismatch;
      result->all_converged = st.all_converged;
    }
  })
}

pf_status pf_solve_forward_device(pf_handle h, const void* sbus_base_re, const void* sbus_base_im,
                                  const void* load_p, const void* load_q, const void* v0_va, const void* v0_vm,
                                  int32_t batched_v0, void* va_out, void* vm_out, int32_t batch, int32_t n_bus,
                                  const char* dtype, const pf_nr_config* config,
                                  const pf_solve_options* solve_options, void* stream, pf_adjoint_result* result) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (!h->eng->initialized())
      throw std::runtime_error("cupf::torch_api::solve_forward(): initialize() must be called first");
    const std::string want = dtype_expected(h->opt);
    if (!dtype || want != dtype)
      throw std::invalid_argument("cupf::torch_api::solve_forward(): dtype must be " + want +
                                  " for this cuPF compute policy");
    if (n_bus != h->n_bus)
      throw std::invalid_argument("cupf::torch_api::solve_forward(): n_bus does not match initialized solver");
    if (batch <= 0) throw std::invalid_argument("cupf::torch_api::solve_forward(): batch_size must be positive");
    const pf_nr_config cfg = config ? *config : pf_nr_config{1e-8, 50};
    const int prep = solve_options ? solve_options->prepare_adjoint_cache : 0;
    const auto st = h->eng->solve_from_load(sbus_base_re, sbus_base_im, load_p, load_q, v0_va, v0_vm, batched_v0,
                                            va_out, vm_out, batch, want == "float64", cfg.tolerance, cfg.max_iter,
                                            prep, caller_stream(stream), nullptr);
    if (result) {
      std::memset(result, 0, sizeof(*result));
      result->n_bus = n_bus;
      result->batch_size = batch;
      result->dim_f = h->eng->dim();
      result->success = 1;
      result->iterations = st.iterations;
      result->max_final_mismatch = st.max_final_mismatch;
      result->all_converged = st.all_converged;
    }
  })
}

pf_status pf_solve_backward_device(pf_handle h, const void* grad_va, const void* grad_vm, void* grad_load_p,
                                   void* grad_load_q, int32_t batch, int32_t n_bus, const char* dtype,
                                   const pf_adjoint_options* options, void* stream, pf_adjoint_result* result) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    const std::string want = dtype_expected(h->opt);
    if (!dtype || want != dtype)
      throw std::invalid_argument("cupf::torch_api::solve_backward(): dtype must be " + want);
    if (n_bus != h->n_bus) throw std::invalid_argument("cupf::torch_api::solve_backward(): n_bus mismatch");
    if (!grad_load_p || !grad_load_q) throw std::invalid_argument("output gradients must not be null");
    const double res = h->eng->solve_adjoint_device(grad_va, grad_vm, grad_load_p, grad_load_q, nullptr, batch,
                                                    want == "float64", caller_stream(stream),
                                                    options ? options->check_residual != 0 : true);
    if (result) {
      std::memset(result, 0, sizeof(*result));
      result->n_bus = n_bus;
      result->batch_size = batch;
      result->dim_f = h->eng->dim();
      result->success = 1;
      result->used_adjoint_cache = 1;
      result->reused_final_state_factorization = 1;
      result->jt_residual_norm = res;
    }
  })
}

pf_status pf_solve_adjoint(pf_handle h, const double* grad_va, int64_t grad_va_stride, const double* grad_vm,
                           int64_t grad_vm_stride, int32_t batch, const int32_t* pv, int32_t n_pv,
                           const int32_t* pq, int32_t n_pq, const pf_adjoint_options* options, double* lambda,
                           double* grad_load_p, double* grad_load_q, pf_adjoint_result* result) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (!h->eng->initialized())
      throw std::runtime_error("NewtonSolver::solve_adjoint(): initialize() and solve()/solve_batch() must be called first");
    if (batch <= 0) throw std::invalid_argument("NewtonSolver::solve_adjoint(): batch_size must be positive");
    if (!grad_va || !grad_vm) throw std::invalid_argument("NewtonSolver::solve_adjoint(): grad_va/grad_vm must not be null");
    if (grad_va_stride < h->n_bus || grad_vm_stride < h->n_bus)
      throw std::invalid_argument("NewtonSolver::solve_adjoint(): grad strides must be at least n_bus");
    if (n_pv != (int32_t)h->pv.size() || n_pq != (int32_t)h->pq.size() ||
        (n_pv && std::memcmp(pv, h->pv.data(), n_pv * sizeof(int32_t))) ||
        (n_pq && std::memcmp(pq, h->pq.data(), n_pq * sizeof(int32_t))))
      throw std::invalid_argument("NewtonSolver::solve_adjoint(): pv/pq dimensions do not match solver dimF");
    if (options && options->require_cached_factorization && !h->eng->adjoint_cache_valid())
      throw std::runtime_error("NewtonSolver::solve_adjoint(): missing exact final-state adjoint cache");
    if (!h->eng->adjoint_cache_valid())
      throw std::runtime_error(
          "NewtonSolver::solve_adjoint(): no final-state factorization; solve with prepare_adjoint_cache=True");
    const int n = h->n_bus, dim = h->eng->dim();
    // stage the host gradients as dense [batch][n] on the device
    std::vector<double> ga((size_t)batch * n), gm((size_t)batch * n);
    for (int b = 0; b < batch; ++b) {
      std::memcpy(&ga[(size_t)b * n], grad_va + (size_t)b * grad_va_stride, n * sizeof(double));
      std::memcpy(&gm[(size_t)b * n], grad_vm + (size_t)b * grad_vm_stride, n * sizeof(double));
    }
    double *dga = nullptr, *dgm = nullptr, *dgp = nullptr, *dgq = nullptr, *dl = nullptr;
    const size_t bn = (size_t)batch * n * sizeof(double), bd = (size_t)batch * dim * sizeof(double);
    if (cudaMalloc(&dga, bn) || cudaMalloc(&dgm, bn) || cudaMalloc(&dgp, bn) || cudaMalloc(&dgq, bn) ||
        cudaMalloc(&dl, bd)) {
      cudaFree(dga); cudaFree(dgm); cudaFree(dgp); cudaFree(dgq); cudaFree(dl);
      throw std::runtime_error("solve_adjoint: device allocation failed");
    }
    struct Guard {
      double* p[5];
      ~Guard() {
        for (double* q : p) cudaFree(q);
      }
    } guard{{dga, dgm, dgp, dgq, dl}};
    cudaMemcpy(dga, ga.data(), bn, cudaMemcpyHostToDevice);
    cudaMemcpy(dgm, gm.data(), bn, cudaMemcpyHostToDevice);
    const double res = h->eng->solve_adjoint_device(dga, dgm, dgp, dgq, dl, batch, 1, cudaStreamLegacy,
                                                    options ? options->check_residual != 0 : true);
    if (lambda) cudaMemcpy(lambda, dl, bd, cudaMemcpyDeviceToHost);
    if (grad_load_p) cudaMemcpy(grad_load_p, dgp, bn, cudaMemcpyDeviceToHost);
    if (grad_load_q) cudaMemcpy(grad_load_q, dgq, bn, cudaMemcpyDeviceToHost);
    if (result) {
      std::memset(result, 0, sizeof(*result));
      result->n_bus = n;
      result->batch_size = batch;
      result->dim_f = dim;
      result->success = 1;
      result->used_adjoint_cache = 1;
      result->reused_final_state_factorization = 1;
      result->jt_residual_norm = res;
    }
  })
}

pf_status pf_info(pf_handle h, pf_info_t* out) {
  if (!h || !h->eng || !out) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    const auto& ja = h->eng->jacobian();
    const auto& fp = h->eng->program();
    std::memset(out, 0, sizeof(*out));
    out->n_bus = ja.n_bus;
    out->n_pv = ja.n_pv;
    out->n_pq = ja.n_pq;
    out->dim_f = ja.dim;
    out->nnz_ybus = (int32_t)ja.map11.size();
    out->nnz_jacobian = ja.nnz;
    out->num_panels = fp.P;
    out->num_levels = fp.num_levels;
    out->max_front = fp.max_fsz;
    out->max_panel = fp.max_nc;
    out->factor_elements = fp.u_total + fp.l_total + fp.cb_total;
    out->last_kernel_launches = h->eng->last_launches();
  })
}

pf_status pf_plan_array(pf_handle h, const char* name, int32_t* out, int64_t capacity, int64_t* len) {
  if (!h || !h->eng || h->eng->dim() <= 0) return PF_INVALID_ARGUMENT;
  if (!copy_plan_array(*h->eng, name, out, capacity, len)) {
    h->err = std::string("unknown plan array or capacity too small: ") + (name ? name : "");
    return PF_INVALID_ARGUMENT;
  }
  return PF_OK;
}

pf_status pf_dump_fronts_csv(pf_handle h, const char* path) {
  if (!h || !h->eng || h->eng->symbolic().level_ptr.empty()) return PF_INVALID_ARGUMENT;
  if (!path || !write_text_file(path, fronts_csv(h->eng->symbolic()))) {
    h->err = std::string("cannot write the front CSV to ") + (path ? path : "(null)");
    return PF_INVALID_ARGUMENT;
  }
  return PF_OK;
}

pf_status pf_evaluate(pf_handle h, const double* V, const double* sbus, int32_t batch, double* F, double* J) {
  if (!h || !h->eng || !V || !sbus || !F || !J) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    if (!h->eng->initialized()) throw std::runtime_error("pf_evaluate: initialize() must be called first");
    h->eng->evaluate_host(V, sbus, batch, F, J);
  })
}

pf_status pf_set_profiling(pf_handle h, int32_t enabled) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  h->eng->set_profiling(enabled != 0);
  return PF_OK;
}

pf_status pf_stage_times(pf_handle h, double* times_ms, int64_t* launches) {
  if (!h || !h->eng) return PF_INVALID_ARGUMENT;
  h->eng->stage_times_ms(times_ms, launches);
  return PF_OK;
}

pf_status pf_plan_array64(pf_handle h, const char* name, int64_t* out, int64_t capacity, int64_t* len) {
  if (!h || !h->eng || h->eng->dim() <= 0) return PF_INVALID_ARGUMENT;
  const auto& fp = h->eng->program();
  const std::string n(name ? name : "");
  const std::vector<int64_t>* v = nullptr;
  if (n == "fe_split") v = &fp.fe_split;
  if (n == "fe_src") v = &fp.fe_src;
  if (n == "fe_ptr") v = &fp.fe_ptr;
  if (n == "u_off") v = &fp.u_off;
  if (n == "l_off") v = &fp.l_off;
  if (n == "cb_off") v = &fp.cb_off;
  if (!v) {
    h->err = "unknown int64 plan array: " + n;
    return PF_INVALID_ARGUMENT;
  }
  if (len) *len = (int64_t)v->size();
  if (out) {
    if (capacity < (int64_t)v->size()) return PF_INVALID_ARGUMENT;
    if (!v->empty()) std::memcpy(out, v->data(), v->size() * sizeof(int64_t));
  }
  return PF_OK;
}

pf_status pf_singular_flags(pf_handle h, int32_t* out_host, int32_t batch) {
  if (!h || !h->eng || !out_host) return PF_INVALID_ARGUMENT;
  PF_TRY(h, {
    const std::vector<int32_t> f = h->eng->singular_flags();
    for (int32_t b = 0; b < batch; ++b) out_host[b] = b < (int32_t)f.size() ? f[b] : 0;
  })
}

}  // extern "C"
