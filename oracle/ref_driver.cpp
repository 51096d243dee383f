// ref_driver.cpp -- C entry points into the REFERENCE's own CPU NewtonSolver
// (TEST INFRASTRUCTURE ONLY).
//
// Built by oracle/Makefile together with the reference's CPU core sources
// (cuPF/CMakeLists.txt:243-262 CUPF_CORE_SOURCES, compiled where they lie) and
// the KLU shim, into oracle/_ref/libcupf_ref.so.  Each function runs the
// reference's public C++ API (NewtonSolver, cuPF/cpp/inc/newton_solver/core/
// newton_solver.hpp:26-102) on the CPU backend and copies the results out, so
// the oracle restatement and the GPU engine can be checked against the
// reference itself.
#include <complex>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "dump_case_loader.hpp"
#include "newton_solver/core/newton_solver.hpp"
#include "newton_solver/ops/jacobian/jacobian_analysis.hpp"

namespace {
thread_local std::string g_error;

YbusView make_view(int n, const int32_t* indptr, const int32_t* indices, const double* ydata) {
  return YbusView{indptr, indices, reinterpret_cast<const std::complex<double>*>(ydata), n, n, indptr[n]};
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_error.c_str(); }

// NewtonSolver::solve_batch on the CPU backend (batch 1 per call; the CPU
// pipeline rejects batch > 1, newton_solver.cpp:268-276).
int ref_nr_solve(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                 const double* sbus, const double* v0, const int32_t* pv, int n_pv, const int32_t* pq,
                 int n_pq, double tol, int max_iter, double* v_out, int32_t* iterations,
                 double* final_mismatch, int32_t* converged) {
  try {
    NewtonOptions opts;
    opts.backend = BackendKind::CPU;
    opts.cpu_linear_solver = CpuLinearSolverKind::KLU;
    NewtonSolver solver(opts);
    const YbusView y = make_view(n_bus, indptr, indices, ydata);
    solver.initialize(y, pv, n_pv, pq, n_pq);
    NRConfig cfg;
    cfg.tolerance = tol;
    cfg.max_iter = max_iter;
    NRResult res;
    solver.solve(y, reinterpret_cast<const std::complex<double>*>(sbus),
                 reinterpret_cast<const std::complex<double>*>(v0), pv, n_pv, pq, n_pq, cfg, SolveOptions{}, res);
    std::memcpy(v_out, res.V.data(), sizeof(double) * 2 * n_bus);
    *iterations = res.iterations;
    *final_mismatch = res.final_mismatch;
    *converged = res.converged ? 1 : 0;
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

// Forward solve with the adjoint cache, then NewtonSolver::solve_adjoint
// (newton_solver_adjoint.cpp:33-153).
int ref_nr_adjoint(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                   const double* sbus, const double* v0, const int32_t* pv, int n_pv, const int32_t* pq,
                   int n_pq, double tol, int max_iter, const double* grad_va, const double* grad_vm,
                   double* v_out, double* lambda, double* grad_p, double* grad_q, double* residual) {
  try {
    NewtonOptions opts;
    opts.backend = BackendKind::CPU;
    NewtonSolver solver(opts);
    const YbusView y = make_view(n_bus, indptr, indices, ydata);
    solver.initialize(y, pv, n_pv, pq, n_pq);
    NRConfig cfg;
    cfg.tolerance = tol;
    cfg.max_iter = max_iter;
    SolveOptions so;
    so.prepare_adjoint_cache = true;
    NRResult res;
    solver.solve(y, reinterpret_cast<const std::complex<double>*>(sbus),
                 reinterpret_cast<const std::complex<double>*>(v0), pv, n_pv, pq, n_pq, cfg, so, res);
    std::memcpy(v_out, res.V.data(), sizeof(double) * 2 * n_bus);
    AdjointOptions ao;
    AdjointResult ar;
    solver.solve_adjoint(grad_va, n_bus, grad_vm, n_bus, 1, pv, n_pv, pq, n_pq, ao, ar);
    std::memcpy(lambda, ar.lambda.data(), sizeof(double) * ar.lambda.size());
    std::memcpy(grad_p, ar.grad_load_p.data(), sizeof(double) * n_bus);
    std::memcpy(grad_q, ar.grad_load_q.data(), sizeof(double) * n_bus);
    *residual = ar.jt_residual_norm;
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

// `count` independent cases spread over `threads` host threads, one reference
// NewtonSolver per thread (the CPU pipeline is batch-1 only, pipeline.hpp:121).
// sbus / v0 rows have stride 2 * n_bus doubles.
int ref_nr_solve_many(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                      const double* sbus, const double* v0, int count, const int32_t* pv, int n_pv,
                      const int32_t* pq, int n_pq, double tol, int max_iter, int threads, double* v_out,
                      int32_t* iterations, double* final_mismatch) {
  if (threads < 1) threads = 1;
  std::vector<std::thread> pool;
  std::vector<std::string> errs(threads);
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t] {
      try {
        NewtonOptions opts;
        opts.backend = BackendKind::CPU;
        NewtonSolver solver(opts);
        const YbusView y = make_view(n_bus, indptr, indices, ydata);
        solver.initialize(y, pv, n_pv, pq, n_pq);
        NRConfig cfg;
        cfg.tolerance = tol;
        cfg.max_iter = max_iter;
        const size_t stride = 2 * (size_t)n_bus;
        for (int c = t; c < count; c += threads) {
          NRResult res;
          solver.solve(y, reinterpret_cast<const std::complex<double>*>(sbus + c * stride),
                       reinterpret_cast<const std::complex<double>*>(v0 + c * stride), pv, n_pv, pq, n_pq, cfg,
                       SolveOptions{}, res);
          if (v_out) std::memcpy(v_out + c * stride, res.V.data(), sizeof(double) * stride);
          if (iterations) iterations[c] = res.iterations;
          if (final_mismatch) final_mismatch[c] = res.final_mismatch;
        }
      } catch (const std::exception& e) {
        errs[t] = e.what();
      }
    });
  }
  for (auto& th : pool) th.join();
  for (auto& e : errs)
    if (!e.empty()) {
      g_error = e;
      return 1;
    }
  return 0;
}

// make_jacobian_indexing + JacobianPatternGenerator + JacobianMapBuilder
// (jacobian_analysis.cpp:257-445).  Call with row_ptr == nullptr first to get
// dim and nnz.
int ref_jacobian_analysis(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                          const int32_t* pv, int n_pv, const int32_t* pq, int n_pq, int32_t* dim_out,
                          int32_t* nnz_out, int32_t* row_ptr, int32_t* col_idx, int32_t* maps_out) {
  try {
    const YbusView y = make_view(n_bus, indptr, indices, ydata);
    const JacobianIndexing ix = make_jacobian_indexing(n_bus, pv, n_pv, pq, n_pq);
    const JacobianPattern pat = JacobianPatternGenerator().generate(y, ix);
    *dim_out = pat.dim;
    *nnz_out = pat.nnz;
    if (!row_ptr) return 0;
    const JacobianScatterMap m = JacobianMapBuilder().build(y, ix, pat);
    std::memcpy(row_ptr, pat.row_ptr.data(), sizeof(int32_t) * (pat.dim + 1));
    std::memcpy(col_idx, pat.col_idx.data(), sizeof(int32_t) * pat.nnz);
    const int nnz_y = indptr[n_bus];
    const std::vector<int32_t>* per_entry[4] = {&m.mapJ11, &m.mapJ21, &m.mapJ12, &m.mapJ22};
    const std::vector<int32_t>* per_bus[4] = {&m.diagJ11, &m.diagJ21, &m.diagJ12, &m.diagJ22};
    int32_t* w = maps_out;
    for (auto* v : per_entry) {
      std::memcpy(w, v->data(), sizeof(int32_t) * nnz_y);
      w += nnz_y;
    }
    for (auto* v : per_bus) {
      std::memcpy(w, v->data(), sizeof(int32_t) * n_bus);
      w += n_bus;
    }
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

// cupf::tests::load_dump_case (cuPF/tests/dump_case_loader.cpp:210-232):
// sizes when any output pointer is null, else the arrays (complex as re, im).
int ref_load_dump_case(const char* dir, int32_t* rows, int32_t* nnz, int32_t* n_pv, int32_t* n_pq, int32_t* indptr,
                       int32_t* indices, double* ydata, double* sbus, double* v0, int32_t* pv, int32_t* pq) {
  try {
    const auto d = cupf::tests::load_dump_case(dir);
    *rows = d.rows;
    *nnz = (int32_t)d.ybus_data.size();
    *n_pv = (int32_t)d.pv.size();
    *n_pq = (int32_t)d.pq.size();
    if (!indptr || !indices || !ydata || !sbus || !v0 || !pv || !pq) return 0;
    std::memcpy(indptr, d.indptr.data(), d.indptr.size() * sizeof(int32_t));
    std::memcpy(indices, d.indices.data(), d.indices.size() * sizeof(int32_t));
    std::memcpy(ydata, d.ybus_data.data(), d.ybus_data.size() * sizeof(std::complex<double>));
    std::memcpy(sbus, d.sbus.data(), d.sbus.size() * sizeof(std::complex<double>));
    std::memcpy(v0, d.v0.data(), d.v0.size() * sizeof(std::complex<double>));
    if (!d.pv.empty()) std::memcpy(pv, d.pv.data(), d.pv.size() * sizeof(int32_t));
    if (!d.pq.empty()) std::memcpy(pq, d.pq.data(), d.pq.size() * sizeof(int32_t));
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 1;
  }
}

}  // extern "C"
