// ref_gpu_driver.cpp -- a C shim over the reference's own GPU linear solver
// (custom_linear_solver::Solver, custom_linear_solver/src/solver.hpp:80-114),
// compiled from the reference sources by oracle/Makefile (target refgpu) for
// compute_86 PTX, which the driver JIT-compiles for the B200.
//
// TEST INFRASTRUCTURE ONLY: it lets bench.py time the reference's GPU
// factorization and solve beside this engine's on the same GPU and the same
// matrices.  Nothing in the engine links or calls it.
//
// Buffers follow the reference's conventions: device CSR pattern (int32),
// batch-strided values [B][nnz], rhs and solution [B][n].
#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <string>

#include "solver.hpp"

namespace cls = custom_linear_solver;

namespace {
thread_local std::string g_err;

struct Handle {
  cls::Solver solver;
  explicit Handle(const cls::SolverConfig& c) : solver(c) {}
};

int status(cls::Status s, const char* what) {
  if (s == cls::Status::kSuccess) return 0;
  g_err = std::string(what) + ": " + cls::StatusString(s);
  return 1 + static_cast<int>(s);
}
}  // namespace

extern "C" {

const char* rg_last_error() { return g_err.c_str(); }

// precision 0 FP64, 1 FP32, 2 TF32; serial_nd 1 = one METIS_NodeND call
void* rg_create(int precision, int serial_nd) {
  try {
    cls::SolverConfig c;
    c.precision = precision == 0 ? cls::Precision::FP64 : precision == 1 ? cls::Precision::FP32 : cls::Precision::TF32;
    c.use_parallel_nested_dissection = serial_nd == 0;
    return new Handle(c);
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

void rg_destroy(void* h) { delete static_cast<Handle*>(h); }

// device pattern; values (device, [B][nnz]) registered for Factorize, rhs and
// solution (device, [B][n]) for Solve; value_type 0 f64, 1 f32 for each
int rg_setup(void* hv, int n, int nnz, const int32_t* d_row_ptr, const int32_t* d_col_idx, const void* d_values,
             int values_f32, void* d_rhs, int rhs_f32, void* d_x, int x_f32, int batch) {
  auto* h = static_cast<Handle*>(hv);
  cls::CsrMatrixView m;
  m.nrows = m.ncols = n;
  m.nnz = nnz;
  m.index_type = cls::IndexType::kInt32;
  m.location = cls::DataLocation::kDevice;
  m.value_type = values_f32 ? cls::ValueType::kFloat32 : cls::ValueType::kFloat64;
  m.row_offsets = d_row_ptr;
  m.col_indices = d_col_idx;
  m.values = d_values;
  cls::DenseVectorView r, x;
  r.size = x.size = (int64_t)n * batch;
  r.location = x.location = cls::DataLocation::kDevice;
  r.value_type = rhs_f32 ? cls::ValueType::kFloat32 : cls::ValueType::kFloat64;
  x.value_type = x_f32 ? cls::ValueType::kFloat32 : cls::ValueType::kFloat64;
  r.values = d_rhs;
  x.values = d_x;
  if (int e = status(h->solver.SetData(m), "SetData")) return e;
  if (int e = status(h->solver.SetRhs(r), "SetRhs")) return e;
  if (int e = status(h->solver.SetSolution(x), "SetSolution")) return e;
  if (int e = status(h->solver.Analyze(), "Analyze")) return e;
  return status(h->solver.Setup(batch), "Setup");
}

int rg_factorize(void* hv) { return status(static_cast<Handle*>(hv)->solver.Factorize(), "Factorize"); }
int rg_solve(void* hv) { return status(static_cast<Handle*>(hv)->solver.Solve(), "Solve"); }

}  // extern "C"
