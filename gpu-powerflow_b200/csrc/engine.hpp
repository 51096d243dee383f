// engine.hpp -- batched Newton-Raphson power-flow engine (host orchestration).
//
// One Engine = one grid (Ybus pattern + PV/PQ sets) analysed once, solved for
// any number of scenarios.  It is the engine behind the C ABI in
// include/cupf_b200.h and the role the reference's NewtonSolver + cuda-custom
// pipeline play (cuPF/cpp/inc/newton_solver/core/newton_solver.hpp:26-102,
// cuPF/cpp/src/newton_solver/core/pipeline.hpp:350-388).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "analysis.hpp"
#include "device_plan.cuh"
#include "kernels.hpp"

namespace cupf_b200 {

enum ComputeMode : int32_t { kComputeFP64 = 0, kComputeFP32 = 1, kComputeMixed = 2 };
enum FactorPrecision : int32_t { kFactorFP64 = 0, kFactorFP32 = 1, kFactorTF32 = 2 };

struct EngineConfig {
  int32_t compute = kComputeMixed;
  int32_t factor_precision = kFactorFP32;
  int32_t max_panel_width = 8;
  int32_t serial_nd = 1;
  int32_t use_matching = 0;       // structural (Hopcroft-Karp) column matching
  int32_t jacobian_kind = 0;      // CudaJacobianKind: 0 Edge, 1 EdgeAtomic, 2 VertexWarp
  int32_t static_pivot = 1;       // StaticDiagonalShift
  double shift_epsilon = 1e-8;    // threshold and replacement magnitude
  int32_t use_cuda_graph = 0;     // run each solve as one graph (device-side convergence test)
  int32_t adjoint_refine_steps = 2;
  int32_t autotune = 0;           // tune the factor levels' warps per block per batch size
  int32_t par_nd_depth = 4, par_nd_base_small = 4000, par_nd_base_large = 20000;
  int32_t wide_min_front = 65;  // launches with a front this large run the any-size tier
  int32_t tc_min_front = 0;     // TF32: launches with a front this large use the tensor cores (0: 33 / autotuned)
  int32_t batch1_schedule = 0;  // batch 1: 0 the single-system front kernel, 1 the lane kernels
};

struct SolveStats {
  int32_t iterations = 0;
  double max_final_mismatch = 0.0;
  int32_t all_converged = 0;
  int32_t any_shifted_pivot = 0;
};

class Engine {
 public:
  explicit Engine(const EngineConfig& cfg);
  ~Engine();
  Engine(const Engine&) = delete;
  Engine& operator=(const Engine&) = delete;

  // Host CSR Ybus (complex as interleaved doubles), PV/PQ bus lists.
  void initialize(int32_t n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                  const int32_t* pv, int32_t n_pv, const int32_t* pq, int32_t n_pq);
  // Linear-solver use: analyse an n x n CSR pattern (no Ybus / NR state).
  void initialize_matrix(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx);
  // Host-only analysis (no device memory): for plan introspection on machines
  // without a GPU.  The engine cannot solve after this call alone.
  void analyze_host(int32_t n_bus, const int32_t* indptr, const int32_t* indices, const int32_t* pv, int32_t n_pv,
                    const int32_t* pq, int32_t n_pq);
  void analyze_matrix_host(int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx);
  bool initialized() const { return initialized_; }
  // New Ybus values on the analysed pattern (complex interleaved, CSR order).
  void update_ybus_values(const double* ydata);

  // NewtonSolver::solve_batch semantics with host buffers: sbus / v0 are
  // complex [B][stride]; outputs V [B][n] complex, per-scenario stats.
  SolveStats solve_batch_host(const double* sbus, int64_t sbus_stride, const double* v0, int64_t v0_stride,
                              int32_t B, double tol, int32_t max_iter, int32_t prepare_adjoint, double* v_out,
                              int32_t* iterations, double* final_mismatch, uint8_t* converged,
                              const double* ybus = nullptr, int64_t ybus_stride = 0);
  // Same with device-resident inputs/outputs in the same host layout.  With
  // d_ybus (complex [B][ybus_stride], CSR order of the analysed pattern) every
  // scenario has its own Ybus values; otherwise all share the handle's.
  SolveStats solve_batch_device(const double* d_sbus, int64_t sbus_stride, const double* d_v0, int64_t v0_stride,
                                int32_t B, double tol, int32_t max_iter, int32_t prepare_adjoint, double* d_v_out,
                                double* d_final_mismatch, cudaStream_t stream, const double* d_ybus = nullptr,
                                int64_t ybus_stride = 0);
  // solve_batch_device from a predicted state (Jacobian-row order, fp32)
  SolveStats solve_batch_warm_device(const double* d_sbus, int64_t sbus_stride, const double* d_v0, int64_t v0_stride,
                                     const float* d_pred, int64_t pred_ld, const float* d_scale, const float* d_shift,
                                     int32_t B, double tol, int32_t max_iter,
                                     int32_t prepare_adjoint, double* d_v_out, double* d_final_mismatch,
                                     cudaStream_t stream);
  // torch-style: Sbus = base - load, V0 = (va0, vm0); base/v0 shared [n] or
  // v0 batched [B][n]; outputs Va/Vm [B][n]; float or double per is_double.
  SolveStats solve_from_load(const void* base_re, const void* base_im, const void* load_p, const void* load_q,
                             const void* va0, const void* vm0, int32_t batched_v0, void* va_out, void* vm_out,
                             int32_t B, int32_t is_double, double tol, int32_t max_iter, int32_t prepare_adjoint,
                             cudaStream_t stream, double* d_final_mismatch);
  // Adjoint on the cached final-state factors: grads [B][n] device, outputs
  // grad_p / grad_q [B][n]; optional lambda [B][dimF] (double, device).
  // The relative residual ||J^T lambda - g|| / ||g|| is returned when
  // `residual` (else 0).
  double solve_adjoint_device(const void* grad_va, const void* grad_vm, void* grad_p, void* grad_q,
                              double* d_lambda, int32_t B, int32_t is_double, cudaStream_t stream,
                              bool residual = true);

  // Linear-solver boundary: factor caller-supplied Jacobian values and solve.
  void factorize_values(const void* d_values, int32_t values_is_double, int32_t B, cudaStream_t stream);
  // factorize_values with the global front scratch in a fixed caller area;
  // allocates nothing (the workspace must already hold batch B)
  void factorize_values_static_scratch(const void* d_values, int32_t values_is_double, int32_t B, void* scratch,
                                       size_t scratch_bytes, cudaStream_t stream);
  void solve_values(const void* d_rhs, int32_t rhs_is_double, void* d_x, int32_t x_is_double, int32_t B,
                    bool transpose, cudaStream_t stream);

  // Evaluate F and J (fp64) at host states V / Sbus ([B][n] complex).
  void evaluate_host(const double* V, const double* sbus, int32_t B, double* F_out, double* J_out);

  const JacobianAnalysis& jacobian() const { return ja_; }
  const SymbolicPlan& symbolic() const { return sp_; }
  // warps per block of each factor level launch (0: the built-in rule)
  std::vector<int32_t> factor_level_warps() const;
  // factor kernel tier of each launch (0 register rows, 1 any-size, 2 tensor
  // cores) and the tensor-core threshold in use (0 when not TF32)
  std::vector<int32_t> factor_level_tiers() const;
  // where each factor launch keeps its dense fronts: 1 shared memory, 2 the global scratch
  std::vector<int32_t> factor_level_placements() const;
  int32_t tc_threshold() const { return tc_min_; }
  // the same for the backward sweep's launches, tree top first
  std::vector<int32_t> backward_launch_warps() const;
  const FactorProgram& program() const { return fp_; }
  const EngineConfig& config() const { return cfg_; }
  int32_t n_bus() const { return ja_.n_bus; }
  int32_t dim() const { return ja_.dim; }
  bool factor_is_double() const;
  bool adjoint_cache_valid() const { return adjoint_ready_; }
  int32_t cached_batch() const { return B_; }
  std::vector<int32_t> singular_flags() const;  // per scenario of the last factorization
  // kernel launches issued by the last solve (for reporting)
  int64_t last_launches() const { return launches_; }
  // Stage timers (the reference's NR.iteration.* StageScope labels,
  // newton_solver.cpp:521-553) measured with CUDA events on the solve stream.
  // Stages: 0 mismatch (ibus+mismatch+norm), 1 jacobian, 2 factorize,
  // 3 solve, 4 voltage_update.  Enabling adds event records, no host syncs.
  void set_profiling(bool on) { profiling_ = on; }
  void stage_times_ms(double* out5, int64_t* launches5) const;

 private:
  struct Impl;
  std::unique_ptr<Impl> d_;
  EngineConfig cfg_;
  JacobianAnalysis ja_;
  SymbolicPlan sp_;
  FactorProgram fp_;
  bool initialized_ = false;
  bool adjoint_ready_ = false;
  int32_t B_ = 0;
  int64_t launches_ = 0;
  bool profiling_ = false;
  bool tolerate_nonfinite_ = false;  // set during warm-started solves
  int32_t tc_min_ = 0;               // tensor-core tier threshold in use (TF32 factors)
  template <typename T>
  void factor_all_external(cudaStream_t s, const void* J, T* scratch, size_t scratch_elems);
  void stage_begin(int stage, cudaStream_t s);
  void stage_end(int stage, cudaStream_t s);
  void collect_stage_times();

  void ensure_workspace(int32_t B);
  void upload_plan();
  // factor kernel tier of every launch: the any-size tier from wide_min_front
  // rows, and with TF32 factors the tensor-core tier from tc_min rows
  void assign_tiers(int tc_min);
  bool tf32_factors() const;
  // batch 1 with the single-system schedule: one block per front, threads over its rows
  bool single_system() const;
  // ... and the whole factorization as one launch over the front tree
  bool single_tree(size_t elem_bytes) const;
  template <typename T>
  void factor_tree(const FactorArgs<T, T>& a, cudaStream_t s);
  // selects per-scenario (d_ybus != null) or shared Ybus values for this batch
  void use_scenario_ybus(const double* d_ybus, int64_t ybus_stride, int32_t B, cudaStream_t s);
  template <typename T>
  // d_v_out: when given, the final voltages are packed into it (host
  // layout, complex [B][n]) before the loop's closing synchronisation
  SolveStats run_loop(double tol, int32_t max_iter, int32_t prepare_adjoint, cudaStream_t s, double* d_final,
                      double* d_v_out = nullptr);
  template <typename T>
  void ensure_loop_graph(const DevState& st);
  template <typename T>
  void iteration_tail(cudaStream_t s, int store_l);
  template <typename T>
  void factor_all(cudaStream_t s, int store_l, const void* J);
  template <typename T>
  FactorArgs<T, T> factor_args(int store_l, const void* J) const;
  // times every factor level with each candidate block shape on the values J
  // and keeps the fastest per level (once per batch size and precision)
  template <typename T>
  void autotune_factor(cudaStream_t s, const void* J);
  template <typename T>
  void autotune_backward(cudaStream_t s);
  template <typename T>
  SweepArgs<T> sweep_args() const;
  template <typename T>
  void backward_all(cudaStream_t s);
  template <typename T>
  int64_t backward_levels(const SweepArgs<T>& a, cudaStream_t s);
  template <typename T>
  void transpose_solve(const double* d_G, double* d_lam, cudaStream_t s);
};

}  // namespace cupf_b200
