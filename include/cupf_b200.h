/*
 * cupf_b200.h -- C ABI of the B200 batched Newton-Raphson power-flow engine.
 *
 * Plain pointers, sizes and integer status codes; no C++ or torch types cross
 * this boundary.  Two layers, each replacing one reference interface:
 *
 *   cls_*  the batched sparse direct solver behind cuPF's "cuda-custom"
 *          backend: custom_linear_solver::Solver's phase API
 *          (custom_linear_solver/src/solver.hpp:67-114) -- SetData / Analyze /
 *          Setup / SetStream / Factorize / Solve -- plus the transpose solve the
 *          reference lacks (cuda_custom_solver.cpp:268-307 throws) and per-system
 *          singular-pivot flags (the reference never reads d_sing back,
 *          factorize.cu:68).
 *
 *   pf_*   the Newton solver itself: NewtonSolver (cuPF/cpp/inc/newton_solver/
 *          core/newton_solver.hpp:26-102) -- initialize, solve_batch,
 *          solve_adjoint, and the device-pointer entry points behind cuPF's
 *          torch extension (cuPF/bindings/torch_cupf_extension.cpp:81-173).
 *
 * Batch layout at the boundary is the reference's: scenario-major, value
 * (scenario b, element k) at b * stride + k.  Complex arrays are interleaved
 * (re, im) doubles, i.e. std::complex<double>.
 *
 * Streams: the device-pointer entry points (pf_solve_*_device) run on the
 * caller's `stream`; NULL means the legacy default stream, so the engine's
 * kernels stay ordered with whatever the caller queued there before (torch
 * reports its default stream as handle 0).
 *
 * Errors: every function returns a status; *_last_error() gives the message.
 * PF_INVALID_ARGUMENT corresponds to the reference's std::invalid_argument,
 * PF_RUNTIME_ERROR to std::runtime_error.  Handles are not thread-safe.
 */
#ifndef CUPF_B200_H
#define CUPF_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Linear-solver layer (custom_linear_solver::Solver)                        */
/* ------------------------------------------------------------------------ */

/* custom_linear_solver::Status (solver.hpp:21-29), same order. */
typedef enum {
  CLS_SUCCESS = 0,
  CLS_INVALID_VALUE = 1,
  CLS_INVALID_STATE = 2,
  CLS_ALLOCATION_FAILED = 3,
  CLS_ANALYSIS_FAILED = 4,
  CLS_FACTORIZATION_FAILED = 5,
  CLS_SOLVE_FAILED = 6
} cls_status;

/* CustomPrecision / ValueType / DataLocation values */
enum { CLS_PRECISION_FP64 = 0, CLS_PRECISION_FP32 = 1, CLS_PRECISION_TF32 = 2 };
enum { CLS_VALUE_FLOAT64 = 0, CLS_VALUE_FLOAT32 = 1 };
enum { CLS_LOCATION_HOST = 0, CLS_LOCATION_DEVICE = 1 };
enum { CLS_PIVOT_NONE = 0, CLS_PIVOT_STATIC_DIAGONAL_SHIFT = 1 };

/* SolverConfig / CustomSolverConfig (solver.hpp:35-65,
 * cuPF newton_solver_types.hpp:152-159).  matching 1 (Structural) computes a
 * Hopcroft-Karp row -> column matching before the ordering and factors
 * P_r A P_c^T with the columns following their matched rows
 * (analyze/pipeline.cpp:77-160, 222-272); plan arrays "row_iperm",
 * "col_perm" and "row_to_col" expose it. */
typedef struct {
  int32_t precision;            /* CLS_PRECISION_*; TF32 = FP32 factors with tensor-core trailing updates */
  int32_t matching;             /* 0 = None, 1 = Structural */
  int32_t pivot_strategy;       /* CLS_PIVOT_* */
  int32_t serial_nd;            /* 1 = one METIS_NodeND call, 0 = separator recursion */
  int32_t max_panel_width;      /* 1..8 (front kernels are built for panels of at most 8 pivots) */
  double shift_retry_epsilon;   /* static-shift threshold and magnitude */
  int32_t autotune;             /* 1 = at the first factorization of each batch size, time every
                                   factor level with 1, 2, 4 and 8 warps per block on the actual
                                   values and keep the fastest per level (results do not change:
                                   the warps of a block share one front's arithmetic, each
                                   element's operation order is fixed); 0 = built-in rule */
  int32_t parallel_nd_depth;    /* separator recursion when serial_nd = 0 (SolverConfig::
                                   parallel_nd_depth, parallel_nd_base_small, parallel_nd_base_large,
                                   solver.hpp:44-46): recursion depth, and the graph size below */
  int32_t parallel_nd_base_small; /* which a part is ordered by one METIS call, for graphs of fewer */
  int32_t parallel_nd_base_large; /* than 20,000 vertices / otherwise; 0 = the defaults 4, 4000, 20000 */
  int32_t wide_min_front;       /* factor launches whose largest front has at least this many rows run the
                                   wide tier, which takes fronts of any size (the register kernels stop at
                                   64 rows); 1..65, 0 = 65.  Both give the same factors. */
  int32_t tc_min_front;         /* precision TF32: launches whose largest front has at least this many rows
                                   run their trailing update CB = A22 - L21 U12 on the tensor cores
                                   (tcgen05 kind::tf32, operands split hi + lo, fp32 accumulation); 0 = 65,
                                   or the fastest of 33, 49 and 65 when autotune is on */
  int32_t batch1_schedule;      /* a batch of one system: 0 = one block per front with its threads over the
                                   front's rows and elements (the reference's single-system path,
                                   factorize/single.cuh); 1 = the batched kernels, whose lanes are scenarios
                                   (31 of 32 then copy the one system).  Both give the same factors. */
} cls_config;

typedef struct cls_solver_s* cls_handle;

/* Replaces: Solver::Solver(config) / ~Solver (solver.hpp:82-83) */
cls_status cls_create(const cls_config* config, cls_handle* out);
cls_status cls_destroy(cls_handle h);
/* Replaces: Solver::SetData(CsrMatrixView) (solver.hpp:90); int32 CSR pattern
 * of an n x n matrix, on the host or the device. */
cls_status cls_set_data(cls_handle h, int32_t n, int32_t nnz, const int32_t* row_ptr, const int32_t* col_idx,
                        int32_t location);
/* Replaces: Solver::Analyze() (solver.hpp:100) */
cls_status cls_analyze(cls_handle h);
/* Analyze on the host only (no device memory); for plan introspection
 * through cls_plan_array on machines without a GPU.  cls_analyze is still
 * required before factorizing. */
cls_status cls_analyze_host(cls_handle h);
/* Replaces: Solver::Setup(batch_size) (solver.hpp:101) */
cls_status cls_setup(cls_handle h, int32_t batch_size);
/* Replaces: Solver::SetStream(void*) (solver.hpp:109).  NULL selects the
 * legacy default stream; a handle never given a stream uses a private one
 * (its factorize / solve calls synchronise that stream before returning). */
cls_status cls_set_stream(cls_handle h, void* stream);
/* Replaces: Solver::SetValues + Factorize() (solver.hpp:91,102); device values
 * [batch][nnz] in CSR order. */
cls_status cls_factorize(cls_handle h, const void* values, int32_t value_type);
/* New, no reference counterpart: cls_factorize for callers that must not
 * allocate device memory in the call (their memory is pooled or reserved
 * up front, or they cannot afford the implicit synchronisation of an
 * allocation).  The dense fronts that exceed shared memory use a fixed 8 MiB
 * static device area instead of the handle's workspace.  The call allocates
 * nothing; it therefore needs the handle's workspace to exist for this batch
 * size already (one regular cls_factorize at this batch size or larger), and
 * it rejects a batch whose front scratch exceeds 8 MiB (CLS_INVALID_VALUE,
 * message in cls_last_error).  Nothing has to be zeroed beforehand.  The area
 * is shared by all handles of the process on a device: calls must not
 * overlap in time.  The regular call that sizes the handle's workspace
 * looks the area's address up (cudaGetSymbolAddress with the handle's device
 * current), which is when the runtime loads the area's module and reserves
 * its memory, so not even the first call of this entry point does; make
 * that regular call before any stream capture.  The address is cached for
 * the life of the process: after
 * cudaDeviceReset on a device the cache is stale and this entry point must
 * not be used there again.  The launches use the built-in placement of the
 * dense fronts (not an autotuned one), which the 8 MiB bound refers to. */
cls_status cls_factorize_static_scratch(cls_handle h, const void* values, int32_t value_type);
/* Replaces: Solver::SetRhs / SetSolution / Solve() (solver.hpp:93-94,103);
 * device rhs / solution [batch][n]; pairs f64/f64, f64/f32, f32/f32. */
cls_status cls_solve(cls_handle h, const void* rhs, int32_t rhs_type, void* solution, int32_t solution_type);
/* New: A^T x = b on the same factors (no reference counterpart). */
cls_status cls_solve_transpose(cls_handle h, const void* rhs, int32_t rhs_type, void* solution,
                               int32_t solution_type);
/* New: per-system flag, 1 when a pivot was shifted in the last factorization. */
cls_status cls_singular_flags(cls_handle h, int32_t* out_host, int32_t batch);
/* Replaces: StatusString (solver.hpp:116) */
const char* cls_status_string(cls_status s);
const char* cls_last_error(cls_handle h);
/* Plan introspection: copies the named int32 array of the symbolic plan
 * ("perm", "iperm", "parent", "Lp", "Li", "panel_first", "panel_ncols",
 * "panel_width", "panel_of", "front_ptr", "front_rows", "panel_parent",
 * "asm_ptr", "asm_idx", "asm_local", "plevel", "level_ptr", "plcols_level",
 * "front_off", "a_pos_csr", "graph_xadj", "graph_adjncy", "sym_col_ptr",
 * "sym_row_idx"), or of the engine's launch plan: "factor_level_warps" and
 * "backward_launch_warps" (the autotuner's block shapes, 0 = built-in rule),
 * "factor_level_tiers" (per factor launch: 0 register-row kernel, 1 any-size
 * tier, 2 any-size tier with the tensor-core trailing update),
 * "factor_level_placement" (per factor launch: 1 dense fronts in shared
 * memory, 2 in the global scratch, 3 a register-tier launch of large fronts
 * run by the any-size tier instead; the autotuner chooses it with the block
 * shape, and a launch of the any-size tier may take 16 or 32 warps) and
 * "tc_threshold" (one value: the front size from which TF32 factors use the
 * tensor cores, 0 for other precisions).  With out == NULL only *len is set. */
cls_status cls_plan_array(cls_handle h, const char* name, int32_t* out, int64_t capacity, int64_t* len);
/* Writes the per-front structure of the analysed plan to a CSV file:
 * q,p,fsz,nc,uc,level,parent,asm_len,extend_elems, the columns of the
 * reference's front dump (SolverConfig::analyze_dump_fronts_path,
 * custom_linear_solver/src/solver.cpp:120, written by MaybeDumpFronts,
 * analyze/pipeline.cpp:162-193).  Rows follow the panel levels, leaves first,
 * each level's panels ascending: the order of the reference's dump under
 * analyze_fronts_only; its full analysis lists the same rows in its own
 * dispatch order inside each level.  Returns CLS_INVALID_VALUE when the file
 * cannot be written. */
cls_status cls_dump_fronts_csv(cls_handle h, const char* path);

/* ------------------------------------------------------------------------ */
/* Newton layer (NewtonSolver)                                               */
/* ------------------------------------------------------------------------ */

typedef enum { PF_OK = 0, PF_INVALID_ARGUMENT = 1, PF_RUNTIME_ERROR = 2 } pf_status;

/* BackendKind, ComputePolicy, CudaLinearSolverKind, CudaJacobianKind
 * (newton_solver_types.hpp:55-101) */
enum { PF_BACKEND_CPU = 0, PF_BACKEND_CUDA = 1 };
/* FP64: FP64 everywhere; FP32: FP32 state (V, Sbus, Ibus, F, update), Jacobian and factors
 * (FP64 factor precision falls back to FP32); Mixed: FP64 state with FP32 Jacobian and factors */
enum { PF_COMPUTE_FP64 = 0, PF_COMPUTE_FP32 = 1, PF_COMPUTE_MIXED = 2 };
enum { PF_CUDA_SOLVER_CUDSS = 0, PF_CUDA_SOLVER_CUSTOM = 1 };
enum { PF_JACOBIAN_EDGE = 0, PF_JACOBIAN_EDGE_ATOMIC = 1, PF_JACOBIAN_VERTEX_WARP = 2 };

/* NewtonOptions (newton_solver_types.hpp:167-192) */
typedef struct {
  int32_t backend;              /* only PF_BACKEND_CUDA is provided */
  int32_t compute;              /* PF_COMPUTE_* */
  int32_t cuda_linear_solver;   /* only PF_CUDA_SOLVER_CUSTOM is provided */
  int32_t cuda_jacobian;        /* PF_JACOBIAN_*: EDGE writes each slot once and takes the diagonal
                                   from Ibus; EDGE_ATOMIC sums the diagonal from the edges with
                                   atomicAdd (last bits vary run to run); VERTEX_WARP sums each bus
                                   row's diagonal in registers (fill_jacobian_*_kernel.hpp) */
  cls_config custom;
  int32_t use_cuda_graph;       /* capture one iteration, replay per step */
} pf_options;

/* NRConfig (newton_solver_types.hpp:35-38) */
typedef struct {
  double tolerance;
  int32_t max_iter;
} pf_nr_config;

/* SolveOptions (newton_solver_types.hpp:48-52) */
typedef struct {
  int32_t prepare_adjoint_cache;
  int32_t adjoint_cache_mode;                /* 0 None, 1 FinalStateFactorization, 2 Reuse...IfExact */
  int32_t allow_explicit_transpose_fallback; /* accepted; the engine solves J^T natively */
} pf_solve_options;

/* AdjointOptions (newton_solver_types.hpp:227-237) */
typedef struct {
  int32_t reuse_forward_factorization;
  int32_t allow_refactorize;
  int32_t require_cached_factorization;
  int32_t allow_refactorize_for_backward;
  int32_t allow_inexact_last_newton_factorization;
  int32_t use_transpose_solve;
  int32_t allow_explicit_transpose_fallback;
  int32_t compute_load_gradients;
  int32_t check_residual;
} pf_adjoint_options;

/* Scalar part of AdjointResult (newton_solver_types.hpp:239-290) */
typedef struct {
  int32_t n_bus, batch_size, dim_f;
  int32_t success, used_adjoint_cache, reused_final_state_factorization, refactorized_for_backward;
  int32_t iterations;           /* forward entry points: NR iterations run */
  double jt_residual_norm;
  double max_final_mismatch;    /* forward entry points */
  int32_t all_converged;        /* forward entry points */
} pf_adjoint_result;

typedef struct pf_solver_s* pf_handle;

/* Replaces: NewtonSolver::NewtonSolver(options) (newton_solver.cpp:70-175) */
pf_status pf_create(const pf_options* options, pf_handle* out);
pf_status pf_destroy(pf_handle h);
const char* pf_last_error(pf_handle h);
/* Replaces: NewtonSolver::initialize (newton_solver.cpp:184-217); host CSR
 * Ybus (complex values interleaved), PV/PQ bus lists. */
pf_status pf_initialize(pf_handle h, const int32_t* indptr, const int32_t* indices, const double* data,
                        int32_t rows, int32_t cols, int32_t nnz, const int32_t* pv, int32_t n_pv, const int32_t* pq,
                        int32_t n_pq);
/* Host-only analysis of a case (Jacobian pattern, maps, symbolic plan) with
 * no device allocation, for pf_plan_array / pf_info on machines without a
 * GPU.  pf_initialize is still required before solving. */
pf_status pf_analyze_host(pf_handle h, const int32_t* indptr, const int32_t* indices, int32_t rows, int32_t nnz,
                          const int32_t* pv, int32_t n_pv, const int32_t* pq, int32_t n_pq);
/* Replaces: NewtonSolver::solve_batch (newton_solver.cpp:245-342), host
 * buffers.  sbus / V0 [batch][stride] complex; V_out [batch][n_bus] complex;
 * iterations / final_mismatch / converged [batch]. */
pf_status pf_solve_batch(pf_handle h, const int32_t* indptr, const int32_t* indices, const double* data,
                         int32_t rows, int32_t cols, int32_t nnz, const double* sbus, int64_t sbus_stride,
                         const double* V0, int64_t V0_stride, int32_t batch, const int32_t* pv, int32_t n_pv,
                         const int32_t* pq, int32_t n_pq, const pf_nr_config* config,
                         const pf_solve_options* solve_options, double* V_out, int32_t* iterations,
                         double* final_mismatch, uint8_t* converged);
/* Device-resident variant of pf_solve_batch (same layouts, device pointers,
 * Ybus values as initialized); V_out / final_mismatch device, may be NULL. */
pf_status pf_solve_batch_device(pf_handle h, const double* sbus, int64_t sbus_stride, const double* V0,
                                int64_t V0_stride, int32_t batch, const pf_nr_config* config,
                                const pf_solve_options* solve_options, double* V_out, double* final_mismatch,
                                void* stream, pf_adjoint_result* result);
/* Per-scenario Ybus values (contingency and parameter sweeps on one pattern).
 * The reference's storage carries ybus_values_batched / ybus_value_stride
 * (cuda_batched_storage.hpp:84-89, .cpp:262-293; solver_contexts.hpp:42-43)
 * but its Ibus kernel rejects them (compute_ibus.cu:45-48) and
 * newton_solver.cpp:294 always passes false.  Here ybus_data is complex
 * [batch][ybus_stride] in the CSR order of the pattern given to
 * pf_initialize (ybus_stride >= nnz); scenario b solves with row b.  The
 * pattern, pv and pq are the initialized ones.  A later solve without these
 * entry points uses the shared values again; an adjoint after this solve
 * uses the per-scenario values of its forward solve.  Host buffers: */
pf_status pf_solve_batch_ybus(pf_handle h, const double* ybus_data, int64_t ybus_stride, const double* sbus,
                              int64_t sbus_stride, const double* V0, int64_t V0_stride, int32_t batch,
                              const pf_nr_config* config, const pf_solve_options* solve_options, double* V_out,
                              int32_t* iterations, double* final_mismatch, uint8_t* converged);
/* ... device buffers (as pf_solve_batch_device): */
pf_status pf_solve_batch_ybus_device(pf_handle h, const double* ybus_data, int64_t ybus_stride, const double* sbus,
                                     int64_t sbus_stride, const double* V0, int64_t V0_stride, int32_t batch,
                                     const pf_nr_config* config, const pf_solve_options* solve_options,
                                     double* V_out, double* final_mismatch, void* stream, pf_adjoint_result* result);
/* New (learned warm start, no reference counterpart): pf_solve_batch_device
 * started from a predicted state.  pred [batch][pred_ld] fp32 holds, in
 * Jacobian-row order, Va at the angle rows (PV then PQ buses) and Vm at the
 * magnitude rows (PQ buses); the other buses keep V0.  V0_stride 0 uses one
 * V0 row for every scenario.  pred_scale / pred_shift (fp32 [dim_f] each,
 * may be NULL together) map a standardized prediction to the state:
 * value = pred * scale + shift per Jacobian row.  result->all_converged is 0
 * whenever a scenario failed (final mismatch above tol or not finite). */
pf_status pf_solve_batch_warm_device(pf_handle h, const double* sbus, int64_t sbus_stride, const double* V0,
                                     int64_t V0_stride, const float* pred, int64_t pred_ld, const float* pred_scale,
                                     const float* pred_shift, int32_t batch,
                                     const pf_nr_config* config, const pf_solve_options* solve_options,
                                     double* V_out, double* final_mismatch, void* stream, pf_adjoint_result* result);
/* Replaces: NewtonSolver::solve_torch_forward (core/torch_bridge.cpp:309-482).
 * Device pointers: sbus_base_re/im, v0_va/vm [n_bus] (or [batch][n_bus] when
 * batched_v0 = 1, used for per-scenario warm starts), load_p/q and
 * va_out/vm_out [batch][n_bus]; dtype "float64" for FP64 compute, "float32"
 * for FP32/Mixed, as in the reference. */
pf_status pf_solve_forward_device(pf_handle h, const void* sbus_base_re, const void* sbus_base_im,
                                  const void* load_p, const void* load_q, const void* v0_va, const void* v0_vm,
                                  int32_t batched_v0, void* va_out, void* vm_out, int32_t batch, int32_t n_bus,
                                  const char* dtype, const pf_nr_config* config,
                                  const pf_solve_options* solve_options, void* stream, pf_adjoint_result* result);
/* Replaces: NewtonSolver::solve_torch_backward (core/torch_bridge.cpp:209-303).
 * Device pointers [batch][n_bus]. */
pf_status pf_solve_backward_device(pf_handle h, const void* grad_va, const void* grad_vm, void* grad_load_p,
                                   void* grad_load_q, int32_t batch, int32_t n_bus, const char* dtype,
                                   const pf_adjoint_options* options, void* stream, pf_adjoint_result* result);
/* Replaces: NewtonSolver::solve_adjoint (newton_solver.cpp:345-381), host
 * buffers: grads [batch][stride]; lambda [batch][dim_f], grad_load_p/q
 * [batch][n_bus]. */
pf_status pf_solve_adjoint(pf_handle h, const double* grad_va, int64_t grad_va_stride, const double* grad_vm,
                           int64_t grad_vm_stride, int32_t batch, const int32_t* pv, int32_t n_pv,
                           const int32_t* pq, int32_t n_pq, const pf_adjoint_options* options, double* lambda,
                           double* grad_load_p, double* grad_load_q, pf_adjoint_result* result);

/* Sizes of the analysed case. */
typedef struct {
  int32_t n_bus, n_pv, n_pq, dim_f, nnz_ybus, nnz_jacobian;
  int32_t num_panels, num_levels, max_front, max_panel;
  int64_t factor_elements;      /* U + L21 + CB elements per scenario */
  int64_t last_kernel_launches; /* launches of the last solve call */
} pf_info_t;
pf_status pf_info(pf_handle h, pf_info_t* out);
/* Jacobian analysis and plan introspection: "jac_row_ptr", "jac_col_idx",
 * "map11", "map21", "map12", "map22", "diag11", "diag21", "diag12", "diag22",
 * plus every cls_plan_array name. */
pf_status pf_plan_array(pf_handle h, const char* name, int32_t* out, int64_t capacity, int64_t* len);
/* The front CSV of cls_dump_fronts_csv for the Newton handle's Jacobian plan. */
pf_status pf_dump_fronts_csv(pf_handle h, const char* path);
/* New (verification): evaluate the mismatch F and the Jacobian values at the
 * given voltages with the engine's own kernels.  Host buffers: V [batch][n_bus]
 * complex, sbus [batch][n_bus] complex; outputs F [batch][dim_f] and J
 * [batch][nnz_jacobian] (CSR order of "jac_col_idx"), both double. */
pf_status pf_evaluate(pf_handle h, const double* V, const double* sbus, int32_t batch, double* F, double* J);
/* Stage timers of the last solve (the reference's NR.iteration.* stage
 * labels, newton_solver.cpp:521-553): times_ms[5] and launches[5] for
 * 0 mismatch, 1 jacobian, 2 factorize, 3 solve, 4 voltage_update, measured
 * with CUDA events on the solve stream when enabled (no extra host syncs). */
pf_status pf_set_profiling(pf_handle h, int32_t enabled);
pf_status pf_stage_times(pf_handle h, double* times_ms, int64_t* launches);
/* int64 plan arrays of the engine's factor program: "fe_split", "fe_src",
 * "u_off", "l_off", "cb_off" (same calling convention as pf_plan_array). */
pf_status pf_plan_array64(pf_handle h, const char* name, int64_t* out, int64_t capacity, int64_t* len);
/* Per-scenario static-pivot flags of the last factorization. */
pf_status pf_singular_flags(pf_handle h, int32_t* out_host, int32_t batch);

/* ---- Case I/O: the reference's dump-case directory format ----------------
 * Replaces: cupf::tests::load_dump_case (cuPF/tests/dump_case_loader.cpp:210-232,
 * dump_case_loader.hpp:14-42), the loader of the case directories that
 * benchmark/common/matpower_data.py:341-359 (save_dump_case) writes:
 * dump_Ybus.mtx (MatrixMarket coordinate complex), dump_Sbus.txt, dump_V.txt,
 * dump_pv.txt, dump_pq.txt, and, when present, dump_Vref.txt.  Complex arrays
 * come out interleaved (re, im) as double[2 * n]; Ybus as sorted CSR.
 * pf_case_load returns PF_RUNTIME_ERROR with the reference's message (read
 * with pf_case_last_error, per thread) for a missing directory or file,
 * a malformed line, an unsupported header, an out-of-range entry or
 * mismatched sizes. */
typedef struct pf_case_s* pf_case;
pf_status pf_case_load(const char* case_dir, pf_case* out);
const char* pf_case_last_error(void);
pf_status pf_case_dims(pf_case c, int32_t* rows, int32_t* cols, int32_t* nnz, int32_t* n_pv, int32_t* n_pq,
                       int32_t* has_vref);
/* Directory name of the case (DumpCaseData::case_name). */
const char* pf_case_name(pf_case c);
/* Copies the case into caller buffers sized by pf_case_dims; any pointer may
 * be NULL to skip that array (vref must be NULL when has_vref is 0). */
pf_status pf_case_copy(pf_case c, int32_t* indptr, int32_t* indices, double* ybus, double* sbus, double* v0,
                       int32_t* pv, int32_t* pq, double* vref);
void pf_case_destroy(pf_case c);

#ifdef __cplusplus
}
#endif

#endif /* CUPF_B200_H */
