// kernels.hpp -- host-side launchers of the engine's CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "device_plan.cuh"

namespace cupf_b200 {

// One level of the front tree as the launchers see it.
struct LevelLaunch {
  int begin = 0;   // offset into DevPlan::level_fronts
  int count = 0;   // fronts in the level
  int max_fsz = 0; // largest front of the level (selects the register bucket)
  int max_nc = 0;  // widest panel of the level
  int max_src = 0; // longest assembly source list of the level
  // the launch's source lists, padded to max_src entries each (front q of
  // the launch starts at fe_base + (q - begin) * max_src), so a block finds
  // its list without reading the launch record first
  long long fe_base = 0;
  int warps = 0;   // warps per block of the factor launch (0: the built-in rule)
  int bw_wpb = 0;  // warps per block of the backward-sweep launch (0: the built-in rule)
  // factor kernel: 0 register rows (fronts of at most 64 rows), 1 the wide
  // tier on the FP32/FP64 pipes (any size), 2 the wide tier with the trailing
  // update on the tensor cores (FP32 factors only)
  int tier = 0;
  // register tier: where the dense fronts live -- 0 the built-in rule
  // (front_in_shared_memory), 1 shared memory, 2 the global scratch (chosen
  // by the engine's autotuner; a choice that does not fit falls back to the
  // rule); 3 the wide tier instead of register rows (fronts of at least
  // kWideOptionRows rows; same factors)
  int placement = 0;
};

template <typename T, typename TJ>
struct FactorArgs {
  DevPlan plan;
  int groups = 0, Bp = 0;
  const TJ* J = nullptr;
  const T* Fp = nullptr;  // right-hand side rows in pivot order
  T* U = nullptr;
  T* L = nullptr;
  T* CB = nullptr;
  T* Y = nullptr;
  int store_l = 0;
  double eps = 1e-8;
  int static_pivot = 1;
  int* sing = nullptr;
  T* front_scratch = nullptr;       // global dense fronts for levels whose front exceeds shared memory
  size_t front_scratch_elems = 0;   // capacity in elements per scenario lane group (x 32)
  int single = 0;                   // batch 1: the single-system schedule where a front fits shared memory
};

constexpr size_t kSmemLimit = 227 * 1024;  // opt-in dynamic shared memory per block on sm_100

// Header of the single-system kernels' shared memory: pivot reciprocal (0),
// shift flag (8), tree item (12).
constexpr int kSingleHeader = 32;

// The single-system schedule's shared memory: the header, the dense front
// [fs][fs + 1], and a source list of up to list_cap entries with their values
// (value, source, destination per entry; +16: the list's 16-byte alignment).
inline size_t single_smem_bytes(int max_fsz, int list_cap, size_t elem_bytes) {
  return kSingleHeader + 16 + ((size_t)max_fsz * (max_fsz + 1) + (size_t)list_cap) * elem_bytes +
         (size_t)list_cap * (sizeof(long long) + sizeof(int));
}

// The front tree for the single-system factorization launch, in level order
// (q): parent[q] (-1 at a root), nchild[q], the start of q's source list in
// the padded lists, the leaves (fronts without children) in level order;
// done: P + 1 ints zeroed before each launch (per-front child counts, then
// the leaf counter).
struct SingleTree {
  const int* parent = nullptr;
  const int* nchild = nullptr;
  const long long* q_e0 = nullptr;
  const int* leaves = nullptr;
  int* done = nullptr;
  int P = 0, n_leaves = 0, max_fsz = 0, list_cap = 0;
};

// Shared-memory plan of one factor-level launch (same for every block):
// staged source list (src, dst), pivot reciprocals, staged source rows,
// dense front.
struct FrontSmem {
  int chunk = 0;        // staged source rows per buffer
  int nbuf = 1;         // 1, or 2 when a front's sources need more than one chunk
  int idx_cap = 0;      // source entries whose (src, dst) are staged (0: read from global memory)
  size_t idx_bytes = 0, inv_bytes = 0, stage_bytes = 0, front_bytes = 0;
  size_t us_bytes = 0;  // wide tier: the pivot rows [nc][fs + 1][32] (0: kept in the global scratch)
  size_t total() const { return idx_bytes + inv_bytes + stage_bytes + front_bytes + us_bytes; }
};

// The whole source list staged at once when it fits next to the dense front,
// else two alternating chunk buffers of 128 / 64 / 32 rows.  With
// front_in_smem = false the dense front lives in global scratch.
inline FrontSmem plan_front_smem(const LevelLaunch& lv, size_t elem_bytes, bool front_in_smem) {
  FrontSmem sm;
  const size_t row = 32 * elem_bytes;
  sm.idx_cap = lv.max_src > 0 ? lv.max_src : 1;
  sm.idx_bytes = ((size_t)sm.idx_cap * (sizeof(long long) + sizeof(int)) + 15) / 16 * 16;
  sm.inv_bytes = 8 * row;  // reciprocals of the (at most 8) pivots, per scenario lane
  sm.front_bytes = front_in_smem ? (size_t)lv.max_fsz * (lv.max_fsz + 1) * row : 0;
  sm.chunk = sm.idx_cap;
  sm.nbuf = 1;
  sm.stage_bytes = (size_t)sm.chunk * row;
  for (int c : {128, 64, 32}) {
    if (sm.total() <= kSmemLimit) break;
    if (c >= sm.chunk && sm.nbuf == 1) continue;
    sm.chunk = c;
    sm.nbuf = 2;
    sm.stage_bytes = 2 * (size_t)c * row;
  }
  return sm;
}

// Round trips to memory a launch's blocks spend staging their source rows.
inline int staging_round_trips(const LevelLaunch& lv, const FrontSmem& sm) {
  const int n = lv.max_src > 0 ? lv.max_src : 1;
  return (n + sm.chunk - 1) / sm.chunk;
}

// Where a register-kernel launch keeps its dense fronts.  In shared memory
// when the front and all its staged source rows fit.  A large front leaves
// room only for small double-buffered chunks of the source rows, and each
// chunk is one more dependent memory round trip before the front is
// assembled; with the front in the global scratch (L2-resident) the whole
// list is staged in one round trip, at the price of reading the front from
// L2 during the elimination.  The front moves to the scratch when that
// saves more than two staging round trips.
inline bool front_in_shared_memory(const LevelLaunch& lv, size_t elem_bytes) {
  const FrontSmem a = plan_front_smem(lv, elem_bytes, true);
  if (a.total() > kSmemLimit) return false;
  const FrontSmem b = plan_front_smem(lv, elem_bytes, false);
  if (b.total() > kSmemLimit) return true;
  if (lv.placement == 1) return true;
  if (lv.placement == 2) return false;
  return !(staging_round_trips(lv, b) + 2 < staging_round_trips(lv, a));
}

// Launches whose fronts have at least this many rows always run a wide tier
// (no compile-time bound on the front size); the register kernels are built
// for fronts of up to 64 rows.
constexpr int kWideFrontRows = 65;
// TF32 factors: the tensor cores take the trailing updates of launches with
// fronts of at least this many rows (the fronts past the register kernels),
// unless configured or autotuned otherwise; the autotuner tries 33, 49 and 65.
constexpr int kTcDefaultMinFront = 65;
constexpr int kTcSmallestMinFront = 33;  // the smallest threshold the autotuner tries
// Register-tier launches whose fronts reach this many rows may run the wide
// tier instead (placement 3, an autotuner choice): a few large fronts per
// launch go faster with up to 32 warps over their columns and rows than with
// at most 8 warps of register rows.
constexpr int kWideOptionRows = 17;


// Shared-memory plan of a wide-tier launch: pivot reciprocals, the staged
// source rows, and `reserve` bytes after them for the kernel's other arrays
// (the source list itself is read from global memory: it can be thousands of
// entries long; the dense front is in the global scratch).  The whole list is
// staged at once when it fits, else two alternating chunks as large as fit
// (multiples of 32 rows, at least 32); 0 chunk rows when even that fails.
inline FrontSmem plan_wide_staging(const LevelLaunch& lv, size_t elem_bytes, size_t reserve) {
  FrontSmem sm;
  const size_t row = 32 * elem_bytes;
  sm.idx_cap = 0;
  sm.idx_bytes = 0;
  sm.inv_bytes = 8 * row;
  sm.front_bytes = 0;
  const int nsrc = lv.max_src > 0 ? lv.max_src : 1;
  const size_t avail = kSmemLimit > sm.inv_bytes + reserve ? kSmemLimit - sm.inv_bytes - reserve : 0;
  if ((size_t)nsrc * row <= avail) {
    sm.chunk = nsrc;
    sm.nbuf = 1;
  } else {
    sm.chunk = (int)(avail / (2 * row)) / 32 * 32;
    sm.nbuf = 2;
  }
  sm.stage_bytes = (size_t)sm.nbuf * sm.chunk * row;
  return sm;
}

// The any-size tier's plan: the pivot rows Us [nc][fs + 1][32] in shared
// memory when at least 32-row staging chunks fit beside them, else in the
// scratch after the front.
inline FrontSmem plan_wide_smem(const LevelLaunch& lv, size_t elem_bytes) {
  const size_t us = (size_t)lv.max_nc * (lv.max_fsz + 1) * 32 * elem_bytes;
  FrontSmem sm = plan_wide_staging(lv, elem_bytes, us);
  if (sm.chunk >= 32 || sm.nbuf == 1) {
    sm.us_bytes = us;
    return sm;
  }
  sm = plan_wide_staging(lv, elem_bytes, 0);
  sm.us_bytes = 0;
  return sm;
}

inline bool wide_option(const LevelLaunch& lv) { return lv.tier == 0 && lv.max_fsz >= kWideOptionRows; }

// Whether a factor launch runs the wide tier: its own tier, fronts past the
// register kernels, the autotuner's placement 3, or -- the built-in rule --
// large fronts that would not fit in shared memory (register rows over a
// front in the L2 scratch are the slowest of the choices there).
inline bool runs_wide(const LevelLaunch& lv, size_t elem_bytes) {
  if (lv.tier == 1 || lv.max_fsz >= kWideFrontRows) return true;
  if (!wide_option(lv)) return false;
  if (lv.placement == 3) return true;
  return lv.placement == 0 && !front_in_shared_memory(lv, elem_bytes);
}

// Elements (x 32 scenario lanes) of global scratch one block of a wide-tier
// launch uses: its dense front, plus the pivot rows when they are not in
// shared memory.
inline size_t wide_block_elems(const LevelLaunch& lv, size_t elem_bytes) {
  const size_t rw = (size_t)lv.max_fsz + 1;
  return (size_t)lv.max_fsz * rw + (plan_wide_smem(lv, elem_bytes).us_bytes ? 0 : (size_t)lv.max_nc * rw);
}

// Global front scratch (elements x 32) a factor launch needs for all its
// blocks (groups = 32-scenario groups of the batch) with its current tier
// and placement; 0 when its fronts live in shared memory.
inline size_t level_scratch_elems(const LevelLaunch& lv, size_t elem_bytes, int groups) {
  if (lv.tier > 0 || runs_wide(lv, elem_bytes)) return wide_block_elems(lv, elem_bytes) * lv.count * groups;
  if (front_in_shared_memory(lv, elem_bytes)) return 0;
  return (size_t)lv.max_fsz * (lv.max_fsz + 1) * lv.count * groups;
}

// The most a register-tier launch can need whatever placement the autotuner
// gives it (the workspace is sized for this).
inline size_t level_scratch_capacity(const LevelLaunch& lv, size_t elem_bytes, int groups) {
  if (lv.tier > 0) return level_scratch_elems(lv, elem_bytes, groups);
  size_t c = plan_front_smem(lv, elem_bytes, false).total() > kSmemLimit
                 ? 0
                 : (size_t)lv.max_fsz * (lv.max_fsz + 1) * lv.count * groups;
  if (wide_option(lv)) c = std::max(c, wide_block_elems(lv, elem_bytes) * lv.count * groups);
  return c;
}

template <typename T>
struct SweepArgs {
  DevPlan plan;
  int groups = 0, Bp = 0;
  const T* U = nullptr;
  const T* Y = nullptr;
  T* X = nullptr;
};

template <typename T>
struct AdjointSweepArgs {
  DevPlan plan;
  int groups = 0, Bp = 0;
  const T* U = nullptr;
  const T* L = nullptr;
  const double* G = nullptr;  // rhs in Jacobian-row order
  T* TV = nullptr;            // update vectors [tv_total][Bp]
  T* W = nullptr;             // U^T solution (permuted order)
  T* Z = nullptr;             // L^T solution (permuted order)
};

template <typename T, typename TJ>
void configure_front_kernels();
template <typename T, typename TJ>
void launch_factor_level(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s);
template <typename T, typename TJ>
void launch_factor_single_tree(const FactorArgs<T, TJ>& a, const SingleTree& t, cudaStream_t s);
template <typename T>
void launch_backward_level(const LevelLaunch& lv, const SweepArgs<T>& a, cudaStream_t s);
// The narrow top levels as one launch (block = 32 scenarios walking the
// levels root-down); lv_bounds: device array of nlev + 1 descending level
// boundaries in level order; top: the levels' extent (max_fsz, max_nc).
template <typename T>
void launch_backward_top(const LevelLaunch& top, const int* lv_bounds, int nlev, const SweepArgs<T>& a,
                         cudaStream_t s);
template <typename T>
void launch_ut_forward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s);
// L y = P g for a rhs given after factorization (y written to a.W)
template <typename T>
void launch_l_forward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s);
template <typename T>
void launch_lt_backward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s);

// ---- element-wise NR stages (kernels_nr.cu) ----
void launch_ibus_mismatch(const DevGrid& g, const DevState& st, cudaStream_t s);
template <typename TJ>
void launch_jacobian(const DevGrid& g, const DevState& st, TJ* J, cudaStream_t s);
template <typename T>
void launch_voltage_update(const DevGrid& g, const DevPlan& pl, const DevState& st, const T* X, cudaStream_t s);
// seed from host-layout complex arrays [B][stride] (interleaved re/im) staged on device
void launch_seed_state(const DevGrid& g, const DevState& st, const double* sbus_c, long long sbus_stride,
                       const double* v0_c, long long v0_stride, cudaStream_t s);
void launch_pack_voltage(const DevGrid& g, const DevState& st, double* v_c, cudaStream_t s);
// launch_seed_state with the state taken from a prediction pred[B][ld] in
// Jacobian-row order (fp32) where it has rows: the warm start's seed
void launch_seed_warm(const DevGrid& g, const DevState& st, const double* sbus_c, long long sbus_stride,
                      const double* v0_c, long long v0_stride, const float* pred, long long ld, const float* scale,
                      const float* shift, cudaStream_t s);
// torch-style inputs: base injection [n], loads [B][n], flat start [n]; dtype float or double
void launch_set_inputs_from_load(const DevGrid& g, const DevState& st, const void* base_re, const void* base_im,
                                 const void* load_p, const void* load_q, const void* va0, const void* vm0,
                                 int is_double, cudaStream_t s);
void launch_set_inputs_batched(const DevGrid& g, const DevState& st, const void* base_re, const void* base_im,
                               const void* load_p, const void* load_q, const void* va0, const void* vm0,
                               int is_double, cudaStream_t s);
void launch_copy_voltage_outputs(const DevGrid& g, const DevState& st, void* va_out, void* vm_out, int is_double,
                                 cudaStream_t s);
// adjoint helpers
void launch_gather_adjoint_rhs(const DevGrid& g, const DevState& st, const void* grad_va, const void* grad_vm,
                               int is_double, double* G, cudaStream_t s);
template <typename T>
void launch_permuted_to_rows(const int* inv, int dim, int Bp, const T* Z, double* lam, cudaStream_t s);
void launch_project_load_gradients(const DevGrid& g, const DevState& st, const double* lam, void* grad_p,
                                   void* grad_q, int is_double, cudaStream_t s);
// r = g - J^T lambda, J given by its CSR values [nnz_j][Bp] (fp64)
void launch_jt_residual(const DevGrid& g, int Bp, const double* Jd, const double* lam, const double* G, double* R,
                        cudaStream_t s);
void launch_axpy(double* y, const double* x, long long n, cudaStream_t s);
// scratch[0] = sum r^2, scratch[1] = sum g^2 over f < dim, b < B of [dim][Bp]
// arrays R and G; scratch holds 2 + 2 * 296 doubles
// Per-scenario Ybus values complex [B][stride] -> re/im [nnz][Bp]
void launch_ybus_to_rows(const double* yc, long long stride, int nnz, int B, int Bp, double* yr, double* yi,
                         cudaStream_t s);
// Convergence test of the device-side Newton loop (one CUDA graph per solve,
// a WHILE node around the iteration).  The host writes tol / max_iter / B /
// tolerate before each launch; the check kernel keeps the rest.
struct LoopCtl {
  double tol = 0.0;
  int max_iter = 0;
  int B = 0;
  int tolerate = 0;   // a non-finite scenario norm ends that scenario (inf) instead of the solve
  int completed = 0;  // norm evaluations so far
  int status = 0;     // 1: a non-finite norm that was not tolerated
  int nonfinite = 0;  // 1: some scenario's norm was non-finite (tolerated: that scenario failed)
  double gmax = 0.0;  // max over the batch of the last evaluated norms
};
// Reads the per-scenario norms of the last mismatch, records them as the
// final mismatches, counts the evaluation and sets the loop's condition to
// 1 (iterate again) or 0 (converged, iteration cap, or non-finite).
// The graph-mode solve's control block and results travel through pinned
// host memory that the kernels read and write directly (unified addressing),
// not through copies: small copies would queue on the copy engines behind a
// stream of batch uploads and downloads.  load: host control -> device;
// store: device control -> host, final norms -> host and (if given) to the
// caller's device buffer.
void launch_ctl_load(const LoopCtl* host_ctl, LoopCtl* ctl, cudaStream_t s);
void launch_ctl_store(const LoopCtl* ctl, LoopCtl* host_ctl, const double* final_norm, double* host_final,
                      double* d_final, int B, cudaStream_t s);
void launch_loop_check(cudaGraphConditionalHandle h, LoopCtl* ctl, const unsigned long long* norm_bits,
                       double* final_norm, cudaStream_t s);
void launch_sumsq2(const double* R, const double* G, int dim, int B, int Bp, double* scratch, cudaStream_t s);
// [B][rows] (TS) -> [rows][Bp] (TD) and back; pad scenarios copy scenario B - 1
template <typename TS, typename TD>
void launch_batch_to_rows(const TS* src, TD* dst, int rows, int B, int Bp, cudaStream_t s);
template <typename TS, typename TD>
void launch_rows_to_batch(const TS* src, TD* dst, int rows, int B, int Bp, cudaStream_t s);

}  // namespace cupf_b200
