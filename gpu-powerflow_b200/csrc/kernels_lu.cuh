// kernels_lu.cuh -- batched multifrontal LU of the Newton Jacobian, fused with
// the forward substitution, and the triangular sweeps that use its factors.
//
// Work unit: one warp = one front x 32 consecutive scenarios; lane = scenario.
// Every scenario of a batch shares the sparsity pattern and the symbolic plan,
// so all plan indices are warp-uniform and every value access is a coalesced
// 32-scenario row of the [element][Bp] layout.  A lane factors its own
// scenario's front with the front row held in registers (FMAX = front-size
// bucket, compile time), which removes the per-element shared-memory traffic
// of a block-per-front layout; only the nc pivot rows of the front are staged
// in shared memory, where each lane reads its own column (bank-conflict free).
//
// Numerics follow the reference's dense front kernels (custom_linear_solver/
// src/factorize/front_ops.cuh:146-185): right-looking LU without pivoting over
// the nc pivot columns of the front, static diagonal shift of pivots with
// |piv| <= eps to +-eps (GuardedPivot), contribution block CB = A22 - L21 U12
// extend-added into the parent front.  Differences by design:
//   * extend-add is a deterministic pull: a front gathers its children's CB
//     rows (the reference pushes with atomicAdd, factorize/assemble.cuh:14-27);
//   * the right-hand side rides along as an extra column of every front row,
//     so factorization also performs L y = P F (the reference runs a separate
//     forward sweep, solve/phases.cuh);
//   * a front is row-eliminated (each row applies the previous pivot rows),
//     which yields the same L and U as the right-looking form.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "device_plan.cuh"
#include "kernels.hpp"

namespace cupf_b200 {
namespace {

constexpr int kFactorWarps = 4;       // independent (front, scenario-group) items per block, at most
constexpr size_t kSmemLimit = 227 * 1024;  // opt-in dynamic shared memory per block on sm_100

template <typename T>
__device__ __forceinline__ T guarded_pivot(T piv, bool static_pivot, double eps, bool& shifted) {
  if (piv == T(0)) {
    shifted = true;
    if (!static_pivot) return T(1);
  }
  if (static_pivot && (piv < T(0) ? -piv : piv) <= static_cast<T>(eps)) {
    shifted = true;
    return piv < T(0) ? static_cast<T>(-eps) : static_cast<T>(eps);
  }
  return piv;
}

// ---------------------------------------------------------------------------
// Factor + forward substitution of one level of the front tree.
//   U  [u_total][Bp]  : pivot rows k of every front, fsz entries (L11 left of
//                       the diagonal, U11 | U12 from it)
//   L  [l_total][Bp]  : L21 rows (only when store_l; needed by the adjoint)
//   CB [cb_total][Bp] : uc rows of uc + 1 entries (last = rhs update)
//   Y  [dim][Bp]      : y = L^-1 P F at the pivot rows (permuted order)
// ---------------------------------------------------------------------------
template <typename T, typename TJ, int FMAX, int NCMAX>
__global__ void __launch_bounds__(kFactorWarps * kWarp)
    k_factor_level(DevPlan pl, int level_begin, int level_count, int groups, int Bp, int ub_rows,
                   const TJ* __restrict__ J, const double* __restrict__ F, T* __restrict__ U, T* __restrict__ L,
                   T* __restrict__ CB, T* __restrict__ Y, int store_l, double eps, int static_pivot,
                   int* __restrict__ sing) {
  extern __shared__ unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long item = (long)blockIdx.x * (blockDim.x >> 5) + warp;
  if (item >= (long)level_count * groups) return;
  const int p = pl.level_fronts[level_begin + item / groups];
  const int g = (int)(item % groups);
  const size_t b = (size_t)g * kWarp + lane;

  constexpr int RW = FMAX + 1;  // row width incl. the rhs slot
  T* ub = reinterpret_cast<T*>(smem_raw) + (size_t)warp * (ub_rows + 1) * RW * kWarp;
  T* rb = ub + (size_t)ub_rows * RW * kWarp;

  const int fs = pl.fsz[p], nc = pl.nc[p], uc = fs - nc;
  const int fr0 = pl.front_ptr[p], first = pl.first[p];
  const long long uo = pl.u_off[p], lo = pl.l_off[p], co = pl.cb_off[p];
  bool shifted = false;

  for (int i = 0; i < fs; ++i) {
    // ---- assemble row i: original entries, children's CB rows, rhs ----
#pragma unroll
    for (int j = 0; j < RW; ++j) rb[j * kWarp + lane] = T(0);
    for (int e = pl.arow_ptr[fr0 + i]; e < pl.arow_ptr[fr0 + i + 1]; ++e)
      rb[pl.arow_col[e] * kWarp + lane] += static_cast<T>(J[(size_t)pl.arow_q[e] * Bp + b]);
    if (i < nc) rb[FMAX * kWarp + lane] = static_cast<T>(F[(size_t)pl.perm[first + i] * Bp + b]);
    for (int e = pl.crow_ptr[fr0 + i]; e < pl.crow_ptr[fr0 + i + 1]; ++e) {
      const int c = pl.crow_child[e], r = pl.crow_r[e];
      const int ucc = pl.fsz[c] - pl.nc[c];
      const T* src = CB + (size_t)(pl.cb_off[c] + (long long)r * (ucc + 1)) * Bp + b;
      const int* al = pl.asm_local + pl.asm_ptr[c];
      for (int cc = 0; cc < ucc; ++cc) rb[al[cc] * kWarp + lane] += src[(size_t)cc * Bp];
      rb[FMAX * kWarp + lane] += src[(size_t)ucc * Bp];
    }
    T row[RW];
#pragma unroll
    for (int j = 0; j < RW; ++j) row[j] = rb[j * kWarp + lane];

    // ---- eliminate with the previous pivot rows ----
    const int kmax = i < nc ? i : nc;
#pragma unroll
    for (int k = 0; k < NCMAX; ++k) {
      if (k < kmax) {
        const T* uk = ub + (size_t)k * RW * kWarp + lane;
        const T l = row[k] / uk[k * kWarp];
        row[k] = l;
#pragma unroll
        for (int j = k + 1; j < FMAX; ++j)
          if (j < fs) row[j] -= l * uk[j * kWarp];
        row[FMAX] -= l * uk[FMAX * kWarp];
      }
    }

    if (i < nc) {
      // ---- pivot row: guard the pivot, keep it for later rows, write U / y ----
#pragma unroll
      for (int k = 0; k < NCMAX; ++k)
        if (k == i) row[k] = guarded_pivot(row[k], static_pivot != 0, eps, shifted);
      T* ui = ub + (size_t)i * RW * kWarp + lane;
#pragma unroll
      for (int j = 0; j < RW; ++j) ui[j * kWarp] = row[j];
      T* urow = U + (size_t)(uo + (long long)i * fs) * Bp + b;
#pragma unroll
      for (int j = 0; j < FMAX; ++j)
        if (j < fs) urow[(size_t)j * Bp] = row[j];
      Y[(size_t)(first + i) * Bp + b] = row[FMAX];
    } else {
      // ---- contribution row: L21 part (optional) and CB part + rhs update ----
      const int ii = i - nc;
      if (store_l) {
        T* lrow = L + (size_t)(lo + (long long)ii * nc) * Bp + b;
#pragma unroll
        for (int j = 0; j < NCMAX; ++j)
          if (j < nc) lrow[(size_t)j * Bp] = row[j];
      }
      T* cbrow = CB + (size_t)(co + (long long)ii * (uc + 1)) * Bp + b;
#pragma unroll
      for (int j = 0; j < FMAX; ++j)
        if (j >= nc && j < fs) cbrow[(size_t)(j - nc) * Bp] = row[j];
      cbrow[(size_t)uc * Bp] = row[FMAX];
    }
  }
  if (shifted) sing[b] = 1;
}

// ---------------------------------------------------------------------------
// Backward substitution U x = y of one level (root first).  X is in permuted
// order; a front reads the x of its CB rows, which belong to ancestors.
// ---------------------------------------------------------------------------
template <typename T, int FMAX, int NCMAX>
__global__ void __launch_bounds__(128)
    k_backward_level(DevPlan pl, int level_begin, int level_count, int groups, int Bp, const T* __restrict__ U,
                     const T* __restrict__ Y, T* __restrict__ X) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long item = (long)blockIdx.x * (blockDim.x >> 5) + warp;
  if (item >= (long)level_count * groups) return;
  const int p = pl.level_fronts[level_begin + item / groups];
  const size_t b = (size_t)(item % groups) * kWarp + lane;
  const int fs = pl.fsz[p], nc = pl.nc[p];
  const int fr0 = pl.front_ptr[p], first = pl.first[p];
  const long long uo = pl.u_off[p];
  T xs[FMAX];
#pragma unroll
  for (int j = 0; j < FMAX; ++j)
    xs[j] = (j >= nc && j < fs) ? X[(size_t)pl.front_rows[fr0 + j] * Bp + b] : T(0);
#pragma unroll
  for (int k = NCMAX - 1; k >= 0; --k) {
    if (k < nc) {
      const T* urow = U + (size_t)(uo + (long long)k * fs) * Bp + b;
      T s = Y[(size_t)(first + k) * Bp + b];
#pragma unroll
      for (int j = k + 1; j < FMAX; ++j)
        if (j < fs) s -= urow[(size_t)j * Bp] * xs[j];
      xs[k] = s / urow[(size_t)k * Bp];
      X[(size_t)(first + k) * Bp + b] = xs[k];
    }
  }
}

// ---------------------------------------------------------------------------
// Standalone forward substitution L y = P b (leaves first) for a right-hand
// side supplied after factorization (linear-solver boundary).  A front gathers
// its children's update vectors (extend-add of sum_m L21[.][m] y_m), solves its
// unit-lower pivot block and emits its own update vector.
// ---------------------------------------------------------------------------
template <typename T, int FMAX, int NCMAX>
__global__ void __launch_bounds__(128)
    k_l_forward_level(DevPlan pl, int level_begin, int level_count, int groups, int Bp, const T* __restrict__ U,
                      const T* __restrict__ L, const double* __restrict__ G, T* __restrict__ TV, T* __restrict__ Yo) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long item = (long)blockIdx.x * (blockDim.x >> 5) + warp;
  if (item >= (long)level_count * groups) return;
  const int p = pl.level_fronts[level_begin + item / groups];
  const size_t b = (size_t)(item % groups) * kWarp + lane;
  const int fs = pl.fsz[p], nc = pl.nc[p];
  const int fr0 = pl.front_ptr[p], first = pl.first[p];
  const long long uo = pl.u_off[p], lo = pl.l_off[p];
  T t[FMAX];
#pragma unroll
  for (int j = 0; j < FMAX; ++j) t[j] = T(0);
  for (int i = 0; i < fs; ++i) {
    T acc = T(0);
    for (int e = pl.crow_ptr[fr0 + i]; e < pl.crow_ptr[fr0 + i + 1]; ++e)
      acc += TV[(size_t)(pl.tv_off[pl.crow_child[e]] + pl.crow_r[e]) * Bp + b];
#pragma unroll
    for (int j = 0; j < FMAX; ++j)
      if (j == i) t[j] = acc;
  }
  T y[NCMAX];
#pragma unroll
  for (int k = 0; k < NCMAX; ++k) {
    y[k] = T(0);
    if (k < nc) {
      T s = static_cast<T>(G[(size_t)pl.perm[first + k] * Bp + b]) - t[k];
#pragma unroll
      for (int m = 0; m < k; ++m) s -= U[(size_t)(uo + (long long)k * fs + m) * Bp + b] * y[m];
      y[k] = s;
      Yo[(size_t)(first + k) * Bp + b] = s;
    }
  }
  const long long to = pl.tv_off[p];
#pragma unroll
  for (int j = 0; j < FMAX; ++j) {
    if (j >= nc && j < fs) {
      T s = t[j];
#pragma unroll
      for (int m = 0; m < NCMAX; ++m)
        if (m < nc) s += L[(size_t)(lo + (long long)(j - nc) * nc + m) * Bp + b] * y[m];
      TV[(size_t)(to + (j - nc)) * Bp + b] = s;
    }
  }
}

// ---------------------------------------------------------------------------
// Adjoint sweeps.  With P J P^T = L U, J^T lambda = g becomes
//   U^T w = P g (leaves first) and L^T z = w (root first), lambda = P^T z.
// U^T forward: a front gathers its children's update vectors t (extend-add of
// sum_m U12[m][.] w_m), solves its pivots and emits its own t for the parent.
// ---------------------------------------------------------------------------
template <typename T, int FMAX, int NCMAX>
__global__ void __launch_bounds__(128)
    k_ut_forward_level(DevPlan pl, int level_begin, int level_count, int groups, int Bp, const T* __restrict__ U,
                       const double* __restrict__ G, T* __restrict__ TV, T* __restrict__ W) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long item = (long)blockIdx.x * (blockDim.x >> 5) + warp;
  if (item >= (long)level_count * groups) return;
  const int p = pl.level_fronts[level_begin + item / groups];
  const size_t b = (size_t)(item % groups) * kWarp + lane;
  const int fs = pl.fsz[p], nc = pl.nc[p];
  const int fr0 = pl.front_ptr[p], first = pl.first[p];
  const long long uo = pl.u_off[p];
  T t[FMAX];
#pragma unroll
  for (int j = 0; j < FMAX; ++j) t[j] = T(0);
  // gather children's update vectors into this front's rows
  for (int i = 0; i < fs; ++i) {
    T acc = T(0);
    for (int e = pl.crow_ptr[fr0 + i]; e < pl.crow_ptr[fr0 + i + 1]; ++e)
      acc += TV[(size_t)(pl.tv_off[pl.crow_child[e]] + pl.crow_r[e]) * Bp + b];
#pragma unroll
    for (int j = 0; j < FMAX; ++j)
      if (j == i) t[j] = acc;
  }
  T w[NCMAX];
#pragma unroll
  for (int k = 0; k < NCMAX; ++k) {
    w[k] = T(0);
    if (k < nc) {
      T s = static_cast<T>(G[(size_t)pl.perm[first + k] * Bp + b]) - t[k];
#pragma unroll
      for (int m = 0; m < k; ++m) s -= U[(size_t)(uo + (long long)m * fs + k) * Bp + b] * w[m];
      w[k] = s / U[(size_t)(uo + (long long)k * fs + k) * Bp + b];
      W[(size_t)(first + k) * Bp + b] = w[k];
    }
  }
  const long long to = pl.tv_off[p];
#pragma unroll
  for (int j = 0; j < FMAX; ++j) {
    if (j >= nc && j < fs) {
      T s = t[j];
#pragma unroll
      for (int m = 0; m < NCMAX; ++m)
        if (m < nc) s += U[(size_t)(uo + (long long)m * fs + j) * Bp + b] * w[m];
      TV[(size_t)(to + (j - nc)) * Bp + b] = s;
    }
  }
}

// L^T backward: z_k = w_k - sum_{m>k} L11[m][k] z_m - sum_jj L21[jj][k] z(row jj)
template <typename T, int FMAX, int NCMAX>
__global__ void __launch_bounds__(128)
    k_lt_backward_level(DevPlan pl, int level_begin, int level_count, int groups, int Bp, const T* __restrict__ U,
                        const T* __restrict__ L, const T* __restrict__ W, T* __restrict__ Z) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long item = (long)blockIdx.x * (blockDim.x >> 5) + warp;
  if (item >= (long)level_count * groups) return;
  const int p = pl.level_fronts[level_begin + item / groups];
  const size_t b = (size_t)(item % groups) * kWarp + lane;
  const int fs = pl.fsz[p], nc = pl.nc[p];
  const int fr0 = pl.front_ptr[p], first = pl.first[p];
  const long long uo = pl.u_off[p], lo = pl.l_off[p];
  T zc[FMAX];
#pragma unroll
  for (int j = 0; j < FMAX; ++j)
    zc[j] = (j >= nc && j < fs) ? Z[(size_t)pl.front_rows[fr0 + j] * Bp + b] : T(0);
  T z[NCMAX];
#pragma unroll
  for (int k = NCMAX - 1; k >= 0; --k) {
    z[k] = T(0);
    if (k < nc) {
      T s = W[(size_t)(first + k) * Bp + b];
#pragma unroll
      for (int m = k + 1; m < NCMAX; ++m)
        if (m < nc) s -= U[(size_t)(uo + (long long)m * fs + k) * Bp + b] * z[m];
#pragma unroll
      for (int j = 0; j < FMAX; ++j)
        if (j >= nc && j < fs) s -= L[(size_t)(lo + (long long)(j - nc) * nc + k) * Bp + b] * zc[j];
      z[k] = s;
      Z[(size_t)(first + k) * Bp + b] = s;
    }
  }
}

// ---------------------------------------------------------------------------
// Launch helpers: pick the front-size bucket of a level.
// ---------------------------------------------------------------------------
inline int bucket_of(int fmax) {
  if (fmax <= 8) return 8;
  if (fmax <= 16) return 16;
  if (fmax <= 32) return 32;
  if (fmax <= 64) return 64;
  if (fmax <= 128) return 128;
  return -1;
}

template <typename T, typename TJ, int FMAX, int NCMAX>
void launch_factor_t(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s) {
  constexpr int RW = FMAX + 1;
  // per warp: the level's pivot rows plus one assembly row, 32 scenarios wide
  const size_t per_warp = (size_t)(lv.max_nc + 1) * RW * kWarp * sizeof(T);
  const int warps = (int)std::min<size_t>(kFactorWarps, kSmemLimit / per_warp);
  if (warps < 1) throw std::runtime_error("front too large for the shared-memory budget of the factor kernel");
  const size_t smem = per_warp * warps;
  auto kern = k_factor_level<T, TJ, FMAX, NCMAX>;
  static size_t configured = 0;
  if (smem > configured) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) throw std::runtime_error(std::string("factor kernel smem attribute: ") + cudaGetErrorString(e));
    configured = smem;
  }
  const long items = (long)lv.count * a.groups;
  const unsigned blocks = (unsigned)((items + warps - 1) / warps);
  kern<<<blocks, warps * kWarp, smem, s>>>(a.plan, lv.begin, lv.count, a.groups, a.Bp, lv.max_nc, a.J, a.F, a.U,
                                          a.L, a.CB, a.Y, a.store_l, a.eps, a.static_pivot, a.sing);
}

template <typename T, int FMAX, int NCMAX>
void launch_backward_t(const LevelLaunch& lv, const SweepArgs<T>& a, cudaStream_t s) {
  const long items = (long)lv.count * a.groups;
  const unsigned blocks = (unsigned)((items + 3) / 4);
  k_backward_level<T, FMAX, NCMAX><<<blocks, 128, 0, s>>>(a.plan, lv.begin, lv.count, a.groups, a.Bp, a.U, a.Y, a.X);
}

template <typename T, int FMAX, int NCMAX>
void launch_lf_t(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  const long items = (long)lv.count * a.groups;
  const unsigned blocks = (unsigned)((items + 3) / 4);
  k_l_forward_level<T, FMAX, NCMAX><<<blocks, 128, 0, s>>>(a.plan, lv.begin, lv.count, a.groups, a.Bp, a.U, a.L,
                                                          a.G, a.TV, a.W);
}

template <typename T, int FMAX, int NCMAX>
void launch_ut_t(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  const long items = (long)lv.count * a.groups;
  const unsigned blocks = (unsigned)((items + 3) / 4);
  k_ut_forward_level<T, FMAX, NCMAX><<<blocks, 128, 0, s>>>(a.plan, lv.begin, lv.count, a.groups, a.Bp, a.U, a.G,
                                                           a.TV, a.W);
}

template <typename T, int FMAX, int NCMAX>
void launch_lt_t(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  const long items = (long)lv.count * a.groups;
  const unsigned blocks = (unsigned)((items + 3) / 4);
  k_lt_backward_level<T, FMAX, NCMAX><<<blocks, 128, 0, s>>>(a.plan, lv.begin, lv.count, a.groups, a.Bp, a.U, a.L,
                                                            a.W, a.Z);
}

#define CUPF_BUCKET_SWITCH(NCMAX, CALL)                                        \
  switch (bucket_of(lv.max_fsz)) {                                             \
    case 8: CALL(8, NCMAX); break;                                             \
    case 16: CALL(16, NCMAX); break;                                           \
    case 32: CALL(32, NCMAX); break;                                           \
    case 64: CALL(64, NCMAX); break;                                           \
    case 128: CALL(128, NCMAX); break;                                         \
    default: throw std::runtime_error("front larger than 128 rows is not supported"); \
  }

}  // namespace

template <typename T, typename TJ>
void launch_factor_level(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc <= 8) {
#define CALL(F, N) launch_factor_t<T, TJ, (F < 8 ? 8 : F), N>(lv, a, s)
    CUPF_BUCKET_SWITCH(8, CALL)
#undef CALL
  } else {
    throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  }
}

template <typename T>
void launch_backward_level(const LevelLaunch& lv, const SweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc <= 8) {
#define CALL(F, N) launch_backward_t<T, (F < 8 ? 8 : F), N>(lv, a, s)
    CUPF_BUCKET_SWITCH(8, CALL)
#undef CALL
  } else {
    throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  }
}

template <typename T>
void launch_ut_forward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc <= 8) {
#define CALL(F, N) launch_ut_t<T, (F < 8 ? 8 : F), N>(lv, a, s)
    CUPF_BUCKET_SWITCH(8, CALL)
#undef CALL
  } else {
    throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  }
}

template <typename T>
void launch_l_forward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc <= 8) {
#define CALL(F, N) launch_lf_t<T, (F < 8 ? 8 : F), N>(lv, a, s)
    CUPF_BUCKET_SWITCH(8, CALL)
#undef CALL
  } else {
    throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  }
}

template <typename T>
void launch_lt_backward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc <= 8) {
#define CALL(F, N) launch_lt_t<T, (F < 8 ? 8 : F), N>(lv, a, s)
    CUPF_BUCKET_SWITCH(8, CALL)
#undef CALL
  } else {
    throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  }
}

}  // namespace cupf_b200
