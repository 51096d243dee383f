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
//
// One block = one front x 32 scenarios (lane = scenario).  The block
// assembles the dense front [fsz][fsz + 1] (last column = right-hand side) in
// shared memory from the front's destination-sorted source list -- original
// Jacobian entries, the mismatch rows of its pivots and its children's
// contribution blocks -- each warp accumulating its own destination chunk with
// eight independent loads in flight, then runs the right-looking LU over the
// nc pivot columns with the rows split across the warps, and writes
//   U  [u_total][Bp]  : pivot rows k (L11 left of the diagonal, U11 | U12 from it)
//   L  [l_total][Bp]  : L21 rows (only when store_l; the adjoint needs them)
//   CB [cb_total][Bp] : uc rows of uc + 1 entries (last = right-hand-side update)
//   Y  [dim][Bp]      : y = L^-1 P F at the pivot rows (permuted order)
// Fronts whose dense block does not fit the shared-memory budget use a
// caller-provided global scratch area (front_scratch), same code.
// ---------------------------------------------------------------------------
template <typename T, typename TJ>
__global__ void __launch_bounds__(256)
    k_front_factor(DevPlan pl, int level_begin, int groups, int Bp, int front_elems, const TJ* __restrict__ J,
                   const double* __restrict__ F, T* __restrict__ U, T* __restrict__ L, T* __restrict__ CB,
                   T* __restrict__ Y, int store_l, double eps, int static_pivot, int* __restrict__ sing,
                   T* __restrict__ front_scratch) {
  extern __shared__ unsigned char smem_raw[];
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x;
  const int p = pl.level_fronts[level_begin + item / groups];
  const size_t b = (size_t)(item % groups) * kWarp + lane;
  const int fs = pl.fsz[p], nc = pl.nc[p], uc = fs - nc, rw = fs + 1;
  T* Fm = front_scratch ? front_scratch + (size_t)item * front_elems * kWarp : reinterpret_cast<T*>(smem_raw);

  for (int e = threadIdx.x; e < fs * rw * kWarp; e += blockDim.x) Fm[e] = T(0);
  __syncthreads();

  // ---- assembly ----
  const long long* split = pl.fe_split + (size_t)p * 9;
  for (int ch = warp; ch < 8; ch += W) {
    const long long e1 = split[ch + 1];
    for (long long e = split[ch]; e < e1; e += 8) {
      T v[8];
      int d[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        v[u] = T(0);
        d[u] = -1;
        if (e + u < e1) {
          const long long src = pl.fe_src[e + u];
          d[u] = pl.fe_dst[e + u];
          const int kind = (int)((unsigned long long)src >> 62);
          const size_t idx = (size_t)(src & 0x3FFFFFFFFFFFFFFFll);
          v[u] = kind == 0 ? static_cast<T>(J[idx * Bp + b])
                           : (kind == 1 ? CB[idx * Bp + b] : static_cast<T>(F[idx * Bp + b]));
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (d[u] >= 0) Fm[(size_t)d[u] * kWarp + lane] += v[u];
    }
  }
  __syncthreads();

  // ---- right-looking LU over the pivot columns ----
  bool shifted = false;
  for (int k = 0; k < nc; ++k) {
    T* Fk = Fm + (size_t)k * rw * kWarp + lane;
    if (warp == 0) Fk[k * kWarp] = guarded_pivot(Fk[k * kWarp], static_pivot != 0, eps, shifted);
    __syncthreads();
    const T piv = Fk[k * kWarp];
    for (int i = k + 1 + warp; i < fs; i += W) {
      T* Fi = Fm + (size_t)i * rw * kWarp + lane;
      const T l = Fi[k * kWarp] / piv;
      Fi[k * kWarp] = l;
      for (int j = k + 1; j < rw; ++j) Fi[j * kWarp] -= l * Fk[j * kWarp];
    }
    __syncthreads();
  }

  // ---- write U, y, L21, CB ----
  const long long uo = pl.u_off[p], lo = pl.l_off[p], co = pl.cb_off[p];
  const int first = pl.first[p];
  for (int e = warp; e < nc * fs; e += W) {
    const int k = e / fs, j = e - k * fs;
    U[(size_t)(uo + e) * Bp + b] = Fm[(size_t)(k * rw + j) * kWarp + lane];
  }
  for (int k = warp; k < nc; k += W) Y[(size_t)(first + k) * Bp + b] = Fm[(size_t)(k * rw + fs) * kWarp + lane];
  if (store_l) {
    for (int e = warp; e < uc * nc; e += W) {
      const int ii = e / nc, j = e - ii * nc;
      L[(size_t)(lo + e) * Bp + b] = Fm[(size_t)((nc + ii) * rw + j) * kWarp + lane];
    }
  }
  for (int e = warp; e < uc * (uc + 1); e += W) {
    const int ii = e / (uc + 1), jj = e - ii * (uc + 1);
    CB[(size_t)(co + e) * Bp + b] = Fm[(size_t)((nc + ii) * rw + nc + jj) * kWarp + lane];
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
  const int fmax = lv.max_fsz;
  const size_t elems = (size_t)fmax * (fmax + 1);
  const size_t smem = elems * kWarp * sizeof(T);
  const int warps = fmax <= 8 ? 2 : (fmax <= 20 ? 4 : 8);
  const bool in_smem = smem <= kSmemLimit;
  auto kern = k_front_factor<T, TJ>;
  if (in_smem) {
    static size_t configured = 0;
    if (smem > configured) {
      const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess)
        throw std::runtime_error(std::string("factor kernel smem attribute: ") + cudaGetErrorString(e));
      configured = smem;
    }
  } else if (!a.front_scratch || a.front_scratch_elems < elems * (size_t)lv.count * a.groups) {
    throw std::runtime_error("front larger than the shared-memory budget and no scratch area provided");
  }
  const unsigned blocks = (unsigned)((long)lv.count * a.groups);
  kern<<<blocks, warps * kWarp, in_smem ? smem : 0, s>>>(a.plan, lv.begin, a.groups, a.Bp, (int)elems, a.J, a.F, a.U,
                                                        a.L, a.CB, a.Y, a.store_l, a.eps, a.static_pivot, a.sing,
                                                        in_smem ? nullptr : a.front_scratch);
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
