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
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

#include "device_plan.cuh"
#include "kernels.hpp"
#include "tcgen05.cuh"

namespace cupf_b200 {
namespace {

constexpr int kFactorWarps = 4;       // independent (front, scenario-group) items per block, at most

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

// Opt a kernel into the full 227 KB of dynamic shared memory, once per
// (device, kernel); the attribute is per device and per function.
inline void allow_full_smem(const void* fn) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("cudaGetDevice failed");
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({dev, fn})) return;
  const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemLimit);
  if (e != cudaSuccess) throw std::runtime_error(std::string("shared-memory attribute: ") + cudaGetErrorString(e));
  done.insert({dev, fn});
}

inline void check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + " launch: " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Programmatic dependent launch between consecutive level kernels: a level
// kernel lets the next one be scheduled as soon as all of its own blocks are
// running (launch_dependents), and the next one runs the part of its work
// that reads only the static plan (launch record, assembly list, zeroing its
// shared-memory front) before it waits for the previous grid to finish and
// its writes to be visible (griddepcontrol.wait, a hardware wait that ends
// when that grid completes).  Launched without the attribute, both are
// no-ops.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void chain_allow_next() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void chain_wait_previous() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Launch with programmatic stream serialization (the kernel's prologue may
// overlap the tail of the kernel before it on the stream).
template <typename... KArgs, typename... Args>
void launch_chained(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, const char* what,
                    Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + " launch: " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async, sm_80+ form; the copy
// completes in the background and cp.async.wait_group is a hardware wait, so
// no software spin is involved).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// ---------------------------------------------------------------------------
// Factor + forward substitution of one level of the front tree.
//
// One block = one front x 32 scenarios (lane = scenario).  Three phases:
//  1. staging: the front's destination-sorted source list (indices) is copied
//     into shared memory, then every source row -- 32 scenarios of one
//     Jacobian entry or one child contribution-block element, a contiguous
//     128 B (fp32) / 256 B (fp64) segment of the [element][Bp] arrays -- is
//     requested with cp.async in one sweep, so a front costs two memory round
//     trips however many sources it has (large lists go through two
//     alternating buffers, chunk by chunk);
//  2. assembly into the dense front [fsz][fsz + 1] (last column = right-hand
//     side, seeded with the pivots' mismatch rows), each warp owning whole
//     destinations so the sums run in list order without atomics;
//  3. right-looking LU over the nc pivot columns with the rows split across
//     the warps, then
//       U  [u_total][Bp]  : pivot rows k (L11 left of the diagonal, U11 | U12 from it)
//       L  [l_total][Bp]  : L21 rows (only when store_l; the adjoint needs them)
//       CB [cb_total][Bp] : uc rows of uc + 1 entries (last = right-hand-side update)
//       Y  [dim][Bp]      : y = L^-1 P F at the pivot rows (permuted order)
// Fronts whose dense block does not fit next to the staging buffers live in a
// caller-provided global scratch area (front_scratch), same code.
// ---------------------------------------------------------------------------
// Phases 1 and 2 of a factor block, shared by the front kernels: stage the
// front's source list (STAGE_LIST: in shared memory; else it is read from
// global memory where it is used, for lists too long to stage) and its
// source rows, zero the dense front Fm (shared memory, or this block's slice
// of the global scratch, whose per-block stride is front_elems x 32) and
// assemble it.  Returns the launch record; *Fm_out is the assembled front
// [fs][fs + 1][32].
// The first entry at or after x of the destination-sorted list d that
// starts a new destination within the range [A0, Z0) (A0 itself counts as a
// start; x >= A0), or Z0: a warp-wide scan, 32 entries a step.
__device__ __forceinline__ int run_start(const int* d, int x, int A0, int Z0) {
  const int lane = threadIdx.x & 31;
  for (int base = x; base < Z0; base += kWarp) {
    const int y = base + lane;
    const bool cut = y >= Z0 || y <= A0 || d[y] != d[y - 1];
    const unsigned m = __ballot_sync(0xffffffffu, cut);
    if (m) return base + __ffs(m) - 1;
  }
  return Z0;
}

template <typename T, typename TJ, bool SMEM_FRONT, bool STAGE_LIST = true>
__device__ __forceinline__ FrontMeta stage_and_assemble(const DevPlan& pl, int level_begin, long long fe_base,
                                                        int fe_pad, int groups, int Bp, int front_elems,
                                                        const FrontSmem& sm, const TJ* __restrict__ J,
                                                        const T* __restrict__ Fp, const T* __restrict__ CB,
                                                        T* __restrict__ front_scratch, unsigned char* smem_raw,
                                                        T** Fm_out) {
  static_assert(sizeof(TJ) == sizeof(T), "Jacobian and factor rows are staged in the same slots");
  constexpr int kRowBytes = kWarp * sizeof(T);
  constexpr int kPieces = kRowBytes / 16;  // 16-byte cp.async pieces per source row
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int item = blockIdx.x;
  const int q = level_begin + item / groups;
  const int grp = item - (item / groups) * groups;
  const size_t col0 = (size_t)grp * kWarp;
  chain_allow_next();
  const long long e0 = fe_base + (long long)(q - level_begin) * fe_pad;
  const long long* s_src = pl.fe_src + e0;
  const int* s_dst = pl.fe_dst + e0;
  // phase 1a: the source list -> shared memory.  Its place follows from the
  // item alone (padded lists), so it is requested together with the launch
  // record: one memory round trip for both.
  if constexpr (STAGE_LIST) {
    long long* ss = reinterpret_cast<long long*>(smem_raw);
    int* sd = reinterpret_cast<int*>(smem_raw + (size_t)sm.idx_cap * sizeof(long long));
    for (int e = threadIdx.x; e < fe_pad; e += blockDim.x) {
      cp_async8(ss + e, pl.fe_src + e0 + e);
      cp_async4(sd + e, pl.fe_dst + e0 + e);
    }
    cp_async_commit();
    s_src = ss;
    s_dst = sd;
  }
  const FrontMeta m = load_front_meta(pl.front_meta, q);
  const int fs = m.fs, rw = fs + 1;
  const int nsrc = m.split[8];

  unsigned char* stage = smem_raw + sm.idx_bytes + sm.inv_bytes;
  T* Fm;
  if constexpr (SMEM_FRONT)
    Fm = reinterpret_cast<T*>(stage + sm.stage_bytes);
  else
    Fm = front_scratch + (size_t)item * front_elems * kWarp;
  *Fm_out = Fm;

  // (the dense front is zeroed while the list arrives)
  // fs * rw * 32 elements is a multiple of 16 bytes: zero with 16-byte stores
  auto zero_front = [&]() {
    float4* z4 = reinterpret_cast<float4*>(Fm);
    const int n4 = fs * rw * kWarp * (int)sizeof(T) / 16;
    for (int e = threadIdx.x; e < n4; e += blockDim.x) z4[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  };
  if constexpr (SMEM_FRONT) zero_front();
  // everything below reads what earlier kernels wrote (J, CB, Fp), and a
  // global scratch front may still be in use by the previous level's blocks
  chain_wait_previous();
  if constexpr (!SMEM_FRONT) zero_front();
  cp_async_wait<0>();
  __syncthreads();

  // phase 1b: request the source rows (Jacobian entries, right-hand-side rows,
  // children's contribution-block elements), one row per thread, chunk by chunk
  const int nchunks = (nsrc + sm.chunk - 1) / sm.chunk;
  auto issue = [&](int c) {
    const int cs = c * sm.chunk, ce = min(nsrc, cs + sm.chunk);
    unsigned char* buf = stage + (size_t)(c % sm.nbuf) * sm.chunk * kRowBytes;
    for (int e = cs + (int)threadIdx.x; e < ce; e += blockDim.x) {
      const unsigned long long src = (unsigned long long)s_src[e];
      const int kind = (int)(src >> 62);
      const size_t off = (size_t)(src & 0x3FFFFFFFFFFFFFFFull) * Bp + col0;
      const unsigned char* g = kind == 0   ? reinterpret_cast<const unsigned char*>(J + off)
                               : kind == 1 ? reinterpret_cast<const unsigned char*>(CB + off)
                                           : reinterpret_cast<const unsigned char*>(Fp + off);
      unsigned char* d = buf + (size_t)(e - cs) * kRowBytes;
#pragma unroll
      for (int piece = 0; piece < kPieces; ++piece) cp_async16(d + piece * 16, g + piece * 16);
    }
    cp_async_commit();
  };
  if (nchunks > 0) issue(0);
  if (nchunks > 1) issue(1);

  // phase 2: assembly.  Warp w owns the destination-disjoint range
  // [split[8w/W], split[8(w+1)/W]); consecutive entries with one destination
  // are summed in a register (in list order) and stored once.  With more
  // than 8 warps (W a multiple of 8) the W/8 warps of a range divide it
  // evenly, each cut moved forward to the next change of destination.
  int A, Z;
  if (W <= 8) {
    const int wa = warp * 8 / W, wz = (warp + 1) * 8 / W;
    A = wa == 0 ? 0 : pl.front_meta[(size_t)q * kFrontMetaInts + 11 + wa];
    Z = pl.front_meta[(size_t)q * kFrontMetaInts + 11 + wz];
  } else {
    const int G = W / 8, g = warp / G, sub = warp - g * G;
    const int A0 = g == 0 ? 0 : pl.front_meta[(size_t)q * kFrontMetaInts + 11 + g];
    const int Z0 = pl.front_meta[(size_t)q * kFrontMetaInts + 11 + g + 1];
    A = sub == 0 ? A0 : run_start(s_dst, A0 + (int)((long long)(Z0 - A0) * sub / G), A0, Z0);
    Z = sub == G - 1 ? Z0 : run_start(s_dst, A0 + (int)((long long)(Z0 - A0) * (sub + 1) / G), A0, Z0);
  }
  int cur = -1;
  T acc = T(0);
  for (int c = 0; c < nchunks; ++c) {
    if (c + 1 < nchunks)
      cp_async_wait<1>();
    else
      cp_async_wait<0>();
    __syncthreads();
    const int cs = c * sm.chunk, ce = min(nsrc, cs + sm.chunk);
    const T* buf = reinterpret_cast<const T*>(stage + (size_t)(c % sm.nbuf) * sm.chunk * kRowBytes) + lane;
    const int a = max(cs, A), z = min(ce, Z);
    auto add8 = [&](const int (&d)[8], const T (&v)[8]) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        if (d[u] >= 0) {
          if (d[u] != cur) {
            if (cur >= 0) Fm[cur * kWarp + lane] = acc;
            cur = d[u];
            acc = T(0);
          }
          acc += v[u];
        }
      }
    };
    if constexpr (STAGE_LIST) {
      for (int e = a; e < z; e += 8) {
        T v[8];
        int d[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const bool in = e + u < z;
          d[u] = in ? s_dst[e + u] : -1;
          v[u] = in ? buf[(e + u - cs) * kWarp] : T(0);
        }
        add8(d, v);
      }
    } else {
      // the list is in global memory: the lanes fetch 32 destinations in one
      // request (the next 32 already in flight) and pass them round by shuffle
      int dl = a + lane < z ? s_dst[a + lane] : -1;
      for (int e0 = a; e0 < z; e0 += kWarp) {
        const int n = min(kWarp, z - e0);
        const int dl_next = e0 + kWarp + lane < z ? s_dst[e0 + kWarp + lane] : -1;
        for (int u0 = 0; u0 < n; u0 += 8) {  // u0 + u <= 31
          T v[8];
          int d[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            d[u] = __shfl_sync(0xffffffffu, dl, u0 + u);
            v[u] = d[u] >= 0 ? buf[(e0 + u0 + u - cs) * kWarp] : T(0);
          }
          add8(d, v);
        }
        dl = dl_next;
      }
    }
    __syncthreads();
    if (c + 2 < nchunks) issue(c + 2);
  }
  if (cur >= 0) Fm[cur * kWarp + lane] = acc;
  __syncthreads();
  return m;
}

template <typename T, typename TJ, int FMAX, bool SMEM_FRONT>
__global__ void __launch_bounds__(256)
    k_front_factor(DevPlan pl, int level_begin, long long fe_base, int fe_pad, int groups, int Bp, int front_elems,
                   FrontSmem sm,
                   const TJ* __restrict__ J, const T* __restrict__ Fp, T* __restrict__ U, T* __restrict__ L,
                   T* __restrict__ CB, T* __restrict__ Y, int store_l, double eps, int static_pivot,
                   int* __restrict__ sing, T* __restrict__ front_scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t col0 = (size_t)(blockIdx.x % groups) * kWarp;
  T* Fm = nullptr;
  const FrontMeta m = stage_and_assemble<T, TJ, SMEM_FRONT>(pl, level_begin, fe_base, fe_pad, groups, Bp, front_elems,
                                                            sm, J, Fp, CB, front_scratch, smem_raw, &Fm);
  const int fs = m.fs, nc = m.nc, uc = fs - nc, rw = fs + 1;
  T* s_inv = reinterpret_cast<T*>(smem_raw + sm.idx_bytes);  // [8][32] pivot reciprocals

  // phase 3a: the nc pivot rows.  A pivot is guarded once and its reciprocal
  // kept in s_inv, so every elimination is a multiply (l = a * (1 / u_kk)).
  // With at least nc warps, warp k holds pivot row k in registers and the
  // block runs the nc right-looking steps (warp m publishes its final row,
  // warps k > m apply it); otherwise warp 0 eliminates the rows in order.
  // The eliminated pivot rows go to Pl: the front itself when it is in
  // shared memory; for a front in the global scratch, the staging area
  // (free once the front is assembled) when they fit there, so that every
  // row's elimination reads them from shared memory instead of L2.
  bool shifted = false;
  T* Fl = Fm + lane;
  T* inv_l = s_inv + lane;
  T* Pl = Fl;
  if constexpr (!SMEM_FRONT) {
    if ((size_t)nc * rw * kWarp * sizeof(T) <= sm.stage_bytes)
      Pl = reinterpret_cast<T*>(smem_raw + sm.idx_bytes + sm.inv_bytes) + lane;
  }
  if (W >= nc) {
    T r[FMAX + 1];
    const bool own = warp < nc;
    if (own) {
      const T* Rw = Fl + warp * rw * kWarp;
#pragma unroll
      for (int j = 0; j <= FMAX; ++j) r[j] = j < rw ? Rw[j * kWarp] : T(0);
    }
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if (m >= nc) break;
      if (warp == m) {
        r[m] = guarded_pivot(r[m], static_pivot != 0, eps, shifted);
        inv_l[m * kWarp] = T(1) / r[m];
        T* Rm = Pl + m * rw * kWarp;
#pragma unroll
        for (int j = 0; j <= FMAX; ++j)
          if (j < rw) Rm[j * kWarp] = r[j];
      }
      __syncthreads();
      if (own && warp > m) {
        const T* Um = Pl + m * rw * kWarp;
        const T l = r[m] * inv_l[m * kWarp];
        r[m] = l;
#pragma unroll
        for (int j = m + 1; j <= FMAX; ++j)
          if (j < rw) r[j] -= l * Um[j * kWarp];
      }
    }
  } else {
    if (warp == 0) {
      for (int k = 0; k < nc; ++k) {
        const T* Rk = Fl + (size_t)k * rw * kWarp;
        T r[FMAX + 1];
#pragma unroll
        for (int j = 0; j <= FMAX; ++j) r[j] = j < rw ? Rk[(size_t)j * kWarp] : T(0);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
          if (m < k) {
            const T* Um = Pl + (size_t)m * rw * kWarp;
            const T l = r[m] * inv_l[m * kWarp];
            r[m] = l;
#pragma unroll
            for (int j = m + 1; j <= FMAX; ++j)
              if (j < rw) r[j] -= l * Um[(size_t)j * kWarp];
          }
        }
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (j == k) {
            r[j] = guarded_pivot(r[j], static_pivot != 0, eps, shifted);
            inv_l[j * kWarp] = T(1) / r[j];
          }
        T* Pk = Pl + (size_t)k * rw * kWarp;
#pragma unroll
        for (int j = 0; j <= FMAX; ++j)
          if (j < rw) Pk[(size_t)j * kWarp] = r[j];
      }
    }
    __syncthreads();
  }

  // phase 3b: outputs of the pivot rows (U rows, y) ...
  const size_t b = col0 + lane;
  const long long uo = m.uo, lo = m.lo, co = m.co;
  const int first = m.first;
  {
    const size_t step = (size_t)W * Bp;
    for (int k = 0; k < nc; ++k) {
      T* Ub = U + (size_t)(uo + (long long)k * fs + warp) * Bp + b;
      const T* src = Pl + (k * rw + warp) * kWarp;
      for (int j = warp; j < fs; j += W, Ub += step, src += W * kWarp) *Ub = *src;
    }
    for (int k = warp; k < nc; k += W) Y[(size_t)(first + k) * Bp + b] = Pl[(k * rw + fs) * kWarp];
  }
  // ... and the uc non-pivot rows, independent of each other: row i applies
  // the nc pivot rows in registers and goes straight out as L21 | CB.  FP32
  // fronts of up to 16 rows take two rows per pass (two independent chains,
  // and each pivot-row element read once for both; in FP64 the second row's
  // registers cost more residency than the pass saves).
  auto store_row = [&](const T (&r)[FMAX + 1], int i) {
    const int ii = i - nc;
    if (store_l) {
      T* Lb = L + (size_t)(lo + (long long)ii * nc) * Bp + b;
#pragma unroll
      for (int m = 0; m < 8; ++m)
        if (m < nc) Lb[(size_t)m * Bp] = r[m];
    }
    T* Cb = CB + (size_t)(co + (long long)ii * (uc + 1)) * Bp + b;
#pragma unroll
    for (int j = 0; j <= FMAX; ++j)
      if (j >= nc && j < rw) Cb[(size_t)(j - nc) * Bp] = r[j];
  };
  if constexpr (FMAX <= 16 && sizeof(T) == 4) {
    for (int i = nc + warp; i < fs; i += 2 * W) {
      const int i2 = i + W;
      const bool two = i2 < fs;
      const T* Ri = Fl + i * rw * kWarp;
      const T* Ri2 = Fl + (two ? i2 : i) * rw * kWarp;
      T r[FMAX + 1], r2[FMAX + 1];
#pragma unroll
      for (int j = 0; j <= FMAX; ++j) {
        r[j] = j < rw ? Ri[j * kWarp] : T(0);
        r2[j] = j < rw ? Ri2[j * kWarp] : T(0);
      }
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        if (m < nc) {
          const T* Um = Pl + m * rw * kWarp;
          const T inv = inv_l[m * kWarp];
          const T l = r[m] * inv, l2 = r2[m] * inv;
          r[m] = l;
          r2[m] = l2;
#pragma unroll
          for (int j = m + 1; j <= FMAX; ++j)
            if (j < rw) {
              const T u = Um[j * kWarp];
              r[j] -= l * u;
              r2[j] -= l2 * u;
            }
        }
      }
      store_row(r, i);
      if (two) store_row(r2, i2);
    }
  } else {
    for (int i = nc + warp; i < fs; i += W) {
      const T* Ri = Fl + i * rw * kWarp;
      T r[FMAX + 1];
#pragma unroll
      for (int j = 0; j <= FMAX; ++j) r[j] = j < rw ? Ri[j * kWarp] : T(0);
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        if (m < nc) {
          const T* Um = Pl + m * rw * kWarp;
          const T l = r[m] * inv_l[m * kWarp];
          r[m] = l;
#pragma unroll
          for (int j = m + 1; j <= FMAX; ++j)
            if (j < rw) r[j] -= l * Um[j * kWarp];
        }
      }
      store_row(r, i);
    }
  }
  if (shifted) sing[b] = 1;
}

// ---------------------------------------------------------------------------
// The single-system schedule (batch 1): one block per front, its threads
// spread over the front's rows and elements instead of over scenarios (the
// lane kernels above would keep 31 of every 32 lanes on padding copies).
//   1. the dense front [fs][fs + 1] in shared memory, zeroed;
//   2. assembly: each run of list entries with one destination is summed in
//      list order by one thread (the lane kernels sum the same runs in the
//      same order);
//   3. right-looking elimination of the nc pivot columns: per pivot, one
//      thread guards it and takes its reciprocal, the rows below take their
//      multiplier l = a_ik * (1 / u_kk), then every trailing element
//      a_ij -= l_i u_kj.  Each element sees the lane kernels' operations in
//      the same order, so the factors are the same bits;
//   4. U rows, y, L21 (store_l) and the contribution block out, each value
//      written to all 32 lanes of its row: every lane of the batch-innermost
//      arrays then holds what the lane kernels leave there for a batch of 1
//      (whose padding lanes copy scenario 0), and the backward sweep and the
//      adjoint read them unchanged.
// ---------------------------------------------------------------------------
// Shared memory of a single-system block: [header | kSingleHeader B]
// [front fs x (fs + 1)][values x list_cap][sources, destinations x list_cap,
// from a 16-byte boundary].
template <typename T>
struct SingleSmem {
  T* F;
  T* vals;
  long long* srcs;
  int* dsts;
  __device__ SingleSmem(unsigned char* raw, int fs, int list_cap) {
    F = reinterpret_cast<T*>(raw + kSingleHeader);
    vals = F + fs * (fs + 1);
    const size_t list_off = (kSingleHeader + ((size_t)fs * (fs + 1) + list_cap) * sizeof(T) + 15) & ~(size_t)15;
    srcs = reinterpret_cast<long long*>(raw + list_off);
    dsts = reinterpret_cast<int*>(srcs + list_cap);
  }
};

// Phase 1 of front q (whole block): its source list (starting at e0, at most
// list_cap entries) into shared memory, the front zeroed, and the values
// that earlier kernels wrote (Jacobian entries, right-hand-side rows); the
// children's contribution-block values wait for single_finish.
// wait_previous: wait for the previous kernel before reading those values.
template <typename T, typename TJ>
__device__ __forceinline__ FrontMeta single_load(const DevPlan& pl, int q, long long e0, int list_cap, int Bp,
                                                 const TJ* __restrict__ J, const T* __restrict__ Fp,
                                                 unsigned char* smem_raw, bool wait_previous) {
  const int nt = blockDim.x, tid = threadIdx.x;
  const FrontMeta m = load_front_meta(pl.front_meta, q);
  const int fs = m.fs, rw = fs + 1, nsrc = m.split[8];
  const SingleSmem<T> sm(smem_raw, fs, list_cap);
  for (int e = tid; e < fs * rw; e += nt) sm.F[e] = T(0);
  if (wait_previous) chain_wait_previous();
  for (int e = tid; e < nsrc; e += nt) {
    const unsigned long long sv = (unsigned long long)pl.fe_src[e0 + e];
    sm.srcs[e] = (long long)sv;
    sm.dsts[e] = pl.fe_dst[e0 + e];
    const int kind = (int)(sv >> 62);
    const size_t off = (size_t)(sv & 0x3FFFFFFFFFFFFFFFull) * Bp;
    if (kind != 1) sm.vals[e] = kind == 0 ? static_cast<T>(J[off]) : Fp[off];
  }
  return m;
}

// Phase 2 (whole block, after single_load): the contribution-block values
// (read through L2 only, ld.global.cg: in the tree launch another SM wrote
// them during this kernel), the assembly, the elimination and the outputs.
// Returns after the outputs are stored (no barrier at the end).
template <typename T>
__device__ __forceinline__ void single_finish(const FrontMeta& m, int list_cap, int Bp, T* __restrict__ U,
                                              T* __restrict__ L, T* __restrict__ CB, T* __restrict__ Y,
                                              int store_l, double eps, int static_pivot, int* __restrict__ sing,
                                              unsigned char* smem_raw) {
  T& s_inv = *reinterpret_cast<T*>(smem_raw);
  int& s_shift = *reinterpret_cast<int*>(smem_raw + 8);
  const int nt = blockDim.x, tid = threadIdx.x, W = nt >> 5, warp = tid >> 5, lane = tid & 31;
  const int fs = m.fs, nc = m.nc, uc = fs - nc, rw = fs + 1, nsrc = m.split[8];
  const SingleSmem<T> sm(smem_raw, fs, list_cap);
  T* F = sm.F;
  if (tid == 0) s_shift = 0;
  __syncthreads();
  for (int e = tid; e < nsrc; e += nt) {
    const unsigned long long sv = (unsigned long long)sm.srcs[e];
    if ((int)(sv >> 62) == 1) sm.vals[e] = __ldcg(CB + (size_t)(sv & 0x3FFFFFFFFFFFFFFFull) * Bp);
  }
  __syncthreads();
  // each run of entries with one destination summed in list order by one thread
  for (int e = tid; e < nsrc; e += nt) {
    const int d = sm.dsts[e];
    if (d < 0 || (e > 0 && sm.dsts[e - 1] == d)) continue;  // not the first entry of its run
    T acc = T(0);
    for (int f = e; f < nsrc && sm.dsts[f] == d; ++f) acc += sm.vals[f];
    F[d] = acc;
  }
  // right-looking elimination: warp w takes rows k + 1 + w, k + 1 + w + W, ...
  // (every lane forms the row's multiplier, lane j its columns)
  for (int k = 0; k < nc; ++k) {
    __syncthreads();
    if (tid == 0) {
      bool sh = false;
      const T p = guarded_pivot(F[k * rw + k], static_pivot != 0, eps, sh);
      F[k * rw + k] = p;
      s_inv = T(1) / p;
      if (sh) s_shift = 1;
    }
    __syncthreads();
    const T inv = s_inv;
    for (int i = k + 1 + warp; i < fs; i += W) {
      const T l = F[i * rw + k] * inv;
      for (int j = k + 1 + lane; j < rw; j += 32) F[i * rw + j] -= l * F[k * rw + j];
      __syncwarp();
      if (lane == 0) F[i * rw + k] = l;
    }
  }
  __syncthreads();
  // every output value to all 32 lanes of its row (one coalesced store per
  // warp); warp w takes rows w, w + W, ...
  for (int k = warp; k < nc; k += W) {
    T* Uk = U + (size_t)(m.uo + (long long)k * fs) * Bp + lane;
    for (int j = 0; j < fs; ++j) Uk[(size_t)j * Bp] = F[k * rw + j];
    Y[(size_t)(m.first + k) * Bp + lane] = F[k * rw + fs];
  }
  for (int ii = warp; ii < uc; ii += W) {
    const T* Fi = F + (nc + ii) * rw;
    if (store_l) {
      T* Li = L + (size_t)(m.lo + (long long)ii * nc) * Bp + lane;
      for (int mm = 0; mm < nc; ++mm) Li[(size_t)mm * Bp] = Fi[mm];
    }
    T* Ci = CB + (size_t)(m.co + (long long)ii * (uc + 1)) * Bp + lane;
    for (int jj = 0; jj <= uc; ++jj) Ci[(size_t)jj * Bp] = Fi[nc + jj];
  }
  if (s_shift && warp == 0) sing[lane] = 1;
}

// One launch per level: block b factors front level_begin + b.
template <typename T, typename TJ>
__global__ void __launch_bounds__(256)
    k_front_factor_single(DevPlan pl, int level_begin, long long fe_base, int fe_pad, int Bp,
                          const TJ* __restrict__ J, const T* __restrict__ Fp, T* __restrict__ U, T* __restrict__ L,
                          T* __restrict__ CB, T* __restrict__ Y, int store_l, double eps, int static_pivot,
                          int* __restrict__ sing) {
  static_assert(sizeof(TJ) == sizeof(T), "Jacobian and factor rows share one element type");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  chain_allow_next();
  const int q = level_begin + blockIdx.x;
  const FrontMeta m = single_load<T, TJ>(pl, q, fe_base + (long long)(q - level_begin) * fe_pad, fe_pad, Bp, J, Fp,
                                         smem_raw, true);
  single_finish<T>(m, fe_pad, Bp, U, L, CB, Y, store_l, eps, static_pivot, sing, smem_raw);
}

// The whole factorization of a single system as one launch over the front
// tree.  Persistent blocks take the tree's leaves in level order from a
// counter (next).  A block that has stored a front's outputs counts it done
// at the parent (done[parent]); the block whose count completes the parent's
// children goes on with the parent itself, so no block ever waits for
// another: a front starts as soon as its last child is stored.  While the
// count is in flight, every block loads the parent's list and its Jacobian
// and right-hand-side values (kept only by the block that goes on).  done
// and next start at zero.
template <typename T, typename TJ>
__global__ void __launch_bounds__(128)
    k_factor_single_tree(DevPlan pl, const int* __restrict__ parent, const int* __restrict__ nchild,
                         const long long* __restrict__ q_e0, const int* __restrict__ leaves, int n_leaves,
                         int* __restrict__ done, int* __restrict__ next, int list_cap, int Bp,
                         const TJ* __restrict__ J, const T* __restrict__ Fp, T* __restrict__ U, T* __restrict__ L,
                         T* __restrict__ CB, T* __restrict__ Y, int store_l, double eps, int static_pivot,
                         int* __restrict__ sing) {
  static_assert(sizeof(TJ) == sizeof(T), "Jacobian and factor rows share one element type");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  int& s_item = *reinterpret_cast<int*>(smem_raw + 12);
  chain_allow_next();
  chain_wait_previous();  // J and Fp come from earlier kernels
  int q = -1;             // the front this block goes on with (-1: take the next leaf)
  FrontMeta m;
  for (;;) {
    if (q < 0) {
      __syncthreads();  // every thread has read s_item
      if (threadIdx.x == 0) {
        const int i = atomicAdd(next, 1);
        s_item = i < n_leaves ? leaves[i] : -1;
      }
      __syncthreads();
      q = s_item;
      if (q < 0) break;
      m = single_load<T, TJ>(pl, q, q_e0[q], list_cap, Bp, J, Fp, smem_raw, false);
    }
    single_finish<T>(m, list_cap, Bp, U, L, CB, Y, store_l, eps, static_pivot, sing, smem_raw);
    __threadfence();  // this front's stores before its count at the parent
    __syncthreads();  // (also: the front's shared memory is free)
    const int p = parent[q];
    int last = 0;
    if (threadIdx.x == 0 && p >= 0) last = atomicAdd(done + p, 1) == nchild[p] - 1;
    if (p >= 0) m = single_load<T, TJ>(pl, p, q_e0[p], list_cap, Bp, J, Fp, smem_raw, false);
    if (threadIdx.x == 0) {
      if (last) __threadfence();  // the other children's stores, counted before ours, before our reads
      s_item = last ? p : -1;
    }
    __syncthreads();
    q = s_item;
  }
}

// ---------------------------------------------------------------------------
// The wide tier: fronts of any size.  Same block shape (one front x 32
// scenarios) and phases 1-2 as k_front_factor, with the source list read
// from global memory, the dense front always in this block's slice of the
// global scratch, and the nc pivot rows Us [nc][fs + 1][32] in shared memory
// (or after the front in the scratch when they do not fit).  No row is held
// in registers, so the front size has no compile-time bound:
//  3a. pivot rows k = 0 .. nc-1 in order: every warp forms the row's
//      multipliers l_km (m < k) for its lane, then its share of the row's
//      columns j >= k (j = fs is the right-hand side); warp 0 guards the
//      pivot and keeps 1 / u_kk;
//  3b. U rows and y out;
//  3c. non-pivot rows, one warp per row: the nc multipliers (L21, stored
//      when store_l), then CB row = A22 row - L21 row * U12, streamed out.
// Every element sees the register kernel's operations in the same order, so
// both tiers produce the same factors.
// ---------------------------------------------------------------------------

// Multipliers of front row Ri against the first n pivot rows (n <= 8):
// l_m = (a_m - sum_{m' < m} l_m' u_m'm) / u_mm, in the register kernel's order.
// Us holds the pivot rows with lane stride LS (32, or 33 where other code
// reads one scenario's column of it).
template <typename T, int LS = kWarp>
__device__ __forceinline__ void row_multipliers(const T* Ri, const T* Us, const T* inv_l, int rw, int n, T (&l)[8]) {
#pragma unroll
  for (int mm = 0; mm < 8; ++mm) {
    l[mm] = T(0);
    if (mm < n) {
      T r = Ri[(size_t)mm * kWarp];
#pragma unroll
      for (int m2 = 0; m2 < 8; ++m2)
        if (m2 < mm) r -= l[m2] * Us[(size_t)(m2 * rw + mm) * LS];
      l[mm] = r * inv_l[mm * kWarp];
    }
  }
}

// Phase 3a/3b of the wide tier: the pivot rows into Us (lane stride LS), then
// U rows and y out.
template <typename T, int LS = kWarp>
__device__ __forceinline__ void wide_pivot_rows(const FrontMeta& m, const T* Fl, T* Us, T* inv_l, int Bp, size_t b,
                                                T* __restrict__ U, T* __restrict__ Y, double eps, int static_pivot,
                                                bool& shifted) {
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const int fs = m.fs, nc = m.nc, rw = fs + 1;
  for (int k = 0; k < nc; ++k) {
    const T* Rk = Fl + (size_t)k * rw * kWarp;
    T l[8];
    row_multipliers<T, LS>(Rk, Us, inv_l, rw, k, l);
    T* Uk = Us + (size_t)k * rw * LS;
    for (int j = warp; j <= fs; j += W) {
      T r = T(0);
      if (j < k) {
#pragma unroll
        for (int mm = 0; mm < 8; ++mm)
          if (mm == j) r = l[mm];
      } else {
        r = Rk[(size_t)j * kWarp];
#pragma unroll
        for (int mm = 0; mm < 8; ++mm)
          if (mm < k) r -= l[mm] * Us[(size_t)(mm * rw + j) * LS];
      }
      Uk[(size_t)j * LS] = r;
    }
    __syncthreads();
    if (warp == 0) {
      const T p = guarded_pivot(Uk[(size_t)k * LS], static_pivot != 0, eps, shifted);
      Uk[(size_t)k * LS] = p;
      inv_l[k * kWarp] = T(1) / p;
    }
    __syncthreads();
  }
  // U rows: elements uo + k * fs + j (j < fs), then y from the rhs column
  for (int e = warp; e < nc * fs; e += W) {
    const int k = e / fs, j = e - k * fs;
    U[(size_t)(m.uo + e) * Bp + b] = Us[(size_t)(k * rw + j) * LS];
  }
  for (int k = warp; k < nc; k += W) Y[(size_t)(m.first + k) * Bp + b] = Us[(size_t)(k * rw + fs) * LS];
}

// MAXW: the most warps a launch of this instance may have (8, 16 or 32;
// 32 leaves 64 registers a thread).
template <typename T, typename TJ, int MAXW = 8>
__global__ void __launch_bounds__(MAXW * 32)
    k_front_factor_wide(DevPlan pl, int level_begin, long long fe_base, int fe_pad, int groups, int Bp,
                        int front_elems, FrontSmem sm, const TJ* __restrict__ J, const T* __restrict__ Fp,
                        T* __restrict__ U, T* __restrict__ L, T* __restrict__ CB, T* __restrict__ Y, int store_l,
                        double eps, int static_pivot, int* __restrict__ sing, T* __restrict__ front_scratch) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t col0 = (size_t)(blockIdx.x % groups) * kWarp;
  const size_t b = col0 + lane;
  T* Fm = nullptr;
  const FrontMeta m = stage_and_assemble<T, TJ, false, false>(pl, level_begin, fe_base, fe_pad, groups, Bp,
                                                              front_elems, sm, J, Fp, CB, front_scratch, smem_raw,
                                                              &Fm);
  const int fs = m.fs, nc = m.nc, uc = fs - nc, rw = fs + 1;
  T* inv_l = reinterpret_cast<T*>(smem_raw + sm.idx_bytes) + lane;
  T* Us = (sm.us_bytes ? reinterpret_cast<T*>(smem_raw + sm.idx_bytes + sm.inv_bytes + sm.stage_bytes)
                       : Fm + (size_t)fs * rw * kWarp) + lane;
  const T* Fl = Fm + lane;
  bool shifted = false;
  wide_pivot_rows<T>(m, Fl, Us, inv_l, Bp, b, U, Y, eps, static_pivot, shifted);
  for (int i = nc + warp; i < fs; i += W) {
    const int ii = i - nc;
    const T* Ri = Fl + (size_t)i * rw * kWarp;
    T l[8];
    row_multipliers(Ri, Us, inv_l, rw, nc, l);
    if (store_l) {
      T* Lb = L + (size_t)(m.lo + (long long)ii * nc) * Bp + b;
#pragma unroll
      for (int mm = 0; mm < 8; ++mm)
        if (mm < nc) Lb[(size_t)mm * Bp] = l[mm];
    }
    T* Cb = CB + (size_t)(m.co + (long long)ii * (uc + 1)) * Bp + b;
#pragma unroll 4
    for (int j = nc; j <= fs; ++j) {
      T r = Ri[(size_t)j * kWarp];
#pragma unroll
      for (int mm = 0; mm < 8; ++mm)
        if (mm < nc) r -= l[mm] * Us[(size_t)(mm * rw + j) * kWarp];
      Cb[(size_t)(j - nc) * Bp] = r;
    }
  }
  if (shifted) sing[b] = 1;
}

// ---------------------------------------------------------------------------
// The wide tier with the trailing update on the tensor cores (FP32 factors;
// CustomPrecision::TF32).  Phases 1-3b as k_front_factor_wide, with the
// pivot rows in shared memory at lane stride 33 (so that one scenario's
// column is read across the banks); then
//  3c. the L21 multipliers of every non-pivot row, for the block's 32
//      scenarios, into shared memory (Ls [uc][8][33]);
//  3d. in rounds of S scenarios (as many as the shared-memory tiles and the
//      512 tensor-memory columns allow): each scenario's L21 block (uc x nc,
//      padded to M = 128 rows) and U12^T ((uc + 1) x nc: the trailing
//      columns and the right-hand side, padded to N rows) are packed as
//      K-major tf32 tiles, each operand split as x = hi + lo (both tf32,
//      about 21 bits of the fp32 value); three tcgen05.mma kind::tf32 with
//      K = 8 -- hi*hi + hi*lo + lo*hi, the Ozaki-style split -- accumulate
//      D = L21 U12 in the scenario's own tensor-memory columns (fp32), one
//      commit per round.  The epilogue reads D back (tcgen05.ld: TMEM lane =
//      front row) and subtracts it from the trailing block of the front in
//      the scratch;
//  3e. the trailing block, now A22 - L21 U12 with the updated right-hand
//      side, is copied to CB, 32 scenarios per coalesced row.
// One thread issues the MMAs; the wait for their commit is bounded.  When it
// runs out, the block flags its systems (singular flag 2) and writes NaN to
// their y and CB rows, so a solve on these factors is visibly non-finite.
// Limits (checked by the launcher, which uses the FP32 wide tier otherwise):
// uc <= 128 (one M tile), uc + 1 <= 256 (one N tile), shared memory.
// ---------------------------------------------------------------------------
constexpr int kTcLS = kWarp + 1;  // lane stride of Us and Ls in the tensor-core tier

// Shared-memory layout of a tensor-core launch (byte offsets from the base).
// A round packs the operands of `spr` scenarios and issues their products
// together (3 MMAs each into its own TMEM columns, one commit).
struct TcLayout {
  int n_pad = 0;      // N of the MMA: the trailing columns + rhs, rounded up to 16
  int spr = 1;        // scenarios per round (1, 2, 4 or 8)
  int tmem_cols = 0;  // tensor-memory columns allocated (power of 2 >= 32, >= spr * n_pad)
  unsigned us_off = 0, ls_off = 0, a_off = 0, b_off = 0, bar_off = 0, total = 0;
};

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

inline int tc_n_pad(const LevelLaunch& lv) { return (int)align_up((size_t)std::max(lv.max_fsz, 16), 16); }

// Bytes the tensor-core tier needs beside the staging (rounding included)
// for `spr` scenarios per round.
inline size_t tc_reserve_bytes(const LevelLaunch& lv, int spr) {
  const int rw = lv.max_fsz + 1, max_uc = lv.max_fsz - 1;
  return 16 + (size_t)lv.max_nc * rw * kTcLS * sizeof(float) + 16 +
         (size_t)std::max(max_uc, 1) * 8 * kTcLS * sizeof(float) + 128 + (size_t)spr * 2 * 128 * 32 +
         (size_t)spr * 2 * tc_n_pad(lv) * 32 + 8 + 16 + 16;
}

inline TcLayout plan_tc_layout(const LevelLaunch& lv, const FrontSmem& sm, int spr) {
  TcLayout t;
  const int rw = lv.max_fsz + 1;
  const int max_uc = lv.max_fsz - 1;  // nc >= 1
  t.n_pad = tc_n_pad(lv);
  t.spr = spr;
  t.tmem_cols = 32;
  while (t.tmem_cols < spr * t.n_pad) t.tmem_cols *= 2;
  size_t off = sm.idx_bytes + sm.inv_bytes + sm.stage_bytes;
  off = align_up(off, 16);
  t.us_off = (unsigned)off;
  off += (size_t)lv.max_nc * rw * kTcLS * sizeof(float);
  off = align_up(off, 16);
  t.ls_off = (unsigned)off;
  off += (size_t)std::max(max_uc, 1) * 8 * kTcLS * sizeof(float);
  off = align_up(off, 128);
  t.a_off = (unsigned)off;
  off += (size_t)spr * 2 * 128 * 32;  // per scenario: A hi, A lo (128 rows x 8 tf32)
  t.b_off = (unsigned)off;
  off += (size_t)spr * 2 * t.n_pad * 32;  // per scenario: B hi, B lo (n_pad rows x 8 tf32)
  off = align_up(off, 8);
  t.bar_off = (unsigned)off;
  off += 8 + 4 + 4;  // mbarrier, TMEM address slot, failure flag
  t.total = (unsigned)align_up(off, 16);
  return t;
}

inline bool tc_tier_fits(const LevelLaunch& lv, const TcLayout& t) {
  return lv.max_fsz - 1 <= 128 && t.n_pad <= 256 && t.spr * t.n_pad <= 512 && t.total <= kSmemLimit;
}

// Staging and layout of a tensor-core launch: the most scenarios per round
// (8, 4, 2, 1) whose tiles and tensor memory fit, with staging chunks of at
// least 32 rows beside them.
inline bool plan_tc(const LevelLaunch& lv, FrontSmem* sm, TcLayout* tl) {
  for (int spr : {8, 4, 2, 1}) {
    if (spr * tc_n_pad(lv) > 512) continue;
    *sm = plan_wide_staging(lv, sizeof(float), tc_reserve_bytes(lv, spr));
    sm->us_bytes = 0;  // the pivot rows have their own padded place
    if (sm->nbuf == 2 && sm->chunk < 32) continue;
    *tl = plan_tc_layout(lv, *sm, spr);
    if (tc_tier_fits(lv, *tl)) return true;
  }
  return false;
}

// byte offset of element (r, k) in a K-major tile of 8-row x 16-byte core
// matrices, K = 8 tf32: core matrices 128 B apart along K, 8-row groups 256 B
__device__ __forceinline__ unsigned tc_tile_off(int r, int k) {
  return (unsigned)((r >> 3) * 256 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

__global__ void __launch_bounds__(256)
    k_front_factor_tc(DevPlan pl, int level_begin, long long fe_base, int fe_pad, int groups, int Bp,
                      int front_elems, FrontSmem sm, TcLayout tl, const float* __restrict__ J,
                      const float* __restrict__ Fp, float* __restrict__ U, float* __restrict__ L,
                      float* __restrict__ CB, float* __restrict__ Y, int store_l, double eps, int static_pivot,
                      int* __restrict__ sing, float* __restrict__ front_scratch, long long spin_limit) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t col0 = (size_t)(blockIdx.x % groups) * kWarp;
  const size_t b = col0 + lane;
  float* Fm = nullptr;
  const FrontMeta m = stage_and_assemble<float, float, false, false>(pl, level_begin, fe_base, fe_pad, groups, Bp,
                                                                      front_elems, sm, J, Fp, CB, front_scratch,
                                                                      smem_raw, &Fm);
  const int fs = m.fs, nc = m.nc, uc = fs - nc, rw = fs + 1, nb = uc + 1;
  float* inv_l = reinterpret_cast<float*>(smem_raw + sm.idx_bytes) + lane;
  float* Us = reinterpret_cast<float*>(smem_raw + tl.us_off);  // [nc][rw][33]
  float* Ls = reinterpret_cast<float*>(smem_raw + tl.ls_off);  // [uc][8][33]
  unsigned char* tA = smem_raw + tl.a_off;
  unsigned char* tB = smem_raw + tl.b_off;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + tl.bar_off);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem_raw + tl.bar_off + 8);
  int* s_fail = reinterpret_cast<int*>(smem_raw + tl.bar_off + 12);
  const float* Fl = Fm + lane;
  if (threadIdx.x == 0) {
    tc::mbar_init(bar, 1);
    *s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  bool shifted = false;
  wide_pivot_rows<float, kTcLS>(m, Fl, Us + lane, inv_l, Bp, b, U, Y, eps, static_pivot, shifted);
  // 3c: multipliers of the non-pivot rows (L21), 32 scenarios at a time
  for (int i = nc + warp; i < fs; i += W) {
    const int ii = i - nc;
    float l[8];
    row_multipliers<float, kTcLS>(Fl + (size_t)i * rw * kWarp, Us + lane, inv_l, rw, nc, l);
    float* Lr = Ls + (size_t)ii * 8 * kTcLS + lane;
#pragma unroll
    for (int k = 0; k < 8; ++k) Lr[k * kTcLS] = l[k];
    if (store_l) {
      float* Lb = L + (size_t)(m.lo + (long long)ii * nc) * Bp + b;
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k < nc) Lb[(size_t)k * Bp] = l[k];
    }
  }
  if (warp == 0) tc::tmem_alloc(tslot, (uint32_t)tl.tmem_cols);
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = tc::idesc_tf32(128, tl.n_pad);
  const int qtr = warp & 3, nsplit = W >> 2, part = warp >> 2;
  const int row = qtr * 32 + lane;  // this thread's TMEM lane = front row of the trailing block
  int failed_at = -1;  // the round whose products did not complete
  const int S = tl.spr;
  const size_t a_stride = 2 * 128 * 32, b_stride = 2 * (size_t)tl.n_pad * 32;  // bytes per scenario
  for (int rnd = 0; rnd < (uc > 0 ? kWarp / S : 0); ++rnd) {  // (a root front has no trailing block)
    const int sc0 = rnd * S;
    // 3d: the operands of scenarios sc0 .. sc0 + S - 1 as hi + lo tf32 tiles
    for (int e = threadIdx.x; e < S * 128 * 8; e += blockDim.x) {
      const int s_ = e / (128 * 8), r = (e >> 3) & 127, k = e & 7;
      const float x = r < uc ? Ls[((size_t)r * 8 + k) * kTcLS + sc0 + s_] : 0.0f;
      const float hi = tc::to_tf32(x);
      unsigned char* a = tA + (size_t)s_ * a_stride + tc_tile_off(r, k);
      *reinterpret_cast<float*>(a) = hi;
      *reinterpret_cast<float*>(a + 4096) = tc::to_tf32(x - hi);
    }
    for (int e = threadIdx.x; e < S * tl.n_pad * 8; e += blockDim.x) {
      const int s_ = e / (tl.n_pad * 8), j = (e >> 3) % tl.n_pad, k = e & 7;
      const float x = (j < nb && k < nc) ? Us[((size_t)k * rw + nc + j) * kTcLS + sc0 + s_] : 0.0f;
      const float hi = tc::to_tf32(x);
      unsigned char* bp = tB + (size_t)s_ * b_stride + tc_tile_off(j, k);
      *reinterpret_cast<float*>(bp) = hi;
      *reinterpret_cast<float*>(bp + (size_t)tl.n_pad * 32) = tc::to_tf32(x - hi);
    }
    tc::fence_smem_to_async();
    __syncthreads();
    if (threadIdx.x == 0) {
      tc::tc_fence_after();
      for (int s_ = 0; s_ < S; ++s_) {
        const unsigned char* a = tA + (size_t)s_ * a_stride;
        const unsigned char* bp = tB + (size_t)s_ * b_stride;
        const uint64_t ah = tc::smem_desc_plain(a, 128, 256), al = tc::smem_desc_plain(a + 4096, 128, 256);
        const uint64_t bh = tc::smem_desc_plain(bp, 128, 256);
        const uint64_t bl = tc::smem_desc_plain(bp + (size_t)tl.n_pad * 32, 128, 256);
        const uint32_t d = tmem + (uint32_t)(s_ * tl.n_pad);  // this scenario's accumulator columns
        tc::tc_mma_tf32(d, ah, bh, idesc, 0u);
        tc::tc_mma_tf32(d, ah, bl, idesc, 1u);
        tc::tc_mma_tf32(d, al, bh, idesc, 1u);
      }
      tc::tc_commit(bar);
    }
    const bool have = __all_sync(0xffffffffu, tc::mbar_wait(bar, (uint32_t)(rnd & 1), spin_limit));
    if (!have && lane == 0) atomicExch(s_fail, 1);
    __syncthreads();
    tc::tc_fence_after();
    if (*s_fail) {
      failed_at = rnd;
      break;
    }
    // epilogue: the W / 4 warps of a TMEM lane quarter split the (scenario,
    // 16-column chunk) pairs
    const int nch = tl.n_pad / 16;
    for (int w = part; w < S * nch; w += nsplit) {
      const int s_ = w / nch, c = w - s_ * nch;
      float v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(qtr * 32) << 16) + (uint32_t)(s_ * tl.n_pad + c * 16), v);
      if (row < uc) {
        float* Fr = Fm + ((size_t)(nc + row) * rw + nc) * kWarp + sc0 + s_;
#pragma unroll
        for (int t = 0; t < 16; ++t)
          if (c * 16 + t < nb) Fr[(size_t)(c * 16 + t) * kWarp] -= v[t];
      }
    }
    tc::tc_fence_before();
    __syncthreads();
  }
  if (failed_at >= 0) tc::mbar_wait(bar, (uint32_t)(failed_at & 1), spin_limit);  // the MMAs still in flight
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, (uint32_t)tl.tmem_cols);
  // 3e: the updated trailing block -> CB (NaN when the products did not complete)
  const float nan = __int_as_float(0x7fc00000);
  for (int ii = warp; ii < uc; ii += W) {
    const float* Fr = Fl + ((size_t)(nc + ii) * rw + nc) * kWarp;
    float* Cb = CB + (size_t)(m.co + (long long)ii * nb) * Bp + b;
    for (int j = 0; j < nb; ++j) Cb[(size_t)j * Bp] = failed_at < 0 ? Fr[(size_t)j * kWarp] : nan;
  }
  if (failed_at >= 0) {
    for (int k = warp; k < nc; k += W) Y[(size_t)(m.first + k) * Bp + b] = nan;
    if (warp == 0) sing[b] = 2;
  } else if (shifted) {
    sing[b] = 1;
  }
}

// ---------------------------------------------------------------------------
// Backward substitution U x = y of one level (root first).  X is in permuted
// order; a front reads the x of its CB rows, which belong to ancestors.
// One warp = one front x 32 scenarios.  The warp stages its front's U rows
// (contiguous elements) and the x rows of its CB rows (gathered through
// front_rows) with cp.async, then solves the nc pivots from shared memory.
// ---------------------------------------------------------------------------
// One front x 32 scenarios (starting at col0), by one warp, with its
// staging area Us.
// STAGED = false (fronts whose U rows do not fit in shared memory): the same
// substitution reading U and x straight from global memory.
template <typename T, bool STAGED = true>
__device__ __forceinline__ void backward_front(const DevPlan& pl, const FrontMeta& m, size_t col0, int Bp, T* Us,
                                               const T* __restrict__ U, const T* __restrict__ Y,
                                               T* __restrict__ X) {
  constexpr int kPieces = kWarp * sizeof(T) / 16;
  const int lane = threadIdx.x & 31;
  const size_t b = col0 + lane;
  const int fs = m.fs, nc = m.nc, uc = fs - nc;
  const int fr0 = m.fr0, first = m.first;
  const long long uo = m.uo;
  if constexpr (!STAGED) {
    // x_k = (y_k - sum_{j > k} u_kj x(row j)) / u_kk, k from the last pivot
    // down; the pivots' x rows are first + k, written by this thread
    for (int k = nc - 1; k >= 0; --k) {
      const T* urow = U + (size_t)(uo + (long long)k * fs) * Bp + b;
      T s = Y[(size_t)(first + k) * Bp + b];
      for (int j = k + 1; j < fs; ++j) s -= urow[(size_t)j * Bp] * X[(size_t)pl.front_rows[fr0 + j] * Bp + b];
      X[(size_t)(first + k) * Bp + b] = s / urow[(size_t)k * Bp];
    }
    return;
  }
  T* Xs = Us + (size_t)nc * fs * kWarp;  // [fs][32]
  // U rows: contiguous elements uo .. uo + nc * fs
  for (int t = lane; t < nc * fs * kPieces; t += kWarp) {
    const int e = t / kPieces, piece = t % kPieces;
    cp_async16(reinterpret_cast<unsigned char*>(Us + (size_t)e * kWarp) + piece * 16,
               reinterpret_cast<const unsigned char*>(U + (size_t)(uo + e) * Bp + col0) + piece * 16);
  }
  // x of the CB rows: lane j fetches row front_rows[fr0 + nc + j]
  for (int j = lane; j < uc; j += kWarp) {
    const size_t row = (size_t)pl.front_rows[fr0 + nc + j];
#pragma unroll
    for (int piece = 0; piece < kPieces; ++piece)
      cp_async16(reinterpret_cast<unsigned char*>(Xs + (size_t)(nc + j) * kWarp) + piece * 16,
                 reinterpret_cast<const unsigned char*>(X + row * Bp + col0) + piece * 16);
  }
  cp_async_commit();
  T yk[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) yk[k] = k < nc ? Y[(size_t)(first + k) * Bp + b] : T(0);
  cp_async_wait<0>();
  __syncwarp();
#pragma unroll
  for (int k = 7; k >= 0; --k) {
    if (k < nc) {
      const T* urow = Us + (size_t)k * fs * kWarp + lane;
      T s = yk[k];
      for (int j = k + 1; j < fs; ++j) s -= urow[(size_t)j * kWarp] * Xs[(size_t)j * kWarp + lane];
      const T xk = s / urow[(size_t)k * kWarp];
      Xs[(size_t)k * kWarp + lane] = xk;
      X[(size_t)(first + k) * Bp + b] = xk;
    }
  }
  __syncwarp();  // the staging area is reused by the warp's next front
}

template <typename T, bool STAGED = true>
__global__ void __launch_bounds__(256)
    k_backward_level(DevPlan pl, int level_begin, int level_count, int groups, int Bp, int warp_elems,
                     const T* __restrict__ U, const T* __restrict__ Y, T* __restrict__ X) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5;
  const long item = (long)blockIdx.x * (blockDim.x >> 5) + warp;
  if (item >= (long)level_count * groups) return;
  const int q = level_begin + (int)(item / groups);
  const size_t col0 = (size_t)(item % groups) * kWarp;
  chain_allow_next();
  const FrontMeta m = load_front_meta(pl.front_meta, q);  // (plan data: before the wait)
  chain_wait_previous();  // U, Y and the x of ancestors come from earlier kernels
  T* Us = reinterpret_cast<T*>(smem_raw) + (size_t)warp * warp_elems * kWarp;  // [nc * fs][32]
  backward_front<T, STAGED>(pl, m, col0, Bp, Us, U, Y, X);
}

// The narrow top of the tree in one launch: block = one group of 32
// scenarios, walking the levels from the root down; the warps of the block
// share out each level's fronts and meet at a block barrier between levels
// (the x a front reads come from its ancestors, written by this block).
// lv_lo[t] .. lv_lo[t + 1]: level-order fronts of the t-th level from the
// root (descending boundaries, nlev + 1 entries).
template <typename T, bool STAGED = true>
__global__ void __launch_bounds__(256)
    k_backward_top(DevPlan pl, const int* __restrict__ lv_bounds, int nlev, int Bp, int warp_elems,
                   const T* __restrict__ U, const T* __restrict__ Y, T* __restrict__ X) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const size_t col0 = (size_t)blockIdx.x * kWarp;
  chain_allow_next();
  chain_wait_previous();
  T* Us = reinterpret_cast<T*>(smem_raw) + (size_t)warp * warp_elems * kWarp;
  for (int t = 0; t < nlev; ++t) {
    const int hi = lv_bounds[t], lo = lv_bounds[t + 1];
    for (int q = lo + warp; q < hi; q += W)
      backward_front<T, STAGED>(pl, load_front_meta(pl.front_meta, q), col0, Bp, Us, U, Y, X);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Triangular sweeps for right-hand sides given after factorization: the
// standalone forward substitution and the two adjoint sweeps.  One block per
// (front, 32 scenarios), one launch per level, chained.  The block's warps
// split the front's rows: two on wide levels, up to 8 on the narrow top of the
// tree, so the latency of a large front's loads is spread over more warps.
//
// Children's update vectors are gathered into a front's rows (extend-add)
// from one list per front, sorted by row: each entry holds its absolute
// update-vector element (crow_src) and its row in the front (crow_dst).  A
// warp gathers its rows [r0, r1): the lanes fetch 32 list entries in one
// request, the values of 8 entries are requested together, and each row's
// entries are summed in list order into ts[row * 32] (ts: this lane's column
// of the block's [fs][32] area in shared memory; rows without entries get 0).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void gather_child_updates(const DevPlan& pl, int fr0, int r0, int r1, size_t b, int Bp,
                                                     const T* __restrict__ TV, T* __restrict__ ts) {
  const int lane = threadIdx.x & 31;
  for (int i = r0; i < r1; ++i) ts[i * kWarp] = T(0);
  const int e0 = pl.crow_ptr[fr0 + r0], e1 = pl.crow_ptr[fr0 + r1];
  int cur = -1;
  T acc = T(0);
  for (int c = e0; c < e1; c += kWarp) {
    const int n = min(kWarp, e1 - c);
    long long src = 0;
    int dst = -1;
    if (lane < n) {
      src = pl.crow_src[c + lane];
      dst = pl.crow_dst[c + lane];
    }
    for (int u0 = 0; u0 < n; u0 += 8) {  // u0 + u <= 31
      T v[8];
      int d[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const long long sv = __shfl_sync(0xffffffffu, src, u0 + u);
        d[u] = __shfl_sync(0xffffffffu, dst, u0 + u);
        v[u] = d[u] >= 0 ? TV[(size_t)sv * Bp + b] : T(0);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
        if (d[u] >= 0) {
          if (d[u] != cur) {
            if (cur >= 0) ts[cur * kWarp] = acc;
            cur = d[u];
            acc = T(0);
          }
          acc += v[u];
        }
    }
  }
  if (cur >= 0) ts[cur * kWarp] = acc;
}

// A sweep block's item: front p of the level, scenario b of this lane.
struct SweepItem {
  int p, fs, nc, fr0, first;
  size_t b;
};

__device__ __forceinline__ SweepItem sweep_item(const DevPlan& pl, int level_begin, int groups) {
  SweepItem it;
  it.p = pl.level_fronts[level_begin + blockIdx.x / groups];
  it.b = (size_t)(blockIdx.x % groups) * kWarp + (threadIdx.x & 31);
  it.fs = pl.fsz[it.p];
  it.nc = pl.nc[it.p];
  it.fr0 = pl.front_ptr[it.p];
  it.first = pl.first[it.p];
  return it;
}

// Standalone forward substitution L y = P b (leaves first), for a right-hand
// side supplied after factorization (linear-solver boundary).  A front gathers
// its children's update vectors (extend-add of sum_m L21[.][m] y_m), solves its
// unit-lower pivot block and emits its own update vector.
// Shared memory: [fs_cap][32] gathered rows, [8][32] pivot values.
template <typename T, int NCMAX>
__global__ void __launch_bounds__(256)
    k_l_forward_level(DevPlan pl, int level_begin, int groups, int Bp, int fs_cap, const T* __restrict__ U,
                      const T* __restrict__ L, const double* __restrict__ G, T* __restrict__ TV,
                      T* __restrict__ Yo) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  chain_allow_next();
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const SweepItem it = sweep_item(pl, level_begin, groups);
  const int fs = it.fs, nc = it.nc;
  const size_t b = it.b;
  const long long uo = pl.u_off[it.p], lo = pl.l_off[it.p], to = pl.tv_off[it.p];
  T* ts = reinterpret_cast<T*>(smem_raw) + (threadIdx.x & 31);
  T* ys = ts + (size_t)fs_cap * kWarp;
  chain_wait_previous();
  gather_child_updates(pl, it.fr0, warp * fs / W, (warp + 1) * fs / W, b, Bp, TV, ts);
  __syncthreads();
  if (warp == 0) {
    T y[NCMAX];
#pragma unroll
    for (int k = 0; k < NCMAX; ++k) {
      y[k] = T(0);
      if (k < nc) {
        T s = static_cast<T>(G[(size_t)pl.perm[it.first + k] * Bp + b]) - ts[k * kWarp];
#pragma unroll
        for (int m = 0; m < k; ++m) s -= U[(size_t)(uo + (long long)k * fs + m) * Bp + b] * y[m];
        y[k] = s;
        ys[k * kWarp] = s;
        Yo[(size_t)(it.first + k) * Bp + b] = s;
      }
    }
  }
  __syncthreads();
  T y[NCMAX];
#pragma unroll
  for (int m = 0; m < NCMAX; ++m) y[m] = m < nc ? ys[m * kWarp] : T(0);
#pragma unroll 4
  for (int j = nc + warp; j < fs; j += W) {
    T s = ts[j * kWarp];
#pragma unroll
    for (int m = 0; m < NCMAX; ++m)
      if (m < nc) s += L[(size_t)(lo + (long long)(j - nc) * nc + m) * Bp + b] * y[m];
    TV[(size_t)(to + (j - nc)) * Bp + b] = s;
  }
}

// ---------------------------------------------------------------------------
// Adjoint sweeps.  With P J P^T = L U, J^T lambda = g becomes
//   U^T w = P g (leaves first) and L^T z = w (root first), lambda = P^T z.
// U^T forward: a front gathers its children's update vectors t (extend-add of
// sum_m U12[m][.] w_m), solves its pivots and emits its own t for the parent.
// Shared memory: [fs_cap][32] gathered rows, [8][32] pivot values.
// ---------------------------------------------------------------------------
template <typename T, int NCMAX>
__global__ void __launch_bounds__(256)
    k_ut_forward_level(DevPlan pl, int level_begin, int groups, int Bp, int fs_cap, const T* __restrict__ U,
                       const double* __restrict__ G, T* __restrict__ TV, T* __restrict__ Wv) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  chain_allow_next();
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const SweepItem it = sweep_item(pl, level_begin, groups);
  const int fs = it.fs, nc = it.nc;
  const size_t b = it.b;
  const long long uo = pl.u_off[it.p], to = pl.tv_off[it.p];
  T* ts = reinterpret_cast<T*>(smem_raw) + (threadIdx.x & 31);
  T* wsm = ts + (size_t)fs_cap * kWarp;
  chain_wait_previous();
  gather_child_updates(pl, it.fr0, warp * fs / W, (warp + 1) * fs / W, b, Bp, TV, ts);
  __syncthreads();
  if (warp == 0) {
    T w[NCMAX];
#pragma unroll
    for (int k = 0; k < NCMAX; ++k) {
      w[k] = T(0);
      if (k < nc) {
        // J^T's right-hand side is indexed by Jacobian columns
        T s = static_cast<T>(G[(size_t)pl.col_perm[it.first + k] * Bp + b]) - ts[k * kWarp];
#pragma unroll
        for (int m = 0; m < k; ++m) s -= U[(size_t)(uo + (long long)m * fs + k) * Bp + b] * w[m];
        w[k] = s / U[(size_t)(uo + (long long)k * fs + k) * Bp + b];
        wsm[k * kWarp] = w[k];
        Wv[(size_t)(it.first + k) * Bp + b] = w[k];
      }
    }
  }
  __syncthreads();
  T w[NCMAX];
#pragma unroll
  for (int m = 0; m < NCMAX; ++m) w[m] = m < nc ? wsm[m * kWarp] : T(0);
#pragma unroll 4
  for (int j = nc + warp; j < fs; j += W) {
    T s = ts[j * kWarp];
#pragma unroll
    for (int m = 0; m < NCMAX; ++m)
      if (m < nc) s += U[(size_t)(uo + (long long)m * fs + j) * Bp + b] * w[m];
    TV[(size_t)(to + (j - nc)) * Bp + b] = s;
  }
}

// L^T backward: z_k = w_k - sum_{m>k} L11[m][k] z_m - sum_jj L21[jj][k] z(row jj).
// The warps split the non-pivot rows jj (ancestors' z, from earlier launches)
// and each sums its rows' L21 terms for every k; warp 0 then solves the pivot
// block with those partial sums (shared memory [W][8][32]).
template <typename T, int NCMAX>
__global__ void __launch_bounds__(256)
    k_lt_backward_level(DevPlan pl, int level_begin, int groups, int Bp, const T* __restrict__ U,
                        const T* __restrict__ L, const T* __restrict__ Wv, T* __restrict__ Z) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  chain_allow_next();
  const int W = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const SweepItem it = sweep_item(pl, level_begin, groups);
  const int fs = it.fs, nc = it.nc;
  const size_t b = it.b;
  const long long uo = pl.u_off[it.p], lo = pl.l_off[it.p];
  T* ps = reinterpret_cast<T*>(smem_raw) + (threadIdx.x & 31);
  chain_wait_previous();
  T acc[NCMAX];
#pragma unroll
  for (int k = 0; k < NCMAX; ++k) acc[k] = T(0);
#pragma unroll 2
  for (int j = nc + warp; j < fs; j += W) {
    const T zj = Z[(size_t)pl.front_rows[it.fr0 + j] * Bp + b];
#pragma unroll
    for (int k = 0; k < NCMAX; ++k)
      if (k < nc) acc[k] += L[(size_t)(lo + (long long)(j - nc) * nc + k) * Bp + b] * zj;
  }
#pragma unroll
  for (int k = 0; k < NCMAX; ++k) ps[(warp * NCMAX + k) * kWarp] = acc[k];
  __syncthreads();
  if (warp == 0) {
    T z[NCMAX];
#pragma unroll
    for (int k = NCMAX - 1; k >= 0; --k) {
      z[k] = T(0);
      if (k < nc) {
        T s = Wv[(size_t)(it.first + k) * Bp + b];
#pragma unroll
        for (int m = k + 1; m < NCMAX; ++m)
          if (m < nc) s -= U[(size_t)(uo + (long long)m * fs + k) * Bp + b] * z[m];
        for (int w = 0; w < W; ++w) s -= ps[(w * NCMAX + k) * kWarp];
        z[k] = s;
        Z[(size_t)(it.first + k) * Bp + b] = s;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Sweep launches.
// ---------------------------------------------------------------------------
// Warps per block of a sweep launch: two where the level has many items
// (fronts x scenario groups; at most 32 blocks are resident on an SM, so one
// warp per block would leave half of its warp slots empty), up to 8 on the
// narrow levels.
inline int sweep_warps(long items) {
  if (items >= 512) return 2;
  if (items >= 128) return 4;
  return 8;
}

template <typename... KArgs, typename... Args>
void launch_sweep(void (*kern)(KArgs...), long items, int warps, size_t smem, cudaStream_t s, const char* what,
                  Args&&... args) {
  if (smem > kSmemLimit) throw std::runtime_error(std::string(what) + ": front too large for shared memory");
  allow_full_smem(reinterpret_cast<const void*>(kern));
  launch_chained(kern, dim3((unsigned)items), dim3(warps * kWarp), smem, s, what, std::forward<Args>(args)...);
}

}  // namespace

template <typename T, typename TJ, int FMAX>
void launch_factor_t(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s) {
  const int fmax = lv.max_fsz;
  const size_t elems = (size_t)fmax * (fmax + 1);
  const bool in_smem = front_in_shared_memory(lv, sizeof(T));
  FrontSmem sm = plan_front_smem(lv, sizeof(T), in_smem);
  if (!in_smem) {
    if (sm.total() > kSmemLimit) throw std::runtime_error("factor level: source staging exceeds shared memory");
    if (!a.front_scratch || a.front_scratch_elems < elems * (size_t)lv.count * a.groups)
      throw std::runtime_error("front larger than the shared-memory budget and no scratch area provided");
  }
  const long items = (long)lv.count * a.groups;
  // latency-bound levels (few fronts): every warp of the block helps.  Wide
  // levels are limited by the shared memory of the dense fronts (a handful
  // of blocks per SM), not by warps, so even small fronts get two warps: the
  // assembly and the non-pivot rows split between them (measured on the
  // 2,000-bus grid: 0.624 ms per factorization against 0.663 ms with one warp
  // for fronts of at most 10 rows; eight warps: 0.891 ms)
  int warps = fmax <= 16 ? 2 : (fmax <= 24 ? 4 : 8);
  if (items < 4L * 148) warps = 8;
  if (lv.warps > 0) warps = std::min(lv.warps, 8);  // chosen by the engine's autotuner (the wide tier's 16 and 32
                                                   // warps are not register-kernel shapes)
  const size_t smem = sm.total();
  auto run = [&](auto kern) {
    allow_full_smem(reinterpret_cast<const void*>(kern));
    launch_chained(kern, dim3((unsigned)items), dim3(warps * kWarp), smem, s, "front factor", a.plan, lv.begin,
                   lv.fe_base, lv.max_src, a.groups, a.Bp, (int)elems, sm, a.J, a.Fp, a.U, a.L, a.CB, a.Y, a.store_l, a.eps, a.static_pivot,
                   a.sing, a.front_scratch);
  };
  if (in_smem) run(k_front_factor<T, TJ, FMAX, true>);
  else run(k_front_factor<T, TJ, FMAX, false>);
}

// Opt every front kernel of this precision into the full dynamic shared
// memory up front (outside any stream capture).
template <typename T, typename TJ>
void configure_front_kernels() {
  allow_full_smem(reinterpret_cast<const void*>(k_backward_level<T>));
  allow_full_smem(reinterpret_cast<const void*>(k_backward_top<T>));
#define CUPF_ALLOW(F)                                                                  \
  allow_full_smem(reinterpret_cast<const void*>(k_front_factor<T, TJ, F, true>));    \
  allow_full_smem(reinterpret_cast<const void*>(k_front_factor<T, TJ, F, false>));
  CUPF_ALLOW(8) CUPF_ALLOW(12) CUPF_ALLOW(16) CUPF_ALLOW(20) CUPF_ALLOW(24) CUPF_ALLOW(32) CUPF_ALLOW(48)
  CUPF_ALLOW(64)
#undef CUPF_ALLOW
  allow_full_smem(reinterpret_cast<const void*>(k_front_factor_wide<T, TJ, 8>));
  allow_full_smem(reinterpret_cast<const void*>(k_front_factor_wide<T, TJ, 16>));
  allow_full_smem(reinterpret_cast<const void*>(k_front_factor_wide<T, TJ, 32>));
  if constexpr (std::is_same<T, float>::value) allow_full_smem(reinterpret_cast<const void*>(k_front_factor_tc));
}

// A wide-tier launch: one block per front x 32 scenarios, 8 to 32 warps
// (the rule below unless the autotuner chose), dense fronts in the global
// scratch.
template <typename T, typename TJ>
void launch_factor_wide(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s) {
  const FrontSmem sm = plan_wide_smem(lv, sizeof(T));
  if (sm.total() > kSmemLimit) throw std::runtime_error("wide front tier: staging exceeds shared memory");
  const size_t per_block = wide_block_elems(lv, sizeof(T));
  const long items = (long)lv.count * a.groups;
  if (!a.front_scratch || a.front_scratch_elems < per_block * (size_t)items)
    throw std::runtime_error("wide front tier: the front scratch area is missing or too small");
  if (per_block > (size_t)INT32_MAX) throw std::runtime_error("wide front tier: front too large");
  // built-in rule: the fewer the blocks, the more warps share a front (a
  // launch of at most one block per SM gets 32)
  const int rule = items <= 148 ? 32 : items <= 4 * 148 ? 16 : 8;
  const int warps = lv.warps > 0 ? std::min(lv.warps, 32) : rule;
  auto run = [&](auto kern) {
    allow_full_smem(reinterpret_cast<const void*>(kern));
    launch_chained(kern, dim3((unsigned)items), dim3(warps * kWarp), sm.total(), s, "front factor (wide tier)",
                   a.plan, lv.begin, lv.fe_base, lv.max_src, a.groups, a.Bp, (int)per_block, sm, a.J, a.Fp, a.U, a.L,
                   a.CB, a.Y, a.store_l, a.eps, a.static_pivot, a.sing, a.front_scratch);
  };
  // more than 8 warps split each assembly range at destination changes,
  // which needs a multiple of 8
  if (warps > 8 && warps % 8) throw std::runtime_error("wide front tier: more than 8 warps must be a multiple of 8");
  if (warps <= 8) run(k_front_factor_wide<T, TJ, 8>);
  else if (warps <= 16) run(k_front_factor_wide<T, TJ, 16>);
  else run(k_front_factor_wide<T, TJ, 32>);
}

inline size_t single_front_bytes(const LevelLaunch& lv, size_t elem_bytes) {
  return single_smem_bytes(lv.max_fsz, lv.max_src, elem_bytes);
}

// One block per front of the launch; 64 threads for fronts of up to 12 rows,
// 128 up to 24, else 256 (the trailing update has about fs^2 / 2 elements).
template <typename T, typename TJ>
void launch_factor_single(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s) {
  const size_t smem = single_front_bytes(lv, sizeof(T));
  auto kern = k_front_factor_single<T, TJ>;
  allow_full_smem(reinterpret_cast<const void*>(kern));
  const int threads = lv.max_fsz <= 12 ? 64 : lv.max_fsz <= 24 ? 128 : 256;
  launch_chained(kern, dim3((unsigned)lv.count), dim3(threads), smem, s, "front factor (single system)", a.plan,
                 lv.begin, lv.fe_base, lv.max_src, a.Bp, a.J, a.Fp, a.U, a.L, a.CB, a.Y, a.store_l, a.eps,
                 a.static_pivot, a.sing);
}

// The whole single-system factorization as one launch (k_factor_single_tree):
// persistent blocks of 128 threads, at most 8 per SM's worth.
template <typename T, typename TJ>
void launch_factor_single_tree(const FactorArgs<T, TJ>& a, const SingleTree& t, cudaStream_t s) {
  const size_t smem = single_smem_bytes(t.max_fsz, t.list_cap, sizeof(T));
  if (smem > kSmemLimit) throw std::runtime_error("single-system tree: a front exceeds shared memory");
  auto kern = k_factor_single_tree<T, TJ>;
  allow_full_smem(reinterpret_cast<const void*>(kern));
  const int blocks = std::max(1, std::min(t.n_leaves, 148 * 8));
  launch_chained(kern, dim3((unsigned)blocks), dim3(128), smem, s, "front factor (single-system tree)", a.plan,
                 t.parent, t.nchild, t.q_e0, t.leaves, t.n_leaves, t.done, t.done + t.P, t.list_cap, a.Bp, a.J,
                 a.Fp, a.U, a.L, a.CB, a.Y, a.store_l, a.eps, a.static_pivot, a.sing);
}

// A tensor-core launch (FP32 factors): 4 or 8 warps (every TMEM lane
// quarter needs its warp); falls back to the FP32 wide tier where the fronts
// exceed its limits.
template <typename T, typename TJ>
void launch_factor_tc(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s) {
  if constexpr (!std::is_same<T, float>::value || !std::is_same<TJ, float>::value) {
    launch_factor_wide<T, TJ>(lv, a, s);  // the tensor-core tier is built for FP32 factors
  } else {
    FrontSmem sm;
    TcLayout tl;
    if (!plan_tc(lv, &sm, &tl)) {
      launch_factor_wide<T, TJ>(lv, a, s);
      return;
    }
    const int front_elems = lv.max_fsz * (lv.max_fsz + 1);
    const long items = (long)lv.count * a.groups;
    if (!a.front_scratch || a.front_scratch_elems < (size_t)front_elems * (size_t)items)
      throw std::runtime_error("tensor-core front tier: the front scratch area is missing or too small");
    const int warps = lv.warps >= 8 || lv.warps == 0 ? 8 : 4;
    allow_full_smem(reinterpret_cast<const void*>(k_front_factor_tc));
    launch_chained(k_front_factor_tc, dim3((unsigned)items), dim3(warps * kWarp), (size_t)tl.total, s,
                   "front factor (tensor-core tier)", a.plan, lv.begin, lv.fe_base, lv.max_src, a.groups, a.Bp,
                   front_elems, sm, tl, a.J, a.Fp, a.U, a.L, a.CB, a.Y, a.store_l, a.eps, a.static_pivot, a.sing,
                   a.front_scratch, tc::kSpinLimit);
  }
}

template <typename T, typename TJ>
void launch_factor_level(const LevelLaunch& lv, const FactorArgs<T, TJ>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc > 8) throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  if (a.single && lv.tier != 2 && single_front_bytes(lv, sizeof(T)) <= kSmemLimit) {
    launch_factor_single<T, TJ>(lv, a, s);  // batch 1 (the tensor-core tier keeps its own kernel)
    return;
  }
  if (lv.tier == 2) {
    launch_factor_tc<T, TJ>(lv, a, s);
    return;
  }
  if (runs_wide(lv, sizeof(T))) {
    launch_factor_wide<T, TJ>(lv, a, s);
    return;
  }
  const int f = lv.max_fsz;
  if (f <= 8) launch_factor_t<T, TJ, 8>(lv, a, s);
  else if (f <= 12) launch_factor_t<T, TJ, 12>(lv, a, s);
  else if (f <= 16) launch_factor_t<T, TJ, 16>(lv, a, s);
  else if (f <= 20) launch_factor_t<T, TJ, 20>(lv, a, s);
  else if (f <= 24) launch_factor_t<T, TJ, 24>(lv, a, s);
  else if (f <= 32) launch_factor_t<T, TJ, 32>(lv, a, s);
  else if (f <= 48) launch_factor_t<T, TJ, 48>(lv, a, s);
  else launch_factor_t<T, TJ, 64>(lv, a, s);
}

template <typename T>
void launch_backward_level(const LevelLaunch& lv, const SweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc > 8) throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  const int warp_elems = lv.max_nc * lv.max_fsz + lv.max_fsz;
  const size_t per_warp = (size_t)warp_elems * kWarp * sizeof(T);
  const long items = (long)lv.count * a.groups;
  if (per_warp > kSmemLimit) {  // U rows too large to stage: read them from global memory
    const int w = lv.bw_wpb > 0 ? lv.bw_wpb : 4;
    launch_chained(k_backward_level<T, false>, dim3((unsigned)((items + w - 1) / w)), dim3(w * kWarp), 0, s,
                   "backward sweep", a.plan, lv.begin, lv.count, a.groups, a.Bp, warp_elems, a.U, a.Y, a.X);
    return;
  }
  int wpb = (int)std::min<size_t>(8, kSmemLimit / per_warp);
  const int cap = wpb;
  wpb = (int)std::min<long>(wpb, std::max<long>(1, items / 148));
  wpb = std::max(1, std::min(wpb, 4));
  if (lv.bw_wpb > 0) wpb = std::min(lv.bw_wpb, cap);  // chosen by the engine's autotuner
  const size_t smem = per_warp * wpb;
  auto kern = k_backward_level<T>;
  allow_full_smem(reinterpret_cast<const void*>(kern));
  const unsigned blocks = (unsigned)((items + wpb - 1) / wpb);
  launch_chained(kern, dim3(blocks), dim3(wpb * kWarp), smem, s, "backward sweep", a.plan, lv.begin, lv.count,
                 a.groups, a.Bp, warp_elems, a.U, a.Y, a.X);
}

// The top levels [top.begin, top.begin + top.count) of the launch list given
// by lv_bounds (device, descending level boundaries, nlev + 1 entries).
template <typename T>
void launch_backward_top(const LevelLaunch& top, const int* lv_bounds, int nlev, const SweepArgs<T>& a,
                         cudaStream_t s) {
  if (top.count == 0 || nlev == 0) return;
  const int warp_elems = top.max_nc * top.max_fsz + top.max_fsz;
  const size_t per_warp = (size_t)warp_elems * kWarp * sizeof(T);
  if (per_warp > kSmemLimit) {  // U rows too large to stage: read them from global memory
    const int w = top.bw_wpb > 0 ? top.bw_wpb : 4;
    launch_chained(k_backward_top<T, false>, dim3((unsigned)a.groups), dim3(w * kWarp), 0, s,
                   "backward sweep (tree top)", a.plan, lv_bounds, nlev, a.Bp, warp_elems, a.U, a.Y, a.X);
    return;
  }
  const int cap = (int)std::min<size_t>(8, kSmemLimit / per_warp);
  const int wpb = top.bw_wpb > 0 ? std::min(top.bw_wpb, cap) : std::min(4, cap);
  auto kern = k_backward_top<T>;
  allow_full_smem(reinterpret_cast<const void*>(kern));
  launch_chained(kern, dim3((unsigned)a.groups), dim3(wpb * kWarp), per_warp * wpb, s, "backward sweep (tree top)",
                 a.plan, lv_bounds, nlev, a.Bp, warp_elems, a.U, a.Y, a.X);
}

template <typename T>
void launch_ut_forward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc > 8) throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  const long items = (long)lv.count * a.groups;
  launch_sweep(k_ut_forward_level<T, 8>, items, sweep_warps(items), (size_t)(lv.max_fsz + 8) * kWarp * sizeof(T), s,
               "adjoint sweep (U^T)", a.plan, lv.begin, a.groups, a.Bp, lv.max_fsz, a.U, a.G, a.TV, a.W);
}

template <typename T>
void launch_l_forward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc > 8) throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  const long items = (long)lv.count * a.groups;
  launch_sweep(k_l_forward_level<T, 8>, items, sweep_warps(items), (size_t)(lv.max_fsz + 8) * kWarp * sizeof(T), s,
               "forward substitution", a.plan, lv.begin, a.groups, a.Bp, lv.max_fsz, a.U, a.L, a.G, a.TV, a.W);
}

template <typename T>
void launch_lt_backward_level(const LevelLaunch& lv, const AdjointSweepArgs<T>& a, cudaStream_t s) {
  if (lv.count == 0) return;
  if (lv.max_nc > 8) throw std::runtime_error("panels wider than 8 columns are not supported (max_panel_width <= 8)");
  const long items = (long)lv.count * a.groups;
  const int warps = sweep_warps(items);
  launch_sweep(k_lt_backward_level<T, 8>, items, warps, (size_t)warps * 8 * kWarp * sizeof(T), s,
               "adjoint sweep (L^T)", a.plan, lv.begin, a.groups, a.Bp, a.U, a.L, a.W, a.Z);
}

}  // namespace cupf_b200
