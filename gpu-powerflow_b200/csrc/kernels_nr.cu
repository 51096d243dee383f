// kernels_nr.cu -- element-wise stages of one Newton-Raphson iteration and
// the host<->engine layout conversions.
//
// All per-scenario state is [element][Bp] with the scenario innermost: a warp
// covers 32 scenarios of one bus or one Ybus entry, so Ybus values and map
// indices are warp-uniform broadcasts and the state accesses are coalesced.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "device_plan.cuh"
#include "kernels.hpp"

namespace cupf_b200 {
namespace {

constexpr int kRows = 8;  // warps per block in the (lane, row) kernels

__device__ __forceinline__ double dmax_nan(double m, double a, bool& bad) {
  if (!(a == a) || a > 1.7976931348623157e308) bad = true;
  return a > m ? a : m;
}

// The state arrays of a DevState in their element type S: double under the
// FP64 and Mixed compute policies, float under ComputePolicy::FP32 (the
// reference's CudaFp32Storage: V, Sbus, Ibus and F all single precision,
// newton_solver_types.hpp:67-80).
template <typename S>
struct StateArrays {
  S *v_re, *v_im, *va, *vm, *s_re, *s_im, *i_re, *i_im, *F;
  __device__ __forceinline__ explicit StateArrays(const DevState& st)
      : v_re(reinterpret_cast<S*>(st.v_re)), v_im(reinterpret_cast<S*>(st.v_im)), va(reinterpret_cast<S*>(st.va)),
        vm(reinterpret_cast<S*>(st.vm)), s_re(reinterpret_cast<S*>(st.s_re)), s_im(reinterpret_cast<S*>(st.s_im)),
        i_re(reinterpret_cast<S*>(st.i_re)), i_im(reinterpret_cast<S*>(st.i_im)), F(reinterpret_cast<S*>(st.F)) {}
};

__device__ __forceinline__ void sin_cos(double a, double* s, double* c) { sincos(a, s, c); }
__device__ __forceinline__ void sin_cos(float a, float* s, float* c) { sincosf(a, s, c); }

// ---------------------------------------------------------------------------
// Ibus = Ybus V, F = [Re mis@pv, Re mis@pq, Im mis@pq] with mis = V conj(I) - S,
// and per-scenario ||F||_inf (cuPF compute_ibus.cu:58-95,
// compute_mismatch_from_ibus.cu:32-85, reduce_mismatch_norm.cu:49-119 fused).
// The norm is an atomicMax on the IEEE bits of |F| (order preserving for
// non-negative doubles); a non-finite entry forces NaN bits.  S is the
// state's type: under ComputePolicy::FP32 the Ybus values are rounded to
// float and Ibus and F are computed in float (compute_ibus.cu with
// CudaFp32Storage); the norm of the float entries is exact in double.
// F goes out in pivot order and the factor's type (Fp, the LU's right-hand
// side); the Jacobian-row-order copy st.F is written only when it is set
// (evaluate), since the Newton loop never reads it.
// ---------------------------------------------------------------------------
template <typename S>
__global__ void k_ibus_mismatch(DevGrid g, DevState st) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int Bp = st.Bp;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  const StateArrays<S> v(st);
  double nmax = 0.0;
  bool bad = false;
  // Ybus value of entry k: shared y[k], or this scenario's yb[k * Bp + b]
  const double* yre = st.yb_re ? st.yb_re + b : g.y_re;
  const double* yim = st.yb_re ? st.yb_im + b : g.y_im;
  const size_t ys = st.yb_re ? (size_t)Bp : 1;
  for (int i = blockIdx.x * kRows + wy; i < g.n_bus; i += gridDim.x * kRows) {
    S ir = S(0), ii = S(0);
    for (int k = g.y_ptr[i]; k < g.y_ptr[i + 1]; ++k) {
      const size_t c = (size_t)g.y_col[k] * Bp + b;
      const S yr = static_cast<S>(yre[k * ys]), yi = static_cast<S>(yim[k * ys]);
      const S vr = v.v_re[c], vi = v.v_im[c];
      ir += yr * vr - yi * vi;
      ii += yr * vi + yi * vr;
    }
    const size_t o = (size_t)i * Bp + b;
    v.i_re[o] = ir;
    v.i_im[o] = ii;
    const S vr = v.v_re[o], vi = v.v_im[o];
    const S mr = (vr * ir + vi * ii) - v.s_re[o];
    const S mi = (vi * ir - vr * ii) - v.s_im[o];
    const int fa = g.bus_fa[i], fm = g.bus_fm[i];
    if (fa >= 0) {
      if (v.F) v.F[(size_t)fa * Bp + b] = mr;
      nmax = dmax_nan(nmax, fabs(static_cast<double>(mr)), bad);
    }
    if (fm >= 0) {
      if (v.F) v.F[(size_t)fm * Bp + b] = mi;
      nmax = dmax_nan(nmax, fabs(static_cast<double>(mi)), bad);
    }
    if (st.Fp) {
      const int pa = g.bus_fa_p[i], pm = g.bus_fm_p[i];
      if (st.fp_double) {
        if (pa >= 0) static_cast<double*>(st.Fp)[(size_t)pa * Bp + b] = mr;
        if (pm >= 0) static_cast<double*>(st.Fp)[(size_t)pm * Bp + b] = mi;
      } else {
        if (pa >= 0) static_cast<float*>(st.Fp)[(size_t)pa * Bp + b] = static_cast<float>(mr);
        if (pm >= 0) static_cast<float*>(st.Fp)[(size_t)pm * Bp + b] = static_cast<float>(mi);
      }
    }
  }
  __shared__ double red[kRows][kWarp];
  __shared__ int redbad[kRows][kWarp];
  red[wy][lane] = nmax;
  redbad[wy][lane] = bad ? 1 : 0;
  __syncthreads();
  if (wy == 0) {
    double m = red[0][lane];
    int anybad = redbad[0][lane];
    for (int r = 1; r < kRows; ++r) {
      m = red[r][lane] > m ? red[r][lane] : m;
      anybad |= redbad[r][lane];
    }
    const unsigned long long bits =
        anybad ? 0x7FF8000000000000ull : (unsigned long long)__double_as_longlong(m);
    atomicMax(&st.norm_bits[b], bits);
  }
}

// ---------------------------------------------------------------------------
// Jacobian values into the fixed CSR pattern through the scatter maps
// (cuPF fill_jacobian_edge_kernel.hpp:30-197, jacobian_gpu_common.hpp:96-127):
//   off-diagonal  dS/dVa = -j V_i conj(y V_j),  dS/dVm = V_i conj(y V_j / |V_j|)
//   diagonal adds          j V_i conj(I_i)   and         conj(I_i) V_i / |V_i|
// J11/J21 take the real/imaginary parts of dS/dVa, J12/J22 of dS/dVm.  The
// diagonal terms are added by the thread of the Ybus diagonal entry, so every
// slot is written exactly once (no memset, no atomics).
// ---------------------------------------------------------------------------
template <typename S, typename TJ>
__global__ void k_jacobian(DevGrid g, DevState st, TJ* __restrict__ J) {
  // arithmetic in the Jacobian's own type, as the reference's fill does
  // (fill_jacobian_edge_kernel.hpp:58-60: AccumScalar = JScalar); the state
  // is read and rounded once
  using A = TJ;
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int Bp = st.Bp;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  const StateArrays<S> v(st);
  const double* yre = st.yb_re ? st.yb_re + b : g.y_re;
  const double* yim = st.yb_re ? st.yb_im + b : g.y_im;
  const size_t ys = st.yb_re ? (size_t)Bp : 1;
  for (int k = blockIdx.x * kRows + wy; k < g.nnz_y; k += gridDim.x * kRows) {
    const int i = g.y_row[k], c = g.y_col[k];
    const A yr = static_cast<A>(yre[k * ys]), yi = static_cast<A>(yim[k * ys]);
    const size_t oi = (size_t)i * Bp + b, oc = (size_t)c * Bp + b;
    const A vir = static_cast<A>(v.v_re[oi]), vii = static_cast<A>(v.v_im[oi]);
    const A vcr = static_cast<A>(v.v_re[oc]), vci = static_cast<A>(v.v_im[oc]);
    const A yvr = yr * vcr - yi * vci, yvi = yr * vci + yi * vcr;  // y V_c
    // -j V_i conj(y V_c)
    A var = vii * yvr - vir * yvi;
    A vai = -(vii * yvi + vir * yvr);
    // V_i conj(y V_c / |V_c|), with |V_c| the stored magnitude Vm_c (V is
    // built as Vm e^{j Va}, so they agree to rounding); one reciprocal
    A mc = static_cast<A>(v.vm[oc]);
    mc = mc < A(1e-8) ? A(1e-8) : mc;
    const A inv = A(1) / mc;
    const A ynr = yvr * inv, yni = yvi * inv;
    A vmr = vir * ynr + vii * yni;
    A vmi = vii * ynr - vir * yni;
    if (i == c) {
      const A ir = static_cast<A>(v.i_re[oi]), ii = static_cast<A>(v.i_im[oi]);
      // j V conj(I)
      var += -(vii * ir - vir * ii);
      vai += vir * ir + vii * ii;
      // conj(I) V / |V|
      const A nr = vir * inv, ni = vii * inv;
      vmr += ir * nr + ii * ni;
      vmi += ir * ni - ii * nr;
    }
    const int p11 = g.map11[k], p21 = g.map21[k], p12 = g.map12[k], p22 = g.map22[k];
    if (p11 >= 0) J[(size_t)p11 * Bp + b] = var;
    if (p21 >= 0) J[(size_t)p21 * Bp + b] = vai;
    if (p12 >= 0) J[(size_t)p12 * Bp + b] = vmr;
    if (p22 >= 0) J[(size_t)p22 * Bp + b] = vmi;
  }
}

// ---------------------------------------------------------------------------
// The two other fills of CudaJacobianKind (fill_jacobian_edge_atomic_kernel.hpp,
// fill_jacobian_vertex_warp_kernel.hpp).  Both build the diagonal from the
// edges instead of from Ibus:
//   dS_i/dVa_i = sum_{c != i} j V_i conj(y_ic V_c)            (= -sum of the off-diagonal angle terms)
//   dS_i/d|V_i| = sum_c conj(y_ic V_c) V_i / |V_i| + V_i conj(y_ii V_i / |V_i|)
// The off-diagonal entries are those of k_jacobian.
// ---------------------------------------------------------------------------
struct EdgeTerms {
  double var, vai, vmr, vmi;  // -j V_i conj(y V_c) and V_i conj(y V_c / |V_c|)
  double dmr, dmi;            // conj(y V_c) V_i / |V_i|
};

__device__ __forceinline__ EdgeTerms edge_terms(double yr, double yi, double vir, double vii, double vcr, double vci) {
  EdgeTerms t;
  const double yvr = yr * vcr - yi * vci, yvi = yr * vci + yi * vcr;
  t.var = vii * yvr - vir * yvi;
  t.vai = -(vii * yvi + vir * yvr);
  double mc = hypot(vcr, vci);
  mc = mc < 1e-8 ? 1e-8 : mc;
  const double ynr = yvr / mc, yni = yvi / mc;
  t.vmr = vir * ynr + vii * yni;
  t.vmi = vii * ynr - vir * yni;
  double mi = hypot(vir, vii);
  mi = mi < 1e-8 ? 1e-8 : mi;
  const double nr = vir / mi, ni = vii / mi;
  t.dmr = yvr * nr + yvi * ni;
  t.dmi = yvr * ni - yvi * nr;
  return t;
}

// Vertex fill: a warp takes one bus row for 32 scenarios and walks its Ybus
// entries, storing the off-diagonal slots and summing the diagonal in
// registers (each lane owns its scenario, so no reduction is needed).
template <typename S, typename TJ>
__global__ void k_jacobian_vertex(DevGrid g, DevState st, TJ* __restrict__ J) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int Bp = st.Bp;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  const StateArrays<S> v(st);
  const double* yre = st.yb_re ? st.yb_re + b : g.y_re;
  const double* yim = st.yb_re ? st.yb_im + b : g.y_im;
  const size_t ys = st.yb_re ? (size_t)Bp : 1;
  for (int i = blockIdx.x * kRows + wy; i < g.n_bus; i += gridDim.x * kRows) {
    const size_t oi = (size_t)i * Bp + b;
    const double vir = v.v_re[oi], vii = v.v_im[oi];
    double d11 = 0.0, d21 = 0.0, d12 = 0.0, d22 = 0.0;
    int kd = -1;
    for (int k = g.y_ptr[i]; k < g.y_ptr[i + 1]; ++k) {
      const int c = g.y_col[k];
      const size_t oc = (size_t)c * Bp + b;
      const EdgeTerms t = edge_terms(yre[k * ys], yim[k * ys], vir, vii, v.v_re[oc], v.v_im[oc]);
      d12 += t.dmr;
      d22 += t.dmi;
      if (c == i) {
        kd = k;
        d12 += t.vmr;
        d22 += t.vmi;
        continue;
      }
      d11 -= t.var;
      d21 -= t.vai;
      const int p11 = g.map11[k], p21 = g.map21[k], p12 = g.map12[k], p22 = g.map22[k];
      if (p11 >= 0) J[(size_t)p11 * Bp + b] = static_cast<TJ>(t.var);
      if (p21 >= 0) J[(size_t)p21 * Bp + b] = static_cast<TJ>(t.vai);
      if (p12 >= 0) J[(size_t)p12 * Bp + b] = static_cast<TJ>(t.vmr);
      if (p22 >= 0) J[(size_t)p22 * Bp + b] = static_cast<TJ>(t.vmi);
    }
    if (kd >= 0) {
      const int p11 = g.map11[kd], p21 = g.map21[kd], p12 = g.map12[kd], p22 = g.map22[kd];
      if (p11 >= 0) J[(size_t)p11 * Bp + b] = static_cast<TJ>(d11);
      if (p21 >= 0) J[(size_t)p21 * Bp + b] = static_cast<TJ>(d21);
      if (p12 >= 0) J[(size_t)p12 * Bp + b] = static_cast<TJ>(d12);
      if (p22 >= 0) J[(size_t)p22 * Bp + b] = static_cast<TJ>(d22);
    }
  }
}

// Edge fill with atomic diagonal accumulation: a warp takes one Ybus entry
// for 32 scenarios, stores its off-diagonal slots and adds its share of the
// row's diagonal with atomicAdd in the Jacobian's own type (the diagonal
// slots are zeroed first).  The summation order of the diagonal depends on
// scheduling, so results may differ in the last bits from run to run.
template <typename TJ>
__global__ void k_jacobian_zero_diag(DevGrid g, DevState st, TJ* __restrict__ J) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int Bp = st.Bp;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  for (int i = blockIdx.x * kRows + wy; i < g.n_bus; i += gridDim.x * kRows)
    for (int k = g.y_ptr[i]; k < g.y_ptr[i + 1]; ++k)
      if (g.y_col[k] == i) {
        const int p[4] = {g.map11[k], g.map21[k], g.map12[k], g.map22[k]};
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (p[q] >= 0) J[(size_t)p[q] * Bp + b] = TJ(0);
      }
}

template <typename S, typename TJ>
__global__ void k_jacobian_edge_atomic(DevGrid g, DevState st, TJ* __restrict__ J) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int Bp = st.Bp;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  const StateArrays<S> v(st);
  const double* yre = st.yb_re ? st.yb_re + b : g.y_re;
  const double* yim = st.yb_re ? st.yb_im + b : g.y_im;
  const size_t ys = st.yb_re ? (size_t)Bp : 1;
  for (int k = blockIdx.x * kRows + wy; k < g.nnz_y; k += gridDim.x * kRows) {
    const int i = g.y_row[k], c = g.y_col[k];
    const size_t oi = (size_t)i * Bp + b, oc = (size_t)c * Bp + b;
    const EdgeTerms t = edge_terms(yre[k * ys], yim[k * ys], v.v_re[oi], v.v_im[oi], v.v_re[oc], v.v_im[oc]);
    const int kd = g.y_diag[i];
    if (kd < 0) continue;
    const int q11 = g.map11[kd], q21 = g.map21[kd], q12 = g.map12[kd], q22 = g.map22[kd];
    double a12 = t.dmr, a22 = t.dmi;
    if (c == i) {
      a12 += t.vmr;
      a22 += t.vmi;
    } else {
      const int p11 = g.map11[k], p21 = g.map21[k], p12 = g.map12[k], p22 = g.map22[k];
      if (p11 >= 0) J[(size_t)p11 * Bp + b] = static_cast<TJ>(t.var);
      if (p21 >= 0) J[(size_t)p21 * Bp + b] = static_cast<TJ>(t.vai);
      if (p12 >= 0) J[(size_t)p12 * Bp + b] = static_cast<TJ>(t.vmr);
      if (p22 >= 0) J[(size_t)p22 * Bp + b] = static_cast<TJ>(t.vmi);
      if (q11 >= 0) atomicAdd(&J[(size_t)q11 * Bp + b], static_cast<TJ>(-t.var));
      if (q21 >= 0) atomicAdd(&J[(size_t)q21 * Bp + b], static_cast<TJ>(-t.vai));
    }
    if (q12 >= 0) atomicAdd(&J[(size_t)q12 * Bp + b], static_cast<TJ>(a12));
    if (q22 >= 0) atomicAdd(&J[(size_t)q22 * Bp + b], static_cast<TJ>(a22));
  }
}

// ---------------------------------------------------------------------------
// Va/Vm -= dx at the pv/pq rows, V = Vm (cos Va + j sin Va)
// (cuPF voltage_update_kernels.hpp:44-104).  dx is read from the permuted
// solution X (x_perm[iperm[row]]).  The bus-0 thread clears the scenario's
// norm for the next mismatch evaluation.
// ---------------------------------------------------------------------------
template <typename S, typename T>
__global__ void k_voltage_update(DevGrid g, DevPlan pl, DevState st, const T* __restrict__ X) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const int Bp = st.Bp;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  const StateArrays<S> v(st);
  for (int i = blockIdx.x * kRows + wy; i < g.n_bus; i += gridDim.x * kRows) {
    const size_t o = (size_t)i * Bp + b;
    S va = v.va[o], vm = v.vm[o];
    const int fa = g.bus_fa[i], fm = g.bus_fm[i];
    if (fa >= 0) va -= static_cast<S>(X[(size_t)pl.iperm[fa] * Bp + b]);
    if (fm >= 0) vm -= static_cast<S>(X[(size_t)pl.iperm[fm] * Bp + b]);
    S s, c;
    sin_cos(va, &s, &c);
    v.va[o] = va;
    v.vm[o] = vm;
    v.v_re[o] = vm * c;
    v.v_im[o] = vm * s;
    if (i == 0) st.norm_bits[b] = 0ull;
  }
}

// ---------------------------------------------------------------------------
// Layout conversions through a 32 x 32 shared tile: host arrays are
// scenario-major [B][stride], the engine is bus-major [n][Bp].
// Pad scenarios (B <= b < Bp) replicate scenario B - 1.
// ---------------------------------------------------------------------------
// Seed of a warm-started solve in one pass: Sbus as k_seed_state converts it,
// and the state from a prediction pred[b][row] in Jacobian-row order (fp32,
// un-standardized as pred * scale + shift when scale is given): Va at the
// angle rows of the PV and PQ buses, Vm at the magnitude rows of the PQ
// buses, V0's angle and magnitude where the prediction has no row, and V
// rebuilt from them (a bus the prediction does not touch keeps V0's value).
// The inputs are read along the buses (a warp reads 32 buses of one
// scenario, so the prediction's rows arrive in runs of consecutive columns)
// and transposed through shared memory to the bus-major state.
template <typename S>
__global__ void k_seed_warm(DevGrid g, DevState st, const double* __restrict__ sbus_c, long long sbus_stride,
                            const double* __restrict__ v0_c, long long v0_stride, const float* __restrict__ pred,
                            long long ld, const float* __restrict__ scale, const float* __restrict__ shift) {
  __shared__ double t[4][kWarp][kWarp + 1];  // s_re, s_im, va, vm
  const StateArrays<S> v(st);
  const int tx = threadIdx.x, ty = threadIdx.y;  // (32, 8)
  const int bus0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  const int bus = bus0 + tx;
  const int fa = bus < g.n_bus ? g.bus_fa[bus] : -1, fm = bus < g.n_bus ? g.bus_fm[bus] : -1;
  float sa = 1.f, ha = 0.f, sm = 1.f, hm = 0.f;
  if (scale) {
    if (fa >= 0) sa = scale[fa], ha = shift[fa];
    if (fm >= 0) sm = scale[fm], hm = shift[fm];
  }
  for (int r = ty; r < kWarp; r += kRows) {
    const long long bb = min(b0 + r, st.B - 1);
    if (bus < g.n_bus) {
      const size_t so = ((size_t)bb * sbus_stride + bus) * 2, vo = ((size_t)bb * v0_stride + bus) * 2;
      t[0][r][tx] = sbus_c[so];
      t[1][r][tx] = sbus_c[so + 1];
      const double vr = v0_c[vo], vi = v0_c[vo + 1];
      double va = 0.0, vm = 0.0;
      if (fa < 0) va = atan2(vi, vr);
      if (fm < 0) vm = hypot(vr, vi);
      if (fa >= 0) va = (double)(scale ? pred[bb * ld + fa] * sa + ha : pred[bb * ld + fa]);
      if (fm >= 0) vm = (double)(scale ? pred[bb * ld + fm] * sm + hm : pred[bb * ld + fm]);
      t[2][r][tx] = va;
      t[3][r][tx] = vm;
    }
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int i = bus0 + r;
    if (i >= g.n_bus) continue;
    const bool predicted = g.bus_fa[i] >= 0 || g.bus_fm[i] >= 0;
    const size_t o = (size_t)i * st.Bp + b0 + tx;
    const S va = static_cast<S>(t[2][tx][r]), vm = static_cast<S>(t[3][tx][r]);
    v.s_re[o] = static_cast<S>(t[0][tx][r]);
    v.s_im[o] = static_cast<S>(t[1][tx][r]);
    v.va[o] = va;
    v.vm[o] = vm;
    if (predicted) {
      S sn, cs;
      sin_cos(va, &sn, &cs);
      v.v_re[o] = vm * cs;
      v.v_im[o] = vm * sn;
    } else {  // a slack bus (no Jacobian row; few per grid): V0 read again
      const size_t vo = ((size_t)min(b0 + tx, st.B - 1) * v0_stride + i) * 2;
      v.v_re[o] = static_cast<S>(v0_c[vo]);
      v.v_im[o] = static_cast<S>(v0_c[vo + 1]);
    }
  }
}

// ---------------------------------------------------------------------------
template <typename S>
__global__ void k_seed_state(DevGrid g, DevState st, const double* __restrict__ sbus_c, long long sbus_stride,
                             const double* __restrict__ v0_c, long long v0_stride) {
  __shared__ double t[4][kWarp][kWarp + 1];
  const StateArrays<S> v(st);
  const int tx = threadIdx.x, ty = threadIdx.y;  // (32, 8)
  const int bus0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  for (int r = ty; r < kWarp; r += kRows) {
    const int bb = min(b0 + r, st.B - 1);
    const int bus = bus0 + tx;
    if (bus < g.n_bus) {
      const size_t so = ((size_t)bb * sbus_stride + bus) * 2, vo = ((size_t)bb * v0_stride + bus) * 2;
      t[0][r][tx] = sbus_c[so];
      t[1][r][tx] = sbus_c[so + 1];
      t[2][r][tx] = v0_c[vo];
      t[3][r][tx] = v0_c[vo + 1];
    }
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int bus = bus0 + r;
    if (bus >= g.n_bus) continue;
    const size_t o = (size_t)bus * st.Bp + b0 + tx;
    const double vr = t[2][tx][r], vi = t[3][tx][r];
    v.s_re[o] = static_cast<S>(t[0][tx][r]);
    v.s_im[o] = static_cast<S>(t[1][tx][r]);
    v.v_re[o] = static_cast<S>(vr);
    v.v_im[o] = static_cast<S>(vi);
    v.va[o] = static_cast<S>(atan2(vi, vr));
    v.vm[o] = static_cast<S>(hypot(vr, vi));
  }
}

template <typename S>
__global__ void k_pack_voltage(DevGrid g, DevState st, double* __restrict__ v_c) {
  __shared__ double t[2][kWarp][kWarp + 1];
  const StateArrays<S> v(st);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int bus0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  for (int r = ty; r < kWarp; r += kRows) {
    const int bus = bus0 + r;
    if (bus < g.n_bus) {
      const size_t o = (size_t)bus * st.Bp + b0 + tx;
      t[0][r][tx] = static_cast<double>(v.v_re[o]);
      t[1][r][tx] = static_cast<double>(v.v_im[o]);
    }
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int bb = b0 + r, bus = bus0 + tx;
    if (bb < st.B && bus < g.n_bus) {
      const size_t o = ((size_t)bb * g.n_bus + bus) * 2;
      v_c[o] = t[0][tx][r];
      v_c[o + 1] = t[1][tx][r];
    }
  }
}

template <typename TI>
__device__ __forceinline__ double ld_in(const void* p, size_t i) {
  return static_cast<double>(static_cast<const TI*>(p)[i]);
}

// Sbus = base - load, V0 from (va0, vm0); torch_bridge_kernels.cu:116-152.
// batched_v0 = 1: va0/vm0 are [B][n] (warm starts), else [n] shared.
template <typename TI, typename S>
__global__ void k_set_inputs(DevGrid g, DevState st, const void* base_re, const void* base_im, const void* load_p,
                             const void* load_q, const void* va0, const void* vm0, int batched_v0) {
  __shared__ double t[4][kWarp][kWarp + 1];
  const StateArrays<S> v(st);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int bus0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  const int bus = bus0 + tx;
  for (int r = ty; r < kWarp; r += kRows) {
    const int bb = min(b0 + r, st.B - 1);
    if (bus < g.n_bus) {
      const size_t o = (size_t)bb * g.n_bus + bus;
      t[0][r][tx] = ld_in<TI>(load_p, o);
      t[1][r][tx] = ld_in<TI>(load_q, o);
      t[2][r][tx] = batched_v0 ? ld_in<TI>(va0, o) : 0.0;
      t[3][r][tx] = batched_v0 ? ld_in<TI>(vm0, o) : 0.0;
    }
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int bs = bus0 + r;
    if (bs >= g.n_bus) continue;
    const size_t o = (size_t)bs * st.Bp + b0 + tx;
    const S a = static_cast<S>(batched_v0 ? t[2][tx][r] : ld_in<TI>(va0, bs));
    const S m = static_cast<S>(batched_v0 ? t[3][tx][r] : ld_in<TI>(vm0, bs));
    v.s_re[o] = static_cast<S>(ld_in<TI>(base_re, bs) - t[0][tx][r]);
    v.s_im[o] = static_cast<S>(ld_in<TI>(base_im, bs) - t[1][tx][r]);
    S s, c;
    sin_cos(a, &s, &c);
    v.va[o] = a;
    v.vm[o] = m;
    v.v_re[o] = m * c;
    v.v_im[o] = m * s;
  }
}

template <typename TO, typename S>
__global__ void k_copy_voltage_outputs(DevGrid g, DevState st, TO* __restrict__ va_out, TO* __restrict__ vm_out) {
  __shared__ double t[2][kWarp][kWarp + 1];
  const StateArrays<S> v(st);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int bus0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  for (int r = ty; r < kWarp; r += kRows) {
    const int bus = bus0 + r;
    if (bus < g.n_bus) {
      const size_t o = (size_t)bus * st.Bp + b0 + tx;
      t[0][r][tx] = static_cast<double>(v.va[o]);
      t[1][r][tx] = static_cast<double>(v.vm[o]);
    }
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int bb = b0 + r, bus = bus0 + tx;
    if (bb < st.B && bus < g.n_bus) {
      const size_t o = (size_t)bb * g.n_bus + bus;
      va_out[o] = static_cast<TO>(t[0][tx][r]);
      vm_out[o] = static_cast<TO>(t[1][tx][r]);
    }
  }
}

// dL/dx = [grad_va@pv, grad_va@pq, grad_vm@pq] (torch_bridge_kernels.cu:32-54)
template <typename TI>
__global__ void k_gather_adjoint_rhs(DevGrid g, DevState st, const void* grad_va, const void* grad_vm,
                                     double* __restrict__ G) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  const int bb = min((int)b, st.B - 1);
  const int npvpq = g.n_pv + g.n_pq;
  for (int f = blockIdx.x * kRows + wy; f < g.dim; f += gridDim.x * kRows) {
    double v;
    if (f < g.n_pv) v = ld_in<TI>(grad_va, (size_t)bb * g.n_bus + g.pv[f]);
    else if (f < npvpq) v = ld_in<TI>(grad_va, (size_t)bb * g.n_bus + g.pq[f - g.n_pv]);
    else v = ld_in<TI>(grad_vm, (size_t)bb * g.n_bus + g.pq[f - npvpq]);
    G[(size_t)f * st.Bp + b] = v;
  }
}

// lam[f] = Z[inv[f]]: a solution in pivot order back to Jacobian order
// (inv = the column inverse for J x = b, the row inverse for J^T x = b)
template <typename T>
__global__ void k_permuted_to_rows(const int* __restrict__ inv, int dim, int Bp, const T* __restrict__ Z,
                                   double* __restrict__ lam) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  for (int f = blockIdx.x * kRows + wy; f < dim; f += gridDim.x * kRows)
    lam[(size_t)f * Bp + b] = static_cast<double>(Z[(size_t)inv[f] * Bp + b]);
}

// grad_load = -lambda at the bus's rows (adjoint_math.cpp:189-216)
template <typename TO>
__global__ void k_project_load_gradients(DevGrid g, DevState st, const double* __restrict__ lam, TO* grad_p,
                                         TO* grad_q) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  if ((int)b >= st.B) return;
  for (int i = blockIdx.x * kRows + wy; i < g.n_bus; i += gridDim.x * kRows) {
    const int fa = g.bus_fa[i], fm = g.bus_fm[i];
    const size_t o = b * g.n_bus + i;
    grad_p[o] = static_cast<TO>(fa >= 0 ? -lam[(size_t)fa * st.Bp + b] : 0.0);
    grad_q[o] = static_cast<TO>(fm >= 0 ? -lam[(size_t)fm * st.Bp + b] : 0.0);
  }
}

// R = G - J^T lambda: row j of J^T is column j of J
__global__ void k_jt_residual(DevGrid g, int Bp, const double* __restrict__ Jd, const double* __restrict__ lam,
                              const double* __restrict__ G, double* __restrict__ R) {
  const int lane = threadIdx.x, wy = threadIdx.y;
  const size_t b = (size_t)blockIdx.y * kWarp + lane;
  for (int j = blockIdx.x * kRows + wy; j < g.dim; j += gridDim.x * kRows) {
    double acc = 0.0;
    for (int e = g.jt_ptr[j]; e < g.jt_ptr[j + 1]; ++e)
      acc += Jd[(size_t)g.jt_q[e] * Bp + b] * lam[(size_t)g.jt_row[e] * Bp + b];
    R[(size_t)j * Bp + b] = G[(size_t)j * Bp + b] - acc;
  }
}

// Convergence test of the device-side Newton loop, with the semantics of the
// host loop of newton_solver.cpp:245-342: every iteration evaluates the norm
// (the iteration count is the number of evaluations), stops when
// max_b ||F_b||inf <= tol, and otherwise updates V, also after the last
// allowed evaluation; a non-finite norm ends the solve with an error (or, for
// warm-started solves, only that scenario).  The condition it sets means
// "run one more update".  A mismatch evaluated after the cap was reached is
// not counted.  One block; the max is reduced in a fixed order.
constexpr int kCheckThreads = 1024;
__global__ void __launch_bounds__(kCheckThreads)
    k_loop_check(cudaGraphConditionalHandle h, LoopCtl* __restrict__ ctl,
                 const unsigned long long* __restrict__ norm_bits, double* __restrict__ final_norm) {
  __shared__ double sm[kCheckThreads / kWarp];
  __shared__ int sb[kCheckThreads / kWarp];
  if (ctl->completed >= ctl->max_iter) {  // the cap was reached before this evaluation
    if (threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
    return;
  }
  const int B = ctl->B, tolerate = ctl->tolerate;
  double m = 0.0;
  int bad = 0;  // bit 0: a non-finite norm, bit 1: one that is not tolerated
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const double v = __longlong_as_double((long long)norm_bits[b]);
    const bool finite = v == v && v <= 1.7976931348623157e308;
    if (!finite) {
      final_norm[b] = tolerate ? __longlong_as_double(0x7FF0000000000000ll) : v;
      bad |= tolerate ? 1 : 3;
      continue;
    }
    final_norm[b] = v;
    m = v > m ? v : m;
  }
  for (int o = kWarp / 2; o > 0; o >>= 1) {
    const double mo = __shfl_down_sync(0xffffffffu, m, o);
    m = mo > m ? mo : m;
    bad |= __shfl_down_sync(0xffffffffu, bad, o);
  }
  const int w = threadIdx.x / kWarp, l = threadIdx.x % kWarp;
  if (l == 0) {
    sm[w] = m;
    sb[w] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x / kWarp); ++i) {
      m = sm[i] > m ? sm[i] : m;
      bad |= sb[i];
    }
    const int done = ctl->completed + 1;
    ctl->completed = done;
    ctl->gmax = m;
    ctl->nonfinite = bad & 1;
    if (bad & 2) ctl->status = 1;
    const bool stop = (bad & 2) || m <= ctl->tol;
    cudaGraphSetConditional(h, stop ? 0u : 1u);
  }
}

// Relative residual of the adjoint: per-block partial sums of r^2 and g^2
// over the real scenarios (b < B) of two [dim][Bp] arrays, then one block
// adds the partials in a fixed order (deterministic).
constexpr int kNormBlocks = 296;
__global__ void k_sumsq_partials(const double* __restrict__ R, const double* __restrict__ G, int dim, int B, int Bp,
                                 double* __restrict__ partials) {
  __shared__ double sr[256], sg[256];
  double ar = 0.0, ag = 0.0;
  const long long n = (long long)dim * B;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long f = i / B, b = i - f * B;
    const double r = R[f * Bp + b], g = G[f * Bp + b];
    ar += r * r;
    ag += g * g;
  }
  sr[threadIdx.x] = ar;
  sg[threadIdx.x] = ag;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sr[threadIdx.x] += sr[threadIdx.x + o];
      sg[threadIdx.x] += sg[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = sr[0];
    partials[2 * blockIdx.x + 1] = sg[0];
  }
}

__global__ void k_sumsq_final(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double r = 0.0, g = 0.0;
    for (int i = 0; i < nblocks; ++i) {
      r += partials[2 * i];
      g += partials[2 * i + 1];
    }
    out[0] = r;
    out[1] = g;
  }
}

__global__ void k_axpy(double* y, const double* x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] += x[i];
}

template <typename TS, typename TD>
__global__ void k_batch_to_rows(const TS* __restrict__ src, TD* __restrict__ dst, int rows, int B, int Bp) {
  __shared__ double t[kWarp][kWarp + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int r0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  for (int r = ty; r < kWarp; r += kRows) {
    const int bb = min(b0 + r, B - 1), row = r0 + tx;
    if (row < rows) t[r][tx] = static_cast<double>(src[(size_t)bb * rows + row]);
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int row = r0 + r;
    if (row < rows) dst[(size_t)row * Bp + b0 + tx] = static_cast<TD>(t[tx][r]);
  }
}

template <typename TS, typename TD>
__global__ void k_rows_to_batch(const TS* __restrict__ src, TD* __restrict__ dst, int rows, int B, int Bp) {
  __shared__ double t[kWarp][kWarp + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int r0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  for (int r = ty; r < kWarp; r += kRows) {
    const int row = r0 + r;
    if (row < rows) t[r][tx] = static_cast<double>(src[(size_t)row * Bp + b0 + tx]);
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int bb = b0 + r, row = r0 + tx;
    if (bb < B && row < rows) dst[(size_t)bb * rows + row] = static_cast<TD>(t[tx][r]);
  }
}

// Per-scenario Ybus values, complex [B][stride] (CSR order) -> re/im
// [nnz][Bp]: 32 x 32 tiles through shared memory; padding scenarios repeat
// the last one.
__global__ void k_ybus_to_rows(const double* __restrict__ yc, long long stride, int nnz, int B, int Bp,
                               double* __restrict__ yr, double* __restrict__ yi) {
  __shared__ double tr[kWarp][kWarp + 1], ti[kWarp][kWarp + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int k0 = blockIdx.x * kWarp, b0 = blockIdx.y * kWarp;
  for (int r = ty; r < kWarp; r += kRows) {
    const int bb = min(b0 + r, B - 1), k = k0 + tx;
    if (k < nnz) {
      const double* src = yc + 2 * ((size_t)bb * stride + k);
      tr[r][tx] = src[0];
      ti[r][tx] = src[1];
    }
  }
  __syncthreads();
  for (int r = ty; r < kWarp; r += kRows) {
    const int k = k0 + r;
    if (k < nnz) {
      yr[(size_t)k * Bp + b0 + tx] = tr[tx][r];
      yi[(size_t)k * Bp + b0 + tx] = ti[tx][r];
    }
  }
}

dim3 rows_grid(int rows, int Bp) {
  int bx = (rows + kRows * 4 - 1) / (kRows * 4);
  if (bx < 1) bx = 1;
  return dim3(bx, Bp / kWarp);
}

}  // namespace

void launch_ibus_mismatch(const DevGrid& g, const DevState& st, cudaStream_t s) {
  if (st.state_f32)
    k_ibus_mismatch<float><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st);
  else
    k_ibus_mismatch<double><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st);
}

template <typename S, typename TJ>
void launch_jacobian_s(const DevGrid& g, const DevState& st, TJ* J, cudaStream_t s) {
  if (g.jac_kind == 2) {
    k_jacobian_vertex<S, TJ><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st, J);
    return;
  }
  if (g.jac_kind == 1) {
    k_jacobian_zero_diag<TJ><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st, J);
    k_jacobian_edge_atomic<S, TJ><<<rows_grid(g.nnz_y, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st, J);
    return;
  }
  k_jacobian<S, TJ><<<rows_grid(g.nnz_y, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st, J);
}

template <typename TJ>
void launch_jacobian(const DevGrid& g, const DevState& st, TJ* J, cudaStream_t s) {
  if (st.state_f32)
    launch_jacobian_s<float, TJ>(g, st, J, s);
  else
    launch_jacobian_s<double, TJ>(g, st, J, s);
}
template void launch_jacobian<float>(const DevGrid&, const DevState&, float*, cudaStream_t);
template void launch_jacobian<double>(const DevGrid&, const DevState&, double*, cudaStream_t);

template <typename T>
void launch_voltage_update(const DevGrid& g, const DevPlan& pl, const DevState& st, const T* X, cudaStream_t s) {
  if (st.state_f32)
    k_voltage_update<float, T><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, pl, st, X);
  else
    k_voltage_update<double, T><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, pl, st, X);
}
template void launch_voltage_update<float>(const DevGrid&, const DevPlan&, const DevState&, const float*,
                                           cudaStream_t);
template void launch_voltage_update<double>(const DevGrid&, const DevPlan&, const DevState&, const double*,
                                            cudaStream_t);

void launch_seed_state(const DevGrid& g, const DevState& st, const double* sbus_c, long long sbus_stride,
                       const double* v0_c, long long v0_stride, cudaStream_t s) {
  dim3 grid((g.n_bus + kWarp - 1) / kWarp, st.Bp / kWarp);
  if (st.state_f32)
    k_seed_state<float><<<grid, dim3(kWarp, kRows), 0, s>>>(g, st, sbus_c, sbus_stride, v0_c, v0_stride);
  else
    k_seed_state<double><<<grid, dim3(kWarp, kRows), 0, s>>>(g, st, sbus_c, sbus_stride, v0_c, v0_stride);
}

void launch_seed_warm(const DevGrid& g, const DevState& st, const double* sbus_c, long long sbus_stride,
                      const double* v0_c, long long v0_stride, const float* pred, long long ld, const float* scale,
                      const float* shift, cudaStream_t s) {
  dim3 grid((g.n_bus + kWarp - 1) / kWarp, st.Bp / kWarp);
  if (st.state_f32)
    k_seed_warm<float><<<grid, dim3(kWarp, kRows), 0, s>>>(g, st, sbus_c, sbus_stride, v0_c, v0_stride, pred, ld, scale,
                                                           shift);
  else
    k_seed_warm<double><<<grid, dim3(kWarp, kRows), 0, s>>>(g, st, sbus_c, sbus_stride, v0_c, v0_stride, pred, ld,
                                                            scale, shift);
}

void launch_pack_voltage(const DevGrid& g, const DevState& st, double* v_c, cudaStream_t s) {
  dim3 grid((g.n_bus + kWarp - 1) / kWarp, st.Bp / kWarp);
  if (st.state_f32)
    k_pack_voltage<float><<<grid, dim3(kWarp, kRows), 0, s>>>(g, st, v_c);
  else
    k_pack_voltage<double><<<grid, dim3(kWarp, kRows), 0, s>>>(g, st, v_c);
}

// (input type) x (state type) of the torch bridge's input kernel
static void launch_set_inputs(const DevGrid& g, const DevState& st, const void* base_re, const void* base_im,
                       const void* load_p, const void* load_q, const void* va0, const void* vm0, int is_double,
                       int batched_v0, cudaStream_t s) {
  dim3 grid((g.n_bus + kWarp - 1) / kWarp, st.Bp / kWarp);
  const dim3 blk(kWarp, kRows);
  if (is_double && !st.state_f32)
    k_set_inputs<double, double><<<grid, blk, 0, s>>>(g, st, base_re, base_im, load_p, load_q, va0, vm0, batched_v0);
  else if (is_double)
    k_set_inputs<double, float><<<grid, blk, 0, s>>>(g, st, base_re, base_im, load_p, load_q, va0, vm0, batched_v0);
  else if (!st.state_f32)
    k_set_inputs<float, double><<<grid, blk, 0, s>>>(g, st, base_re, base_im, load_p, load_q, va0, vm0, batched_v0);
  else
    k_set_inputs<float, float><<<grid, blk, 0, s>>>(g, st, base_re, base_im, load_p, load_q, va0, vm0, batched_v0);
}

void launch_set_inputs_from_load(const DevGrid& g, const DevState& st, const void* base_re, const void* base_im,
                                 const void* load_p, const void* load_q, const void* va0, const void* vm0,
                                 int is_double, cudaStream_t s) {
  launch_set_inputs(g, st, base_re, base_im, load_p, load_q, va0, vm0, is_double, 0, s);
}

void launch_set_inputs_batched(const DevGrid& g, const DevState& st, const void* base_re, const void* base_im,
                               const void* load_p, const void* load_q, const void* va0, const void* vm0,
                               int is_double, cudaStream_t s) {
  launch_set_inputs(g, st, base_re, base_im, load_p, load_q, va0, vm0, is_double, 1, s);
}

void launch_copy_voltage_outputs(const DevGrid& g, const DevState& st, void* va_out, void* vm_out, int is_double,
                                 cudaStream_t s) {
  dim3 grid((g.n_bus + kWarp - 1) / kWarp, st.Bp / kWarp);
  const dim3 blk(kWarp, kRows);
  double* dva = static_cast<double*>(va_out);
  double* dvm = static_cast<double*>(vm_out);
  float* fva = static_cast<float*>(va_out);
  float* fvm = static_cast<float*>(vm_out);
  if (is_double && !st.state_f32)
    k_copy_voltage_outputs<double, double><<<grid, blk, 0, s>>>(g, st, dva, dvm);
  else if (is_double)
    k_copy_voltage_outputs<double, float><<<grid, blk, 0, s>>>(g, st, dva, dvm);
  else if (!st.state_f32)
    k_copy_voltage_outputs<float, double><<<grid, blk, 0, s>>>(g, st, fva, fvm);
  else
    k_copy_voltage_outputs<float, float><<<grid, blk, 0, s>>>(g, st, fva, fvm);
}

void launch_gather_adjoint_rhs(const DevGrid& g, const DevState& st, const void* grad_va, const void* grad_vm,
                               int is_double, double* G, cudaStream_t s) {
  if (is_double)
    k_gather_adjoint_rhs<double><<<rows_grid(g.dim, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st, grad_va, grad_vm, G);
  else
    k_gather_adjoint_rhs<float><<<rows_grid(g.dim, st.Bp), dim3(kWarp, kRows), 0, s>>>(g, st, grad_va, grad_vm, G);
}

template <typename T>
void launch_permuted_to_rows(const int* inv, int dim, int Bp, const T* Z, double* lam, cudaStream_t s) {
  k_permuted_to_rows<T><<<rows_grid(dim, Bp), dim3(kWarp, kRows), 0, s>>>(inv, dim, Bp, Z, lam);
}
template void launch_permuted_to_rows<float>(const int*, int, int, const float*, double*, cudaStream_t);
template void launch_permuted_to_rows<double>(const int*, int, int, const double*, double*, cudaStream_t);

void launch_project_load_gradients(const DevGrid& g, const DevState& st, const double* lam, void* grad_p,
                                   void* grad_q, int is_double, cudaStream_t s) {
  if (is_double)
    k_project_load_gradients<double><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(
        g, st, lam, static_cast<double*>(grad_p), static_cast<double*>(grad_q));
  else
    k_project_load_gradients<float><<<rows_grid(g.n_bus, st.Bp), dim3(kWarp, kRows), 0, s>>>(
        g, st, lam, static_cast<float*>(grad_p), static_cast<float*>(grad_q));
}

void launch_jt_residual(const DevGrid& g, int Bp, const double* Jd, const double* lam, const double* G, double* R,
                        cudaStream_t s) {
  k_jt_residual<<<rows_grid(g.dim, Bp), dim3(kWarp, kRows), 0, s>>>(g, Bp, Jd, lam, G, R);
}

template <typename TS, typename TD>
void launch_batch_to_rows(const TS* src, TD* dst, int rows, int B, int Bp, cudaStream_t s) {
  dim3 grid((rows + kWarp - 1) / kWarp, Bp / kWarp);
  k_batch_to_rows<TS, TD><<<grid, dim3(kWarp, kRows), 0, s>>>(src, dst, rows, B, Bp);
}
template <typename TS, typename TD>
void launch_rows_to_batch(const TS* src, TD* dst, int rows, int B, int Bp, cudaStream_t s) {
  dim3 grid((rows + kWarp - 1) / kWarp, Bp / kWarp);
  k_rows_to_batch<TS, TD><<<grid, dim3(kWarp, kRows), 0, s>>>(src, dst, rows, B, Bp);
}
template void launch_batch_to_rows<double, double>(const double*, double*, int, int, int, cudaStream_t);
template void launch_batch_to_rows<double, float>(const double*, float*, int, int, int, cudaStream_t);
template void launch_batch_to_rows<float, float>(const float*, float*, int, int, int, cudaStream_t);
template void launch_batch_to_rows<float, double>(const float*, double*, int, int, int, cudaStream_t);
template void launch_rows_to_batch<double, double>(const double*, double*, int, int, int, cudaStream_t);
template void launch_rows_to_batch<float, double>(const float*, double*, int, int, int, cudaStream_t);
template void launch_rows_to_batch<double, float>(const double*, float*, int, int, int, cudaStream_t);

void launch_sumsq2(const double* R, const double* G, int dim, int B, int Bp, double* scratch, cudaStream_t s) {
  k_sumsq_partials<<<kNormBlocks, 256, 0, s>>>(R, G, dim, B, Bp, scratch + 2);
  k_sumsq_final<<<1, 32, 0, s>>>(scratch + 2, kNormBlocks, scratch);
}

void launch_axpy(double* y, const double* x, long long n, cudaStream_t s) {
  long long blocks = (n + 255) / 256;
  if (blocks > 4096) blocks = 4096;
  k_axpy<<<(unsigned)blocks, 256, 0, s>>>(y, x, n);
}

void launch_ybus_to_rows(const double* yc, long long stride, int nnz, int B, int Bp, double* yr, double* yi,
                         cudaStream_t s) {
  k_ybus_to_rows<<<dim3((nnz + kWarp - 1) / kWarp, Bp / kWarp), dim3(kWarp, kRows), 0, s>>>(yc, stride, nnz, B, Bp,
                                                                                          yr, yi);
}

void launch_loop_check(cudaGraphConditionalHandle h, LoopCtl* ctl, const unsigned long long* norm_bits,
                       double* final_norm, cudaStream_t s) {
  k_loop_check<<<1, kCheckThreads, 0, s>>>(h, ctl, norm_bits, final_norm);
}

namespace {
__global__ void k_ctl_load(const LoopCtl* __restrict__ host_ctl, LoopCtl* __restrict__ ctl) {
  if (threadIdx.x == 0) *ctl = *host_ctl;
}
__global__ void k_ctl_store(const LoopCtl* __restrict__ ctl, LoopCtl* __restrict__ host_ctl,
                            const double* __restrict__ final_norm, double* __restrict__ host_final,
                            double* __restrict__ d_final, int B) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    const double v = final_norm[b];
    host_final[b] = v;
    if (d_final) d_final[b] = v;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *host_ctl = *ctl;
  __threadfence_system();
}
}  // namespace

void launch_ctl_load(const LoopCtl* host_ctl, LoopCtl* ctl, cudaStream_t s) {
  k_ctl_load<<<1, 32, 0, s>>>(host_ctl, ctl);
}

void launch_ctl_store(const LoopCtl* ctl, LoopCtl* host_ctl, const double* final_norm, double* host_final,
                      double* d_final, int B, cudaStream_t s) {
  const int blocks = std::max(1, std::min((B + 255) / 256, 64));
  k_ctl_store<<<blocks, 256, 0, s>>>(ctl, host_ctl, final_norm, host_final, d_final, B);
}

}  // namespace cupf_b200
