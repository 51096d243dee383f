// device_plan.cuh -- device views shared by the kernels.
//
// Per-scenario arrays are stored element-major with the scenario index
// innermost: value (element e, scenario b) lives at e * Bp + b, where Bp is the
// batch rounded up to a multiple of 32.  A warp therefore always reads the same
// element for 32 consecutive scenarios: one coalesced 128 B (fp32) or 256 B
// (fp64) transaction, with every plan index warp-uniform.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cupf_b200 {

constexpr int kWarp = 32;
constexpr int kFrontMetaInts = 24;  // int32 per front launch record (front_meta)

// The factor program of one grid (see analysis.hpp FactorProgram).
struct DevPlan {
  int P = 0, dim = 0, nnz = 0;
  const int* fsz = nullptr;
  const int* nc = nullptr;
  const int* first = nullptr;
  const int* front_ptr = nullptr;
  const int* front_rows = nullptr;
  const long long* u_off = nullptr;
  const long long* l_off = nullptr;
  const long long* cb_off = nullptr;
  const long long* tv_off = nullptr;  // adjoint update vectors: prefix sum of uc
  const int* arow_ptr = nullptr;
  const int* arow_q = nullptr;
  const int* arow_col = nullptr;
  const int* crow_ptr = nullptr;
  const int* crow_child = nullptr;
  const int* crow_r = nullptr;
  const long long* crow_src = nullptr;  // per child entry: its update-vector element, tv_off[child] + row
  const int* crow_dst = nullptr;        // per child entry: its row in the parent front
  const int* asm_ptr = nullptr;
  const int* asm_local = nullptr;
  const int* perm = nullptr;   // permuted index -> Jacobian row
  const int* iperm = nullptr;  // Jacobian column -> permuted index
  const int* row_iperm = nullptr;  // Jacobian row -> permuted index (= iperm without matching)
  const int* col_perm = nullptr;   // permuted index -> Jacobian column (= perm without matching)
  const int* level_fronts = nullptr;
  // dense-front assembly program (analysis.hpp FactorProgram::fe_*)
  const long long* fe_split = nullptr;  // 9 per front
  const int* fe_dst = nullptr;
  const long long* fe_src = nullptr;
  const int* front_meta = nullptr;  // 24 int32 per front, in level order
};

// One front's launch record (front_meta), read with six 16-byte loads.
struct FrontMeta {
  int fs, nc, first, p, fr0;
  long long e0, uo, lo, co;
  int split[9];  // assembly-list cuts relative to e0 (split[0] = 0)
};

__device__ __forceinline__ long long meta_ll(int lo, int hi) {
  return (long long)(((unsigned long long)(unsigned)hi << 32) | (unsigned)lo);
}

__device__ __forceinline__ FrontMeta load_front_meta(const int* meta, int q) {
  const int4* m4 = reinterpret_cast<const int4*>(meta) + (size_t)q * 6;
  const int4 a = m4[0], b = m4[1], c = m4[2], d = m4[3], e = m4[4], f = m4[5];
  FrontMeta m;
  m.fs = a.x;
  m.nc = a.y;
  m.first = a.z;
  m.p = a.w;
  m.e0 = meta_ll(b.x, b.y);
  m.uo = meta_ll(b.z, b.w);
  m.lo = meta_ll(c.x, c.y);
  m.co = meta_ll(c.z, c.w);
  m.split[0] = 0;
  m.split[1] = d.x;
  m.split[2] = d.y;
  m.split[3] = d.z;
  m.split[4] = d.w;
  m.split[5] = e.x;
  m.split[6] = e.y;
  m.split[7] = e.z;
  m.split[8] = e.w;
  m.fr0 = f.x;
  return m;
}

// Ybus and the Jacobian maps of one grid.
struct DevGrid {
  int n_bus = 0, nnz_y = 0, dim = 0, nnz_j = 0, n_pv = 0, n_pq = 0;
  int jac_kind = 0;  // Jacobian fill: 0 edge, 1 edge with atomic diagonal sums, 2 vertex (one bus row per warp)
  const int* y_ptr = nullptr;
  const int* y_col = nullptr;
  const int* y_row = nullptr;
  const int* y_diag = nullptr;  // position of the diagonal entry of each row, -1 if absent
  const double* y_re = nullptr;
  const double* y_im = nullptr;
  const int* map11 = nullptr;
  const int* map21 = nullptr;
  const int* map12 = nullptr;
  const int* map22 = nullptr;
  const int* bus_fa = nullptr;  // bus -> angle row (P equation), -1 for slack
  const int* bus_fm = nullptr;  // bus -> magnitude row (Q equation), -1 for slack/PV
  const int* bus_fa_p = nullptr;  // the same rows in the factor's pivot order (iperm applied)
  const int* bus_fm_p = nullptr;
  const int* pv = nullptr;
  const int* pq = nullptr;
  const int* jt_ptr = nullptr;  // J^T as CSR over J's CSR positions: column j of J
  const int* jt_row = nullptr;  //   rows i and positions q of column j
  const int* jt_q = nullptr;
};

// Per-batch state (all [rows][Bp]).  The voltage, injection, current and
// mismatch arrays are typed double below; under ComputePolicy::FP32
// (state_f32 = 1) the same buffers hold float, and the stage kernels read
// them through StateArrays<float>.
struct DevState {
  int B = 0, Bp = 0;
  int state_f32 = 0;
  double* v_re = nullptr;
  double* v_im = nullptr;
  double* va = nullptr;
  double* vm = nullptr;
  double* s_re = nullptr;
  double* s_im = nullptr;
  double* i_re = nullptr;
  double* i_im = nullptr;
  double* F = nullptr;
  void* Fp = nullptr;   // F again, in pivot order and the factor's type (the LU's right-hand side)
  int fp_double = 0;    // Fp holds double (FP64 factors) or float
  unsigned long long* norm_bits = nullptr;  // [Bp] max |F| per scenario as IEEE bits
  int* sing = nullptr;                      // [Bp] static-pivot shift applied
  // per-scenario Ybus values [nnz_y][Bp] (null: every scenario uses DevGrid's)
  const double* yb_re = nullptr;
  const double* yb_im = nullptr;
};

}  // namespace cupf_b200
