// refit_kernels.cu -- FP64 kernels of the warm start's least-squares output
// layer: the normal equations and their Cholesky solve.
//
// The output layer W is refit in closed form on the hidden features a that
// the network's own kernels compute for every training row:
//     (A^T A + ridge I) W^T = A^T Y,   A = [a | 1]  (n rows, p + 1 columns).
// A holds bf16 activations and Y fp32 standardized targets; everything here
// accumulates and factors in FP64 on the CUDA cores (sm_100 has no FP64
// tensor-core instruction in the tcgen05 family):
//
//   k_gemm_tn_f64   C (+)= alpha * A^T B over a range of rows: the Gram
//                   matrix A^T A (upper triangle only), A^T Y, and the
//                   trailing and right-hand-side updates of the blocked
//                   Cholesky solve.  128 x 128 output tiles, 8 x 8 per
//                   thread, 8 rows per step staged in shared memory as FP64.
//                   A is read as A(r, i) = A[r * lda + i] (row layout) or
//                   A[i * lda + r] (column layout); an implicit all-ones
//                   column i == ones_col gives the bias.
//   k_potrf_upper   M_kk = U_kk^T U_kk for one 64 x 64 diagonal block.
//   k_trsm_ut       X = U_kk^-T B (forward substitution), one column a thread.
//   k_trsm_u        X = U_kk^-1 B (back substitution), one column a thread.
//
// mlp_cholesky_solve_f64 drives them: right-looking blocked Cholesky of the
// upper triangle (M = U^T U, block 64), then U^T Y = R and U X = Y.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "cupf_mlp.h"

namespace cupf_b200 {
namespace {

constexpr int kTile = 128, kStep = 8, kThreadsGemm = 256, kNb = 64;

template <typename T>
__device__ __forceinline__ double as_f64(T v) {
  return static_cast<double>(v);
}
template <>
__device__ __forceinline__ double as_f64<__nv_bfloat16>(__nv_bfloat16 v) {
  return static_cast<double>(__bfloat162float(v));
}

// C[i][j] = beta_one ? C + alpha * sum_r A(r, i) B(r, j) : alpha * sum ...,
// i < p, j < q, r < n.  upper: only tiles with i-tile <= j-tile (and only
// i <= j written inside the diagonal tiles).
template <typename TA, typename TB, bool A_COLS>
__global__ void __launch_bounds__(kThreadsGemm)
    k_gemm_tn_f64(const TA* __restrict__ A, long long lda, const TB* __restrict__ B, long long ldb, int n, int p,
                  int q, int ones_col_a, int ones_col_b, double alpha, double* __restrict__ C, long long ldc,
                  int upper) {
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (upper && ti > tj) return;
  __shared__ double As[kStep][kTile];
  __shared__ double Bs[kStep][kTile];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;  // 16 x 16 threads, 8 x 8 outputs each
  const int i0 = ti * kTile, j0 = tj * kTile;
  double acc[8][8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
#pragma unroll
    for (int b = 0; b < 8; ++b) acc[a][b] = 0.0;
  for (int r0 = 0; r0 < n; r0 += kStep) {
    // stage 8 rows x 128 columns of A and of B (FP64)
    for (int e = threadIdx.x; e < kStep * kTile; e += kThreadsGemm) {
      int rr, ii;
      if (A_COLS) {  // consecutive threads walk r, so a column's 8 rows are contiguous
        rr = e % kStep;
        ii = e / kStep;
      } else {
        rr = e / kTile;
        ii = e % kTile;
      }
      const int r = r0 + rr, i = i0 + ii;
      double v = 0.0;
      if (r < n && i < p) {
        if (i == ones_col_a)
          v = 1.0;
        else
          v = as_f64(A_COLS ? A[(size_t)i * lda + r] : A[(size_t)r * lda + i]);
      }
      As[rr][ii] = v;
    }
    for (int e = threadIdx.x; e < kStep * kTile; e += kThreadsGemm) {
      const int rr = e / kTile, jj = e % kTile;
      const int r = r0 + rr, j = j0 + jj;
      double v = 0.0;
      if (r < n && j < q) v = j == ones_col_b ? 1.0 : as_f64(B[(size_t)r * ldb + j]);
      Bs[rr][jj] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kStep; ++k) {
      double a[8], b[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        a[u] = As[k][ty + 16 * u];
        b[u] = Bs[k][tx + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int v = 0; v < 8; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int i = i0 + ty + 16 * u;
    if (i >= p) continue;
#pragma unroll
    for (int v = 0; v < 8; ++v) {
      const int j = j0 + tx + 16 * v;
      if (j >= q || (upper && i > j)) continue;
      double* c = C + (size_t)i * ldc + j;
      *c += alpha * acc[u][v];
    }
  }
}

// M_kk (64 x 64, upper triangle, leading dimension ld) = U^T U in place;
// info[0] = first non-positive pivot (global index + 1) or left as is.
__global__ void __launch_bounds__(256) k_potrf_upper(double* __restrict__ M, long long ld, int k0, int nb,
                                                     int* __restrict__ info) {
  __shared__ double a[kNb][kNb + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e % nb;
    a[i][j] = i <= j ? M[(size_t)(k0 + i) * ld + k0 + j] : 0.0;
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    if (threadIdx.x == 0) {
      const double d = a[j][j];
      if (!(d > 0.0)) {
        if (info[0] == 0) info[0] = k0 + j + 1;
        a[j][j] = 1.0;
      } else {
        a[j][j] = sqrt(d);
      }
    }
    __syncthreads();
    const double inv = 1.0 / a[j][j];
    for (int c = j + 1 + (int)threadIdx.x; c < nb; c += blockDim.x) a[j][c] *= inv;
    __syncthreads();
    // trailing update of rows j+1.. (upper part): a[r][c] -= a[j][r] a[j][c], r <= c
    const int m = nb - j - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int r = j + 1 + e / m, c = j + 1 + e % m;
      if (r <= c) a[r][c] -= a[j][r] * a[j][c];
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, j = e % nb;
    if (i <= j) M[(size_t)(k0 + i) * ld + k0 + j] = a[i][j];
  }
}

// B (nb rows x ncols, leading dimension ldb) <- U^-T B: forward substitution
// with U the nb x nb upper block at U0 (leading dimension ldu).
__global__ void __launch_bounds__(128) k_trsm_ut(const double* __restrict__ U0, long long ldu, int nb,
                                                 double* __restrict__ B, long long ldb, int ncols) {
  __shared__ double u[kNb][kNb + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) u[e / nb][e % nb] = U0[(size_t)(e / nb) * ldu + e % nb];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  double x[kNb];
#pragma unroll
  for (int i = 0; i < kNb; ++i)
    if (i < nb) {
      double s = B[(size_t)i * ldb + c];
#pragma unroll
      for (int m = 0; m < kNb; ++m)
        if (m < i) s -= u[m][i] * x[m];
      x[i] = s / u[i][i];
    }
#pragma unroll
  for (int i = 0; i < kNb; ++i)
    if (i < nb) B[(size_t)i * ldb + c] = x[i];
}

// B <- U^-1 B: back substitution with the same block.
__global__ void __launch_bounds__(128) k_trsm_u(const double* __restrict__ U0, long long ldu, int nb,
                                                double* __restrict__ B, long long ldb, int ncols) {
  __shared__ double u[kNb][kNb + 1];
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) u[e / nb][e % nb] = U0[(size_t)(e / nb) * ldu + e % nb];
  __syncthreads();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  double x[kNb];
#pragma unroll
  for (int i = kNb - 1; i >= 0; --i)
    if (i < nb) {
      double s = B[(size_t)i * ldb + c];
#pragma unroll
      for (int m = 0; m < kNb; ++m)
        if (m > i && m < nb) s -= u[i][m] * x[m];
      x[i] = s / u[i][i];
    }
#pragma unroll
  for (int i = 0; i < kNb; ++i)
    if (i < nb) B[(size_t)i * ldb + c] = x[i];
}

// diag += shift, shift = rel * mean of the positive diagonal entries (one block)
__global__ void k_add_ridge(double* __restrict__ M, long long ld, int D, double rel) {
  __shared__ double s_sum[256];
  __shared__ int s_cnt[256];
  double sum = 0.0;
  int cnt = 0;
  for (int i = threadIdx.x; i < D; i += blockDim.x) {
    const double d = M[(size_t)i * ld + i];
    if (d > 0.0) {
      sum += d;
      ++cnt;
    }
  }
  s_sum[threadIdx.x] = sum;
  s_cnt[threadIdx.x] = cnt;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + o];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + o];
    }
    __syncthreads();
  }
  const double shift = s_cnt[0] > 0 ? rel * s_sum[0] / s_cnt[0] : rel;
  for (int i = threadIdx.x; i < D; i += blockDim.x) M[(size_t)i * ld + i] += shift;
}

thread_local std::string g_refit_err;

template <typename TA, typename TB, bool A_COLS>
void gemm_tn(const TA* A, long long lda, const TB* B, long long ldb, int n, int p, int q, int ones_a, int ones_b,
             double alpha, double* C, long long ldc, bool upper, cudaStream_t s) {
  if (n <= 0 || p <= 0 || q <= 0) return;
  const dim3 grid((unsigned)((q + kTile - 1) / kTile), (unsigned)((p + kTile - 1) / kTile));
  k_gemm_tn_f64<TA, TB, A_COLS><<<grid, kThreadsGemm, 0, s>>>(A, lda, B, ldb, n, p, q, ones_a, ones_b, alpha, C, ldc,
                                                              upper ? 1 : 0);
}

void check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace
}  // namespace cupf_b200

using namespace cupf_b200;

extern "C" {

const char* mlp_refit_last_error() { return g_refit_err.c_str(); }

int mlp_gram_f64(const void* A, long long lda, int a_type, const void* Y, long long ldy, int y_type, int n, int p,
                 int q, double* AtA, long long ld_ata, double* AtY, long long ld_aty, void* stream) {
  try {
    if (!A || !AtA || n < 0 || p <= 0 || lda < p || ld_ata < p + 1 || (a_type != 0 && a_type != 1))
      throw std::invalid_argument("mlp_gram_f64: invalid A / AtA arguments");
    if (AtY && (!Y || q <= 0 || ldy < q || ld_aty < q || (y_type != 0 && y_type != 1)))
      throw std::invalid_argument("mlp_gram_f64: invalid Y / AtY arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // [A | 1]^T [A | 1], upper triangle (the ones column is column p)
    if (a_type == 0)
      gemm_tn<__nv_bfloat16, __nv_bfloat16, false>(static_cast<const __nv_bfloat16*>(A), lda,
                                                   static_cast<const __nv_bfloat16*>(A), lda, n, p + 1, p + 1, p, p,
                                                   1.0, AtA, ld_ata, true, s);
    else
      gemm_tn<float, float, false>(static_cast<const float*>(A), lda, static_cast<const float*>(A), lda, n, p + 1,
                                   p + 1, p, p, 1.0, AtA, ld_ata, true, s);
    check("gram A^T A");
    if (AtY) {
      if (a_type == 0 && y_type == 0)
        gemm_tn<__nv_bfloat16, float, false>(static_cast<const __nv_bfloat16*>(A), lda, static_cast<const float*>(Y),
                                             ldy, n, p + 1, q, p, -1, 1.0, AtY, ld_aty, false, s);
      else if (a_type == 0)
        gemm_tn<__nv_bfloat16, double, false>(static_cast<const __nv_bfloat16*>(A), lda,
                                              static_cast<const double*>(Y), ldy, n, p + 1, q, p, -1, 1.0, AtY, ld_aty,
                                              false, s);
      else if (y_type == 0)
        gemm_tn<float, float, false>(static_cast<const float*>(A), lda, static_cast<const float*>(Y), ldy, n, p + 1,
                                     q, p, -1, 1.0, AtY, ld_aty, false, s);
      else
        gemm_tn<float, double, false>(static_cast<const float*>(A), lda, static_cast<const double*>(Y), ldy, n,
                                      p + 1, q, p, -1, 1.0, AtY, ld_aty, false, s);
      check("gram A^T Y");
    }
    return 0;
  } catch (const std::invalid_argument& e) {
    g_refit_err = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_refit_err = e.what();
    return 2;
  }
}

int mlp_cholesky_solve_f64(double* M, long long ldm, int D, double* R, long long ldr, int q, double ridge_rel,
                           int* d_info, void* stream) {
  try {
    if (!M || !R || !d_info || D <= 0 || q <= 0 || ldm < D || ldr < q || ridge_rel < 0.0)
      throw std::invalid_argument("mlp_cholesky_solve_f64: invalid arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(d_info, 0, sizeof(int), s) != cudaSuccess) throw std::runtime_error("info reset failed");
    if (ridge_rel > 0.0) k_add_ridge<<<1, 256, 0, s>>>(M, ldm, D, ridge_rel);
    check("ridge");
    // M = U^T U (upper triangle), right-looking, 64-column panels
    for (int k = 0; k < D; k += kNb) {
      const int nb = std::min(kNb, D - k), rest = D - k - nb;
      k_potrf_upper<<<1, 256, 0, s>>>(M, ldm, k, nb, d_info);
      check("potrf");
      if (rest > 0) {
        double* Ukk = M + (size_t)k * ldm + k;
        double* Urow = M + (size_t)k * ldm + k + nb;  // U[k..k+nb)[k+nb..D)
        k_trsm_ut<<<(rest + 127) / 128, 128, 0, s>>>(Ukk, ldm, nb, Urow, ldm, rest);
        check("trsm");
        // trailing M[j1][j2] -= sum_r U[r][j1] U[r][j2], r in this panel (upper part)
        gemm_tn<double, double, false>(Urow, ldm, Urow, ldm, nb, rest, rest, -1, -1, -1.0,
                                       M + (size_t)(k + nb) * ldm + k + nb, ldm, true, s);
        check("trailing update");
      }
    }
    // U^T Y = R (forward), row panels top-down
    for (int k = 0; k < D; k += kNb) {
      const int nb = std::min(kNb, D - k), rest = D - k - nb;
      k_trsm_ut<<<(q + 127) / 128, 128, 0, s>>>(M + (size_t)k * ldm + k, ldm, nb, R + (size_t)k * ldr, ldr, q);
      check("forward solve");
      if (rest > 0)
        gemm_tn<double, double, false>(M + (size_t)k * ldm + k + nb, ldm, R + (size_t)k * ldr, ldr, nb, rest, q, -1,
                                       -1, -1.0, R + (size_t)(k + nb) * ldr, ldr, false, s);
      check("forward update");
    }
    // U X = Y (backward), row panels bottom-up
    const int last = (D - 1) / kNb * kNb;
    for (int k = last; k >= 0; k -= kNb) {
      const int nb = std::min(kNb, D - k);
      k_trsm_u<<<(q + 127) / 128, 128, 0, s>>>(M + (size_t)k * ldm + k, ldm, nb, R + (size_t)k * ldr, ldr, q);
      check("backward solve");
      if (k > 0)  // R[0..k) -= U[0..k)[k..k+nb) X_k: A(r, i) = U[i][k + r], column layout
        gemm_tn<double, double, true>(M + k, ldm, R + (size_t)k * ldr, ldr, nb, k, q, -1, -1, -1.0, R, ldr, false,
                                      s);
      check("backward update");
    }
    return 0;
  } catch (const std::invalid_argument& e) {
    g_refit_err = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_refit_err = e.what();
    return 2;
  }
}

}  // extern "C"
