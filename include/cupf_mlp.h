/*
 * cupf_mlp.h -- C ABI of the warm-start network's BF16 kernels.
 *
 * No reference counterpart.  The reference has only a torch MLP analog in its
 * PINN benchmark harness (benchmark/pinn/model.py:13-38).  The engine trains
 * and runs its warm-start network with these kernels; the Python driver is
 * gpu-powerflow_b200/cupf/warm_start.py.
 *
 * All pointers are device pointers; row-major matrices; bf16 = IEEE bfloat16.
 * Every function returns 0 on success, 1 for an invalid argument, 2 for a
 * CUDA error; mlp_last_error() gives the message.  Launches are asynchronous
 * on `stream` (NULL = legacy default stream).
 */
#ifndef CUPF_MLP_H
#define CUPF_MLP_H

#ifdef __cplusplus
extern "C" {
#endif

const char* mlp_last_error(void);

/* C[M][N] = A[M][K] * B[N][K]^T on the tcgen05 tensor cores (bf16 in, fp32
 * accumulate).  M and N multiples of 128, K a multiple of 64; row strides
 * lda, ldb, ldo (elements, multiples of 8, at least the row length); A, B and
 * out 16-byte aligned.  epi: 0 out = C (fp32); 1 out = C + bias (fp32);
 * 2 aux = C + bias, out = gelu(aux) (both bf16; aux may be NULL when the
 * pre-activations are not needed, as in inference); 3 out = C * gelu'(aux)
 * (bf16).  aux has row stride ldaux. */
int mlp_gemm_bf16(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K, int epi,
                  void* out, long long ldo, const float* bias, void* aux, long long ldaux, void* stream);
/* Split-weight GEMM: out = A (B_hi + B_lo)^T (+ bias), fp32 out [M][ldo].
 * A is [M][lda] bf16 with K columns; B is [N][ldb] bf16 holding B_hi in
 * columns [0, K) and B_lo in [K, 2K) (B_lo = bf16(W - B_hi) of fp32 weights
 * W), so the product carries about 16 mantissa bits of W at the cost of a
 * GEMM with 2K.  epi: 0 (out = C) or 1 (out = C + bias). */
int mlp_gemm_bf16_split(const void* A, long long lda, const void* B, long long ldb, int M, int N, int K, int epi,
                        void* out, long long ldo, const float* bias, void* stream);
/* Device error flag of the GEMM (1 or 2 after a bounded wait gave up); copied
 * to *out_host with a synchronising copy, optionally reset. */
int mlp_error_flag(int* out_host, int reset);
/* Failure-path test of the GEMM's bounded waits (process-wide, read at each
 * launch).  spin_limit: mbarrier polls before a wait gives up (default
 * 4,194,304).  stall_loads = 1 makes the producer issue no tile loads, so the
 * MMA thread's wait for the first tile runs out: the kernel then raises the
 * error flag (1), writes NaN into its output tiles, frees its tensor memory
 * and returns.  Nothing faults or hangs; set (4194304, 0) to restore. */
int mlp_set_wait_test(long long spin_limit, int stall_loads);
/* Least-squares output layer of the warm start, in FP64 on the CUDA cores
 * (refit_kernels.cu).  These report their own errors through
 * mlp_refit_last_error (same return codes).
 *
 * Normal equations of [A | 1] (n rows; the ones column is the bias), added
 * to what AtA and AtY hold:  AtA[(p+1)][(p+1)] += [A|1]^T [A|1] (upper
 * triangle only, i <= j), AtY[(p+1)][q] += [A|1]^T Y (AtY may be NULL).
 * A [n][lda] is bf16 (a_type 0) or fp32 (1); Y [n][ldy] fp32 (y_type 0) or
 * fp64 (1).  Asynchronous on `stream`. */
int mlp_gram_f64(const void* A, long long lda, int a_type, const void* Y, long long ldy, int y_type, int n, int p,
                 int q, double* AtA, long long ld_ata, double* AtY, long long ld_aty, void* stream);
/* Solves (M + ridge) X = R in place for symmetric positive definite M
 * [D][ldm] given by its upper triangle: ridge = ridge_rel x the mean of the
 * positive diagonal entries, added to the diagonal; blocked Cholesky
 * M = U^T U (U overwrites the upper triangle, 64-column panels), then
 * U^T Y = R and U X = Y with R [D][ldr] (q columns) overwritten by X.
 * d_info (device int) is set to the first non-positive pivot's index + 1
 * (0: none).  Asynchronous on `stream`. */
int mlp_cholesky_solve_f64(double* M, long long ldm, int D, double* R, long long ldr, int q, double ridge_rel,
                           int* d_info, void* stream);
const char* mlp_refit_last_error(void);
/* out[cols][rows] = in[rows][cols] (bf16; in has row stride ld). */
int mlp_transpose_bf16(const void* in, long long ld, void* out, int rows, int cols, void* stream);
/* x[b][k] = bf16((raw[b][k] - mean[k]) * inv_std[k]) for k < n_in, 0 for
 * n_in <= k < width; x has row stride ldx >= width, raw [B][n_in] fp32. */
int mlp_standardize(const float* raw, const float* mean, const float* inv_std, void* x, long long ldx, int B,
                    int n_in, int width, void* stream);
/* Standardized power-flow load features straight from Sbus (complex128
 * [B][sbus_stride]) and the grid's generation sgen (complex128 [n]):
 * x[r][k] = bf16((f_k - mean[k]) * inv_std[k]) with f_k = Re(sgen_k - S_rk)
 * for k < n, Im(sgen - S) at k - n for n <= k < 2n, extra[k - 2n] for the
 * next n_extra columns; 0 up to width.  Rows B <= r < rows repeat row B - 1.
 * x has row stride ldx >= width; sbus and sgen start on 16-byte boundaries
 * (whole complex128 elements); rows <= 65535. */
int mlp_load_features(const double* sbus, long long sbus_stride, const double* sgen, const float* extra, int n,
                      int n_extra, const float* mean, const float* inv_std, void* x, long long ldx, int B, int rows,
                      int width, void* stream);
/* Mean-squared error on the first n_out of ld columns: grad (bf16 [B][ld]) and
 * *loss += mean squared difference (fp32, may be NULL). */
int mlp_mse_grad(const float* pred, int ld, const float* target, int n_out, int B, void* grad, float* loss,
                 void* stream);
/* out[c] = sum_r g[r][c] (g bf16 [rows][cols], out fp32). */
int mlp_col_sum_bf16(const void* g, int rows, int cols, float* out, void* stream);
/* Adam step on fp32 master weights w (n elements) with moments m, v; writes
 * the bf16 copy w_bf16 when not NULL.  step counts from 1. */
int mlp_adam(float* w, const float* grad, float* m, float* v, void* w_bf16, long long n, float lr, float b1, float b2,
             float eps, int step, float weight_decay, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CUPF_MLP_H */
