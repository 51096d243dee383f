/*
 * pf_oracle.h -- CPU FP64 oracle for the batched Newton-Raphson power flow.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * cpu-klu path (cuPF CpuFp64Pipeline, cuPF/cpp/src/newton_solver/core/
 * pipeline.hpp:86-122).  Only tests/, the smoke check and the CPU-baseline leg
 * of bench.py may load it, and only as the checker; the product never links or
 * calls it.
 *
 * The reference factors J with SuiteSparse KLU, which is not installed here.
 * The LU below is this oracle's own left-looking Gilbert-Peierls sparse LU with
 * threshold partial pivoting (the algorithm KLU applies to each diagonal block,
 * as published by Gilbert & Peierls 1988 and Davis 2006), on a METIS
 * nested-dissection column order.  It is not KLU and is labelled that way.
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Jacobian symbolic analysis (cuPF ops/jacobian/jacobian_analysis.cpp) ---- */

/* Sizes first: returns dimF, sets *nnz_j.  Returns -1 on invalid input. */
int orc_jacobian_nnz(int n_bus, const int32_t* indptr, const int32_t* indices,
                     const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                     int* nnz_j);

/* Fills the CSR pattern (row_ptr[dimF+1], col_idx[nnz_j]) and the eight
 * scatter maps: map11/21/12/22[nnz_y] per Ybus entry, diag11/21/12/22[n_bus].
 * Returns 0 on success. */
int orc_jacobian_analysis(int n_bus, const int32_t* indptr, const int32_t* indices,
                          const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                          int32_t* row_ptr, int32_t* col_idx,
                          int32_t* map11, int32_t* map21, int32_t* map12, int32_t* map22,
                          int32_t* diag11, int32_t* diag21, int32_t* diag12, int32_t* diag22);

/* ---- Sparse LU (Gilbert-Peierls, threshold partial pivoting) ---- */

typedef struct orc_lu orc_lu;

/* Factor the CSC matrix (Ap, Ai, Ax), n x n.  col_order may be NULL (natural)
 * or a permutation new -> old.  tol in (0, 1]: a diagonal pivot is kept when
 * |a_diag| >= tol * max|column|.  Returns NULL on a structurally or
 * numerically singular matrix. */
orc_lu* orc_lu_factor(int n, const int32_t* Ap, const int32_t* Ai, const double* Ax,
                      const int32_t* col_order, double tol);
/* Refactor with the same ordering and pivot sequence search (values change). */
int orc_lu_refactor(orc_lu* lu, const int32_t* Ap, const int32_t* Ai, const double* Ax);
void orc_lu_solve(const orc_lu* lu, double* b);   /* A x = b, in place */
void orc_lu_tsolve(const orc_lu* lu, double* b);  /* A^T x = b, in place */
int orc_lu_nnz(const orc_lu* lu);
int orc_lu_dim(const orc_lu* lu);
void orc_lu_free(orc_lu* lu);

/* METIS nested-dissection order (serial METIS_NodeND, seed 42) of the
 * symmetric pattern A + A^T of a CSC matrix; perm[new] = old. */
int orc_nd_order(int n, const int32_t* Ap, const int32_t* Ai, int32_t* perm);

/* ---- Newton-Raphson FP64, batch 1 (cuPF core/newton_solver.cpp:497-558) ---- */

typedef struct {
  double tolerance;      /* NRConfig::tolerance (default 1e-8) */
  int32_t max_iter;      /* NRConfig::max_iter  (default 50)   */
} orc_nr_config;

typedef struct {
  int32_t iterations;
  double final_mismatch;
  int32_t converged;
  int32_t status;        /* 0 ok, 1 non-finite mismatch, 2 singular J, 3 bad input */
} orc_nr_result;

/* Solve one case.  Complex arrays are interleaved (re, im) doubles.
 * v_out[2*n_bus].  Optionally returns J at the final state (CSC values in the
 * pattern order of orc_jacobian_analysis's CSR -> CSC remap) when jac_out is
 * non-NULL (size nnz_j). */
int orc_nr_solve(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                 const double* sbus, const double* v0,
                 const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                 orc_nr_config cfg, double* v_out, orc_nr_result* res);

/* Adjoint at the converged state of the last orc_nr_solve call arguments:
 * rebuilds Ibus/J at v (interleaved complex), solves J^T lambda = dL/dx with
 * dL/dx = [grad_va@pv, grad_va@pq, grad_vm@pq]
 * (cuPF core/adjoint_math.cpp:62-122) and returns lambda[dimF],
 * grad_p[n_bus] = grad_q[n_bus] = -lambda projected to buses.
 * Returns the relative residual ||J^T lambda - rhs|| / ||rhs|| (< 0 on error). */
double orc_adjoint(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                   const double* v, const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                   const double* grad_va, const double* grad_vm,
                   double* lambda, double* grad_p, double* grad_q);

/* Pieces of one NR iteration, exposed for element-wise parity tests:
 * mismatch F(V) [dimF] and its infinity norm; the Jacobian CSR values at V
 * (in the CSR order of orc_jacobian_analysis). */
double orc_mismatch(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                    const double* sbus, const double* v,
                    const int32_t* pv, int n_pv, const int32_t* pq, int n_pq, double* F);
int orc_jacobian_values(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                        const double* v, const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                        double* jvals_csr);

/* Run `count` independent cases (sbus/v0 rows of stride 2*n_bus doubles) on
 * `threads` host threads, one solver per thread.  Used as the CPU baseline. */
int orc_nr_solve_many(int n_bus, const int32_t* indptr, const int32_t* indices, const double* ydata,
                      const double* sbus, const double* v0, int count,
                      const int32_t* pv, int n_pv, const int32_t* pq, int n_pq,
                      orc_nr_config cfg, int threads, double* v_out,
                      int32_t* iterations, double* final_mismatch);

#ifdef __cplusplus
}
#endif

#endif /* PF_ORACLE_H */
