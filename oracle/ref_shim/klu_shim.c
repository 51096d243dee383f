/*
 * klu_shim.c -- KLU / UMFPACK entry points over the oracle's sparse LU
 * (TEST INFRASTRUCTURE ONLY; see klu.h).  Ordering: METIS nested dissection
 * on A + A^T (KLU would use AMD after a BTF pre-pass); pivoting: threshold
 * partial pivoting with tol 0.001 preferring the diagonal, KLU's default.
 */
#include "klu.h"
#include "umfpack.h"

#include <stdlib.h>
#include <string.h>

#include "../pf_oracle.h"

struct klu_symbolic_struct {
  int32_t n;
  int32_t* order;
};
struct klu_numeric_struct {
  orc_lu* lu;
};

int klu_defaults(klu_common* c) {
  if (!c) return 0;
  c->status = 0;
  c->tol = 0.001;
  return 1;
}

klu_symbolic* klu_analyze(int32_t n, int32_t* Ap, int32_t* Ai, klu_common* c) {
  klu_symbolic* s = (klu_symbolic*)calloc(1, sizeof(klu_symbolic));
  s->n = n;
  s->order = (int32_t*)malloc(sizeof(int32_t) * n);
  orc_nd_order(n, Ap, Ai, s->order);
  if (c) c->status = 0;
  return s;
}

klu_numeric* klu_factor(int32_t* Ap, int32_t* Ai, double* Ax, klu_symbolic* s, klu_common* c) {
  orc_lu* lu = orc_lu_factor(s->n, Ap, Ai, Ax, s->order, c ? c->tol : 0.001);
  if (!lu) {
    if (c) c->status = 1;
    return NULL;
  }
  klu_numeric* num = (klu_numeric*)calloc(1, sizeof(klu_numeric));
  num->lu = lu;
  return num;
}

int klu_solve(klu_symbolic* s, klu_numeric* num, int32_t ldim, int32_t nrhs, double* B, klu_common* c) {
  (void)s; (void)c;
  for (int r = 0; r < nrhs; ++r) orc_lu_solve(num->lu, B + (size_t)r * ldim);
  return 1;
}

int klu_tsolve(klu_symbolic* s, klu_numeric* num, int32_t ldim, int32_t nrhs, double* B, klu_common* c) {
  (void)s; (void)c;
  for (int r = 0; r < nrhs; ++r) orc_lu_tsolve(num->lu, B + (size_t)r * ldim);
  return 1;
}

int klu_free_symbolic(klu_symbolic** s, klu_common* c) {
  (void)c;
  if (s && *s) {
    free((*s)->order);
    free(*s);
    *s = NULL;
  }
  return 1;
}

int klu_free_numeric(klu_numeric** num, klu_common* c) {
  (void)c;
  if (num && *num) {
    orc_lu_free((*num)->lu);
    free(*num);
    *num = NULL;
  }
  return 1;
}

/* ---- UMFPACK over the same LU ---- */

typedef struct { int32_t n; int32_t* order; } umf_sym;

int umfpack_di_defaults(double Control[UMFPACK_CONTROL]) {
  for (int i = 0; i < UMFPACK_CONTROL; ++i) Control[i] = 0.0;
  return UMFPACK_OK;
}

int umfpack_di_symbolic(int32_t n_row, int32_t n_col, const int32_t Ap[], const int32_t Ai[], const double Ax[],
                        void** Symbolic, const double Control[UMFPACK_CONTROL], double Info[UMFPACK_INFO]) {
  (void)Ax; (void)Control; (void)Info;
  if (n_row != n_col || n_row <= 0) return UMFPACK_ERROR_invalid_matrix;
  umf_sym* s = (umf_sym*)calloc(1, sizeof(umf_sym));
  s->n = n_row;
  s->order = (int32_t*)malloc(sizeof(int32_t) * n_row);
  orc_nd_order(n_row, Ap, Ai, s->order);
  *Symbolic = s;
  return UMFPACK_OK;
}

int umfpack_di_numeric(const int32_t Ap[], const int32_t Ai[], const double Ax[], void* Symbolic, void** Numeric,
                       const double Control[UMFPACK_CONTROL], double Info[UMFPACK_INFO]) {
  (void)Control; (void)Info;
  umf_sym* s = (umf_sym*)Symbolic;
  orc_lu* lu = orc_lu_factor(s->n, Ap, Ai, Ax, s->order, 0.1);
  if (!lu) return UMFPACK_ERROR_invalid_matrix;
  *Numeric = lu;
  return UMFPACK_OK;
}

int umfpack_di_solve(int sys, const int32_t Ap[], const int32_t Ai[], const double Ax[], double X[],
                     const double B[], void* Numeric, const double Control[UMFPACK_CONTROL],
                     double Info[UMFPACK_INFO]) {
  (void)Ap; (void)Ai; (void)Ax; (void)Control; (void)Info;
  orc_lu* lu = (orc_lu*)Numeric;
  int n = orc_lu_dim(lu);
  memcpy(X, B, sizeof(double) * n);
  if (sys == UMFPACK_At) orc_lu_tsolve(lu, X); else orc_lu_solve(lu, X);
  return UMFPACK_OK;
}

void umfpack_di_free_symbolic(void** Symbolic) {
  if (Symbolic && *Symbolic) {
    umf_sym* s = (umf_sym*)*Symbolic;
    free(s->order);
    free(s);
    *Symbolic = NULL;
  }
}

void umfpack_di_free_numeric(void** Numeric) {
  if (Numeric && *Numeric) {
    orc_lu_free((orc_lu*)*Numeric);
    *Numeric = NULL;
  }
}
