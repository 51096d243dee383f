/*
 * klu.h -- stand-in for SuiteSparse KLU, used only to compile the reference's
 * CPU pipeline into the oracle library (TEST INFRASTRUCTURE ONLY).
 *
 * Declares the six KLU entry points the reference calls
 * (cuPF/cpp/src/newton_solver/ops/linear_solve/cpu_klu.cpp:63,104,135,178,201,225)
 * with the signatures of the published KLU C API.  They are implemented in
 * klu_shim.c over the oracle's own Gilbert-Peierls LU (oracle/pf_oracle.c);
 * numerics differ from real KLU in pivot order and rounding, not in meaning.
 */
#ifndef ORACLE_KLU_SHIM_H
#define ORACLE_KLU_SHIM_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef struct klu_common_struct {
  int status;
  double tol;
} klu_common;
typedef struct klu_symbolic_struct klu_symbolic;
typedef struct klu_numeric_struct klu_numeric;
int klu_defaults(klu_common* Common);
klu_symbolic* klu_analyze(int32_t n, int32_t* Ap, int32_t* Ai, klu_common* Common);
klu_numeric* klu_factor(int32_t* Ap, int32_t* Ai, double* Ax, klu_symbolic* Symbolic, klu_common* Common);
int klu_solve(klu_symbolic* Symbolic, klu_numeric* Numeric, int32_t ldim, int32_t nrhs, double* B,
              klu_common* Common);
int klu_tsolve(klu_symbolic* Symbolic, klu_numeric* Numeric, int32_t ldim, int32_t nrhs, double* B,
               klu_common* Common);
int klu_free_symbolic(klu_symbolic** Symbolic, klu_common* Common);
int klu_free_numeric(klu_numeric** Numeric, klu_common* Common);
#ifdef __cplusplus
}
#endif
#endif
