/*
 * umfpack.h -- stand-in for SuiteSparse UMFPACK (TEST INFRASTRUCTURE ONLY).
 * Declares the entry points and constants the reference's alternate CPU solver
 * uses (cuPF/cpp/src/newton_solver/ops/linear_solve/cpu_umfpack.cpp:29-252),
 * implemented in klu_shim.c over the same oracle LU.
 */
#ifndef ORACLE_UMFPACK_SHIM_H
#define ORACLE_UMFPACK_SHIM_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
#define UMFPACK_CONTROL 20
#define UMFPACK_INFO 90
#define UMFPACK_OK 0
#define UMFPACK_A 0
#define UMFPACK_At 1
#define UMFPACK_ERROR_invalid_matrix (-8)
int umfpack_di_defaults(double Control[UMFPACK_CONTROL]);
int umfpack_di_symbolic(int32_t n_row, int32_t n_col, const int32_t Ap[], const int32_t Ai[], const double Ax[],
                        void** Symbolic, const double Control[UMFPACK_CONTROL], double Info[UMFPACK_INFO]);
int umfpack_di_numeric(const int32_t Ap[], const int32_t Ai[], const double Ax[], void* Symbolic, void** Numeric,
                       const double Control[UMFPACK_CONTROL], double Info[UMFPACK_INFO]);
int umfpack_di_solve(int sys, const int32_t Ap[], const int32_t Ai[], const double Ax[], double X[],
                     const double B[], void* Numeric, const double Control[UMFPACK_CONTROL],
                     double Info[UMFPACK_INFO]);
void umfpack_di_free_symbolic(void** Symbolic);
void umfpack_di_free_numeric(void** Numeric);
#ifdef __cplusplus
}
#endif
#endif
