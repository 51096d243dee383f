/*
 * metis.h -- METIS 5.1 API for compiling the reference's ordering code into the
 * oracle library (TEST INFRASTRUCTURE ONLY).  Names, option indices and
 * signatures follow the public METIS 5.1 manual.
 *
 * The reference is written for a 32-bit idx_t build (its metis_nd.cpp:296-303
 * only compiles when idx_t is int), while the METIS library shipped with the
 * CUDA toolkit is a 64-bit idx_t build.  The three entry points are therefore
 * renamed here to 32-bit adapters (metis32_shim.c) that widen the arrays and
 * call the toolkit library, so the reference and the product order with the
 * same library and options.
 */
#ifndef ORACLE_METIS_SHIM_H
#define ORACLE_METIS_SHIM_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int32_t idx_t;
typedef float real_t;
#define METIS_NOPTIONS 40
#define METIS_OK 1
enum {
  METIS_OPTION_PTYPE, METIS_OPTION_OBJTYPE, METIS_OPTION_CTYPE, METIS_OPTION_IPTYPE,
  METIS_OPTION_RTYPE, METIS_OPTION_DBGLVL, METIS_OPTION_NITER, METIS_OPTION_NCUTS,
  METIS_OPTION_SEED, METIS_OPTION_NO2HOP, METIS_OPTION_MINCONN, METIS_OPTION_CONTIG,
  METIS_OPTION_COMPRESS, METIS_OPTION_CCORDER, METIS_OPTION_PFACTOR, METIS_OPTION_NSEPS,
  METIS_OPTION_UFACTOR, METIS_OPTION_NUMBERING
};
#define METIS_SetDefaultOptions oracle_metis32_SetDefaultOptions
#define METIS_NodeND oracle_metis32_NodeND
#define METIS_ComputeVertexSeparator oracle_metis32_ComputeVertexSeparator
int METIS_SetDefaultOptions(idx_t* options);
int METIS_NodeND(idx_t* nvtxs, idx_t* xadj, idx_t* adjncy, idx_t* vwgt, idx_t* options, idx_t* perm,
                 idx_t* iperm);
int METIS_ComputeVertexSeparator(idx_t* nvtxs, idx_t* xadj, idx_t* adjncy, idx_t* vwgt, idx_t* options,
                                 idx_t* sepsize, idx_t* part);
#ifdef __cplusplus
}
#endif
#endif
