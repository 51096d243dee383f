/*
 * metis32_shim.c -- 32-bit idx_t adapters over the toolkit's 64-bit METIS 5.1
 * library (TEST INFRASTRUCTURE ONLY; see metis.h).
 */
#include <stdint.h>
#include <stdlib.h>

typedef int64_t m64;
int METIS_SetDefaultOptions(m64* options);
int METIS_NodeND(m64* nvtxs, m64* xadj, m64* adjncy, m64* vwgt, m64* options, m64* perm, m64* iperm);
int METIS_ComputeVertexSeparator(m64* nvtxs, m64* xadj, m64* adjncy, m64* vwgt, m64* options, m64* sepsize,
                                 m64* part);

static m64* widen(const int32_t* a, long n) {
  m64* w = (m64*)malloc(sizeof(m64) * (n > 0 ? n : 1));
  for (long i = 0; i < n; ++i) w[i] = a ? a[i] : 0;
  return w;
}

int oracle_metis32_SetDefaultOptions(int32_t* options) {
  m64 o[40];
  int rc = METIS_SetDefaultOptions(o);
  for (int i = 0; i < 40; ++i) options[i] = (int32_t)o[i];
  return rc;
}

int oracle_metis32_NodeND(int32_t* nvtxs, int32_t* xadj, int32_t* adjncy, int32_t* vwgt, int32_t* options,
                          int32_t* perm, int32_t* iperm) {
  long n = *nvtxs, m = xadj[n];
  m64 nv = n;
  m64 *x = widen(xadj, n + 1), *a = widen(adjncy, m), *w = vwgt ? widen(vwgt, n) : NULL;
  m64 o[40];
  for (int i = 0; i < 40; ++i) o[i] = options ? options[i] : -1;
  m64 *p = (m64*)malloc(sizeof(m64) * n), *ip = (m64*)malloc(sizeof(m64) * n);
  int rc = METIS_NodeND(&nv, x, a, w, options ? o : NULL, p, ip);
  for (long i = 0; i < n; ++i) {
    perm[i] = (int32_t)p[i];
    iperm[i] = (int32_t)ip[i];
  }
  free(x); free(a); free(w); free(p); free(ip);
  return rc;
}

int oracle_metis32_ComputeVertexSeparator(int32_t* nvtxs, int32_t* xadj, int32_t* adjncy, int32_t* vwgt,
                                          int32_t* options, int32_t* sepsize, int32_t* part) {
  long n = *nvtxs, m = xadj[n];
  m64 nv = n, sep = 0;
  m64 *x = widen(xadj, n + 1), *a = widen(adjncy, m), *w = vwgt ? widen(vwgt, n) : NULL;
  m64 o[40];
  for (int i = 0; i < 40; ++i) o[i] = options ? options[i] : -1;
  m64* pt = (m64*)malloc(sizeof(m64) * n);
  int rc = METIS_ComputeVertexSeparator(&nv, x, a, w, options ? o : NULL, &sep, pt);
  *sepsize = (int32_t)sep;
  for (long i = 0; i < n; ++i) part[i] = (int32_t)pt[i];
  free(x); free(a); free(w); free(pt);
  return rc;
}
