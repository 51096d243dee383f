/*
 * metis_lock_shim.c -- serialises the reference's METIS calls
 * (TEST INFRASTRUCTURE ONLY).
 *
 * The reference's parallel nested dissection (metis_nd.cpp:241-278) runs the
 * two halves of every separator in two threads, and METIS keeps state in
 * process globals, so concurrent calls race: METIS draws from the C library's
 * rand(), which each METIS call seeds from its options at its start, and the
 * reference reseeds it (std::srand) before every call in every thread.  Calls
 * that never overlap, with no reseeding from another thread in the middle of
 * one, give the result of a race-free run whatever their order.  The oracle's
 * reference library is linked with --wrap for the two METIS entry points and
 * for srand; these wrappers hold one process-wide (recursive) lock around
 * each of them.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>

typedef int64_t m64;
int __real_METIS_NodeND(m64* nvtxs, m64* xadj, m64* adjncy, m64* vwgt, m64* options, m64* perm, m64* iperm);
int __real_METIS_ComputeVertexSeparator(m64* nvtxs, m64* xadj, m64* adjncy, m64* vwgt, m64* options, m64* sepsize,
                                        m64* part);

void __real_srand(unsigned int seed);

static pthread_mutex_t g_metis_lock = PTHREAD_RECURSIVE_MUTEX_INITIALIZER_NP;

void __wrap_srand(unsigned int seed) {
  pthread_mutex_lock(&g_metis_lock);
  __real_srand(seed);
  pthread_mutex_unlock(&g_metis_lock);
}

int __wrap_METIS_NodeND(m64* nvtxs, m64* xadj, m64* adjncy, m64* vwgt, m64* options, m64* perm, m64* iperm) {
  pthread_mutex_lock(&g_metis_lock);
  int rc = __real_METIS_NodeND(nvtxs, xadj, adjncy, vwgt, options, perm, iperm);
  pthread_mutex_unlock(&g_metis_lock);
  return rc;
}

int __wrap_METIS_ComputeVertexSeparator(m64* nvtxs, m64* xadj, m64* adjncy, m64* vwgt, m64* options, m64* sepsize,
                                        m64* part) {
  pthread_mutex_lock(&g_metis_lock);
  int rc = __real_METIS_ComputeVertexSeparator(nvtxs, xadj, adjncy, vwgt, options, sepsize, part);
  pthread_mutex_unlock(&g_metis_lock);
  return rc;
}
