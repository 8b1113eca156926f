/*
 * Test infrastructure only: the oracle build compiles the reference's C
 * (T) kernels in place and needs a "config.h" on the include path (the
 * reference ships only a CMake template for it).  This shim supplies the
 * OpenMP thread-query functions those kernels call.
 */
#ifndef ORACLE_REF_SHIM_CONFIG_H
#define ORACLE_REF_SHIM_CONFIG_H
#ifdef _OPENMP
#include <omp.h>
#else
static inline int omp_get_thread_num(void) { return 0; }
static inline int omp_get_num_threads(void) { return 1; }
#endif
#endif
