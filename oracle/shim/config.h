/* Build-configuration header for compiling the reference CPU analytics as the
 * test oracle (TEST INFRASTRUCTURE ONLY; never linked into the GPU library).
 *
 * The reference generates this file from its CMake template
 * (include/graptor/config.h.in); its cmake build needs the network, so this
 * project-written stand-in fixes the values for an offline OpenMP build:
 * no NUMA, OpenMP backend, vector length from the target ISA. */
#ifndef GG_ORACLE_SHIM_CONFIG_H
#define GG_ORACLE_SHIM_CONFIG_H

#ifndef MAX_VL
# if defined(__AVX512F__)
#  define MAX_VL 16
# else
#  define MAX_VL 8
# endif
#endif

#if defined(__cplusplus)
constexpr unsigned short VLUpperBound = ~(unsigned short)0;
#endif

#define Graptor_VERSION_MAJOR 0
#define Graptor_VERSION_MINOR 0

/* Backend selector values as the reference's parallel backends test them. */
#define BACKEND_seq 0
#define BACKEND_cilk_numa 1
#define BACKEND_cilk 2
#define BACKEND_openmp_numa 3
#define BACKEND_openmp 4
#define BACKEND_parlay_numa 5
#define BACKEND_parlay 6
#define HAS_NUMA(cfg) ((cfg)&1)

#ifndef GRAPTOR_PARALLEL
# define GRAPTOR_PARALLEL BACKEND_openmp
#endif

#define NUMA 0
static const int num_numa_node = 1;
#define ALT_BOR_ASSIGN 1

#endif
