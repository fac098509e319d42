/* The config.h that the reference's headers include (Utilities/
 * Configuration.h), written for the adapter build in place of the one the
 * reference's CMake generates from src/config.h.cmake.in: its default
 * Release build, 3D, non-orthorhombic, OpenMP, timers on, no MPI, FP64
 * (OHMMS_PRECISION double).  The alignment follows the template's GNU
 * branch for an AVX2 target (32 bytes). */
#ifndef QMCPLUSPLUS_CONFIGURATION_H
#define QMCPLUSPLUS_CONFIGURATION_H
#define QMCPACK_VERSION_MAJOR 0
#define QMCPACK_VERSION_MINOR 2
#define QMCPACK_VERSION_PATCH 0
#define ENABLE_OPENMP 1
#define OHMMS_DIM 3
#define OHMMS_INDEXTYPE int
#define OHMMS_PRECISION double
#define OHMMS_PRECISION_FULL double
#define OHMMS_ORTHO 0
#define HAVE_SINCOS 1
#define HAVE_POSIX_MEMALIGN 1
#define ENABLE_TIMERS 1
#define QMC_CLINE 32
#define QMC_ALIGNAS alignas(32)
#define ASSUME_ALIGNED(x) (x) = (__typeof__(x))__builtin_assume_aligned(x, 32)
#endif
