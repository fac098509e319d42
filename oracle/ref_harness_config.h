/* Hand-written stand-in for the config.h that the reference's CMake would
 * generate from src/config.h.cmake.in: FP64, 3D, non-orthorhombic, no MPI,
 * no timers, 32-byte alignment (the reference's GNU non-AVX512 setting).
 * Used only by oracle/ref_harness.mk when compiling the reference's own
 * sources into oracle/_ref/ (golden-vector generation, test infrastructure). */
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
#define QMC_CLINE 32
#define QMC_ALIGNAS alignas(32)
#define ASSUME_ALIGNED(x) (x) = (__typeof__(x))__builtin_assume_aligned(x, 32)
#endif
