/* Hand-written stand-in for the config.h that the reference's CMake would
 * generate from src/config.h.cmake.in for its default Release build: 3D,
 * non-orthorhombic, OpenMP, internal timers on, no MPI.  The arithmetic is
 * FP64 unless the compile line defines QMC_REF_MIXED (the reference's
 * QMC_MIXED_PRECISION=1: OHMMS_PRECISION float, full precision double).
 * Alignment follows the template's GNU branch (64 bytes with AVX-512, else
 * 32).  Used only by oracle/ref_miniqmc.mk to compile the reference's own
 * miniqmc driver into oracle/_ref/ as the timed CPU baseline. */
#ifndef QMCPLUSPLUS_CONFIGURATION_H
#define QMCPLUSPLUS_CONFIGURATION_H
#define QMCPACK_VERSION_MAJOR 0
#define QMCPACK_VERSION_MINOR 2
#define QMCPACK_VERSION_PATCH 0
#define ENABLE_OPENMP 1
#define OHMMS_DIM 3
#define OHMMS_INDEXTYPE int
#ifdef QMC_REF_MIXED
#define OHMMS_PRECISION float
#define OHMMS_PRECISION_FULL double
#define MIXED_PRECISION 1
#else
#define OHMMS_PRECISION double
#define OHMMS_PRECISION_FULL double
#endif
#define OHMMS_ORTHO 0
#define HAVE_SINCOS 1
#define HAVE_POSIX_MEMALIGN 1
#define ENABLE_TIMERS 1
#if defined(__AVX512F__)
#define QMC_CLINE 64
#define QMC_ALIGNAS alignas(64)
#define ASSUME_ALIGNED(x) (x) = (__typeof__(x))__builtin_assume_aligned(x, 64)
#else
#define QMC_CLINE 32
#define QMC_ALIGNAS alignas(32)
#define ASSUME_ALIGNED(x) (x) = (__typeof__(x))__builtin_assume_aligned(x, 32)
#endif
#endif
