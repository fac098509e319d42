// common.cuh -- shared device/host helpers for the B200 VMC walker hot path.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cuda_runtime.h>

#ifndef QMC_HD
#define QMC_HD __host__ __device__ __forceinline__
#endif

namespace qmc
{
// error bits raised by kernels into the batch status word
enum : unsigned
{
  DEV_ERR_SINGULAR  = 1u,
  DEV_ERR_NONFINITE = 2u,
  DEV_ERR_INDEX     = 4u,
  DEV_ERR_STATE     = 8u,
  DEV_ERR_TIMEOUT   = 16u, // a bounded wait on the tensor-core pipeline gave up
  DEV_ERR_CAPACITY  = 32u  // a fixed-size J3 list or pair buffer was full
};

constexpr double kPi = 3.14159265358979323846;

// ------------------------------------------------------------ mt19937 --
// Mersenne Twister MT19937 (Matsumoto & Nishimura 1998), the engine behind
// std::mt19937 that StdRandom.h:19-110 uses.  Seeding and tempering follow
// the published algorithm; the CTA-parallel twist below regenerates the 624
// state words in four dependency-free phases.
constexpr int MT_N = 624, MT_M = 397;
constexpr uint32_t MT_MATRIX_A = 0x9908b0dfu, MT_UPPER = 0x80000000u, MT_LOWER = 0x7fffffffu;

struct MTState
{
  uint32_t mt[MT_N];
  int mti;
};

inline void mt_seed_host(MTState& s, uint32_t seed)
{
  s.mt[0] = seed;
  for (int i = 1; i < MT_N; ++i)
    s.mt[i] = 1812433253u * (s.mt[i - 1] ^ (s.mt[i - 1] >> 30)) + (uint32_t)i;
  s.mti = MT_N;
}
QMC_HD uint32_t mt_temper(uint32_t y)
{
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}
QMC_HD uint32_t mt_twist_one(uint32_t cur, uint32_t next, uint32_t far)
{
  uint32_t y = (cur & MT_UPPER) | (next & MT_LOWER);
  return far ^ (y >> 1) ^ ((y & 1u) ? MT_MATRIX_A : 0u);
}
inline void mt_twist_host(MTState& s)
{
  for (int i = 0; i < MT_N; ++i)
    s.mt[i] = mt_twist_one(s.mt[i], s.mt[(i + 1) % MT_N], s.mt[(i + MT_M) % MT_N]);
  s.mti = 0;
}
inline uint32_t mt_next_host(MTState& s)
{
  if (s.mti >= MT_N)
    mt_twist_host(s);
  return mt_temper(s.mt[s.mti++]);
}
// libstdc++ generate_canonical<double,53>(mt19937): two 32-bit words,
// (w0 + w1 * 2^32) / 2^64 rounded to nearest, clamped below 1.
QMC_HD double canonical_double(uint32_t w0, uint32_t w1)
{
#ifdef __CUDA_ARCH__
  double s = __dadd_rn((double)w0, __dmul_rn((double)w1, 4294967296.0));
#else
  double s = (double)w0 + (double)w1 * 4294967296.0;
#endif
  double r = s * 5.421010862427522170037e-20; // 2^-64, exact scaling
  if (r >= 1.0)
    r = 0.99999999999999988898; // nextafter(1.0, 0.0)
  return r;
}

// ---------------------------------------------------------- SplitMix64 --
// SplitMix64 (Steele, Lea & Flood 2014) as a counter-based stream.
QMC_HD uint64_t splitmix64(uint64_t seed, uint64_t index)
{
  uint64_t z = seed + (index + 1) * 0x9E3779B97F4A7C15ull;
  z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
QMC_HD double splitmix_uniform(uint64_t seed, uint64_t index)
{
  return (double)(splitmix64(seed, index) >> 11) * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------ vectors --
template <typename T> struct Vec16;
template <> struct Vec16<float>
{
  using type                 = float4;
  static constexpr int width = 4;
};
template <> struct Vec16<double>
{
  using type                 = double2;
  static constexpr int width = 2;
};

// --------------------------------------------------------- reductions --
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum NV doubles over the whole block; result broadcast in out[0..NV).
// scratch must hold 32 * NV doubles.  Contains __syncthreads.
template <int NV>
__device__ __forceinline__ void block_sum(const double (&v)[NV], double* scratch, double* out)
{
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i)
  {
    double s = warp_sum(v[i]);
    if (lane == 0)
      scratch[wid * NV + i] = s;
  }
  __syncthreads();
  if (wid == 0)
  {
#pragma unroll
    for (int i = 0; i < NV; ++i)
    {
      double s = lane < nw ? scratch[lane * NV + i] : 0.0;
      s        = warp_sum(s);
      if (lane == 0)
        out[i] = s;
    }
  }
  __syncthreads();
}

} // namespace qmc
