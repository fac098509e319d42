// tc.cuh -- inline-PTX wrappers for the 5th-generation tensor cores
// (tcgen05: TMEM allocation, MMA, commit, TMEM loads) and the shared-memory
// mbarriers their completion is tracked with.  sm_100a only.
#pragma once

#include <cstdint>

namespace qmc
{
// default limit of a bounded wait, in SM cycles (about one second); a batch
// may set its own (qmc_walkers_set_wait_limit)
constexpr long long kTcWaitCycles = 2000000000LL;
// largest padded delay rank of the tensor-core Woodbury flush
constexpr int TC_KD = 64;

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// one warp: allocate `ncols` TMEM columns (power of two >= 32), write the
// base address to shared memory, and give up the right to allocate again
__device__ __forceinline__ void tc_alloc(uint32_t* dst, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
// one warp: give up the right to allocate without allocating.  A CTA of a
// kernel that contains tcgen05.alloc holds that right until it gives it up
// or exits, and CTAs that still hold it keep further CTAs off their SM.
__device__ __forceinline__ void tc_relinquish()
{
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
// one warp: release the columns
__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// make generic-proxy shared-memory writes visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 16-byte global -> shared copy that does not hold registers (cp.async,
// L2 only); each thread waits for its own copies with tc_cp_async_wait_all
__device__ __forceinline__ void tc_cp_async16(void* dst_smem, const void* src)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst_smem)), "l"(src) : "memory");
}
__device__ __forceinline__ void tc_cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void tc_cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// wait until the phase with parity `parity` of `bar` has completed; gives
// up and returns false once `limit` SM cycles have passed (the clock is read
// before each poll, so a limit of 0 gives up before the first one)
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity, long long limit)
{
  const uint32_t a   = smem_u32(bar);
  const long long t0 = clock64();
  while (true)
  {
    if (clock64() - t0 >= limit)
      return false;
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(a), "r"(parity)
                 : "memory");
    if (ok)
      return true;
  }
}

// shared-memory matrix descriptor, no swizzle (K-major "interleave" layout:
// 8-row x 16-byte core matrices; lbo = byte distance between the two core
// matrices along K of one MMA, sbo = byte distance between 8-row groups)
__device__ __forceinline__ uint64_t tc_desc(const void* p, uint32_t lbo, uint32_t sbo)
{
  const uint32_t a = smem_u32(p);
  return (uint64_t)((a >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// instruction descriptor of kind::tf32: FP32 accumulator, TF32 A and B,
// both K-major, dense, M x N
__host__ __device__ constexpr uint32_t tc_idesc_tf32(int M, int N)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] B[smem]^T, issued by one thread
__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate)
{
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
               : "memory");
}
// arrive once on `bar` when every MMA this thread issued so far completes
__device__ __forceinline__ void tc_commit(unsigned long long* bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// warp-collective: 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
               "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                 "=r"(r[15])
               : "r"(taddr)
               : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i)
    v[i] = __uint_as_float(r[i]);
}

// round to the nearest TF32 (10-bit mantissa)
__device__ __forceinline__ float tf32_round(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}
// 3xTF32 operand split: hi = tf32(x), lo = tf32(x - hi); hi + lo carries
// x to within 2^-22 relative
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo)
{
  hi = tf32_round(x);
  lo = tf32_round(x - hi);
}

// float offset of element (row, k) in a K-major no-swizzle tile whose rows
// hold K elements (K a multiple of 4): core matrices of 8 rows x 4 floats
__host__ __device__ __forceinline__ int canon(int row, int k, int K)
{
  return (((row >> 3) * (K >> 2) + (k >> 2)) << 5) + ((row & 7) << 2) + (k & 3);
}

} // namespace qmc
