// sweep.cuh -- what the two forms of the fused sweep (sweep.cu: one CTA per
// walker; sweep_queue.cu: the work queue) share on the host side: the
// dynamic shared memory of a launch and the CTAs per SM it leaves.
#pragma once
#include "device.cuh"

namespace qmc
{
// dynamic shared memory of a sweep launch: the active spin's Binv, then the
// flush scratch or, between flushes, the J2 candidate lists and the epoch's
// stencil weights (or the J3 move scratch); the tensor-core flush tiles
// overlay the cached Binv
template <typename T> static size_t sweep_smem_bytes(int threads, int max_k, bool tc, bool j3, bool epoch)
{
  const size_t moves = j2_list_bytes() + (epoch ? epoch_smem_bytes<T>() : 0);
  size_t bytes       = bsm_bytes(max_k) + std::max(flush_smem_bytes_for<T>(threads, max_k), moves);
  if (tc && tc_flush_smem_bytes(max_k) > bytes)
    bytes = tc_flush_smem_bytes(max_k);
  if (j3)
    bytes = std::max(bytes, bsm_bytes(max_k) + sizeof(J3Smem<T>));
  return bytes;
}

// CTAs per SM from the kernel's registers and static shared memory and the
// launch's block size and dynamic shared memory (registers are allocated
// per warp in units of 256; every CTA also reserves 1 KB of shared memory)
// (the device figures by cudaDeviceGetAttribute: cudaGetDeviceProperties
// takes milliseconds, and a sweep call asks this on every call)
template <typename K> static int occupancy_of(K kernel, int threads, size_t bytes)
{
  cudaFuncAttributes fa;
  int dev = 0, regs = 0, smem = 0, reserved = 0, max_threads = 0, max_blocks = 0;
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_threads, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&max_blocks, cudaDevAttrMaxBlocksPerMultiprocessor, dev) != cudaSuccess)
    return -1;
  const int warps     = (threads + 31) / 32;
  const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;
  const int by_regs   = regs_warp ? regs / (warps * regs_warp) : max_blocks;
  const size_t cta    = fa.sharedSizeBytes + bytes + (size_t)reserved;
  const int by_smem   = (int)((size_t)smem / cta);
  const int by_warps  = max_threads / (warps * 32);
  return std::min(std::min(by_regs, by_smem), std::min(by_warps, max_blocks));
}
} // namespace qmc
