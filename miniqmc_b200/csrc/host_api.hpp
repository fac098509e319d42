// host_api.hpp -- private host-side declarations shared by the C ABI's
// translation units (api.cu: handles, verbs and sweeps; serve.cu: batch
// groups, the autotuner and the request loop).
#pragma once

#include "kernels.cuh"
#include "../../include/qmcgpu.h"

#include <algorithm>
#include <string>
#include <vector>

// last error message of the calling host thread (qmc_last_error)
extern thread_local std::string g_err;
int fail(int code, const std::string& msg);
#define CK(call)                                                                                          \
  do                                                                                                      \
  {                                                                                                       \
    cudaError_t e_ = (call);                                                                              \
    if (e_ != cudaSuccess)                                                                                \
      return fail(e_ == cudaErrorMemoryAllocation ? QMC_ERR_OOM : QMC_ERR_CUDA,                           \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                                    \
  } while (0)

struct qmc_system_s
{
  qmc::DevSystem h;       // host mirror with device pointers
  qmc::DevSystem* d = nullptr;
  bool fp32    = false;
  std::vector<void*> allocs;
  size_t bytes = 0;
};

struct qmc_walkers_s
{
  qmc_system* sys = nullptr;
  qmc::DevWalkers dw{};
  bool fp32   = false;
  int threads = 128;
  cudaStream_t stream = nullptr;
  bool own_stream     = false;
  std::vector<void*> allocs;
  size_t bytes      = 0;
  int64_t launches  = 0;
  int64_t steps_done = 0; // MC steps swept by this batch over all calls
  bool ratio_moves   = false; // a ratio-only verb ran since the last evaluateLog
  int prefetch_mode  = QMC_PREFETCH_AUTO;
  int64_t nlpp_calls = 0; // NonLocalPP sphere rotations drawn so far
  qmc::SweepTask* d_task = nullptr;
  double* d_ur = nullptr, *d_delta = nullptr, *d_trace = nullptr;
  size_t cap_rng = 0, cap_trace = 0;
  double* d_displ = nullptr;
  double* d_step  = nullptr; // [W][4] qmc_step inputs: ur, delta xyz
  int* d_flags    = nullptr;
  double* d_rows  = nullptr;
  size_t cap_rows = 0;
  long long* d_timers = nullptr;
  bool tc_capable = false; // FP32, >= 128 threads, k <= 32, determinant on
  bool use_tc     = false; // Woodbury flushes on the tensor cores
  int max_moves   = 1; // moves the fused sweep evaluates together (qmc_walkers_set_move_batching)
  // the sweep's schedule (qmc_walkers_set_schedule) and the work-queue
  // form's counters and hand-over ring (launch_sweep_queue)
  int sched_mode   = QMC_SCHED_AUTO;
  int sched_unit   = QMC_SCHED_UNIT_DEFAULT;
  int sched_ctas   = 0;
  int* d_sched     = nullptr;
  size_t cap_sched = 0;
  // CTAs of the work-queue launch for the settings in sched_key (the
  // occupancy query runs once per change of settings, not per sweep call)
  mutable int sched_key[6] = {0, 0, 0, 0, 0, 0};
  mutable int sched_cached = 0;
  // a request-loop job's batch: device memory from the server's pool,
  // allocated and freed stream-ordered on its stream (else both null)
  cudaStream_t alloc_stream = nullptr;
  cudaMemPool_t alloc_pool  = nullptr;
};

// the tensor-core flush keeps (Binv V)^T as 32-row hi/lo tiles of up to 32
// delays: 2 x 32 floats per padded orbital and walker
// the tensor-core flush's image of (Binv V)^T hi / lo tiles for delay ranks
// up to k: npad / 32 tiles of 2 x 32 x Kd floats
inline size_t tc_image_floats(int npad, int k) { return (size_t)2 * (k <= 32 ? 32 : 64) * npad; }

// device error bits of a batch -> status (and message); synchronises
int device_status(qmc_walkers* w);
// device error bits -> status (and message)
int status_from_bits(unsigned bits);
// SPO matrices + FP64 inverse and log-det of every walker (evaluateLog's
// determinant part, also the periodic refresh)
int recompute_dets(qmc_walkers* w);
// device bytes a batch of W walkers with delay k of system s will hold,
// including the lazily allocated FP64 inverse scratch
size_t walkers_footprint(qmc_system* s, int W, int k);
// the sweep's SweepTask of a batch (device RNG streams)
qmc::SweepTask sweep_task(qmc_walkers* w, int first_block);
// request-loop batches: device memory stream-ordered from `pool` on `st`
// (freed the same way by qmc_walkers_destroy); initialisation and
// evaluateLog enqueued on the batch's stream without waiting
int walkers_create_pooled(qmc_system* s, int n_walkers, int delay_rank, cudaStream_t st, cudaMemPool_t pool,
                          qmc_walkers** out);
int walkers_init_random(qmc_walkers* w, const uint32_t* seeds, bool sync);
int evaluate_log_launch(qmc_walkers* w);
