// sweep.cu -- the fused persistent PbyP sweep kernel (one CTA per walker).
//
// One launch = one MC step of miniqmc's driver loop (miniqmc.cpp:406-468)
// for every walker of every task in the launch: per substep the walker's
// random stream is advanced (N uniforms, 3N normals), the N electrons are
// moved in order (evalGrad, makeMove, ratioGrad, threshold accept, the
// delayed-update bookkeeping and its in-CTA Woodbury flush), and the
// remaining delayed rows are flushed (completeUpdates); after the substeps
// donePbyP + evaluateGL.  Walkers never exchange data, so CTAs never wait
// on one another.
#include "device.cuh"

namespace qmc
{
// EPOCH: the moves are evaluated an epoch at a time (do_epoch: a run of
// rejected moves and the accepted move that ends it, up to the task's
// max_moves), else one at a time (do_move); the three-body Jastrow runs one
// at a time.
template <typename T, bool HAS_J3, bool EPOCH>
__global__ void __launch_bounds__(256, 3) sweep_kernel(const SweepTask* __restrict__ tasks, int n_tasks, int n_substeps,
                                                    double accept_thr, int tc)
{
  __shared__ SysSmem<T> ss;
  __shared__ MoveSmem m;
  __shared__ SplineSmem<T> sp;
  // the walker's view (its arrays' device pointers) in shared memory rather
  // than in registers: the move code reads each pointer when it needs it
  __shared__ WV<T> wv;
  extern __shared__ __align__(16) unsigned char dyn[];
  int t = 0;
  while (t + 1 < n_tasks && (int)blockIdx.x >= tasks[t + 1].first_block)
    ++t;
  const SweepTask& task = tasks[t];
  const int w           = blockIdx.x - task.first_block;
  if (w >= task.dw.W)
    return;
  const DevSystem* sys = task.sys;
  if (threadIdx.x == 0)
    wv = make_wv<T>(task.dw, w);
  load_sys(sys, ss); // ends with a barrier
  const int N   = wv.N;
  const T* ions = (const T*)sys->ion_soa;
  long long acc = 0;
  const bool DET = ss.comp & QMC_WF_DET;
  // dynamic shared memory: [Binv of the active spin (k x k FP64)][flush
  // scratch, or between flushes the J2 candidate lists / the J3 move scratch]
  const int k = wv.k;
  T* smem     = reinterpret_cast<T*>(dyn + bsm_bytes(k));
  auto load_binv = [&](int spin) {
    const double* g = wv.Binv + (size_t)spin * k * k;
    double* b       = reinterpret_cast<double*>(dyn);
    for (int i = threadIdx.x; i < k * k; i += blockDim.x)
      b[i] = g[i];
    __syncthreads(); // every thread has read wv.bsm of the previous spin
    if (threadIdx.x == 0)
    {
      wv.bsm      = b;
      wv.bsm_spin = spin;
    }
    __syncthreads();
  };
  if (threadIdx.x == 0)
  {
    m.timing = task.timers != nullptr;
    m.tstamp = clock64();
    for (int p = 0; p < NPHASE; ++p)
      m.tacc[p] = 0;
  }
  if constexpr (sizeof(T) == 4)
    tc_begin(m, tc && task.tc && DET, task.dw.wait_cycles);
  else
    tc_none(m);
  for (int l = 0; l < n_substeps && !m.tc_abort; ++l)
  {
    const double* urp;
    const double* dp;
    if (task.rng_mode == QMC_RNG_DEVICE)
    {
      rng_substep(wv, N);
      urp = wv.ur;
      dp  = wv.delta;
      phase_mark(m, PH_RANDOM);
    }
    else
    {
      urp = task.ur + ((size_t)w * n_substeps + l) * N;
      dp  = task.delta + ((size_t)w * n_substeps + l) * 3 * N;
    }
    if (DET)
      load_binv(0);
    for (int iel = 0; iel < N;)
    {
      if (DET && iel == ss.n_up)
      {
        // completeUpdates of the up determinant, taken as soon as its last
        // electron has moved: the down-spin moves never read it, so this is
        // the same arithmetic as flushing both at the end of the substep
        flush(wv, m, 0, smem);
        load_binv(1);
      }
      double* tr = task.trace ? task.trace + (((size_t)w * n_substeps + l) * N + iel) * 8 : nullptr;
      if constexpr (EPOCH)
      {
        // an epoch stays within one spin's moves
        const int lim = iel < ss.n_up ? ss.n_up : N;
        auto* esp     = reinterpret_cast<SplineSmem<T>*>(reinterpret_cast<unsigned char*>(smem) + j2_list_bytes());
        const int G   = do_epoch<T>(ss, sys, wv, m, esp, ions, iel, lim, task.max_moves, accept_thr, urp + iel,
                                  dp + 3 * iel, tr, smem, task.prefetch);
        iel += G;
      }
      else
      {
        do_move<T, HAS_J3>(ss, sys, wv, m, sp, ions, iel, accept_thr, urp + iel, dp + 3 * iel, tr, smem,
                           task.prefetch && iel + 1 < N);
        ++iel;
      }
      acc += m.accept ? 1 : 0;
      __syncthreads(); // m.accept is rewritten by the next move
      if (m.tc_abort)
        break;
    }
    phase_mark(m, PH_REDUCE);
    if (DET)
    {
      flush(wv, m, 0, smem);
      flush(wv, m, 1, smem);
      __syncthreads();
      if (threadIdx.x == 0)
        wv.bsm = nullptr;
      __syncthreads();
    }
    phase_mark(m, PH_COMPLETE);
  }
  if constexpr (sizeof(T) == 4)
    tc_end(m);
  evaluate_gl(ss, wv, m, task.dw.logpsi + w);
  phase_mark(m, PH_GL);
  if (threadIdx.x == 0)
  {
    // every move of the sweep was a ratioGrad one (DiracDeterminant's
    // UpdateMode ORB_PBYP_PARTIAL)
    wv.ms->partial[0] = wv.ms->partial[1] = 1;
    wv.ms->j_partial                      = 1;
    task.dw.accepted[w] += acc;
    if (task.timers)
      for (int p = 0; p < NPHASE; ++p)
        task.timers[(size_t)w * NPHASE + p] += m.tacc[p];
  }
}

// ------------------------------------------------- queue schedule -----
// With more walkers than SMs the static launch leaves some SMs with one
// walker more than others (512 walkers on 148 SMs: 68 SMs with four, 80
// with three), and the SMs with four set the step while the others idle at
// its end.  The queue form runs every resident CTA slot and cuts each
// walker's step into units of at most `unit` consecutive moves of one spin.
// The spare slots (592 - 512 at that size) are CTAs waiting for a walker.
// When a unit ends on an SM where no CTA waits, its SM runs one walker more
// than the others: the CTA hands the walker to the CTA that has waited
// longest (on a quieter SM) and becomes that SM's waiting CTA; where a CTA
// waits already, the walker goes on in place.  So walkers move from busier
// to quieter SMs only, the roles rotate, every walker spends about the same
// share of its step on busier SMs, and no walker waits for a CTA.
//
// Hand-overs go through a ring: a CTA without a walker takes a ticket; the
// first W tickets are the walkers' first units, and ticket t >= W waits
// (bounded) for ring slot t, which hand-over t - W fills.  A waiting CTA
// leaves when every unit of the launch has ended (or the launch stops), so
// every wait ends; the bound only catches a launch in which no unit has
// ended for kQueueWaitNs.
//
// Between units the walker's state is all in global memory: a unit that
// ends a spin flushes its delayed rows (completeUpdates of that spin, as the
// static form does on the first move of the other spin or at the end of the
// substep), and one that ends inside a spin writes the shared-memory copy of
// that spin's Binv back.  The moves' arithmetic and order are those of the
// static form, so the two give the same results bit for bit.
//
// sched (device ints, zero before the launch; QUEUE_HDR + QUEUE_SMS + W +
// CTAs + units): [0] hand-overs, [1] tickets taken, [2] the stop flag (a
// timed-out wait or an aborted tensor-core flush), [3] units ended; then the
// CTAs waiting on each SM, the units done by each walker, and the ring
// (1 + the walker handed over with each ticket).
// the waits poll with relaxed loads and take one acquire fence when they
// end: an acquire at GPU scope also drops the SM's L1 lines, which the
// walkers running beside a waiting CTA still use
__device__ __forceinline__ int ld_relaxed_gpu(const int* p)
{
  int v;
  asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void fence_acquire_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }
__device__ __forceinline__ void st_release_gpu(int* p, int v)
{
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int sm_id()
{
  int v;
  asm volatile("mov.u32 %0, %%smid;" : "=r"(v));
  return v;
}
// a ticket's wait for its hand-over gives up once no unit of the launch has
// ended for this long (a unit is a few milliseconds of moves at the sizes
// this runs)
constexpr unsigned long long kQueueWaitNs = 10ull * 1000 * 1000 * 1000;

// MAXT: the largest block the instantiation takes.  Three CTAs per SM
// either way: at up to 192 threads that leaves 112 registers a thread (the
// kernel takes 96 and spills a third of what it spills at 80), which at 512
// NiO-128 walkers measured 141 ms per launch against 161.5 ms for four CTAs
// per SM at 80 registers (and 154 ms for two CTAs per SM at 168 registers).
template <typename T, bool HAS_J3, bool EPOCH, int MAXT>
__global__ void __launch_bounds__(MAXT, 3) sweep_queue_kernel(const SweepTask* __restrict__ tasks, int n_substeps,
                                                           double accept_thr, int tc, int unit, int* sched)
{
  __shared__ SysSmem<T> ss;
  __shared__ MoveSmem m;
  __shared__ SplineSmem<T> sp;
  __shared__ WV<T> wv;
  // the unit in hand: walker, substep, spin, first and end move, index j
  __shared__ int q_w, q_l, q_spin, q_i0, q_i1, q_j, q_last;
  // thread 0's hand-over state: the walker this CTA goes on with (or -1),
  // and whether it is already counted among its SM's waiting CTAs
  __shared__ int q_keep, q_waiting;
  extern __shared__ __align__(16) unsigned char dyn[];
  const SweepTask& task = tasks[0];
  const DevSystem* sys  = task.sys;
  load_sys(sys, ss); // ends with a barrier
  const int W = task.dw.W, N = task.dw.N, nup = ss.n_up;
  const int nu0 = (nup + unit - 1) / unit, nus = nu0 + (N - nup + unit - 1) / unit;
  const int total = W * n_substeps * nus;
  int* waiting    = sched + QUEUE_HDR;              // [QUEUE_SMS] CTAs waiting per SM
  int* units_done = waiting + QUEUE_SMS;            // [W]
  int* ring       = units_done + W;                 // [CTAs + units]
  const int sm    = min(sm_id(), QUEUE_SMS - 1);
  const T* ions   = (const T*)sys->ion_soa;
  const bool DET  = ss.comp & QMC_WF_DET;
  const int k     = task.dw.k;
  T* smem         = reinterpret_cast<T*>(dyn + bsm_bytes(k));
  if (threadIdx.x == 0)
  {
    m.timing = task.timers != nullptr;
    for (int p = 0; p < NPHASE; ++p)
      m.tacc[p] = 0;
    q_keep    = -1;
    q_waiting = 0;
  }
  if constexpr (sizeof(T) == 4)
    tc_begin(m, tc && task.tc && DET, task.dw.wait_cycles);
  else
    tc_none(m);
  for (;;)
  {
    if (threadIdx.x == 0)
    {
      int w = q_keep;
      if (w < 0)
      {
        // a ticket: the first W are the walkers' first units, each later
        // one waits for the walker handed over in ring slot `ticket`
        int t = total + (int)gridDim.x;
        if (!m.tc_abort && !ld_relaxed_gpu(sched + 2))
          t = atomicAdd(sched + 1, 1);
        if (t < W)
          w = t;
        else if (t < total + (int)gridDim.x)
        {
          if (!q_waiting)
            atomicAdd(waiting + sm, 1);
          unsigned long long t0 = global_ns();
          int seen              = ld_relaxed_gpu(sched + 3);
          unsigned ns           = 64;
          int v;
          while ((v = ld_relaxed_gpu(ring + t)) == 0)
          {
            const int now = ld_relaxed_gpu(sched + 3);
            if (ld_relaxed_gpu(sched + 2) || now >= total)
              break; // stopped, or every unit of the launch is done
            if (now != seen)
            {
              seen = now;
              t0   = global_ns();
            }
            else if (global_ns() - t0 > kQueueWaitNs)
            {
              atomicOr(task.dw.status, DEV_ERR_TIMEOUT);
              atomicExch(sched + 2, 1);
              break;
            }
            __nanosleep(ns);
            ns = min(2 * ns, 2048u);
          }
          atomicSub(waiting + sm, 1);
          // the hand-over's release pairs with this fence: the walker's
          // state, and the stop flag a unit that stopped the launch raised
          // before it handed its walker on (that walker is not moved on)
          fence_acquire_gpu();
          if (v && !ld_relaxed_gpu(sched + 2))
            w = v - 1;
        }
      }
      q_waiting = 0;
      q_keep    = -1;
      q_j       = -1;
      if (w >= 0)
      {
        const int j = units_done[w]; // published with the hand-over
        const int l = j / nus, r = j - l * nus;
        q_w    = w;
        q_j    = j;
        q_l    = l;
        q_spin = r < nu0 ? 0 : 1;
        q_i0   = r < nu0 ? r * unit : nup + (r - nu0) * unit;
        q_i1   = r < nu0 ? min(q_i0 + unit, nup) : min(q_i0 + unit, N);
        q_last = (l == n_substeps - 1 && r == nus - 1) ? 1 : 0;
        wv       = make_wv<T>(task.dw, w);
        m.tstamp = clock64();
      }
    }
    __syncthreads();
    if (q_j < 0)
      break;
    const int w = q_w, l = q_l, spin = q_spin;
    const double* urp;
    const double* dp;
    if (task.rng_mode == QMC_RNG_DEVICE)
    {
      // the substep's random numbers, drawn by its first unit
      if (q_i0 == 0)
      {
        rng_substep(wv, N);
        phase_mark(m, PH_RANDOM);
      }
      urp = wv.ur;
      dp  = wv.delta;
    }
    else
    {
      urp = task.ur + ((size_t)w * n_substeps + l) * N;
      dp  = task.delta + ((size_t)w * n_substeps + l) * 3 * N;
    }
    if (DET)
    {
      const double* g = wv.Binv + (size_t)spin * k * k;
      double* b       = reinterpret_cast<double*>(dyn);
      for (int i = threadIdx.x; i < k * k; i += blockDim.x)
        b[i] = g[i];
      __syncthreads();
      if (threadIdx.x == 0)
      {
        wv.bsm      = b;
        wv.bsm_spin = spin;
      }
      __syncthreads();
    }
    int acc = 0;
    for (int iel = q_i0; iel < q_i1;)
    {
      double* tr = task.trace ? task.trace + (((size_t)w * n_substeps + l) * N + iel) * 8 : nullptr;
      if constexpr (EPOCH)
      {
        auto* esp   = reinterpret_cast<SplineSmem<T>*>(reinterpret_cast<unsigned char*>(smem) + j2_list_bytes());
        const int G = do_epoch<T>(ss, sys, wv, m, esp, ions, iel, q_i1, task.max_moves, accept_thr, urp + iel,
                                  dp + 3 * iel, tr, smem, task.prefetch);
        iel += G;
      }
      else
      {
        do_move<T, HAS_J3>(ss, sys, wv, m, sp, ions, iel, accept_thr, urp + iel, dp + 3 * iel, tr, smem,
                           task.prefetch && iel + 1 < N);
        ++iel;
      }
      acc += m.accept ? 1 : 0;
      __syncthreads(); // m.accept is rewritten by the next move
      if (m.tc_abort)
        break;
    }
    if (DET)
    {
      phase_mark(m, PH_REDUCE);
      if (q_i1 == N || (spin == 0 && q_i1 == nup))
      {
        // the spin's last unit: completeUpdates of its determinant (and of
        // both at the end of the substep, as the static form does)
        flush(wv, m, 0, smem);
        if (q_i1 == N)
          flush(wv, m, 1, smem);
      }
      else
      {
        double* g = wv.Binv + (size_t)spin * k * k;
        for (int i = threadIdx.x; i < k * k; i += blockDim.x)
          g[i] = wv.bsm[i];
      }
      __syncthreads();
      if (threadIdx.x == 0)
        wv.bsm = nullptr;
      __syncthreads();
      phase_mark(m, PH_COMPLETE);
    }
    if (q_last && !m.tc_abort)
    {
      evaluate_gl(ss, wv, m, task.dw.logpsi + w);
      phase_mark(m, PH_GL);
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
      if (q_last)
      {
        wv.ms->partial[0] = wv.ms->partial[1] = 1;
        wv.ms->j_partial                      = 1;
      }
      task.dw.accepted[w] += acc;
      if (task.timers)
        for (int p = 0; p < NPHASE; ++p)
        {
          task.timers[(size_t)w * NPHASE + p] += m.tacc[p];
          m.tacc[p] = 0;
        }
      units_done[w] = q_j + 1;
      if (m.tc_abort)
        atomicExch(sched + 2, 1);
      if (!q_last)
      {
        if (!m.tc_abort && atomicCAS(waiting + sm, 0, 1) != 0)
          q_keep = w; // another CTA of this SM waits already: go on here
        else
        {
          // no CTA of this SM waits: hand the walker to the one that has
          // waited longest (on a quieter SM) and wait here in its place
          __threadfence();
          st_release_gpu(ring + W + atomicAdd(sched, 1), w + 1);
          q_waiting = !m.tc_abort;
        }
      }
      __threadfence();
      atomicAdd(sched + 3, 1);
    }
  }
  if constexpr (sizeof(T) == 4)
    tc_end(m);
}

// qmc_step: the fused move of one electron for every walker, with the same
// device code as one iteration of the sweep (do_move).  The inverse's
// delayed block stays in global memory between calls and flushes run on the
// CUDA cores, as in the per-call verbs.
template <typename T, bool HAS_J3>
__global__ void __launch_bounds__(256, 3) step_kernel(const DevSystem* __restrict__ sys, DevWalkers dw, int iel,
                                                   double accept_thr, const double* __restrict__ in,
                                                   int* __restrict__ out)
{
  __shared__ SysSmem<T> ss;
  __shared__ MoveSmem m;
  __shared__ SplineSmem<T> sp;
  // the walker's view in shared memory rather than registers, as in the sweep
  __shared__ WV<T> wv;
  extern __shared__ __align__(16) unsigned char dyn[];
  const int w = blockIdx.x;
  if (threadIdx.x == 0)
    wv = make_wv<T>(dw, w);
  load_sys(sys, ss); // ends with a barrier
  const T* ions     = (const T*)sys->ion_soa;
  const double* inw = in + (size_t)4 * w;
  if (threadIdx.x == 0)
  {
    m.tc_on    = 0;
    m.tc_abort = 0;
    m.timing   = 0;
  }
  do_move<T, HAS_J3>(ss, sys, wv, m, sp, ions, iel, accept_thr, inw, inw + 1, nullptr, reinterpret_cast<T*>(dyn),
                     false);
  if (threadIdx.x == 0)
  {
    out[w] = m.accept;
    dw.accepted[w] += m.accept;
  }
}

template <typename T> static void launch_step_t(bool j3, const DevSystem* sys, const DevWalkers& dw, int iel,
                                                double accept, const double* in, int* out, int threads,
                                                cudaStream_t st)
{
  const size_t bytes =
      std::max(std::max(flush_smem_bytes<T>(), sizeof(J3Smem<T>)), j2_list_bytes() + sizeof(double));
  if (j3)
  {
    cudaFuncSetAttribute(step_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    step_kernel<T, true><<<dw.W, threads, bytes, st>>>(sys, dw, iel, accept, in, out);
  }
  else
  {
    cudaFuncSetAttribute(step_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    step_kernel<T, false><<<dw.W, threads, bytes, st>>>(sys, dw, iel, accept, in, out);
  }
}

cudaError_t launch_step(bool fp32, bool j3, const DevSystem* sys, const DevWalkers& dw, int iel, double accept,
                        const double* in, int* out, int threads, cudaStream_t st)
{
  if (dw.k > MAXK)
    return cudaErrorInvalidValue;
  if (fp32)
    launch_step_t<float>(j3, sys, dw, iel, accept, in, out, threads, st);
  else
    launch_step_t<double>(j3, sys, dw, iel, accept, in, out, threads, st);
  return cudaGetLastError();
}

template <typename T, bool HAS_J3, bool EPOCH> static void set_smem_attr(size_t bytes)
{
  static size_t done = 0;
  if (bytes > done)
  {
    cudaFuncSetAttribute(sweep_kernel<T, HAS_J3, EPOCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    done = bytes;
  }
}
template <typename T, bool HAS_J3, bool EPOCH, int MAXT> static void set_queue_smem_attr(size_t bytes)
{
  static size_t done = 0;
  if (bytes > done)
  {
    cudaFuncSetAttribute(sweep_queue_kernel<T, HAS_J3, EPOCH, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)bytes);
    done = bytes;
  }
}
template <typename T>
static void launch_sweep_t(bool j3, bool epoch, size_t bytes, const SweepTask* d_tasks, int n_tasks,
                           int total_blocks, int n_substeps, double accept, int threads, cudaStream_t st, int tc)
{
  if (j3)
  {
    set_smem_attr<T, true, false>(bytes);
    sweep_kernel<T, true, false><<<total_blocks, threads, bytes, st>>>(d_tasks, n_tasks, n_substeps, accept, tc);
  }
  else if (epoch)
  {
    set_smem_attr<T, false, true>(bytes);
    sweep_kernel<T, false, true><<<total_blocks, threads, bytes, st>>>(d_tasks, n_tasks, n_substeps, accept, tc);
  }
  else
  {
    set_smem_attr<T, false, false>(bytes);
    sweep_kernel<T, false, false><<<total_blocks, threads, bytes, st>>>(d_tasks, n_tasks, n_substeps, accept, tc);
  }
}

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

cudaError_t launch_sweep(bool fp32, const SweepTask* d_tasks, int n_tasks, int total_blocks, int n_substeps,
                         double accept, int threads, int max_npad, int max_k, cudaStream_t st, bool tc, bool j3,
                         bool epoch)
{
  (void)max_npad;
  if (max_k > MAXK || (tc && (!fp32 || threads < 128)))
    return cudaErrorInvalidValue;
  epoch = epoch && !j3;
  if (fp32)
    launch_sweep_t<float>(j3, epoch, sweep_smem_bytes<float>(threads, max_k, tc, j3, epoch), d_tasks, n_tasks,
                          total_blocks, n_substeps, accept, threads, st, tc ? 1 : 0);
  else
    launch_sweep_t<double>(j3, epoch, sweep_smem_bytes<double>(threads, max_k, false, j3, epoch), d_tasks, n_tasks,
                           total_blocks, n_substeps, accept, threads, st, 0);
  return cudaGetLastError();
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
template <typename T, bool HAS_J3, bool EPOCH, int MAXT> static int queue_occupancy_t(int threads, size_t bytes)
{
  set_queue_smem_attr<T, HAS_J3, EPOCH, MAXT>(bytes);
  return occupancy_of(sweep_queue_kernel<T, HAS_J3, EPOCH, MAXT>, threads, bytes);
}
template <typename T, bool HAS_J3, bool EPOCH> static int occupancy_t(int threads, size_t bytes, bool queue)
{
  if (queue)
    return threads <= 192 ? queue_occupancy_t<T, HAS_J3, EPOCH, 192>(threads, bytes)
                          : queue_occupancy_t<T, HAS_J3, EPOCH, 256>(threads, bytes);
  set_smem_attr<T, HAS_J3, EPOCH>(bytes);
  return occupancy_of(sweep_kernel<T, HAS_J3, EPOCH>, threads, bytes);
}

int sweep_occupancy(bool fp32, int threads, int max_k, bool tc, bool j3, bool epoch, bool queue)
{
  epoch = epoch && !j3;
  if (fp32)
  {
    const size_t b = sweep_smem_bytes<float>(threads, max_k, tc, j3, epoch);
    return j3      ? occupancy_t<float, true, false>(threads, b, queue)
           : epoch ? occupancy_t<float, false, true>(threads, b, queue)
                   : occupancy_t<float, false, false>(threads, b, queue);
  }
  const size_t b = sweep_smem_bytes<double>(threads, max_k, false, j3, epoch);
  return j3      ? occupancy_t<double, true, false>(threads, b, queue)
         : epoch ? occupancy_t<double, false, true>(threads, b, queue)
                 : occupancy_t<double, false, false>(threads, b, queue);
}

template <typename T, bool HAS_J3, bool EPOCH, int MAXT>
static void queue_launch_tt(size_t bytes, const SweepTask* d_task, int ctas, int n_substeps, double accept,
                            int threads, cudaStream_t st, int tc, int unit, int* sched)
{
  set_queue_smem_attr<T, HAS_J3, EPOCH, MAXT>(bytes);
  sweep_queue_kernel<T, HAS_J3, EPOCH, MAXT>
      <<<ctas, threads, bytes, st>>>(d_task, n_substeps, accept, tc, unit, sched);
}
template <typename T, bool HAS_J3, bool EPOCH>
static void queue_launch_t(size_t bytes, const SweepTask* d_task, int ctas, int n_substeps, double accept,
                           int threads, cudaStream_t st, int tc, int unit, int* sched)
{
  if (threads <= 192)
    queue_launch_tt<T, HAS_J3, EPOCH, 192>(bytes, d_task, ctas, n_substeps, accept, threads, st, tc, unit, sched);
  else
    queue_launch_tt<T, HAS_J3, EPOCH, 256>(bytes, d_task, ctas, n_substeps, accept, threads, st, tc, unit, sched);
}
template <typename T>
static void launch_queue_t(bool j3, bool epoch, size_t bytes, const SweepTask* d_task, int ctas, int n_substeps,
                           double accept, int threads, cudaStream_t st, int tc, int unit, int* sched)
{
  if (j3)
    queue_launch_t<T, true, false>(bytes, d_task, ctas, n_substeps, accept, threads, st, tc, unit, sched);
  else if (epoch)
    queue_launch_t<T, false, true>(bytes, d_task, ctas, n_substeps, accept, threads, st, tc, unit, sched);
  else
    queue_launch_t<T, false, false>(bytes, d_task, ctas, n_substeps, accept, threads, st, tc, unit, sched);
}

cudaError_t launch_sweep_queue(bool fp32, const SweepTask* d_task, int ctas, int n_substeps, double accept,
                               int threads, int max_k, cudaStream_t st, bool tc, bool j3, bool epoch, int unit,
                               int* sched)
{
  if (max_k > MAXK || (tc && (!fp32 || threads < 128)) || ctas < 1 || unit < 1 || !sched)
    return cudaErrorInvalidValue;
  epoch = epoch && !j3;
  if (fp32)
    launch_queue_t<float>(j3, epoch, sweep_smem_bytes<float>(threads, max_k, tc, j3, epoch), d_task, ctas,
                          n_substeps, accept, threads, st, tc ? 1 : 0, unit, sched);
  else
    launch_queue_t<double>(j3, epoch, sweep_smem_bytes<double>(threads, max_k, false, j3, epoch), d_task, ctas,
                           n_substeps, accept, threads, st, 0, unit, sched);
  return cudaGetLastError();
}

} // namespace qmc
