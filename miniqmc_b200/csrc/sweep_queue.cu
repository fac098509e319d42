// sweep_queue.cu -- the fused sweep in the work-queue form, over a list of
// tasks (one batch, or the batches of a group or of the request loop):
// every resident CTA slot takes units of a few moves of a walker, walkers
// passing between CTAs (and SMs) between their units.
#include "sweep.cuh"

namespace qmc
{
// ------------------------------------------------- queue schedule -----
// With more walkers than SMs the static launch leaves some SMs with one
// walker more than others (512 walkers on 148 SMs at four per SM: 68 SMs
// with four, 80 with three), and the SMs with four set the step while the
// others idle at its end.  The queue form runs every resident CTA slot and
// cuts each walker's step into units of at most `unit` consecutive moves of
// one spin.  Where slots outnumber walkers, the spare slots are CTAs waiting
// for a walker.  When a unit ends on an SM where no CTA waits, its SM runs
// one walker more than the others: the CTA hands the walker to the CTA
// that has waited longest (on a quieter SM) and becomes that SM's waiting
// CTA; where a CTA waits already, the walker goes on in place.  So walkers
// move from busier to quieter SMs only, the roles rotate, every walker
// spends about the same share of its step on busier SMs, and no walker
// waits for a CTA.  Where walkers outnumber slots, every unit end hands its
// walker on and the walkers take turns on the slots.
//
// Hand-overs go through a ring: a CTA without a walker takes a ticket; the
// first n_walkers tickets are the walkers' first units, and ticket
// t >= n_walkers waits (bounded) for ring slot t, which hand-over
// t - n_walkers fills.  A waiting CTA leaves when every unit of the launch
// has ended (or the launch stops), so every wait ends; the bound only
// catches a launch in which no unit has ended for kQueueWaitNs.
//
// Between units the walker's state is all in global memory: a unit that
// ends a spin flushes its delayed rows (completeUpdates of that spin, as the
// static form does on the first move of the other spin or at the end of the
// substep), and one that ends inside a spin writes the shared-memory copy of
// that spin's Binv back.  The moves' arithmetic and order are those of the
// static form, so the two give the same results bit for bit.
//
// Walkers are numbered over all tasks (a task's first_block is its first).
// sched (device ints, zero before the launch; sweep_queue_words of them):
// [0] hand-overs, [1] tickets taken, [2] the stop flag (a timed-out wait or
// an aborted tensor-core flush), [3] units ended; then the CTAs waiting on
// each SM, the units done by each walker, and the ring (1 + the walker
// handed over with each ticket).
//
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
__global__ void __launch_bounds__(MAXT, 3)
    sweep_queue_kernel(const SweepTask* __restrict__ tasks, int n_tasks, int n_walkers, int total, int n_substeps,
                       double accept_thr, int tc, int unit, int* sched)
{
  __shared__ SysSmem<T> ss;
  __shared__ MoveSmem m;
  __shared__ SplineSmem<T> sp;
  __shared__ WV<T> wv;
  // the unit in hand: task, walker (in its task), substep, spin, first and
  // end move, index j, and its task's electrons and up electrons
  __shared__ int q_task, q_w, q_l, q_spin, q_i0, q_i1, q_j, q_last, q_N, q_nup;
  // thread 0's hand-over state: the walker (over all tasks) this CTA goes on
  // with (or -1), and whether it is already counted among its SM's waiting
  // CTAs; the task whose system is in `ss`; whether this CTA holds tensor
  // memory
  __shared__ int q_keep, q_waiting, q_loaded, q_tc_alloc;
  extern __shared__ __align__(16) unsigned char dyn[];
  int* waiting    = sched + QUEUE_HDR;   // [QUEUE_SMS] CTAs waiting per SM
  int* units_done = waiting + QUEUE_SMS; // [n_walkers]
  int* ring       = units_done + n_walkers; // [CTAs + units]
  const int sm    = min(sm_id(), QUEUE_SMS - 1);
  if (threadIdx.x == 0)
  {
    for (int p = 0; p < NPHASE; ++p)
      m.tacc[p] = 0;
    q_keep    = -1;
    q_waiting = 0;
    q_loaded  = -1;
  }
  if constexpr (sizeof(T) == 4)
    tc_begin(m, tc, tasks[0].dw.wait_cycles);
  else
    tc_none(m);
  if (threadIdx.x == 0)
    q_tc_alloc = m.tc_on;
  for (;;)
  {
    if (threadIdx.x == 0)
    {
      int g = q_keep;
      if (g < 0)
      {
        // a ticket: the first n_walkers are the walkers' first units, each
        // later one waits for the walker handed over in ring slot `ticket`
        int t = total + (int)gridDim.x;
        if (!m.tc_abort && !ld_relaxed_gpu(sched + 2))
          t = atomicAdd(sched + 1, 1);
        if (t < n_walkers)
          g = t;
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
              for (int i = 0; i < n_tasks; ++i)
                atomicOr(tasks[i].dw.status, DEV_ERR_TIMEOUT);
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
            g = v - 1;
        }
      }
      q_waiting = 0;
      q_keep    = -1;
      q_j       = -1;
      if (g >= 0)
      {
        int ti = 0;
        while (ti + 1 < n_tasks && g >= tasks[ti + 1].first_block)
          ++ti;
        const SweepTask& tk = tasks[ti];
        const int w = g - tk.first_block, N = tk.dw.N, nup = tk.sys->n_up;
        const int nu0 = (nup + unit - 1) / unit, nus = nu0 + (N - nup + unit - 1) / unit;
        const int j = units_done[g]; // published with the hand-over
        const int l = j / nus, r = j - l * nus;
        q_task = ti;
        q_w    = w;
        q_j    = j;
        q_l    = l;
        q_N    = N;
        q_nup  = nup;
        q_spin = r < nu0 ? 0 : 1;
        q_i0   = r < nu0 ? r * unit : nup + (r - nu0) * unit;
        q_i1   = r < nu0 ? min(q_i0 + unit, nup) : min(q_i0 + unit, N);
        q_last = (l == n_substeps - 1 && r == nus - 1) ? 1 : 0;
        wv     = make_wv<T>(tk.dw, w);
        // the unit's flushes on the tensor cores where its task asks
        m.tc_on    = q_tc_alloc && tk.tc && (tk.sys->comp & QMC_WF_DET);
        m.tc_limit = tk.dw.wait_cycles;
        m.timing   = tk.timers != nullptr;
        m.tstamp   = clock64();
      }
    }
    __syncthreads();
    if (q_j < 0)
      break;
    if (q_task != q_loaded)
    {
      load_sys(tasks[q_task].sys, ss); // ends with a barrier
      if (threadIdx.x == 0)
        q_loaded = q_task;
    }
    const SweepTask& task = tasks[q_task];
    const DevSystem* sys  = task.sys;
    const int w = q_w, l = q_l, spin = q_spin, N = q_N, k = task.dw.k;
    const T* ions  = (const T*)sys->ion_soa;
    const bool DET = ss.comp & QMC_WF_DET;
    T* smem        = reinterpret_cast<T*>(dyn + bsm_bytes(k));
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
      if (q_i1 == N || (spin == 0 && q_i1 == q_nup))
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
      const int g = task.first_block + w;
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
      units_done[g] = q_j + 1;
      if (m.tc_abort)
        atomicExch(sched + 2, 1);
      if (!q_last)
      {
        if (!m.tc_abort && atomicCAS(waiting + sm, 0, 1) != 0)
          q_keep = g; // another CTA of this SM waits already: go on here
        else
        {
          // no CTA of this SM waits: hand the walker to the one that has
          // waited longest (on a quieter SM) and wait here in its place
          __threadfence();
          st_release_gpu(ring + n_walkers + atomicAdd(sched, 1), g + 1);
          q_waiting = !m.tc_abort;
        }
      }
      __threadfence();
      atomicAdd(sched + 3, 1);
    }
  }
  if constexpr (sizeof(T) == 4)
  {
    if (threadIdx.x == 0)
      m.tc_on = q_tc_alloc; // tc_end frees what tc_begin took
    tc_end(m);
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
template <typename T, bool HAS_J3, bool EPOCH, int MAXT> static int queue_occupancy_t(int threads, size_t bytes)
{
  set_queue_smem_attr<T, HAS_J3, EPOCH, MAXT>(bytes);
  return occupancy_of(sweep_queue_kernel<T, HAS_J3, EPOCH, MAXT>, threads, bytes);
}
template <typename T, bool HAS_J3, bool EPOCH> static int queue_occupancy_for(int threads, size_t bytes)
{
  return threads <= 192 ? queue_occupancy_t<T, HAS_J3, EPOCH, 192>(threads, bytes)
                        : queue_occupancy_t<T, HAS_J3, EPOCH, 256>(threads, bytes);
}

int sweep_queue_occupancy(bool fp32, int threads, int max_k, bool tc, bool j3, bool epoch)
{
  epoch = epoch && !j3;
  if (fp32)
  {
    const size_t b = sweep_smem_bytes<float>(threads, max_k, tc, j3, epoch);
    return j3      ? queue_occupancy_for<float, true, false>(threads, b)
           : epoch ? queue_occupancy_for<float, false, true>(threads, b)
                   : queue_occupancy_for<float, false, false>(threads, b);
  }
  const size_t b = sweep_smem_bytes<double>(threads, max_k, false, j3, epoch);
  return j3      ? queue_occupancy_for<double, true, false>(threads, b)
         : epoch ? queue_occupancy_for<double, false, true>(threads, b)
                 : queue_occupancy_for<double, false, false>(threads, b);
}

template <typename T, bool HAS_J3, bool EPOCH, int MAXT>
static void queue_launch_tt(size_t bytes, const QueueLaunch& q, cudaStream_t st)
{
  set_queue_smem_attr<T, HAS_J3, EPOCH, MAXT>(bytes);
  sweep_queue_kernel<T, HAS_J3, EPOCH, MAXT><<<q.ctas, q.threads, bytes, st>>>(
      q.tasks, q.n_tasks, q.n_walkers, q.total_units, q.n_substeps, q.accept, q.tc ? 1 : 0, q.unit, q.sched);
}
template <typename T, bool HAS_J3, bool EPOCH>
static void queue_launch_t(size_t bytes, const QueueLaunch& q, cudaStream_t st)
{
  if (q.threads <= 192)
    queue_launch_tt<T, HAS_J3, EPOCH, 192>(bytes, q, st);
  else
    queue_launch_tt<T, HAS_J3, EPOCH, 256>(bytes, q, st);
}
template <typename T> static void launch_queue_t(bool j3, bool epoch, size_t bytes, const QueueLaunch& q, cudaStream_t st)
{
  if (j3)
    queue_launch_t<T, true, false>(bytes, q, st);
  else if (epoch)
    queue_launch_t<T, false, true>(bytes, q, st);
  else
    queue_launch_t<T, false, false>(bytes, q, st);
}

cudaError_t launch_sweep_queue(bool fp32, const QueueLaunch& q, int max_k, bool j3, bool epoch, cudaStream_t st)
{
  if (max_k > MAXK || (q.tc && (!fp32 || q.threads < 128)) || q.ctas < 1 || q.unit < 1 || !q.sched ||
      q.n_tasks < 1 || q.n_walkers < 1)
    return cudaErrorInvalidValue;
  epoch = epoch && !j3;
  if (fp32)
    launch_queue_t<float>(j3, epoch, sweep_smem_bytes<float>(q.threads, max_k, q.tc, j3, epoch), q, st);
  else
  {
    QueueLaunch q64 = q;
    q64.tc          = false;
    launch_queue_t<double>(j3, epoch, sweep_smem_bytes<double>(q.threads, max_k, false, j3, epoch), q64, st);
  }
  return cudaGetLastError();
}

} // namespace qmc
