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
#include "sweep.cuh"

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

template <typename T, bool HAS_J3, bool EPOCH> static int occupancy_t(int threads, size_t bytes)
{
  set_smem_attr<T, HAS_J3, EPOCH>(bytes);
  return occupancy_of(sweep_kernel<T, HAS_J3, EPOCH>, threads, bytes);
}

int sweep_occupancy(bool fp32, int threads, int max_k, bool tc, bool j3, bool epoch, bool queue)
{
  if (queue)
    return sweep_queue_occupancy(fp32, threads, max_k, tc, j3, epoch);
  epoch = epoch && !j3;
  if (fp32)
  {
    const size_t b = sweep_smem_bytes<float>(threads, max_k, tc, j3, epoch);
    return j3 ? occupancy_t<float, true, false>(threads, b)
              : epoch ? occupancy_t<float, false, true>(threads, b) : occupancy_t<float, false, false>(threads, b);
  }
  const size_t b = sweep_smem_bytes<double>(threads, max_k, false, j3, epoch);
  return j3 ? occupancy_t<double, true, false>(threads, b)
            : epoch ? occupancy_t<double, false, true>(threads, b) : occupancy_t<double, false, false>(threads, b);
}

} // namespace qmc
