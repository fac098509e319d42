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
template <typename T>
__global__ void __launch_bounds__(256, 3) sweep_kernel(const SweepTask* __restrict__ tasks, int n_tasks, int n_substeps,
                                                    double accept_thr)
{
  __shared__ SysSmem<T> ss;
  __shared__ MoveSmem m;
  __shared__ SplineSmem<T> sp;
  extern __shared__ __align__(16) unsigned char dyn[];
  T* smem = reinterpret_cast<T*>(dyn);
  int t   = 0;
  while (t + 1 < n_tasks && (int)blockIdx.x >= tasks[t + 1].first_block)
    ++t;
  const SweepTask& task = tasks[t];
  const int w           = blockIdx.x - task.first_block;
  if (w >= task.dw.W)
    return;
  const DevSystem* sys = task.sys;
  load_sys(sys, ss);
  const WV<T> wv = make_wv<T>(task.dw, w);
  const int N    = wv.N;
  const T* ions  = (const T*)sys->ion_soa;
  long long acc  = 0;
  if (threadIdx.x == 0)
  {
    m.timing = task.timers != nullptr;
    m.tstamp = clock64();
    for (int p = 0; p < NPHASE; ++p)
      m.tacc[p] = 0;
  }
  __syncthreads();
  for (int l = 0; l < n_substeps; ++l)
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
    for (int iel = 0; iel < N; ++iel)
    {
      double* tr = task.trace ? task.trace + (((size_t)w * n_substeps + l) * N + iel) * 8 : nullptr;
      do_move(ss, sys, wv, m, sp, ions, iel, accept_thr, urp[iel], dp + 3 * iel, tr, smem);
      acc += m.accept ? 1 : 0;
      __syncthreads(); // m.accept is rewritten by the next move
    }
    phase_mark(m, PH_REDUCE);
    if (ss.comp & QMC_WF_DET)
    {
      flush(wv, m, 0, smem);
      flush(wv, m, 1, smem);
    }
    phase_mark(m, PH_COMPLETE);
  }
  evaluate_gl(ss, wv, m, task.dw.logpsi + w);
  phase_mark(m, PH_GL);
  if (threadIdx.x == 0)
  {
    task.dw.accepted[w] += acc;
    if (task.timers)
      for (int p = 0; p < NPHASE; ++p)
        task.timers[(size_t)w * NPHASE + p] += m.tacc[p];
  }
}

template <typename T> static void set_smem_attr()
{
  static bool done = false;
  if (!done)
  {
    cudaFuncSetAttribute(sweep_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)flush_smem_bytes<T>());
    done = true;
  }
}

cudaError_t launch_sweep(bool fp32, const SweepTask* d_tasks, int n_tasks, int total_blocks, int n_substeps,
                         double accept, int threads, int max_npad, int max_k, cudaStream_t st)
{
  (void)max_npad;
  if (max_k > MAXK)
    return cudaErrorInvalidValue;
  if (fp32)
  {
    set_smem_attr<float>();
    sweep_kernel<float><<<total_blocks, threads, flush_smem_bytes_for<float>(threads, max_k), st>>>(
        d_tasks, n_tasks, n_substeps, accept);
  }
  else
  {
    set_smem_attr<double>();
    sweep_kernel<double><<<total_blocks, threads, flush_smem_bytes_for<double>(threads, max_k), st>>>(
        d_tasks, n_tasks, n_substeps, accept);
  }
  return cudaGetLastError();
}

} // namespace qmc
