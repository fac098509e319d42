// kernels.cuh -- host-side launchers of the device code (sweep.cu, others.cu, nlpp.cu, state.cu).
#pragma once

#include "layout.cuh"

namespace qmc
{
// device phase timers of the fused sweep (names follow the reference's
// timers where one exists: miniqmc.cpp:138-147, WaveFunction.cpp:33-41)
enum Phase
{
  PH_RANDOM = 0,    // random streams of a substep
  PH_INVROW,        // DelayedUpdate::getInvRow ("Current Gradient")
  PH_SPO,           // SPO VGH + determinant dots ("New Gradient")
  PH_JASTROW,       // J1/J2 ratio and gradient sums
  PH_REDUCE,        // block reduction + ratio assembly
  PH_DET_ACCEPT,    // acceptRow bookkeeping ("Update")
  PH_FLUSH,         // Woodbury flush (updateInvMat)
  PH_J2_ACCEPT,     // J2 acceptMove
  PH_POSITION,      // ParticleSet::acceptMove
  PH_COMPLETE,      // completeUpdates ("Complete Updates")
  PH_GL,            // evaluateGL ("Kinetic Energy")
  PH_SETUP,         // a move's serial set-up: positions, stencil location
  PH_FLUSH_U2,      // tensor-core flush: the U2 = Binv V image
  PH_FLUSH_G1,      // tensor-core flush: GEMM1 (Ainv U^T); PH_FLUSH keeps GEMM2
  NPHASE
};

// One batch of walkers in a fused sweep launch.  Several tasks (walkers of
// different systems) may share one launch; each CTA runs one walker.
struct SweepTask
{
  long long* timers;    // device [W][NPHASE] cycle counters, or null
  const DevSystem* sys; // device pointer
  DevWalkers dw;
  int rng_mode;         // QMC_RNG_*
  const double* ur;     // device [W][nsub][N] for QMC_RNG_HOST
  const double* delta;  // device [W][nsub][N][3]
  double* trace;        // device [W][nsub][N][8] or null
  int first_block;      // first CTA of this task in the launch
  int prefetch;         // warm L2 with the next move's coefficients
  int tc;               // Woodbury flushes on the tensor cores (needs dw.tci)
  int max_moves;        // most moves evaluated together (an epoch, do_epoch)
};

struct LaunchCfg
{
  int threads;
  size_t smem;
};

// fused sweep: one MC step (n_substeps x N moves + completeUpdates, then
// evaluateGL) for every walker of every task
// tc: FP32 Woodbury flushes on the tensor cores (every task has dw.tci,
// k <= 32, threads >= 128); j3: some task's wavefunction has the three-body
// Jastrow (its shared-memory scratch is added to the launch)
// epoch: evaluate the moves an epoch at a time (each task's max_moves);
// ignored with j3
cudaError_t launch_sweep(bool fp32, const SweepTask* d_tasks, int n_tasks, int total_blocks, int n_substeps,
                         double accept, int threads, int max_npad, int max_k, cudaStream_t st, bool tc, bool j3,
                         bool epoch);
// CTAs (walkers) of one sweep launch that an SM holds at once, or -1
// queue: of the work-queue form (launch_sweep_queue)
int sweep_occupancy(bool fp32, int threads, int max_k, bool tc, bool j3, bool epoch, bool queue = false);
int sweep_queue_occupancy(bool fp32, int threads, int max_k, bool tc, bool j3, bool epoch);
// the fused sweep in the work-queue form over a list of tasks (one batch,
// or a batch group): `ctas` resident CTAs take units of at most `unit`
// moves of one spin of a walker, a walker passing from CTA to CTA between
// its units.  sched: device ints, zero, sweep_queue_words of them.
constexpr int QUEUE_HDR = 4;   // counters of the work-queue launch
constexpr int QUEUE_SMS = 256; // per-SM words (SM ids above share the last)
// units of one walker's step in the work-queue form
inline int sweep_queue_units(int n_elec, int n_up, int n_substeps, int unit)
{
  return n_substeps * ((n_up + unit - 1) / unit + (n_elec - n_up + unit - 1) / unit);
}
// schedule words of a work-queue launch over n_walkers walkers (all tasks)
// on `ctas` CTAs with total_units units in all
inline size_t sweep_queue_words(int n_walkers, int ctas, size_t total_units)
{
  return (size_t)QUEUE_HDR + QUEUE_SMS + n_walkers + ctas + total_units;
}
struct QueueLaunch
{
  const SweepTask* tasks; // device; first_block = the task's first walker over all tasks
  int n_tasks, n_walkers, total_units, n_substeps, unit, ctas, threads;
  double accept;
  bool tc;     // some task's flushes run on the tensor cores (CTAs allocate TMEM)
  int* sched;  // device, sweep_queue_words(...) ints, zero
};
cudaError_t launch_sweep_queue(bool fp32, const QueueLaunch& q, int max_k, bool j3, bool epoch, cudaStream_t st);

// evaluateLog pieces
// ratio_mode_only: only the derivative rows of the determinants whose last
// move was ratio-only (the evaluateGL re-evaluation)
cudaError_t launch_spo_matrix(bool fp32, const DevSystem* sys, const DevWalkers& dw, bool want_lu,
                              cudaStream_t st, bool ratio_mode_only = false);
cudaError_t launch_gj_inverse(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads, int n_spins,
                              cudaStream_t st);
cudaError_t launch_jastrow_recompute(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads,
                                     cudaStream_t st);
cudaError_t launch_gl(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads, cudaStream_t st);
// ThreeBodyJastrow::recompute: the per-ion electron lists and Uat, dUat, d2Uat
cudaError_t launch_j3_recompute(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads,
                                cudaStream_t st);

// capacity of one J3 electron list (ThreeBodyJastrow::elecs_inside of one
// ion and spin): the electrons of that spin, at most 128
inline int j3_list_capacity(int n_elec, int n_up)
{
  const int m = n_up > n_elec - n_up ? n_up : n_elec - n_up;
  return m < 128 ? m : 128;
}
cudaError_t launch_sync_rs(bool fp32, const DevWalkers& dw, cudaStream_t st);

// drop-in verbs (all walkers of a batch, same electron)
enum VerbOp
{
  VERB_MAKE_MOVE = 0,
  VERB_EVAL_GRAD,
  VERB_RATIO_GRAD,
  VERB_RATIO,
  VERB_WF_ACCEPT,
  VERB_PSET_ACCEPT,
  VERB_COMPLETE,
  VERB_TEMP_ROWS,
  VERB_SET_ACTIVE
};
struct VerbArgs
{
  int op, iat;
  const double* displ;   // [W][3] device
  const int* flags;      // [W] device
  double* aa_r;          // temp-row outputs (device), may be null
  double* aa_dr;
  double* ab_r;
  double* ab_dr;
};
// one fused single-electron move of every walker (qmc_step): in = [W][4]
// (ur, delta xyz) on the device, accepted flags into out [W]
cudaError_t launch_step(bool fp32, bool j3, const DevSystem* sys, const DevWalkers& dw, int iel, double accept,
                        const double* in, int* out, int threads, cudaStream_t st);
cudaError_t launch_verb(bool fp32, const DevSystem* sys, const DevWalkers& dw, const VerbArgs& a, int threads,
                        int max_k, cudaStream_t st);

// ParticleSet::activeR(iat) of every walker into pos[W][3] (device)
cudaError_t launch_active_pos(const DevWalkers& dw, int iat, double* pos, cudaStream_t st);
// standalone SPO evaluation at arbitrary points (check_spo)
cudaError_t launch_spo_points(bool fp32, const DevSystem* sys, int n_pos, const double* pos, double* v,
                              double* g, double* h, bool values_only, cudaStream_t st);

// DelayedUpdate engine on one matrix (W = 1 batch view)
// tc: FP32 Woodbury flush on the tensor cores (needs dw.tci, k <= 32)
cudaError_t launch_det_engine(bool fp32, int op, const DevWalkers& dw, int row, int max_k, cudaStream_t st,
                              bool tc);
enum DetEngineOp
{
  DETENG_GET_INV_ROW = 0,
  DETENG_ACCEPT_ROW  = 1,
  DETENG_UPDATE      = 2
};

} // namespace qmc
