/*
 * qmcgpu.h -- C ABI of the B200 VMC walker hot path.
 *
 * This is the drop-in boundary for miniqmc's particle-by-particle (PbyP) VMC
 * sweep: per-electron moves, electron-electron / electron-ion minimum-image
 * distance rows, tricubic B-spline orbitals (SPO), one- and two-body B-spline
 * Jastrows and the delayed-update Slater-determinant inverse.  Every entry
 * point takes plain pointers and sizes, returns an int status (QMC_OK == 0)
 * and never exits the process.
 *
 * The reference interfaces each group replaces (paths inside QMCPACK/miniqmc):
 *   ParticleSet        src/Particle/ParticleSet.h:190-260, ParticleSet.cpp:280-378
 *   SPOSet             src/QMCWaveFunctions/SPOSet.h:55-127
 *   WaveFunction       src/QMCWaveFunctions/WaveFunction.h:62-96, WaveFunction.cpp:178-499
 *   WaveFunctionComponent  src/QMCWaveFunctions/WaveFunctionComponent.h:127-252
 *   BsplineFunctor     src/QMCWaveFunctions/Jastrow/BsplineFunctor.h:93-130
 *   NiO input          src/Input/nio.hpp:17-169, src/Particle/ParticleSet_builder.cpp:23-53
 *   PbyP sweep driver  src/Drivers/miniqmc.cpp:406-468
 *
 * Units: bohr.  Matrices are row-major.  Lattice tensors hold the lattice
 * vectors as rows (a_i = lattice[3*i .. 3*i+2]), as CrystalLattice::R does.
 *
 * Threading: handles are externally synchronised (one host thread per walker
 * batch at a time); distinct handles may be used concurrently.
 */
#ifndef QMCGPU_H
#define QMCGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference aborts with APP_ABORT -> exit(1);
 *      Configuration.h:35.  Here every failure is a return code) ---- */
enum {
  QMC_OK = 0,
  QMC_ERR_ARG = 1,       /* null handle, size or index out of range        */
  QMC_ERR_CUDA = 2,      /* CUDA runtime failure (launch, copy)             */
  QMC_ERR_OOM = 3,       /* device allocation failed                        */
  QMC_ERR_SINGULAR = 4,  /* zero pivot in the FP64 LU of a Slater matrix    */
  QMC_ERR_NONFINITE = 5, /* NaN / Inf in a ratio or a log value             */
  QMC_ERR_TIMEOUT = 6,   /* a bounded device wait ran out                   */
  QMC_ERR_STATE = 7,     /* call out of protocol order (e.g. accept w/o move)*/
  QMC_ERR_NODEVICE = 8,  /* no sm_100 device / library built for other arch */
  QMC_ERR_ADMISSION = 9, /* job refused: does not fit the memory budget     */
  QMC_ERR_CAPACITY = 10  /* a fixed-size device list overflowed (the J3
                            electron lists of an ion, or the pairs of one
                            move); the walker state is no longer valid     */
};

/* arithmetic forms */
enum {
  QMC_PREC_FP64 = 0,  /* plain form: FP64 everywhere                        */
  QMC_PREC_MIXED = 1  /* FP32 splines/tables/Jastrows/inverse, FP64 LU,
                         log-det and the k x k Woodbury block              */
};

/* spline coefficient fills */
enum {
  QMC_FILL_USER = 0,      /* caller supplies the table                     */
  QMC_FILL_REFERENCE = 1, /* einspline_spo::set: one mt19937(seed) uniform
                             field times cos(2 pi n / norb)
                             (einspline_spo.hpp:145-155,
                              BsplineAllocator.hpp:161-182)                */
  QMC_FILL_UNIFORM = 2,   /* every coefficient independent, uniform
                             [-0.5, 0.5) from SplitMix64(seed, index)      */
  QMC_FILL_UNIFORM_F32 = 3 /* QMC_FILL_UNIFORM rounded to FP32: in an FP64
                             system, the mixed form's table held exactly,
                             the FP64 form to measure the mixed one against */
};

/* what the determinant uses as the orbital "laplacian" */
enum {
  QMC_LAP_HXX = 0,   /* the reference stores hess.xx (einspline_spo.hpp:220) */
  QMC_LAP_TRACE = 1  /* hxx + hyy + hzz                                      */
};

/* wavefunction factors (check_wfc -f Det / J1 / J2 / J3 tests them one by
 * one, check_wfc.cpp:152-156).  The three-body Jastrow is opt-in as in the
 * reference (miniqmc -j, WaveFunction.cpp:97-100): QMC_WF_ALL and a zero
 * mask mean Det * J1 * J2. */
enum { QMC_WF_DET = 1, QMC_WF_J1 = 2, QMC_WF_J2 = 4, QMC_WF_ALL = 7, QMC_WF_J3 = 8 };

/* random streams for the fused sweep */
enum {
  QMC_RNG_DEVICE = 0, /* per-walker device mt19937 streams (seeded at init)  */
  QMC_RNG_HOST = 1    /* caller supplies ur[W][nsub][N], delta[W][nsub][N][3]*/
};

#define QMC_MAX_FUNCTOR_COEFS 32
#define QMC_MAX_ION_GROUPS 4

/* A radial cubic B-spline functor after BsplineFunctor::setupParameters:
 * coefs = SplineCoefs (NumParams + 4 values), cutoff = cutoff_radius,
 * delta_r_inv = DeltaRInv.  (BsplineFunctor.h:93-130) */
typedef struct {
  int n_coefs;
  double cutoff;
  double delta_r_inv;
  double coefs[QMC_MAX_FUNCTOR_COEFS];
} qmc_functor;

/* A three-body (electron-electron-ion) polynomial functor after
 * PolynomialFunctor3D::reset_gamma with N_eI = N_ee = 3 and C = 3
 * (PolynomialFunctor3D.h:61-250): gamma[l*16 + m*4 + n] multiplies
 * r_1I^l r_2I^m r_12^n, and the sum is cut off by ((r_1I - L)(r_2I - L))^3
 * with L = cutoff / 2, the ion's cutoff radius (ThreeBodyJastrow.h:137-162). */
#define QMC_J3_PARAMS 26
typedef struct {
  double cutoff;
  double gamma[64];
} qmc_j3_functor;

/* Everything that defines one physical system (shared by all its walkers). */
typedef struct {
  double lattice[9];       /* simulation cell, rows = lattice vectors        */
  int n_ions;
  int n_ion_groups;        /* species count (<= QMC_MAX_ION_GROUPS)          */
  const double* ion_pos;   /* [n_ions][3] Cartesian, grouped by species      */
  const int* ion_group;    /* [n_ions] species index, non-decreasing         */
  int n_elec;              /* electrons; the first n_up are spin up          */
  int n_up;                /* must equal n_elec - n_up == n_orb              */
  double spo_lattice[9];   /* cell on which the orbitals are periodic        */
  int grid[3];             /* spline grid nx, ny, nz (table has +3 per axis) */
  int n_orb;               /* orbitals per spin determinant                  */
  int spo_fill;            /* QMC_FILL_*                                     */
  uint64_t spo_seed;
  const double* spo_user_coefs; /* QMC_FILL_USER: [nx+3][ny+3][nz+3][n_orb] */
  int lap_mode;            /* QMC_LAP_*                                      */
  int components;          /* QMC_WF_* mask of the factors in the wavefunction;
                              0 means all (Slater determinants, J1, J2)      */
  qmc_functor j1[QMC_MAX_ION_GROUPS]; /* one per ion species                 */
  qmc_functor j2_uu;       /* same-spin pairs (uu and dd)                    */
  qmc_functor j2_ud;       /* opposite-spin pairs                            */
  /* QMC_WF_J3 only: per ion species, the same-spin (uu, dd) and the
   * opposite-spin (ud) functor (ThreeBodyJastrow::addFunc fills every spin
   * pair with uu, then ud overwrites the unlike pairs).  All functors of a
   * species share one cutoff. */
  qmc_j3_functor j3_same[QMC_MAX_ION_GROUPS];
  qmc_j3_functor j3_diff[QMC_MAX_ION_GROUPS];
} qmc_system_desc;

/* NiO builders -------------------------------------------------------- */
enum {
  QMC_NIO_REF32 = 0, /* the reference's 32-atom cell tiled by (na,nb,nc)
                        (nio.hpp:23-79 + ParticleIOUtility.h:30-117)        */
  QMC_NIO_PRIM4 = 1  /* the 4-atom NiO cell (half of each 32-atom lattice
                        vector: O(0,0,1/2), O(1/2,1/2,0), Ni(0,0,0),
                        Ni(1/2,1/2,1/2)) tiled by (na,nb,nc)               */
};
/* quirks of the reference's NiO input, reproduced when asked (REF32 only):
 * bit 0: at tiling (1,1,1) the ion positions stay in lattice units and are
 *        used as Cartesian coordinates (expandSuperCell returns before the
 *        conversion; ParticleIOUtility.h:42-43, nio.hpp:35);
 * bit 1: every ion is in species group 0 (ParticleSet::create(int) sets
 *        GroupID = 0; nio.hpp:33, ParticleSet.cpp:96-101).                 */
enum { QMC_NIO_QUIRK_UNIT_IONS = 1, QMC_NIO_QUIRK_ONE_GROUP = 2 };

/* Number of ions for a NiO tiling (n_ions = 32*na*nb*nc or 4*na*nb*nc). */
int qmc_nio_count(int cell, int na, int nb, int nc, int* n_ions);
/* Fill lattice[9], ion_pos[n_ions*3], ion_group[n_ions], spo_lattice[9]
 * (the untiled cell, as SPOSet_builder.cpp:38-39 uses) and n_groups. */
int qmc_nio_build(int cell, int na, int nb, int nc, int quirks, double* lattice,
                  double* ion_pos, int* ion_group, int* n_groups,
                  double* spo_lattice);
/* The reference's Jastrow tables (nio.hpp:81-168), cutoffs capped by the
 * Wigner-Seitz radius of the given cell: j1[0] = O, j1[1] = Ni. */
int qmc_nio_jastrows(const double* lattice, qmc_functor* j1_O, qmc_functor* j1_Ni,
                     qmc_functor* j2_uu, qmc_functor* j2_ud);
/* The reference's three-body tables (nio.hpp:171-245, buildJeeI), cutoff
 * min(Wigner-Seitz radius, 4.8261684030): same[s] / diff[s] for ion species
 * s = 0, 1 in the order buildJeeI adds them ("uuNi"/"udNi" to species 0,
 * "uuO"/"udO" to species 1). */
int qmc_nio_j3(const double* lattice, qmc_j3_functor* same, qmc_j3_functor* diff);
/* PolynomialFunctor3D::reset_gamma: the 26 free parameters (in the
 * reference's order) -> the 64 gammas satisfying the e-e cusp and the
 * no-e-I-cusp constraints (PolynomialFunctor3D.h:113-250). */
int qmc_j3_functor_setup(double rcut, const double* params, qmc_j3_functor* out);
/* BsplineFunctor::setupParameters(n_params, rcut, cusp, params). */
int qmc_functor_setup(int n_params, double rcut, double cusp, const double* params,
                      qmc_functor* out);
/* Synthetic Jastrows of the NiO workloads (no reference counterpart): knot
 * values uniform in [-0.1, 0.1) from SplitMix64(seed, 64 f + i) for functor
 * f = 0 (uu), 1 (ud), 2 + g (ion species g); cutoff = half the
 * Wigner-Seitz radius of `lattice`; cusp 0 for J2 and -0.25 for J1. */
int qmc_synthetic_jastrows(const double* lattice, int n_groups, uint64_t seed, int n_params,
                           qmc_functor* j1, qmc_functor* j2_uu, qmc_functor* j2_ud);
/* Wigner-Seitz radius of a periodic cell (CrystalLattice.cpp:118-125). */
int qmc_lattice_ws_radius(const double* lattice, double* ws);

/* Library / device ----------------------------------------------------- */
const char* qmc_status_string(int status);
/* Select the CUDA device for the calling thread and check it is sm_100. */
int qmc_init(int device);
/* Text of the last error recorded by this thread (never NULL). */
const char* qmc_last_error(void);

/* Systems (shared, read-only spline table) -------------------------------- */
typedef struct qmc_system_s qmc_system;
int qmc_system_create(const qmc_system_desc* desc, int precision, qmc_system** out);
int qmc_system_destroy(qmc_system* sys);
/* bytes of device memory held by the system (spline table + ions) */
int qmc_system_bytes(const qmc_system* sys, size_t* bytes);

/* SPOSet::evaluate (VGH) at arbitrary Cartesian points, for check_spo.
 * v[n_pos][n_orb], g[n_pos][3][n_orb], h[n_pos][6][n_orb] (xx,xy,xz,yy,yz,zz);
 * any output may be NULL.  (MultiBspline.hpp:165-280, einspline_spo.hpp:194) */
int qmc_spo_evaluate_vgh(qmc_system* sys, int n_pos, const double* pos, double* v,
                         double* g, double* h);
/* SPOSet::evaluate (values only, MultiBspline.hpp:35-63). */
int qmc_spo_evaluate_v(qmc_system* sys, int n_pos, const double* pos, double* v);

/* Walker batches (device-resident walker state) ----------------------- */
typedef struct qmc_walkers_s qmc_walkers;
/* delay_rank k >= 1 (k == 1 is rank-1 Sherman-Morrison, DelayedUpdate.h:166). */
int qmc_walkers_create(qmc_system* sys, int n_walkers, int delay_rank, qmc_walkers** out);
int qmc_walkers_destroy(qmc_walkers* w);
/* device bytes held by the batch */
int qmc_walkers_bytes(const qmc_walkers* w, size_t* bytes);
/* Stream used by every launch on this batch (a cudaStream_t; NULL = the
 * batch's own stream). */
int qmc_walkers_set_stream(qmc_walkers* w, void* stream);
/* Mover(seed) + build_els: walker i's mt19937 is seeded with seeds[i] and its
 * first 3N uniforms place the electrons (Mover.hpp:60-63,
 * ParticleSet_builder.cpp:33-53); the stream then drives the sweep. */
int qmc_walkers_init_random(qmc_walkers* w, const uint32_t* seeds);
int qmc_walkers_set_positions(qmc_walkers* w, const double* R /* [W][N][3] */);
int qmc_walkers_get_positions(qmc_walkers* w, double* R /* [W][N][3] */);
/* SPOSet::evaluate (einspline_spo.hpp:163-223) for electron iat of every
 * walker of a batch, at ParticleSet::activeR(iat): the proposed position
 * after qmc_pset_make_move(iat), else the current one.  The outputs are
 * caller-owned DEVICE buffers, FP64, SoA per walker: v[W][n_orb],
 * g[W][3][n_orb], h[W][6][n_orb] (xx xy xz yy yz zz).  With g and h NULL
 * only the values are evaluated.  Asynchronous on the batch's stream
 * (qmc_walkers_sync waits). */
int qmc_spo_evaluate_batch(qmc_walkers* w, int iat, double* v_dev, double* g_dev, double* h_dev);

/* ParticleSet verbs over all walkers of the batch (the flex_* forms of
 * ParticleSet.cpp:296-346; W == 1 is the single-walker API). */
int qmc_pset_update(qmc_walkers* w);
int qmc_pset_set_active(qmc_walkers* w, int iat);
int qmc_pset_make_move(qmc_walkers* w, int iat, const double* displ /* [W][3] */);
/* accept[i] != 0: acceptMove(iat), else rejectMove(iat) */
int qmc_pset_accept_reject(qmc_walkers* w, int iat, const int* accept);
int qmc_pset_done(qmc_walkers* w);
/* Distance rows of the active move (DistanceTableData Temp_r/Temp_dr):
 * aa_r[W][N], aa_dr[W][N][3], ab_r[W][I], ab_dr[W][I][3]; NULL skips. */
int qmc_pset_get_temp_rows(qmc_walkers* w, double* aa_r, double* aa_dr, double* ab_r,
                           double* ab_dr);

/* WaveFunction verbs (WaveFunction.cpp:178-279) */
/* evaluateLog from scratch: SPO VGH of all electrons, FP64 LU inverse and
 * log|det| per spin, J1/J2 recompute.  logpsi[W] may be NULL. */
int qmc_wf_evaluate_log(qmc_walkers* w, double* logpsi);
/* evalGrad: grad[W][3] = grad log psi at electron iat's current position.
 * The output is assigned with the whole wavefunction's gradient, as
 * WaveFunction::evalGrad returns it (WaveFunction.cpp:197-207). */
int qmc_wf_eval_grad(qmc_walkers* w, int iat, double* grad /* [W][3] */);
/* ratioGrad: ratio[W] = det * J1 * J2 ratio; grad[W][3] = grad log psi at
 * the proposed position, assigned (WaveFunction::ratioGrad zeroes it before
 * the components add their shares, WaveFunction.cpp:209-221). */
int qmc_wf_ratio_grad(qmc_walkers* w, int iat, double* ratio, double* grad);
/* ratio only (SPOSet values, no gradients). */
int qmc_wf_ratio(qmc_walkers* w, int iat, double* ratio);
/* evaluateRatios (WaveFunction::evaluateRatios over a VirtualParticleSet,
 * WaveFunction.h:72, DiracDeterminant.cpp:216-224): ratios[k] =
 * psi(R with electron iat at pos[k]) / psi(R) for ONE walker of the batch,
 * at n_pos absolute positions pos[n_pos][3].  The batch's move state is
 * untouched (no makeMove, and the determinants keep their update mode).
 * Needs completeUpdates done (QMC_ERR_STATE with delayed rows pending). */
int qmc_wf_evaluate_ratios(qmc_walkers* w, int walker, int iat, int n_pos, const double* pos, double* ratios);
/* accept[i] != 0: acceptMove(iat); else restore(iat) (a no-op). */
int qmc_wf_accept_restore(qmc_walkers* w, int iat, const int* accept);
int qmc_wf_complete_updates(qmc_walkers* w);
/* evaluateGL: G[W][N][3], L[W][N] (either may be NULL), logpsi[W]. */
int qmc_wf_evaluate_gl(qmc_walkers* w, double* G, double* L, double* logpsi);
/* Per-component log values and phases after the last evaluateLog /
 * accept / evaluateGL: comp[W][7] = {logdet_up, logdet_dn, phase_up,
 * phase_dn, logJ1, logJ2, logJ3}. */
int qmc_wf_components(qmc_walkers* w, double* comp);
/* Slater-matrix inverse of one walker and spin: (A^{-1})^T, n_orb x n_orb
 * (DiracDeterminant::psiM), with any pending delayed update applied first. */
int qmc_wf_get_inverse(qmc_walkers* w, int walker, int spin, double* psiM);

/* The fused PbyP sweep (miniqmc.cpp:406-468): for each step, n_substeps x
 * (N uniforms, 3N normals, N moves of evalGrad / makeMove / ratioGrad /
 * threshold accept, completeUpdates), then donePbyP + evaluateGL.  One
 * persistent launch per step covers every walker of the batch. */
typedef struct {
  int n_steps;
  int n_substeps;
  double accept;          /* accept if ur < accept (miniqmc.cpp:445)           */
  int rng_mode;           /* QMC_RNG_*                                         */
  const double* ur;       /* QMC_RNG_HOST: [n_steps][W][n_substeps][N]         */
  const double* delta;    /* QMC_RNG_HOST: [n_steps][W][n_substeps][N][3]      */
  int recompute_every;    /* FP64 LU refresh of the inverse after every
                             recompute_every-th MC step of the batch, counted
                             over all sweep calls since creation (0 = never) */
  double* trace;          /* optional [n_steps][W][n_substeps][N][8]:
                             ratio, grad_new[3], grad_now[3], accepted        */
  int64_t* n_accepted;    /* optional [W] accepted-move counts (sum of steps) */
  double* logpsi;         /* optional [W] log|psi| after the last step         */
} qmc_sweep_opts;
int qmc_sweep(qmc_walkers* w, const qmc_sweep_opts* opts);
/* One fused single-electron move of every walker of the batch, the body of
 * the driver's loop (miniqmc.cpp:426-458): evalGrad, makeMove(iat,
 * delta[w]), ratioGrad, the threshold accept ur[w] < accept, acceptMove or
 * restore, the position update and the delayed-update bookkeeping (a
 * Woodbury flush when the delay fills).  ur[W] and delta[W][3] are host
 * arrays; accepted[W] (may be NULL) receives 1 or 0 per walker.  After the
 * last electron of a substep call qmc_wf_complete_updates, and
 * qmc_wf_evaluate_gl after the substeps, as the driver does. */
int qmc_step(qmc_walkers* w, int iat, double accept, const double* ur, const double* delta, int* accepted);
/* Asynchronous form for device-resident callers: no host copies, inputs
 * already on the device (QMC_RNG_DEVICE only); results stay on the device
 * until qmc_walkers_sync + qmc_sweep_results. */
int qmc_sweep_async(qmc_walkers* w, int n_steps, int n_substeps, double accept,
                    int recompute_every);
int qmc_walkers_sync(qmc_walkers* w);
int qmc_sweep_results(qmc_walkers* w, int64_t* n_accepted, double* logpsi);
/* Number of CUDA kernel launches this batch issued since creation. */
int qmc_walkers_launch_count(const qmc_walkers* w, int64_t* count);

/* Device phase timers of the fused sweep (the reference's NewTimer phases,
 * miniqmc.cpp:138-147): when enabled, each walker's CTA accumulates SM
 * cycles per phase.  qmc_walkers_phase_times returns, per phase, the mean
 * over walkers in milliseconds at the device's nominal SM clock:
 * [0] random streams, [1] getInvRow, [2] SPO VGH + determinant dots,
 * [3] J1/J2 sums, [4] reductions and ratio, [5] acceptRow bookkeeping,
 * [6] Woodbury flush, [7] J2 accept, [8] position update,
 * [9] completeUpdates, [10] evaluateGL, [11] a move's set-up, and for the
 * tensor-core flush [12] its U2 = Binv V image and [13] its first GEMM
 * (Ainv U^T), [6] then holding its second GEMM and the Ainv update.
 * ms needs room for n_phases values; n_phases receives 14. */
int qmc_walkers_enable_timers(qmc_walkers* w, int enable);

/* Woodbury flush on the tensor cores (tcgen05, 3xTF32 with FP32
 * accumulation) or on the CUDA cores (FP32 FMA).  The tensor-core flush is
 * on by default wherever it applies: FP32 walkers with the determinant,
 * delay rank <= 64 and >= 128 threads per walker (480 or more orbitals per
 * spin).  Its tiles take 48 KB of shared memory per walker up to delay 32
 * and 96 KB above (two walkers per SM).  QMC_ERR_ARG when asked for where
 * it does not apply.  Both compute DelayedUpdate::updateInvMat
 * (DelayedUpdate.h:184-191). */
int qmc_walkers_set_tensor_cores(qmc_walkers* w, int enable);
/* Limit, in SM cycles, of every bounded wait of the tensor-core flush on the
 * MMAs it issued (no reference counterpart: the reference has no device
 * waits).  Default 2e9 (about one second).  A wait that runs out sets the
 * batch's error bit, the launch unwinds (the CTA drains its own MMAs before
 * it frees its tensor memory) and the call that reads the status returns
 * QMC_ERR_TIMEOUT.  The batch's inverses and delayed rows are then
 * undefined: call qmc_wf_evaluate_log (which rebuilds them from the
 * positions) or destroy the batch.  0 makes the first wait give up at once. */
int qmc_walkers_set_wait_limit(qmc_walkers* w, long long cycles);
/* Moves the fused sweep evaluates together, 1 to 4 (default 1).  The
 * reference's accept rule compares each move's uniform with a fixed
 * threshold (miniqmc.cpp:445), so the moves from one accepted move to the
 * next -- rejected ones that change nothing, then the accepted one -- all see
 * the same walker state.  The sweep evaluates up to max_moves of them in one
 * pass (one getInvRow pass over the delayed rows for all of them, one
 * reduction); the ratios, gradients and trajectory are those of one move at
 * a time, bit for bit.  1 moves one electron at a time.  Fewer dependent
 * round trips per move help when few walkers share an SM; with 3-4 walkers
 * per SM the L2 holds less of each walker's next stencil and one move at a
 * time measured faster, so qmc_autotune chooses.  No reference counterpart
 * (the reference loops over electrons one by one). */
int qmc_walkers_set_move_batching(qmc_walkers* w, int max_moves);
/* Threads (one CTA) per walker: a multiple of 32 in [max(64, 2 delay), 256];
 * the default covers the padded orbitals with 16-byte vectors.  The kernels
 * stride over any block size; >= 128 is needed for the tensor-core flush. */
int qmc_walkers_set_threads(qmc_walkers* w, int threads);
/* L2 prefetch of the next move's 16 spline-stencil rows while the current
 * move runs (no reference counterpart).  AUTO: on while the batch's
 * stencils in flight (16 rows x 4 npad coefficients per walker) stay within
 * 32 MB of the 126 MB L2. */
enum { QMC_PREFETCH_AUTO = 0, QMC_PREFETCH_OFF = 1, QMC_PREFETCH_ON = 2 };
int qmc_walkers_set_prefetch(qmc_walkers* w, int mode);
/* Schedule of the fused sweep's CTAs (no reference counterpart: the
 * reference moves each walker on one host thread).  STATIC: one CTA per
 * walker for the whole step (four per SM at NiO-128, 80 registers a
 * thread).  QUEUE: `ctas` resident CTAs (0: walkers per SM x SMs, every slot
 * of the device) take each walker's step in units of at most unit_moves
 * consecutive moves of one spin (0: QMC_SCHED_UNIT_DEFAULT).  A unit that
 * ends on an SM with no spare CTA hands its walker to the CTA that has
 * waited longest; where a CTA waits already, the walker goes on in place.
 * A walker's state passes between units through device memory, so the
 * results are those of STATIC bit for bit.  Up to 192 threads a walker the
 * queue runs three CTAs per SM at up to 112 registers a thread, and the
 * walkers take turns where they outnumber the slots.  At NiO-128 it measured
 * 141 ms per 512-walker launch against 173 ms static, 80 against 101 ms at
 * 148 walkers.  AUTO (the default) is QUEUE.  Batch groups choose theirs
 * with qmc_group_set_schedule. */
enum { QMC_SCHED_AUTO = 0, QMC_SCHED_STATIC = 1, QMC_SCHED_QUEUE = 2 };
#define QMC_SCHED_UNIT_DEFAULT 16
int qmc_walkers_set_schedule(qmc_walkers* w, int mode, int unit_moves, int ctas);
int qmc_walkers_get_config(const qmc_walkers* w, int* threads, int* delay, int* tensor_cores);
/* Walkers (CTAs) of this batch's fused sweep that one SM holds at once with
 * its present settings (registers, shared memory, block size, and the form
 * its schedule selects): with W walkers a static launch runs in
 * ceil(W / (walkers_per_sm x SMs)) waves. */
int qmc_walkers_occupancy(const qmc_walkers* w, int* walkers_per_sm);

/* Batch groups (no reference counterpart: the reference's flex_ batch,
 * miniqmc_sync_move.cpp:432-521, holds movers of one system).  A group
 * advances batches of possibly different systems and electron counts, all of
 * one precision, with ONE fused launch per MC step covering every walker of
 * every batch; each walker keeps its own device RNG stream, so a batch's
 * trajectory does not depend on what else is in the group (given the same
 * threads per walker).  While the group exists its batches run on the
 * group's stream.  With use_graph, the launch is captured once as a CUDA
 * graph (per n_substeps / accept) and replayed each step. */
typedef struct qmc_group_s qmc_group;
int qmc_group_create(qmc_walkers* const* batches, int n_batches, qmc_group** out);
int qmc_group_destroy(qmc_group* g);
/* launch block size: at least every batch's own threads per walker */
int qmc_group_set_threads(qmc_group* g, int threads);
int qmc_group_use_graph(qmc_group* g, int enable);
/* The group's shared launches in the work-queue form or one CTA per walker
 * (QMC_SCHED_*, as qmc_walkers_set_schedule; unit_moves 0 = the default,
 * ctas 0 = every resident CTA slot): the queue takes units of any batch's
 * walkers.  AUTO (the default) is the queue.  The request loop's shared
 * launches take the queue too. */
int qmc_group_set_schedule(qmc_group* g, int mode, int unit_moves, int ctas);
/* n_steps MC steps (device RNG streams) of every batch; asynchronous.
 * recompute_every: FP64 refresh of a batch's inverses after every
 * recompute_every-th step of that batch (0 = never). */
int qmc_group_sweep(qmc_group* g, int n_steps, int n_substeps, double accept, int recompute_every);
int qmc_group_sync(qmc_group* g);
int qmc_group_stats(const qmc_group* g, int* threads, int64_t* launches, int64_t* graph_launches);
/* the group's cudaStream_t (for events a caller records around its sweeps) */
int qmc_group_stream(const qmc_group* g, void** stream);

/* Autotuner (no reference counterpart): times n_steps sweeps of n_walkers
 * walkers of `sys` for each delay rank in `delays` x threads per walker
 * {default, 128, 192, 256 above it} x flush engine {CUDA cores, tensor cores
 * where it applies} x moves evaluated together {1, 4}
 * (qmc_walkers_set_move_batching), and returns the fastest in `best` (all
 * timings in results[0 .. min(n, max_results)), n in *n_results). */
typedef struct {
  int delay;
  int threads;
  int tensor_cores;
  int max_moves;
  double ms_per_step;
} qmc_tune_result;
int qmc_autotune(qmc_system* sys, int n_walkers, const int* delays, int n_delays, int n_steps,
                 qmc_tune_result* results, int max_results, int* n_results, qmc_tune_result* best);

/* Request loop (no reference counterpart).  Jobs (system, walkers, steps,
 * delay rank, seed) are submitted as they arrive; each tick admits, in
 * arrival order, every waiting job whose device footprint fits the memory
 * budget now (walkers created, seeded and evaluated on the device), moves
 * every walker of every running job by one MC step in ONE shared launch
 * (block size `threads` for all jobs, so a job's results are the same alone
 * and in any mix), and retires jobs that reached their steps (results read
 * back, memory released).  Times are seconds since the server was created;
 * latency = t_done - t_submit. */
enum { QMC_JOB_WAITING = 0, QMC_JOB_RUNNING = 1, QMC_JOB_DONE = 2, QMC_JOB_FAILED = 3 };
typedef struct {
  int state;          /* QMC_JOB_*                                       */
  int status;         /* QMC_OK or the failure of a failed job           */
  int steps_done;
  int64_t n_accepted; /* accepted moves over all walkers and steps       */
  double logpsi_mean; /* mean log|psi| of the walkers after the last step */
  double t_submit, t_start, t_done;
} qmc_job_info;
typedef struct qmc_server_s qmc_server;
int qmc_server_create(size_t memory_budget, int threads, int recompute_every, qmc_server** out);
int qmc_server_destroy(qmc_server* s);
/* QMC_ERR_ADMISSION if the job alone exceeds the budget */
int qmc_server_submit(qmc_server* s, qmc_system* sys, int n_walkers, int n_steps, int delay, uint32_t seed,
                      int64_t* job);
int qmc_server_tick(qmc_server* s, int* n_running, int* n_waiting);
int qmc_server_job(qmc_server* s, int64_t job, qmc_job_info* info);
int qmc_server_stats(const qmc_server* s, size_t* bytes_in_use, int64_t* launches, int64_t* electron_moves);
int qmc_walkers_phase_times(qmc_walkers* w, double* ms, int* n_phases);

/* DelayedUpdate + DiracMatrix on one n x n inverse, FP64 on the device
 * (DelayedUpdate.h:28-231, DiracMatrix.h:59-121): the object the reference's
 * unit tests drive with fake orbital rows (test_dirac_matrix.cpp,
 * test_dirac_det.cpp). */
typedef struct qmc_detengine_s qmc_detengine;
int qmc_detengine_create(int n, int delay, qmc_detengine** out);
/* Same engine with the matrices held in the given precision: QMC_PREC_FP64,
 * or QMC_PREC_MIXED (FP32 Ainv/U/V/psiV rows as in the mixed sweep, FP64
 * k x k Binv and FP64 inverse/log-det).  qmc_detengine_create is this with
 * QMC_PREC_FP64. */
int qmc_detengine_create_prec(int n, int delay, int precision, qmc_detengine** out);
int qmc_detengine_destroy(qmc_detengine* e);
/* DiracMatrix::invert_transpose(logdetT = a): psiM = (a^{-1})^T, log|det a|
 * and its phase (0 or pi). */
int qmc_detengine_invert_transpose(qmc_detengine* e, const double* a, double* logdet,
                                   double* phase);
int qmc_detengine_get_inv_row(qmc_detengine* e, int row, double* inv_row);
int qmc_detengine_accept_row(qmc_detengine* e, int row, const double* psiv);
int qmc_detengine_update_inv_mat(qmc_detengine* e);
int qmc_detengine_get_ainv(qmc_detengine* e, double* ainv);
/* The engine's flushes on the tensor cores (FP32 engines with delay rank
 * <= 64; on by default there) or on the CUDA cores. */
int qmc_detengine_set_tensor_cores(qmc_detengine* e, int enable);

/* Local kinetic energy of every walker, -1/2 sum_i (L_i + |G_i|^2), from
 * the G and L of the last evaluateGL (WaveFunction.cpp:261-279; the fused
 * sweep ends each step with it).  With the accepted-move counts of
 * qmc_sweep_results (acceptance = accepted / (steps x substeps x N)) this is
 * the VMC estimator the reference driver leaves out.  kinetic[W]. */
int qmc_local_kinetic(qmc_walkers* w, double* kinetic);

/* Checkpoint / restore of a batch (no reference counterpart: Walker.h is
 * unused there).  The persistent walker state -- positions, inverses and
 * orbital derivative rows, delayed-update state, log values, Jastrow
 * arrays, RNG streams, move state, G, L, accepted counts, step and NLPP
 * counters -- goes to / comes from a host buffer of
 * qmc_walkers_checkpoint_bytes bytes.  Restore needs a batch of the same
 * system, walker count, delay rank and precision; sweeping on from a
 * restored batch gives exactly what the original would have. */
int qmc_walkers_checkpoint_bytes(qmc_walkers* w, size_t* bytes);
int qmc_walkers_checkpoint(qmc_walkers* w, void* buffer, size_t bytes);
int qmc_walkers_restore(qmc_walkers* w, const void* buffer, size_t bytes);

/* Non-local pseudopotential ratios (NonLocalPP, the step after the
 * diffusion in miniqmc.cpp:472-495): for every electron and every ion within
 * rmax (minimum-image e-I distance), WaveFunction::ratio at the 12 points of
 * NonLocalPP's quadrature sphere (NonLocalPP.hpp:61-80), rotated once per
 * call by NonLocalPP::randomize from a stream seeded with 11 as every
 * mover's is (NonLocalPP.hpp:58, 98-110).  Positions: QMC_NLPP_SPHERE
 * R + displ + r rot_k (NonLocalPP::evaluate: the sphere around the ion);
 * QMC_NLPP_DRIVER R + r rot_k - displ (the driver's makeMove), displ being
 * DistanceTableBA's ion - electron.  Needs completeUpdates done (no pending
 * delayed rows; QMC_ERR_STATE otherwise).  Outputs per walker: n_points and
 * wsum = sum of ratio / 12; `ratios` (may be null) receives walker 0's
 * ratios in (electron, ion, knot) order, at most max_ratios. */
enum { QMC_NLPP_SPHERE = 0, QMC_NLPP_DRIVER = 1 };
int qmc_nlpp_evaluate(qmc_walkers* w, double rmax, int form, int64_t* n_points, double* wsum, double* ratios,
                      int max_ratios);
/* The rotated 12-point spheres of the first n_calls calls: out[n_calls][12][3]. */
int qmc_nlpp_sphere(int n_calls, double* out);

/* Allocation-free inverse.  No reference counterpart: the reference always
 * inverts into memory its DiracMatrix owns.  This is the FP64 Gauss-Jordan
 * of qmc_detengine_invert_transpose on caller-owned device memory: a and
 * psim are n x n row-major FP64 device buffers (row stride n), psim =
 * (a^{-1})^T, *logdet = log|det a| and *phase = 0 or pi (either may be null);
 * results equal qmc_detengine_invert_transpose's bit for bit.
 *
 * It calls no cudaMalloc, cudaFree or allocating library routine.  This is
 * for host codes that cannot take a device allocation mid-run.  One kind
 * reserves the device memory up front in its own pool, so an extra
 * cudaMalloc escapes its accounting or fails outright.  Another is a
 * latency-bound loop: cudaFree waits for the whole device, stalling every
 * stream of the process.
 *
 * The working copy of the matrix lives in one static device array per
 * device, which limits n to QMC_NOALLOC_MAX_N (768: 4.5 MiB).  A larger n
 * returns QMC_ERR_ARG.  The first call on each device, made with that
 * device current, looks the array up (cudaGetSymbolAddress).  Make that
 * first call before any stream capture.  Calls on one device share the
 * array, so calls that overlap (other streams or host threads) race: the
 * caller must serialise them.  Every call, not only the first, copies the
 * log-det, phase and status to the host and waits for `stream` (a
 * cudaStream_t, null for the default stream) to finish.  QMC_ERR_SINGULAR
 * on a zero pivot. */
#define QMC_NOALLOC_MAX_N 768
int qmc_invert_transpose_noalloc(int n, const double* a, double* psim, double* logdet, double* phase,
                                 void* stream);

#ifdef __cplusplus
}
#endif
#endif /* QMCGPU_H */
