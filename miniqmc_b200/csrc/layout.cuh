// layout.cuh -- device-resident data of a system and of a walker batch.
//
// HBM layout (per batch of W walkers of one system, N electrons, n orbitals
// per spin padded to npad = roundup(n, 32), I ions, delay rank k; T is the
// walker precision, float for the mixed form and double for the plain form):
//   R        double [W][N][3]        master positions (FP64 in both forms)
//   Rs       T      [W][3][Npad]     SoA mirror used by the distance rows
//   Ainv     T      [W][2][n][npad]  psiM = (A^-1)^T per spin
//   dpsiM    T      [W][2][n][3][npad]
//   d2psiM   T      [W][2][n][npad]
//   U, V     T      [W][2][k][npad]  delayed rows (DelayedUpdate::U, V)
//   Binv     double [W][2][k][k]     k x k Woodbury block, FP64 in both forms
//   J1 Vat/Lap T [W][N], Grad T [W][3][N]; J2 Uat/d2Uat T [W][N], dUat T [W][3][N]
//   J3 Uat/d2Uat T [W][N], dUat T [W][3][N]; j3_cnt int [W][2][I] and
//            j3_list int [W][2][I][cap]: the electrons of each spin within
//            the J3 cutoff of each ion (ThreeBodyJastrow::elecs_inside)
//   mt       uint32 [W][625]         per-walker mt19937 state + index
// The spline table is shared by every walker of the system:
//   coefs    T [(nx+3)][(ny+3)][(nz+3)][npad]  orbital-fastest (einspline
//            multi_UBspline_3d layout, BsplineAllocator.hpp:126-133)
#pragma once

#include "../../include/qmcgpu.h"
#include "common.cuh"

namespace qmc
{
struct DevFunctor
{
  int n;
  double cutoff, dinv;
  double c[QMC_MAX_FUNCTOR_COEFS];
};

struct DevSystem
{
  // simulation cell: reduced basis, its inverse and the 8 image corners
  // (DTD_BConds<T,3,PPPG+SOA_OFFSET>, ParticleBConds.h:106-151)
  double rb[9], gb[9], corners[24];
  // lower bound of |f . rb|^2 / |f|^2 over fractional vectors f (smallest
  // eigenvalue of rb rb^T, slightly shrunk): pairs whose wrapped fractional
  // displacement is at least rc / sqrt(mi_scale2) from every cell corner
  // have every image beyond rc and skip the corner search
  double mi_scale2;
  double lattice[9];
  // orbital cell: toUnit = r . spoG (CrystalLattice.h:180-196)
  double spoG[9];
  int grid[3];
  double dinv[3];
  long long xs, ys, zs; // element strides of the coefficient table
  int norb, npad;
  int table_fp32;
  const void* coefs;
  size_t coef_bytes;
  int n_ions, n_groups;
  const double* ion_pos; // [I][3]
  const void* ion_soa;   // [3][I] in the walker precision (float or double)
  int gfirst[QMC_MAX_ION_GROUPS], glast[QMC_MAX_ION_GROUPS];
  int n_elec, n_up;
  int lap_mode, comp;
  DevFunctor j1[QMC_MAX_ION_GROUPS], j2uu, j2ud;
  // three-body Jastrow: per ion species the ion cutoff (half the functor
  // cutoff, also the L of its polynomial) and the gammas, in the walker
  // precision, [species][0 same spin, 1 opposite spin][64]
  double j3_icut[QMC_MAX_ION_GROUPS];
  const void* j3_gamma;
};

// most moves the fused sweep evaluates together: one epoch is a run of
// rejected moves and the accepted move that ends it, which all see the same
// walker state (the accept rule compares a uniform with a fixed threshold,
// miniqmc.cpp:445, so the run is known before its ratios are)
constexpr int EPOCH_MAX = 4;

// scalars of the move in progress, per walker (drop-in verb API)
struct MoveState
{
  int active;        // ParticleSet::activePtcl
  int invrow_id[2];  // DiracDeterminant::invRow_id
  int partial[2];    // UpdateMode == ORB_PBYP_PARTIAL (det)
  int j_partial;     // UpdateMode == ORB_PBYP_PARTIAL (Jastrows)
  int pad;
  double pos[3];     // ParticleSet::activePos
  double cur_ratio[2];
  double j1_curAt, j1_curLap, j1_curGrad[3];
  double j2_curUat;
  double j3_curUat, j3_curGrad[3];
};

struct DevWalkers
{
  int W, N, Npad, n, npad, I, k;
  double* R;
  void* Rs;
  void* Ainv;
  void* dpsiM;
  void* d2psiM;
  void* U;
  void* V;
  double* Binv;
  int* delay_list;
  int* delay_count;
  double* det_log;
  double* det_phase;
  void* j1_Vat;
  void* j1_Lap;
  void* j1_Grad;
  void* j2_Uat;
  void* j2_d2Uat;
  void* j2_dUat;
  void* j3_Uat;   // [W][N]      (null without J3)
  void* j3_d2Uat; // [W][N]
  void* j3_dUat;  // [W][3][N]
  int* j3_cnt;    // [W][2][I]
  int* j3_list;   // [W][2][I][j3_cap]
  int j3_cap;
  double* j_log; // [W][3] J1, J2, J3
  uint32_t* mt;  // [W][625]
  uint32_t* words; // [W][8N+4]
  double* ur;      // [W][N]
  double* delta;   // [W][N][3]
  void* invRow;    // [W][EPOCH_MAX][npad] (the verbs use row 0)
  void* psiV;      // [W][npad]
  void* dpsiV;     // [W][3][npad]
  void* d2psiV;    // [W][npad]
  void* U2;        // [W][k][npad] flush scratch (Binv V)
  void* tm;        // [W][n][k] flush scratch (Ainv U^T - E)
  float* tci;      // [W][npad/32][2][32][32 or 64 (k > 32)] tensor-core flush: (Binv V)^T hi/lo tiles, or null
  double* lu;      // [W][2][n][npad] FP64 Slater matrices for the LU (lazily)
  MoveState* ms;   // [W]
  double* G;       // [W][N][3]
  double* L;       // [W][N]
  double* logpsi;  // [W]
  long long* accepted; // [W]
  double* out_grad;    // [W][3] verb outputs
  double* out_ratio;   // [W]
  int* accept_flags;   // [W]
  unsigned* status;    // [1]
  long long wait_cycles; // limit of each bounded tensor-core wait (SM cycles)
};

__host__ __device__ inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

} // namespace qmc
