// device.cuh -- __device__ building blocks of the VMC walker hot path (sm_100a).
//
// One CTA owns one walker.  The fused sweep kernel runs a whole MC step per
// launch: per substep the walker's mt19937 stream is advanced (N uniforms,
// 3N normals), then N single-electron moves (evalGrad, makeMove, ratioGrad,
// threshold accept) and completeUpdates; at the end evaluateGL.  Every phase
// is a __device__ function shared with the drop-in verb kernels, so the
// per-call API and the fused sweep execute the same arithmetic.
//
// Reference algorithms (QMCPACK/miniqmc) restated here:
//   minimum image             ParticleBConds.h:153-217
//   B-spline SPO (VGH / V)    MultiBspline.hpp:34-280, MultiBsplineEvalHelper.hpp:43-113,
//                             MultiBsplineData.hpp:52-80, einspline_spo.hpp:163-223
//   radial functor            BsplineFunctor.h:222-339
//   J1                        OneBodyJastrow.h:110-283
//   J2                        TwoBodyJastrow.h:250-430
//   J3                        ThreeBodyJastrow.h:30-677 (j3.cuh)
//   determinant               DiracDeterminant.cpp:80-187
//   delayed update            DelayedUpdate.h:95-231
//   inverse + log|det|        DiracMatrix.h:25-38, 93-119 (Gauss-Jordan here)
#pragma once
#include "kernels.cuh"
#include "tc.cuh"

#include <cfloat>

namespace qmc
{
constexpr int MAXK = 64; // largest delay rank a launch supports

template <typename T> struct FunctorT
{
  int n;
  T cutoff, dinv;
  T c[QMC_MAX_FUNCTOR_COEFS];
};

template <typename T> struct SysSmem
{
  T rb[9], gb[9], cn[24];
  T mi_scale2;
  FunctorT<T> j1[QMC_MAX_ION_GROUPS], j2uu, j2ud;
  T j3cut[QMC_MAX_ION_GROUPS]; // J3 ion cutoff per species
  // orbital cell and spline grid, for locating a move's stencil without
  // global loads
  double spoG[9], sdinv[3];
  long long sstride[3];
  int sgrid[3];
  int gfirst[QMC_MAX_ION_GROUPS], glast[QMC_MAX_ION_GROUPS];
  int n_groups, n_ions, n_elec, n_up, norb, npad, comp, lap_mode;
};

template <typename T> struct SplineSmem
{
  T a[3][4], da[3][4], d2a[3][4];
  long long base;
};

struct MoveSmem
{
  double red[32 * 16];
  double sums[24];
  double pos_old[3], pos_new[3];
  double p[MAXK + 1], wv[MAXK + 1], col[MAXK + 1];
  double ratio_det, curAt, curLap, curGrad[3], curUat, y;
  long long next_base;
  int accept, dc, ok;
  int eG; // moves in the current epoch (do_epoch)
  // tensor-core flush state: commit barriers (GEMM1 stages 0/1, GEMM2
  // accumulators 0/1, and the drain barrier of an aborted CTA), their phase
  // bits, the TMEM base, the abort flag and the limit of each bounded wait
  unsigned long long tc_bar[5];
  unsigned tc_phase, tc_tmem;
  int tc_on, tc_abort;
  long long tc_limit;
  // per-phase device timers (thread 0, clock64 at phase boundaries)
  int timing;
  long long tstamp;
  long long tacc[NPHASE];
};

// attribute the cycles since the last mark to `phase` (thread 0 only)
__device__ __forceinline__ void phase_mark(MoveSmem& m, int phase)
{
  if (m.timing && threadIdx.x == 0)
  {
    const long long t = clock64();
    m.tacc[phase] += t - m.tstamp;
    m.tstamp = t;
  }
}

// ----------------------------------------------------- typed views ------
template <typename T> struct WV
{
  int N, Npad, n, npad, I, k, w;
  double* R;
  T* Rs;
  T* Ainv;
  T* dpsiM;
  T* d2psiM;
  T* U;
  T* V;
  double* Binv;
  int* dlist;
  int* dcount;
  double* det_log;
  double* det_phase;
  T* Vat;
  T* Lap;
  T* Grad;
  T* Uat;
  T* d2Uat;
  T* dUat;
  T* j3Uat;
  T* j3d2Uat;
  T* j3dUat;
  int* j3cnt;  // [2][I]
  int* j3list; // [2][I][j3cap]
  int j3cap;
  double* jlog; // [3] J1, J2, J3
  uint32_t* mt;
  uint32_t* words;
  double* ur;
  double* delta;
  T* invRow;
  T* psiV;
  T* dpsiV;
  T* d2psiV;
  T* U2;
  T* tm;
  float* tci;
  double* lu;
  MoveState* ms;
  double* G;
  double* L;
  unsigned* status;
  double* bsm;  // Binv of spin bsm_spin held in shared memory (fused sweep), or null
  int bsm_spin;

  __device__ T* ainv(int s) const { return Ainv + (size_t)s * n * npad; }
  __device__ T* dpsi(int s) const { return dpsiM + (size_t)s * n * 3 * npad; }
  __device__ T* d2psi(int s) const { return d2psiM + (size_t)s * n * npad; }
  __device__ T* u(int s) const { return U + (size_t)s * k * npad; }
  __device__ T* v(int s) const { return V + (size_t)s * k * npad; }
  __device__ double* binv(int s) const { return (bsm && s == bsm_spin) ? bsm : Binv + (size_t)s * k * k; }
  __device__ int* dl(int s) const { return dlist + s * k; }
};

template <typename T> __device__ WV<T> make_wv(const DevWalkers& d, int w)
{
  WV<T> v;
  v.N = d.N, v.Npad = d.Npad, v.n = d.n, v.npad = d.npad, v.I = d.I, v.k = d.k, v.w = w;
  const size_t nn = (size_t)d.n * d.npad, kn = (size_t)d.k * d.npad;
  v.R         = d.R + (size_t)w * d.N * 3;
  v.Rs        = (T*)d.Rs + (size_t)w * 3 * d.Npad;
  v.Ainv      = (T*)d.Ainv + (size_t)w * 2 * nn;
  v.dpsiM     = (T*)d.dpsiM + (size_t)w * 2 * 3 * nn;
  v.d2psiM    = (T*)d.d2psiM + (size_t)w * 2 * nn;
  v.U         = (T*)d.U + (size_t)w * 2 * kn;
  v.V         = (T*)d.V + (size_t)w * 2 * kn;
  v.Binv      = d.Binv + (size_t)w * 2 * d.k * d.k;
  v.dlist     = d.delay_list + (size_t)w * 2 * d.k;
  v.dcount    = d.delay_count + (size_t)w * 2;
  v.det_log   = d.det_log + (size_t)w * 2;
  v.det_phase = d.det_phase + (size_t)w * 2;
  v.Vat       = (T*)d.j1_Vat + (size_t)w * d.N;
  v.Lap       = (T*)d.j1_Lap + (size_t)w * d.N;
  v.Grad      = (T*)d.j1_Grad + (size_t)w * 3 * d.N;
  v.Uat       = (T*)d.j2_Uat + (size_t)w * d.N;
  v.d2Uat     = (T*)d.j2_d2Uat + (size_t)w * d.N;
  v.dUat      = (T*)d.j2_dUat + (size_t)w * 3 * d.N;
  v.j3Uat     = d.j3_Uat ? (T*)d.j3_Uat + (size_t)w * d.N : nullptr;
  v.j3d2Uat   = d.j3_d2Uat ? (T*)d.j3_d2Uat + (size_t)w * d.N : nullptr;
  v.j3dUat    = d.j3_dUat ? (T*)d.j3_dUat + (size_t)w * 3 * d.N : nullptr;
  v.j3cnt     = d.j3_cnt ? d.j3_cnt + (size_t)w * 2 * d.I : nullptr;
  v.j3list    = d.j3_list ? d.j3_list + (size_t)w * 2 * d.I * d.j3_cap : nullptr;
  v.j3cap     = d.j3_cap;
  v.jlog      = d.j_log + (size_t)w * 3;
  v.mt        = d.mt + (size_t)w * (MT_N + 1);
  v.words     = d.words + (size_t)w * (8 * (size_t)d.N + 8);
  v.ur        = d.ur + (size_t)w * d.N;
  v.delta     = d.delta + (size_t)w * 3 * d.N;
  v.invRow    = (T*)d.invRow + (size_t)w * EPOCH_MAX * d.npad;
  v.psiV      = (T*)d.psiV + (size_t)w * d.npad;
  v.dpsiV     = (T*)d.dpsiV + (size_t)w * 3 * d.npad;
  v.d2psiV    = (T*)d.d2psiV + (size_t)w * d.npad;
  v.U2        = (T*)d.U2 + (size_t)w * kn;
  v.tm        = (T*)d.tm + (size_t)w * d.n * d.k;
  v.tci       = d.tci ? d.tci + (size_t)w * 2 * (d.k <= 32 ? 32 : 64) * d.npad : nullptr; // tc_image_floats
  v.lu        = d.lu ? d.lu + (size_t)w * 2 * nn : nullptr;
  v.ms        = d.ms + w;
  v.G         = d.G + (size_t)w * d.N * 3;
  v.L         = d.L + (size_t)w * d.N;
  v.status    = d.status;
  v.bsm       = nullptr;
  v.bsm_spin  = -1;
  return v;
}

template <typename T> __device__ void load_sys(const DevSystem* __restrict__ s, SysSmem<T>& ss)
{
  const int tid = threadIdx.x;
  if (tid < 9)
  {
    ss.rb[tid]   = (T)s->rb[tid];
    ss.gb[tid]   = (T)s->gb[tid];
    ss.spoG[tid] = s->spoG[tid];
  }
  if (tid < 3)
  {
    ss.sdinv[tid]   = s->dinv[tid];
    ss.sgrid[tid]   = s->grid[tid];
    ss.sstride[tid] = tid == 0 ? s->xs : (tid == 1 ? s->ys : s->zs);
  }
  if (tid < 24)
    ss.cn[tid] = (T)s->corners[tid];
  for (int i = tid; i < QMC_MAX_ION_GROUPS * QMC_MAX_FUNCTOR_COEFS; i += blockDim.x)
  {
    const int g = i / QMC_MAX_FUNCTOR_COEFS, c = i % QMC_MAX_FUNCTOR_COEFS;
    ss.j1[g].c[c] = (T)s->j1[g].c[c];
  }
  for (int c = tid; c < QMC_MAX_FUNCTOR_COEFS; c += blockDim.x)
  {
    ss.j2uu.c[c] = (T)s->j2uu.c[c];
    ss.j2ud.c[c] = (T)s->j2ud.c[c];
  }
  if (tid == 0)
  {
    for (int g = 0; g < QMC_MAX_ION_GROUPS; ++g)
    {
      ss.j1[g].n      = s->j1[g].n;
      ss.j1[g].cutoff = (T)s->j1[g].cutoff;
      ss.j1[g].dinv   = (T)s->j1[g].dinv;
      ss.gfirst[g]    = s->gfirst[g];
      ss.glast[g]     = s->glast[g];
      ss.j3cut[g]     = (T)s->j3_icut[g];
    }
    ss.j2uu.n = s->j2uu.n, ss.j2uu.cutoff = (T)s->j2uu.cutoff, ss.j2uu.dinv = (T)s->j2uu.dinv;
    ss.j2ud.n = s->j2ud.n, ss.j2ud.cutoff = (T)s->j2ud.cutoff, ss.j2ud.dinv = (T)s->j2ud.dinv;
    ss.n_groups = s->n_groups, ss.n_ions = s->n_ions, ss.n_elec = s->n_elec, ss.n_up = s->n_up;
    ss.norb = s->norb, ss.npad = s->npad, ss.comp = s->comp, ss.lap_mode = s->lap_mode;
    ss.mi_scale2 = (T)s->mi_scale2;
  }
  __syncthreads();
}

// true when every periodic image of the displacement is at least sqrt(rc2)
// away, so the pair is outside the cutoff whatever image the corner search
// would pick (see DevSystem::mi_scale2); exact, no false positives
template <typename T>
__device__ __forceinline__ bool beyond_cutoff(T dx, T dy, T dz, const T* __restrict__ gb, T scale2, T rc2)
{
  T f0 = dx * gb[0] + dy * gb[3] + dz * gb[6];
  T f1 = dx * gb[1] + dy * gb[4] + dz * gb[7];
  T f2 = dx * gb[2] + dy * gb[5] + dz * gb[8];
  f0 -= floor(f0);
  f1 -= floor(f1);
  f2 -= floor(f2);
  const T m0 = min(f0, T(1) - f0), m1 = min(f1, T(1) - f1), m2 = min(f2, T(1) - f2);
  return scale2 * (m0 * m0 + m1 * m1 + m2 * m2) >= rc2;
}

// ------------------------------------------------------ minimum image --
// DTD_BConds<T,3,PPPG+SOA_OFFSET>::computeDistances for one pair; the
// caller has applied `flip` to the displacement and applies it again.
template <typename T>
__device__ __forceinline__ T min_image(T& dx, T& dy, T& dz, const T* __restrict__ rb, const T* __restrict__ gb,
                                       const T* __restrict__ cn)
{
  const T ar0  = -floor(dx * gb[0] + dy * gb[3] + dz * gb[6]);
  const T ar1  = -floor(dx * gb[1] + dy * gb[4] + dz * gb[7]);
  const T ar2  = -floor(dx * gb[2] + dy * gb[5] + dz * gb[8]);
  const T delx = dx + ar0 * rb[0] + ar1 * rb[3] + ar2 * rb[6];
  const T dely = dy + ar0 * rb[1] + ar1 * rb[4] + ar2 * rb[7];
  const T delz = dz + ar0 * rb[2] + ar1 * rb[5] + ar2 * rb[8];
  T rmin       = delx * delx + dely * dely + delz * delz;
  int ic       = 0;
#pragma unroll
  for (int c = 1; c < 8; ++c)
  {
    const T x  = delx + cn[3 * c];
    const T y  = dely + cn[3 * c + 1];
    const T z  = delz + cn[3 * c + 2];
    const T r2 = x * x + y * y + z * z;
    ic         = (r2 < rmin) ? c : ic;
    rmin       = (r2 < rmin) ? r2 : rmin;
  }
  dx = delx + cn[3 * ic];
  dy = dely + cn[3 * ic + 1];
  dz = delz + cn[3 * ic + 2];
  return sqrt(rmin);
}

// ------------------------------------------------------ radial functor --
// BsplineFunctor::evaluateVGL for one pair inside the cutoff: u, du/dr / r, d2u/dr2
template <typename T>
__device__ __forceinline__ void functor_vgl(const FunctorT<T>& f, T r, T& u, T& du, T& d2u)
{
  const T rinv = T(1) / r;
  r *= f.dinv;
  const int i = (int)r;
  const T t = r - T(i), tp1 = t * t, tp0 = tp1 * t, tp2 = t;
  const T s0 = f.c[i], s1 = f.c[i + 1], s2 = f.c[i + 2], s3 = f.c[i + 3];
  // constants of BsplineFunctor's A, dA, d2A tables
  d2u = f.dinv * f.dinv *
      (s0 * (T(-1.0) * tp2 + T(1.0)) + s1 * (T(3.0) * tp2 + T(-2.0)) + s2 * (T(-3.0) * tp2 + T(1.0)) +
       s3 * (T(1.0) * tp2 + T(0.0)));
  du = f.dinv * rinv *
      (s0 * (T(-0.5) * tp1 + T(1.0) * tp2 + T(-0.5)) + s1 * (T(1.5) * tp1 + T(-2.0) * tp2 + T(0.0)) +
       s2 * (T(-1.5) * tp1 + T(1.0) * tp2 + T(0.5)) + s3 * (T(0.5) * tp1 + T(0.0) * tp2 + T(0.0)));
  u = (s0 * (T(-1.0 / 6.0) * tp0 + T(3.0 / 6.0) * tp1 + T(-3.0 / 6.0) * tp2 + T(1.0 / 6.0)) +
       s1 * (T(3.0 / 6.0) * tp0 + T(-6.0 / 6.0) * tp1 + T(0.0 / 6.0) * tp2 + T(4.0 / 6.0)) +
       s2 * (T(-3.0 / 6.0) * tp0 + T(3.0 / 6.0) * tp1 + T(3.0 / 6.0) * tp2 + T(1.0 / 6.0)) +
       s3 * (T(1.0 / 6.0) * tp0 + T(0.0 / 6.0) * tp1 + T(0.0 / 6.0) * tp2 + T(0.0 / 6.0)));
}
// BsplineFunctor::evaluateV for one pair inside the cutoff
template <typename T> __device__ __forceinline__ T functor_v(const FunctorT<T>& f, T r)
{
  r *= f.dinv;
  const int i = (int)r;
  const T t = r - T(i), tp1 = t * t, tp0 = tp1 * t, tp2 = t;
  const T d1 = f.c[i] * (T(-1.0 / 6.0) * tp0 + T(3.0 / 6.0) * tp1 + T(-3.0 / 6.0) * tp2 + T(1.0 / 6.0));
  const T d2 = f.c[i + 1] * (T(3.0 / 6.0) * tp0 + T(-6.0 / 6.0) * tp1 + T(0.0 / 6.0) * tp2 + T(4.0 / 6.0));
  const T d3 = f.c[i + 2] * (T(-3.0 / 6.0) * tp0 + T(3.0 / 6.0) * tp1 + T(3.0 / 6.0) * tp2 + T(1.0 / 6.0));
  const T d4 = f.c[i + 3] * (T(1.0 / 6.0) * tp0 + T(0.0 / 6.0) * tp1 + T(0.0 / 6.0) * tp2 + T(0.0 / 6.0));
  return d1 + d2 + d3 + d4;
}

// --------------------------------------------------------- B-spline SPO --
// One dimension of computeLocationAndFractional + compute_prefactors: u is
// the Cartesian point's fractional coordinate before wrapping (r . spoG
// column d), formed in FP64 in both forms; returns the stencil corner's
// offset along d and, when a is given, the weights a, da, d2a.
template <typename T>
__device__ __forceinline__ long long spline_dim(double u, double dinv, int grid, long long stride, T* a, T* da,
                                                T* d2a)
{
  if (-DBL_EPSILON < u && u < 0)
    u = 0.0;
  else
    u -= floor(u);
  const double x = u * dinv;
  int ind;
  double t;
  if (x < 0)
  {
    ind = 0;
    t   = 0.0;
  }
  else
  {
    const double ip = floor(x);
    t               = x - ip;
    ind             = (int)ip;
    if (ind > grid - 1)
    {
      ind = grid - 1;
      t   = 1.0 - DBL_EPSILON;
    }
  }
  if (a)
  {
    a[0]   = (T)(((-1.0 / 6.0 * t + 3.0 / 6.0) * t + -3.0 / 6.0) * t + 1.0 / 6.0);
    a[1]   = (T)(((3.0 / 6.0 * t + -6.0 / 6.0) * t + 0.0 / 6.0) * t + 4.0 / 6.0);
    a[2]   = (T)(((-3.0 / 6.0 * t + 3.0 / 6.0) * t + 3.0 / 6.0) * t + 1.0 / 6.0);
    a[3]   = (T)(((1.0 / 6.0 * t + 0.0 / 6.0) * t + 0.0 / 6.0) * t + 0.0 / 6.0);
    da[0]  = (T)((-0.5 * t + 1.0) * t + -0.5);
    da[1]  = (T)((1.5 * t + -2.0) * t + 0.0);
    da[2]  = (T)((-1.5 * t + 1.0) * t + 0.5);
    da[3]  = (T)((0.5 * t + 0.0) * t + 0.0);
    d2a[0] = (T)(-1.0 * t + 1.0);
    d2a[1] = (T)(3.0 * t + -2.0);
    d2a[2] = (T)(-3.0 * t + 1.0);
    d2a[3] = (T)(1.0 * t + 0.0);
  }
  return (long long)ind * stride;
}

// the whole stencil location of a Cartesian point (one thread)
template <typename T> __device__ void spline_locate(const DevSystem* __restrict__ s, const double* pos, SplineSmem<T>& sp)
{
  const long long strides[3] = {s->xs, s->ys, s->zs};
  long long base             = 0;
  for (int d = 0; d < 3; ++d)
  {
    const double u = pos[0] * s->spoG[d] + pos[1] * s->spoG[3 + d] + pos[2] * s->spoG[6 + d];
    base += spline_dim<T>(u, s->dinv[d], s->grid[d], strides[d], sp.a[d], sp.da[d], sp.d2a[d]);
  }
  sp.base = base;
}

// L2 prefetch of `bytes` (multiple of 16) at a 16-byte aligned address,
// issued to the bulk-copy (TMA) engine; no register or shared memory used
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes)
{
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// L2 evict-first cache policy, for the data a move streams once (the spline
// stencil, the derivative rows of the moved electron): its lines go before
// those a walker reuses from move to move (U, V, the move vectors, the
// Jastrow arrays).  At NiO-128 with 512 walkers the sweep measured 181 ms
// with it against 187 ms without.  The flush's passes over Ainv keep the
// default policy: GEMM2 re-reads the rows GEMM1 has just read, and
// evict-first on either pass measured slower.
__device__ __forceinline__ uint64_t l2_evict_first()
{
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
// 16-byte load of read-only data under an L2 cache policy
__device__ __forceinline__ float4 ld_stream(const float4* a, uint64_t pol)
{
  float4 v;
  asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
      : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double2 ld_stream(const double2* a, uint64_t pol)
{
  double2 v;
  asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol));
  return v;
}
// 16-byte load of data the kernel also writes, under an L2 cache policy
__device__ __forceinline__ float4 ld_stream_rw(const float4* a, uint64_t pol)
{
  float4 v;
  asm volatile("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(a), "l"(pol)
               : "memory");
  return v;
}
__device__ __forceinline__ double2 ld_stream_rw(const double2* a, uint64_t pol)
{
  double2 v;
  asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(a), "l"(pol) : "memory");
  return v;
}

template <typename T> struct SplineOut
{
  static constexpr int VW = Vec16<T>::width;
  T v[VW], gx[VW], gy[VW], gz[VW], hxx[VW], hxy[VW], hxz[VW], hyy[VW], hyz[VW], hzz[VW];
};

// evaluate_vgh for the VW orbitals starting at element e0 (16-byte vector)
template <typename T, bool FULL>
__device__ __forceinline__ void spline_eval(const T* __restrict__ coefs, long long xs, long long ys, long long zs,
                                            const SplineSmem<T>& sp, const double* dinv, int e0, SplineOut<T>& o)
{
  using V              = typename Vec16<T>::type;
  constexpr int VW     = Vec16<T>::width;
#pragma unroll
  for (int e = 0; e < VW; ++e)
    o.v[e] = o.gx[e] = o.gy[e] = o.gz[e] = o.hxx[e] = o.hxy[e] = o.hxz[e] = o.hyy[e] = o.hyz[e] = o.hzz[e] = T(0);
  const T* c0p    = coefs + sp.base + e0;
  const uint64_t pol = l2_evict_first();
#pragma unroll 1
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
    {
      const T* p = c0p + i * xs + j * ys;
      V c[4];
#pragma unroll
      for (int z = 0; z < 4; ++z)
        c[z] = ld_stream(reinterpret_cast<const V*>(p + z * zs), pol);
      const T pre20 = sp.d2a[0][i] * sp.a[1][j];
      const T pre10 = sp.da[0][i] * sp.a[1][j];
      const T pre00 = sp.a[0][i] * sp.a[1][j];
      const T pre11 = sp.da[0][i] * sp.da[1][j];
      const T pre01 = sp.a[0][i] * sp.da[1][j];
      const T pre02 = sp.a[0][i] * sp.d2a[1][j];
#pragma unroll
      for (int e = 0; e < VW; ++e)
      {
        const T v0 = reinterpret_cast<const T*>(&c[0])[e];
        const T v1 = reinterpret_cast<const T*>(&c[1])[e];
        const T v2 = reinterpret_cast<const T*>(&c[2])[e];
        const T v3 = reinterpret_cast<const T*>(&c[3])[e];
        const T sum0 = sp.a[2][0] * v0 + sp.a[2][1] * v1 + sp.a[2][2] * v2 + sp.a[2][3] * v3;
        const T sum1 = sp.da[2][0] * v0 + sp.da[2][1] * v1 + sp.da[2][2] * v2 + sp.da[2][3] * v3;
        const T sum2 = sp.d2a[2][0] * v0 + sp.d2a[2][1] * v1 + sp.d2a[2][2] * v2 + sp.d2a[2][3] * v3;
        o.hxx[e] += pre20 * sum0;
        o.hyy[e] += pre02 * sum0;
        o.hzz[e] += pre00 * sum2;
        if (FULL)
        {
          o.hxy[e] += pre11 * sum0;
          o.hxz[e] += pre10 * sum1;
          o.hyz[e] += pre01 * sum1;
        }
        o.gx[e] += pre10 * sum0;
        o.gy[e] += pre01 * sum0;
        o.gz[e] += pre00 * sum1;
        o.v[e] += pre00 * sum0;
      }
    }
  const T dx = (T)dinv[0], dy = (T)dinv[1], dz = (T)dinv[2];
#pragma unroll
  for (int e = 0; e < VW; ++e)
  {
    o.gx[e] *= dx;
    o.gy[e] *= dy;
    o.gz[e] *= dz;
    o.hxx[e] *= dx * dx;
    o.hyy[e] *= dy * dy;
    o.hzz[e] *= dz * dz;
    if (FULL)
    {
      o.hxy[e] *= dx * dy;
      o.hxz[e] *= dx * dz;
      o.hyz[e] *= dy * dz;
    }
  }
}

// evaluate_v (values only) for VW orbitals at e0
template <typename T>
__device__ __forceinline__ void spline_eval_v(const T* __restrict__ coefs, long long xs, long long ys, long long zs,
                                              const SplineSmem<T>& sp, int e0, T* out)
{
  using V          = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
#pragma unroll
  for (int e = 0; e < VW; ++e)
    out[e] = T(0);
  const T* c0p    = coefs + sp.base + e0;
  const uint64_t pol = l2_evict_first();
#pragma unroll 1
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
    {
      const T* p = c0p + i * xs + j * ys;
      V c[4];
#pragma unroll
      for (int z = 0; z < 4; ++z)
        c[z] = ld_stream(reinterpret_cast<const V*>(p + z * zs), pol);
      const T pre00 = sp.a[0][i] * sp.a[1][j];
#pragma unroll
      for (int e = 0; e < VW; ++e)
        out[e] += pre00 *
            (sp.a[2][0] * reinterpret_cast<const T*>(&c[0])[e] + sp.a[2][1] * reinterpret_cast<const T*>(&c[1])[e] +
             sp.a[2][2] * reinterpret_cast<const T*>(&c[2])[e] + sp.a[2][3] * reinterpret_cast<const T*>(&c[3])[e]);
    }
}

// ------------------------------------------------------- determinant ----
// DelayedUpdate::getInvRow: invRow = Ainv[r] - V^T (Binv^T (U Ainv[r])).
// Stores the intermediate Binv^T p in row dc of Binv, as the reference does
// (acceptRow reads it back).  Block-wide.
template <typename T> __device__ void get_inv_row(const WV<T>& wv, MoveSmem& m, int s, int r, int dc)
{
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  const int nvec  = wv.npad / VW;
  const T* arow   = wv.ainv(s) + (size_t)r * wv.npad;
  if (dc == 0)
  {
    for (int q = tid; q < nvec; q += NT)
      reinterpret_cast<Vt*>(wv.invRow)[q] = reinterpret_cast<const Vt*>(arow)[q];
    return;
  }
  const T* U = wv.u(s);
  const T* V = wv.v(s);
  for (int d = wid; d < dc; d += nw)
  {
    const Vt* ud = reinterpret_cast<const Vt*>(U + (size_t)d * wv.npad);
    const Vt* av = reinterpret_cast<const Vt*>(arow);
    T acc        = T(0);
#pragma unroll 4
    for (int jv = lane; jv < nvec; jv += 32)
    {
      const Vt x = ud[jv], y = av[jv];
#pragma unroll
      for (int e = 0; e < VW; ++e)
        acc += reinterpret_cast<const T*>(&x)[e] * reinterpret_cast<const T*>(&y)[e];
    }
    const double sum = warp_sum((double)acc);
    if (lane == 0)
      m.p[d] = sum;
  }
  __syncthreads();
  double* B = wv.binv(s);
  for (int a = tid; a < dc; a += NT)
  {
    double acc = 0.0;
    for (int b = 0; b < dc; ++b)
      acc += B[b * wv.k + a] * m.p[b];
    m.wv[a] = acc;
    if (dc < wv.k)
      B[dc * wv.k + a] = acc;
  }
  __syncthreads();
  for (int q = tid; q < nvec; q += NT)
  {
    Vt a = reinterpret_cast<const Vt*>(arow)[q];
    T* ap = reinterpret_cast<T*>(&a);
    double acc[VW];
#pragma unroll
    for (int e = 0; e < VW; ++e)
      acc[e] = 0.0;
#pragma unroll 4
    for (int d = 0; d < dc; ++d)
    {
      Vt vv = reinterpret_cast<const Vt*>(V + (size_t)d * wv.npad)[q];
      const double wd = m.wv[d];
#pragma unroll
      for (int e = 0; e < VW; ++e)
        acc[e] += (double)reinterpret_cast<T*>(&vv)[e] * wd;
    }
#pragma unroll
    for (int e = 0; e < VW; ++e)
      ap[e] = (T)((double)ap[e] - acc[e]);
    reinterpret_cast<Vt*>(wv.invRow)[q] = a;
  }
}

#include "flush.cuh"

// DiracDeterminant::acceptMove + DelayedUpdate::acceptRow.  psiV (and the
// derivative rows when `partial`) come from the move scratch.  Block-wide.
template <typename T>
__device__ void det_accept(const WV<T>& wv, MoveSmem& m, int s, int r, double ratio, bool partial, bool track_log,
                           T* smem)
{
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  const int npad = wv.npad, nvec = npad / VW, k = wv.k;
  const int dc = wv.dcount[s];
  T* arow      = wv.ainv(s) + (size_t)r * npad;
  T* Vd        = wv.v(s) + (size_t)dc * npad;
  T* Ud        = wv.u(s) + (size_t)dc * npad;
  for (int q = tid; q < nvec; q += NT)
  {
    reinterpret_cast<Vt*>(Vd)[q] = reinterpret_cast<const Vt*>(arow)[q];
    reinterpret_cast<Vt*>(Ud)[q] = reinterpret_cast<const Vt*>(wv.psiV)[q];
    if (partial)
    {
      for (int c = 0; c < 3; ++c)
        reinterpret_cast<Vt*>(wv.dpsi(s) + ((size_t)r * 3 + c) * npad)[q] =
            reinterpret_cast<const Vt*>(wv.dpsiV + (size_t)c * npad)[q];
      reinterpret_cast<Vt*>(wv.d2psi(s) + (size_t)r * npad)[q] = reinterpret_cast<const Vt*>(wv.d2psiV)[q];
    }
  }
  if (tid == 0)
  {
    if (track_log)
    {
      wv.det_phase[s] += (ratio > 0) ? 0.0 : kPi;
      wv.det_log[s] += log(fabs(ratio));
    }
    wv.dl(s)[dc] = r;
  }
  __syncthreads();
  // p[d] = -V[d] . psiV  for d <= dc
  const T* Vs = wv.v(s);
  for (int d = wid; d <= dc; d += nw)
  {
    const Vt* vd = reinterpret_cast<const Vt*>(Vs + (size_t)d * npad);
    const Vt* pv = reinterpret_cast<const Vt*>(wv.psiV);
    T acc        = T(0);
#pragma unroll 4
    for (int jv = lane; jv < nvec; jv += 32)
    {
      const Vt x = vd[jv], y = pv[jv];
#pragma unroll
      for (int e = 0; e < VW; ++e)
        acc += reinterpret_cast<const T*>(&x)[e] * reinterpret_cast<const T*>(&y)[e];
    }
    const double sum = warp_sum((double)acc);
    if (lane == 0)
      m.p[d] = -sum;
  }
  __syncthreads();
  double* B = wv.binv(s);
  if (tid == 0)
  {
    double y = -m.p[dc];
    for (int i = 0; i < dc; i++)
      y += B[dc * k + i] * m.p[i];
    y              = 1.0 / y;
    B[dc * k + dc] = y;
    m.y            = y;
  }
  __syncthreads();
  const double y = m.y;
  for (int b = tid; b < dc; b += NT)
  {
    double acc = 0.0;
    for (int a = 0; a < dc; ++a)
      acc += B[b * k + a] * m.p[a];
    m.col[b] = y * acc;
  }
  __syncthreads();
  for (int idx = tid; idx < dc * dc; idx += NT)
  {
    const int b = idx / dc, a = idx % dc;
    B[b * k + a] -= B[dc * k + a] * m.col[b];
  }
  for (int b = tid; b < dc; b += NT)
    B[b * k + dc] = m.col[b];
  __syncthreads();
  for (int i = tid; i < dc; i += NT)
    B[dc * k + i] *= -y;
  if (tid == 0)
    wv.dcount[s] = dc + 1;
  __syncthreads();
  if (dc + 1 == k)
    flush(wv, m, s, smem);
}

// ---------------------------------------------------------- Jastrows ----
template <typename T> __device__ __forceinline__ int ion_group(const SysSmem<T>& ss, int c)
{
  int g = 0;
  for (int h = 0; h < ss.n_groups; ++h)
    if (c >= ss.gfirst[h] && c < ss.glast[h])
      g = h;
  return g;
}

// partial J1 sums over the ions for a position: curAt, grad[3], lap
// (OneBodyJastrow::computeU3 + accumulateGL; the AB row is always flipped)
template <typename T, typename A>
__device__ void j1_partials(const SysSmem<T>& ss, const T* __restrict__ ions /*[3][I]*/, const double* pos, A* part)
{
  const T px = (T)pos[0], py = (T)pos[1], pz = (T)pos[2];
  for (int c = threadIdx.x; c < ss.n_ions; c += blockDim.x)
  {
    T dx = (ions[c] - px) * T(-1), dy = (ions[ss.n_ions + c] - py) * T(-1), dz = (ions[2 * ss.n_ions + c] - pz) * T(-1);
    const FunctorT<T>& f = ss.j1[ion_group(ss, c)];
    if (beyond_cutoff(dx, dy, dz, ss.gb, ss.mi_scale2, f.cutoff * f.cutoff))
      continue;
    const T r = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
    dx *= T(-1), dy *= T(-1), dz *= T(-1);
    if (r < f.cutoff)
    {
      T u, du, d2u;
      functor_vgl(f, r, u, du, d2u);
      part[0] += (A)u;
      part[1] += (A)(du * dx);
      part[2] += (A)(du * dy);
      part[3] += (A)(du * dz);
      part[4] += (A)(d2u + T(2) * du);
    }
  }
}
template <typename T>
__device__ void j1_value(const SysSmem<T>& ss, const T* __restrict__ ions, const double* pos, double* part)
{
  const T px = (T)pos[0], py = (T)pos[1], pz = (T)pos[2];
  for (int c = threadIdx.x; c < ss.n_ions; c += blockDim.x)
  {
    T dx = (ions[c] - px) * T(-1), dy = (ions[ss.n_ions + c] - py) * T(-1), dz = (ions[2 * ss.n_ions + c] - pz) * T(-1);
    const T r = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
    const FunctorT<T>& f = ss.j1[ion_group(ss, c)];
    if (r < f.cutoff)
      part[0] += (double)functor_v(f, r);
  }
}

// J2 pair lists: each warp scans its electrons with the exact cutoff test
// (beyond_cutoff) and compacts the candidates into its slice of `wlist`
// (J2_SCAN chunks of 32 electrons per round), then all lanes work through
// the list.  Only a few per cent of the pairs are within the cutoff in the
// NiO cells, so this replaces a divergent branch on most warp steps with one
// dense pass.
constexpr int J2_SCAN = 8;
// shared-memory bytes of the per-warp candidate lists (up to 8 warps)
__host__ __device__ constexpr size_t j2_list_bytes() { return (size_t)8 * 32 * J2_SCAN * sizeof(int); }

// partial J2 sums over the electrons for electron iel moved to pos:
// sum u, sum du*dr (TwoBodyJastrow::ratioGrad with the move row, flip = iel).
// Rs is not __restrict__: accepted moves rewrite it during a launch (on
// another SM, between units of the work-queue sweep), so its loads must stay
// on the coherent path rather than the read-only one
template <typename T, typename A>
__device__ void j2_partials(const SysSmem<T>& ss, const T* Rs, int Npad, int iel, const double* pos,
                            A* part, bool grads, int* wlist)
{
  const T px = (T)pos[0], py = (T)pos[1], pz = (T)pos[2];
  const int gi = iel < ss.n_up ? 0 : 1;
  const int N = ss.n_elec, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  int* lst             = wlist + wid * 32 * J2_SCAN;
  const int nchunks    = (N + 31) >> 5;
  for (int c0 = wid; c0 < nchunks; c0 += nw * J2_SCAN)
  {
    int cnt = 0;
#pragma unroll
    for (int r = 0; r < J2_SCAN; ++r)
    {
      const int j = ((c0 + r * nw) << 5) + lane;
      bool in     = false;
      if (j < N && j != iel)
      {
        const T flip = j < iel ? T(1) : T(-1);
        const T dx = (Rs[j] - px) * flip, dy = (Rs[Npad + j] - py) * flip, dz = (Rs[2 * Npad + j] - pz) * flip;
        const FunctorT<T>& f = (gi == (j < ss.n_up ? 0 : 1)) ? ss.j2uu : ss.j2ud;
        in = !beyond_cutoff(dx, dy, dz, ss.gb, ss.mi_scale2, f.cutoff * f.cutoff);
      }
      const unsigned b = __ballot_sync(0xffffffffu, in);
      if (in)
        lst[cnt + __popc(b & below)] = j;
      cnt += __popc(b);
    }
    __syncwarp();
    for (int q = lane; q < cnt; q += 32)
    {
      const int j  = lst[q];
      const T flip = j < iel ? T(1) : T(-1);
      T dx = (Rs[j] - px) * flip, dy = (Rs[Npad + j] - py) * flip, dz = (Rs[2 * Npad + j] - pz) * flip;
      const FunctorT<T>& f = (gi == (j < ss.n_up ? 0 : 1)) ? ss.j2uu : ss.j2ud;
      const T r = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
      if (r < f.cutoff)
      {
        if (grads)
        {
          T uu, du, d2u;
          functor_vgl(f, r, uu, du, d2u);
          dx *= flip, dy *= flip, dz *= flip;
          part[0] += (A)uu;
          part[1] += (A)(du * dx);
          part[2] += (A)(du * dy);
          part[3] += (A)(du * dz);
        }
        else
          part[0] += (A)functor_v(f, r);
      }
    }
    __syncwarp(); // the list is rewritten by the next round
  }
}

// TwoBodyJastrow::acceptMove: update every electron's Uat, dUat, d2Uat with
// the old (setActive) and new (move) rows of electron iel.  A pair beyond
// the cutoff at both the old and the new position adds exact zeros to Uat,
// dUat and d2Uat (TwoBodyJastrow.h:307-353 updates every entry with
// new - old), so the scan keeps the pairs within the cutoff at either
// position and only those entries are read and written.  Block-wide.
template <typename T>
__device__ void j2_accept(const SysSmem<T>& ss, const WV<T>& wv, MoveSmem& m, int iel, int* wlist)
{
  const T ox = (T)m.pos_old[0], oy = (T)m.pos_old[1], oz = (T)m.pos_old[2];
  const T nx = (T)m.pos_new[0], ny = (T)m.pos_new[1], nz = (T)m.pos_new[2];
  const int gi = iel < ss.n_up ? 0 : 1;
  const int Npad = wv.Npad, N = wv.N;
  const T* Rs = wv.Rs;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned below = (1u << lane) - 1u;
  int* lst             = wlist + wid * 32 * J2_SCAN;
  const int nchunks    = (N + 31) >> 5;
  T part[4] = {T(0), T(0), T(0), T(0)};
  for (int c0 = wid; c0 < nchunks; c0 += nw * J2_SCAN)
  {
    int cnt = 0;
#pragma unroll
    for (int r = 0; r < J2_SCAN; ++r)
    {
      const int j = ((c0 + r * nw) << 5) + lane;
      bool in     = false;
      if (j < N && j != iel)
      {
        const T flip = j < iel ? T(1) : T(-1);
        const T rx = Rs[j], ry = Rs[Npad + j], rz = Rs[2 * Npad + j];
        const FunctorT<T>& f = (gi == (j < ss.n_up ? 0 : 1)) ? ss.j2uu : ss.j2ud;
        const T rc2 = f.cutoff * f.cutoff;
        in = !beyond_cutoff((rx - ox) * flip, (ry - oy) * flip, (rz - oz) * flip, ss.gb, ss.mi_scale2, rc2) ||
            !beyond_cutoff((rx - nx) * flip, (ry - ny) * flip, (rz - nz) * flip, ss.gb, ss.mi_scale2, rc2);
      }
      const unsigned b = __ballot_sync(0xffffffffu, in);
      if (in)
        lst[cnt + __popc(b & below)] = j;
      cnt += __popc(b);
    }
    __syncwarp();
    for (int q = lane; q < cnt; q += 32)
    {
      const int j  = lst[q];
      const T flip = j < iel ? T(1) : T(-1);
      const T rx = Rs[j], ry = Rs[Npad + j], rz = Rs[2 * Npad + j];
      const T ua = wv.Uat[j], la = wv.d2Uat[j], g0 = wv.dUat[j], g1 = wv.dUat[N + j], g2 = wv.dUat[2 * N + j];
      const FunctorT<T>& f = (gi == (j < ss.n_up ? 0 : 1)) ? ss.j2uu : ss.j2ud;
      T odx = (rx - ox) * flip, ody = (ry - oy) * flip, odz = (rz - oz) * flip;
      T ndx = (rx - nx) * flip, ndy = (ry - ny) * flip, ndz = (rz - nz) * flip;
      T uo = 0, duo = 0, d2uo = 0, un = 0, dun = 0, d2un = 0;
      const T ro = min_image(odx, ody, odz, ss.rb, ss.gb, ss.cn);
      if (ro < f.cutoff)
        functor_vgl(f, ro, uo, duo, d2uo);
      odx *= flip, ody *= flip, odz *= flip;
      const T rn = min_image(ndx, ndy, ndz, ss.rb, ss.gb, ss.cn);
      if (rn < f.cutoff)
        functor_vgl(f, rn, un, dun, d2un);
      ndx *= flip, ndy *= flip, ndz *= flip;
      const T newl = d2un + T(2) * dun;
      const T dl   = d2uo + T(2) * duo - newl;
      wv.Uat[j]   = ua + (un - uo);
      wv.d2Uat[j] = la + dl;
      part[0] -= newl;
      const T ng0 = dun * ndx, ng1 = dun * ndy, ng2 = dun * ndz;
      wv.dUat[j]         = g0 - (ng0 - duo * odx);
      wv.dUat[N + j]     = g1 - (ng1 - duo * ody);
      wv.dUat[2 * N + j] = g2 - (ng2 - duo * odz);
      part[1] += ng0;
      part[2] += ng1;
      part[3] += ng2;
    }
    __syncwarp();
  }
  {
    double dpart[4] = {(double)part[0], (double)part[1], (double)part[2], (double)part[3]};
    block_sum<4>(dpart, m.red, m.sums);
  }
  if (threadIdx.x == 0)
  {
    wv.jlog[1] += (double)wv.Uat[iel] - m.curUat;
    wv.Uat[iel]          = (T)m.curUat;
    wv.dUat[iel]         = (T)m.sums[1];
    wv.dUat[N + iel]     = (T)m.sums[2];
    wv.dUat[2 * N + iel] = (T)m.sums[3];
    wv.d2Uat[iel]        = (T)m.sums[0];
  }
  __syncthreads();
}

} // namespace qmc

#include "j3.cuh"

namespace qmc
{
// ------------------------------------------------------- evaluateGL -----
// WaveFunction::evaluateGL (WaveFunction.cpp:261-279): G, L per electron and
// the log values; warp per electron for the determinant row dots.
template <typename T> __device__ void evaluate_gl(const SysSmem<T>& ss, const WV<T>& wv, MoveSmem& m, double* logpsi)
{
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  const bool DET = ss.comp & QMC_WF_DET, J1 = ss.comp & QMC_WF_J1, J2 = ss.comp & QMC_WF_J2;
  const bool J3 = ss.comp & QMC_WF_J3;
  const int N = wv.N, npad = wv.npad;
  for (int i = wid; i < N; i += nw)
  {
    double rv[3] = {0.0, 0.0, 0.0}, lap = 0.0;
    if (DET)
    {
      const int s = i < ss.n_up ? 0 : 1, r = i - (s ? ss.n_up : 0);
      const T* a  = wv.ainv(s) + (size_t)r * npad;
      const T* dp = wv.dpsi(s) + (size_t)r * 3 * npad;
      const T* d2 = wv.d2psi(s) + (size_t)r * npad;
      for (int j = lane; j < npad; j += 32)
      {
        const double aj = (double)a[j];
        rv[0] += aj * (double)dp[j];
        rv[1] += aj * (double)dp[npad + j];
        rv[2] += aj * (double)dp[2 * npad + j];
        lap += aj * (double)d2[j];
      }
      rv[0] = warp_sum(rv[0]);
      rv[1] = warp_sum(rv[1]);
      rv[2] = warp_sum(rv[2]);
      lap   = warp_sum(lap);
    }
    if (lane == 0)
    {
      double g[3] = {rv[0], rv[1], rv[2]};
      double l    = lap - (rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
      if (J1)
      {
        for (int c = 0; c < 3; ++c)
          g[c] += (double)wv.Grad[c * N + i];
        l -= (double)wv.Lap[i];
      }
      if (J2)
      {
        for (int c = 0; c < 3; ++c)
          g[c] += (double)wv.dUat[c * N + i];
        l += (double)wv.d2Uat[i];
      }
      if (J3)
      {
        for (int c = 0; c < 3; ++c)
          g[c] += (double)wv.j3dUat[c * N + i];
        l += (double)wv.j3d2Uat[i];
      }
      for (int c = 0; c < 3; ++c)
        wv.G[3 * i + c] = g[c];
      wv.L[i] = l;
    }
  }
  double part[3] = {0.0, 0.0, 0.0};
  for (int i = tid; i < N; i += NT)
  {
    if (J1)
      part[0] += (double)wv.Vat[i];
    if (J2)
      part[1] += (double)wv.Uat[i];
    if (J3)
      part[2] += (double)wv.j3Uat[i];
  }
  block_sum<3>(part, m.red, m.sums);
  if (tid == 0)
  {
    wv.jlog[0] = J1 ? -m.sums[0] : 0.0;
    wv.jlog[1] = J2 ? -0.5 * m.sums[1] : 0.0;
    wv.jlog[2] = J3 ? -0.5 * m.sums[2] : 0.0;
    const double lp = (DET ? wv.det_log[0] + wv.det_log[1] : 0.0) + wv.jlog[0] + wv.jlog[1] + wv.jlog[2];
    if (logpsi)
      *logpsi = lp;
  }
  __syncthreads();
}

// ------------------------------------------------------------- RNG ------
// Advance the walker's mt19937 stream by the draws of one substep:
// N uniforms then 3N BoxMuller2 normals (miniqmc.cpp:424-425,
// RandomGenerator.h:49-62).  Block-wide.
__device__ inline void mt_block_twist(uint32_t* mt)
{
  const int tid = threadIdx.x, NT = blockDim.x;
  uint32_t nv[4];
  // phase 1: i in [0,227): old neighbours only
  {
    int c = 0;
    for (int i = tid; i < MT_N - MT_M; i += NT, ++c)
      nv[c] = mt_twist_one(mt[i], mt[i + 1], mt[i + MT_M]);
    __syncthreads();
    c = 0;
    for (int i = tid; i < MT_N - MT_M; i += NT, ++c)
      mt[i] = nv[c];
    __syncthreads();
  }
  // phases 2,3: i in [227,454), [454,623): far operand from an earlier phase
  for (int lo = MT_N - MT_M; lo < MT_N - 1; lo += MT_N - MT_M)
  {
    const int hi = min(lo + (MT_N - MT_M), MT_N - 1);
    int c        = 0;
    for (int i = lo + tid; i < hi; i += NT, ++c)
      nv[c] = mt_twist_one(mt[i], mt[i + 1], mt[i + MT_M - MT_N]);
    __syncthreads();
    c = 0;
    for (int i = lo + tid; i < hi; i += NT, ++c)
      mt[i] = nv[c];
    __syncthreads();
  }
  if (tid == 0)
    mt[MT_N - 1] = mt_twist_one(mt[MT_N - 1], mt[0], mt[MT_M - 1]);
  __syncthreads();
}

template <typename T> __device__ void rng_substep(const WV<T>& wv, int N)
{
  const int tid = threadIdx.x, NT = blockDim.x;
  const int npairs = (3 * N + 1) / 2;
  const int M      = 2 * N + 4 * npairs;
  uint32_t* mt     = wv.mt;
  __shared__ int s_mti;
  if (tid == 0)
    s_mti = (int)mt[MT_N];
  __syncthreads();
  int produced = 0;
  while (produced < M)
  {
    if (s_mti >= MT_N)
    {
      mt_block_twist(mt);
      if (tid == 0)
        s_mti = 0;
      __syncthreads();
    }
    const int mti = s_mti;
    const int cnt = min(MT_N - mti, M - produced);
    for (int t = tid; t < cnt; t += NT)
      wv.words[produced + t] = mt_temper(mt[mti + t]);
    produced += cnt;
    __syncthreads();
    if (tid == 0)
      s_mti = mti + cnt;
    __syncthreads();
  }
  if (tid == 0)
    mt[MT_N] = (uint32_t)s_mti;
  for (int i = tid; i < N; i += NT)
    wv.ur[i] = canonical_double(wv.words[2 * i], wv.words[2 * i + 1]);
  const uint32_t* wn = wv.words + 2 * N;
  for (int p = tid; p < npairs; p += NT)
  {
    const double u1 = canonical_double(wn[4 * p], wn[4 * p + 1]);
    const double u2 = canonical_double(wn[4 * p + 2], wn[4 * p + 3]);
    const double t1 = __dsub_rn(1.0, __dmul_rn(0.9999999999, u1));
    const double rr = sqrt(__dmul_rn(-2.0, log(t1)));
    const double an = __dmul_rn(6.283185306, u2);
    wv.delta[2 * p] = __dmul_rn(rr, cos(an));
    if (2 * p + 1 < 3 * N)
      wv.delta[2 * p + 1] = __dmul_rn(rr, sin(an));
  }
  __syncthreads();
}

// --------------------------------------------------------- one move -----
// evalGrad, makeMove, ratioGrad and the threshold accept of electron iel
// (miniqmc.cpp:426-458).  Block-wide.
// HAS_J3 = false compiles the three-body Jastrow out (launches without it
// keep the smaller register footprint)
template <typename T, bool HAS_J3 = true>
__device__ void do_move(const SysSmem<T>& ss, const DevSystem* __restrict__ sys, const WV<T>& wv, MoveSmem& m,
                        SplineSmem<T>& sp, const T* __restrict__ ions, int iel, double accept_thr, const double* urp,
                        const double* dlt, double* trace, T* smem, bool prefetch_next)
{
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  const int tid = threadIdx.x, NT = blockDim.x;
  const bool DET = ss.comp & QMC_WF_DET, J1 = ss.comp & QMC_WF_J1, J2 = ss.comp & QMC_WF_J2;
  const bool J3 = HAS_J3 && (ss.comp & QMC_WF_J3);
  const int s = iel < ss.n_up ? 0 : 1, r = iel - (s ? ss.n_up : 0);
  const int npad = wv.npad, nvec = npad / VW;
  if (tid < 32)
  {
    // warp 0 sets the move up: lanes 0-2 take the three dimensions of this
    // move's proposed position and stencil, lanes 3-5 those of the next
    // electron's when its stencil is prefetched (its current position does
    // not change during this move); one round trip for the positions, the
    // cell constants from shared memory
    const int lane = tid, d = lane % 3;
    const bool cur = lane < 3, nxt = lane >= 3 && lane < 6 && prefetch_next;
    double r = 0.0, pn = 0.0, urv = 0.0;
    if (cur || nxt)
    {
      r  = wv.R[3 * (cur ? iel : iel + 1) + d];
      pn = r + dlt[(cur ? 0 : 3) + d];
    }
    if (lane == 0)
      urv = urp[0];
    const int g0    = lane < 3 ? 0 : 3;
    const double p0 = __shfl_sync(0xffffffffu, pn, g0), p1 = __shfl_sync(0xffffffffu, pn, g0 + 1),
                 p2 = __shfl_sync(0xffffffffu, pn, g0 + 2);
    const double u  = p0 * ss.spoG[d] + p1 * ss.spoG[3 + d] + p2 * ss.spoG[6 + d];
    long long b     = 0;
    if (DET && (cur || nxt))
      b = spline_dim<T>(u, ss.sdinv[d], ss.sgrid[d], ss.sstride[d], cur ? sp.a[d] : nullptr,
                        cur ? sp.da[d] : nullptr, cur ? sp.d2a[d] : nullptr);
    const long long bc = __shfl_sync(0xffffffffu, b, 0) + __shfl_sync(0xffffffffu, b, 1) + __shfl_sync(0xffffffffu, b, 2);
    const long long bn = __shfl_sync(0xffffffffu, b, 3) + __shfl_sync(0xffffffffu, b, 4) + __shfl_sync(0xffffffffu, b, 5);
    if (cur)
    {
      m.pos_old[d] = r;
      m.pos_new[d] = pn;
    }
    if (lane == 0)
    {
      m.accept = urv < accept_thr;
      m.dc     = DET ? wv.dcount[s] : 0;
      if (DET)
      {
        sp.base = bc;
        if (prefetch_next)
          m.next_base = bn;
      }
    }
  }
  __syncthreads();
  phase_mark(m, PH_SETUP);
  // this move's 16 stencil rows start towards L2 now, so that their HBM
  // latency overlaps getInvRow (they may already be there when the next
  // move was prefetched during the previous one)
  if (DET && tid >= 32 && tid < 48)
    prefetch_l2((const T*)sys->coefs + sp.base + ((tid - 32) >> 2) * sys->xs + ((tid - 32) & 3) * sys->ys,
                (unsigned)(4 * sys->zs * sizeof(T)));
  if (DET && prefetch_next && tid < 18)
  {
    // warm L2 with the next move's 16 stencil rows and its inverse and
    // gradient rows while this move runs
    if (tid < 16)
      prefetch_l2((const T*)sys->coefs + m.next_base + (tid >> 2) * sys->xs + (tid & 3) * sys->ys,
                  (unsigned)(4 * sys->zs * sizeof(T)));
    else
    {
      const int i2 = iel + 1, s2 = i2 < ss.n_up ? 0 : 1, r2 = i2 - (s2 ? ss.n_up : 0);
      if (tid == 16)
        prefetch_l2(wv.ainv(s2) + (size_t)r2 * npad, (unsigned)(npad * sizeof(T)));
      else
        prefetch_l2(wv.dpsi(s2) + (size_t)r2 * 3 * npad, (unsigned)(3 * npad * sizeof(T)));
    }
  }
  if (J3)
  {
    // J3 ratio and gradient sums of the proposed position, reduced on their
    // own into sums[16..19] so that the triple code's registers are not live
    // together with the determinant partials
    double jp[4] = {0.0, 0.0, 0.0, 0.0};
    j3_partials(ss, sys, wv, ions, *reinterpret_cast<J3Smem<T>*>(smem), iel, m.pos_new, jp);
    block_sum<4>(jp, m.red, m.sums + 16);
  }
  // per-thread partial sums cover a few terms each: accumulate in the walker
  // precision, widen to FP64 for the block reduction
  T part[16];
#pragma unroll
  for (int i = 0; i < 16; ++i)
    part[i] = T(0);
  phase_mark(m, PH_REDUCE);
  if (DET)
  {
    get_inv_row(wv, m, s, r, m.dc);
    phase_mark(m, PH_INVROW);
    const T* dprow = wv.dpsi(s) + (size_t)r * 3 * npad;
    const T* coefs = (const T*)sys->coefs;
    const long long xs = sys->xs, ys = sys->ys, zs = sys->zs;
    const double dinv[3] = {sys->dinv[0], sys->dinv[1], sys->dinv[2]};
    const bool trace_lap = ss.lap_mode == QMC_LAP_TRACE;
    const uint64_t dpol  = l2_evict_first();
    for (int q = tid; q < nvec; q += NT)
    {
      Vt iv = reinterpret_cast<const Vt*>(wv.invRow)[q];
      const T* ivp = reinterpret_cast<const T*>(&iv);
      for (int c = 0; c < 3; ++c)
      {
        Vt g = ld_stream_rw(reinterpret_cast<const Vt*>(dprow + (size_t)c * npad) + q, dpol);
#pragma unroll
        for (int e = 0; e < VW; ++e)
          part[4 + c] += ivp[e] * reinterpret_cast<T*>(&g)[e];
      }
      SplineOut<T> o;
      spline_eval<T, false>(coefs, xs, ys, zs, sp, dinv, q * VW, o);
      Vt pv, gxv, gyv, gzv, lv;
#pragma unroll
      for (int e = 0; e < VW; ++e)
      {
        reinterpret_cast<T*>(&pv)[e]  = o.v[e];
        reinterpret_cast<T*>(&gxv)[e] = o.gx[e];
        reinterpret_cast<T*>(&gyv)[e] = o.gy[e];
        reinterpret_cast<T*>(&gzv)[e] = o.gz[e];
        reinterpret_cast<T*>(&lv)[e]  = trace_lap ? o.hxx[e] + o.hyy[e] + o.hzz[e] : o.hxx[e];
        part[0] += ivp[e] * o.v[e];
        part[1] += ivp[e] * o.gx[e];
        part[2] += ivp[e] * o.gy[e];
        part[3] += ivp[e] * o.gz[e];
      }
      reinterpret_cast<Vt*>(wv.psiV)[q]            = pv;
      reinterpret_cast<Vt*>(wv.dpsiV)[q]           = gxv;
      reinterpret_cast<Vt*>(wv.dpsiV + npad)[q]    = gyv;
      reinterpret_cast<Vt*>(wv.dpsiV + 2 * npad)[q] = gzv;
      reinterpret_cast<Vt*>(wv.d2psiV)[q]          = lv;
    }
    phase_mark(m, PH_SPO);
  }
  if (J1)
    j1_partials(ss, ions, m.pos_new, part + 7);
  if (J2)
    j2_partials(ss, wv.Rs, wv.Npad, iel, m.pos_new, part + 12, true, reinterpret_cast<int*>(smem));
  phase_mark(m, PH_JASTROW);
  {
    double dpart[16];
#pragma unroll
    for (int i = 0; i < 16; ++i)
      dpart[i] = (double)part[i];
    block_sum<16>(dpart, m.red, m.sums);
  }
  if (tid == 0)
  {
    const double* S = m.sums;
    const double rdet = DET ? S[0] : 1.0;
    double ratio      = rdet;
    double gn[3], g0[3];
    for (int c = 0; c < 3; ++c)
    {
      gn[c] = DET ? (1.0 / rdet) * S[1 + c] : 0.0;
      g0[c] = DET ? S[4 + c] : 0.0;
    }
    m.ratio_det = rdet;
    if (J1)
    {
      m.curAt  = S[7];
      m.curLap = S[11];
      for (int c = 0; c < 3; ++c)
      {
        m.curGrad[c] = S[8 + c];
        gn[c] += S[8 + c];
        g0[c] += (double)wv.Grad[c * wv.N + iel];
      }
      ratio *= exp((double)wv.Vat[iel] - m.curAt);
    }
    if (J2)
    {
      m.curUat = S[12];
      for (int c = 0; c < 3; ++c)
      {
        gn[c] += S[13 + c];
        g0[c] += (double)wv.dUat[c * wv.N + iel];
      }
      ratio *= exp((double)wv.Uat[iel] - m.curUat);
    }
    if (J3)
    {
      for (int c = 0; c < 3; ++c)
      {
        gn[c] += S[17 + c];
        g0[c] += (double)wv.j3dUat[c * wv.N + iel];
      }
      ratio *= exp((double)wv.j3Uat[iel] - S[16]);
    }
    if (!isfinite(ratio))
      atomicOr(wv.status, DEV_ERR_NONFINITE);
    if (trace)
    {
      trace[0] = ratio;
      trace[1] = gn[0], trace[2] = gn[1], trace[3] = gn[2];
      trace[4] = g0[0], trace[5] = g0[1], trace[6] = g0[2];
      trace[7] = m.accept ? 1.0 : 0.0;
    }
  }
  __syncthreads();
  phase_mark(m, PH_REDUCE);
  if (m.accept)
  {
    if (DET)
      det_accept(wv, m, s, r, m.ratio_det, true, true, smem);
    phase_mark(m, PH_DET_ACCEPT);
    if (J1 && tid == 0)
    {
      wv.jlog[0] += (double)wv.Vat[iel] - m.curAt;
      wv.Vat[iel] = (T)m.curAt;
      for (int c = 0; c < 3; ++c)
        wv.Grad[c * wv.N + iel] = (T)m.curGrad[c];
      wv.Lap[iel] = (T)m.curLap;
    }
    if (J2)
      j2_accept(ss, wv, m, iel, reinterpret_cast<int*>(smem));
    if (J3)
      j3_accept(ss, sys, wv, m, *reinterpret_cast<J3Smem<T>*>(smem), ions, iel);
    __syncthreads();
    phase_mark(m, PH_J2_ACCEPT);
    if (tid == 0)
      for (int c = 0; c < 3; ++c)
      {
        wv.R[3 * iel + c]          = m.pos_new[c];
        wv.Rs[c * wv.Npad + iel]   = (T)m.pos_new[c];
      }
    __syncthreads();
    phase_mark(m, PH_POSITION);
  }
}


// ------------------------------------------------------ move epochs -----
// The accept rule of the reference driver compares a uniform with a fixed
// threshold (miniqmc.cpp:445: ur[iel] < accept), so which moves of a
// substep are accepted is known before any ratio is.  A rejected move
// changes no state (rejectMove / restore), hence the moves from one
// accepted move to the next -- the rejected ones and the accepted one that
// ends the run -- all see the same inverse, delayed rows, Jastrow arrays and
// positions.  The fused sweep evaluates such a run ("epoch", at most
// EPOCH_MAX moves, within one spin) together: one set-up, one getInvRow pass
// over the delayed rows U and V for all its rows, one block reduction, and
// the accept bookkeeping of its last move only.  Per move the arithmetic is
// that of do_move (same loops, same summation order), so the trajectory and
// every ratio are the same bit for bit; what changes is the number of
// dependent round trips and barriers per move and the U/V traffic.

// shared-memory bytes an epoch needs beyond the J2 candidate lists (the
// stencil weights of its moves)
template <typename T> __host__ __device__ constexpr size_t epoch_smem_bytes()
{
  return ((sizeof(SplineSmem<T>) * EPOCH_MAX + 15) / 16) * 16;
}

// DelayedUpdate::getInvRow for the rows r[0..G) of one spin at once, into
// wv.invRow + g npad; with no delayed row the caller reads the Ainv rows
// themselves.  Row dc of Binv receives the last row's Binv^T p (the last
// move of an epoch is the only one that may be accepted, and acceptRow
// reads that row).  Per row the arithmetic of get_inv_row.  Block-wide.
// Scratch: m.red holds p[g][d] (first EPOCH_MAX * MAXK) and w[g][a] (next).
template <typename T> __device__ void get_inv_rows(const WV<T>& wv, MoveSmem& m, int s, const int* r, int G, int dc)
{
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  const int nvec = wv.npad / VW;
  double* P      = m.red;
  double* Wg     = m.red + EPOCH_MAX * MAXK;
  const T* A     = wv.ainv(s);
  const T* U     = wv.u(s);
  const T* V     = wv.v(s);
  const Vt* arow[EPOCH_MAX];
#pragma unroll
  for (int g = 0; g < EPOCH_MAX; ++g)
    arow[g] = reinterpret_cast<const Vt*>(A + (size_t)r[g < G ? g : 0] * wv.npad);
  for (int d = wid; d < dc; d += nw)
  {
    const Vt* ud = reinterpret_cast<const Vt*>(U + (size_t)d * wv.npad);
    T acc[EPOCH_MAX];
#pragma unroll
    for (int g = 0; g < EPOCH_MAX; ++g)
      acc[g] = T(0);
#pragma unroll 4
    for (int jv = lane; jv < nvec; jv += 32)
    {
      const Vt x = ud[jv];
#pragma unroll
      for (int g = 0; g < EPOCH_MAX; ++g)
        if (g < G)
        {
          const Vt y = arow[g][jv];
#pragma unroll
          for (int e = 0; e < VW; ++e)
            acc[g] += reinterpret_cast<const T*>(&x)[e] * reinterpret_cast<const T*>(&y)[e];
        }
    }
#pragma unroll
    for (int g = 0; g < EPOCH_MAX; ++g)
      if (g < G)
      {
        const double sum = warp_sum((double)acc[g]);
        if (lane == 0)
          P[g * MAXK + d] = sum;
      }
  }
  __syncthreads();
  double* B = wv.binv(s);
  for (int idx = tid; idx < G * dc; idx += NT)
  {
    const int g = idx / dc, a = idx - g * dc;
    double acc = 0.0;
    for (int b = 0; b < dc; ++b)
      acc += B[b * wv.k + a] * P[g * MAXK + b];
    Wg[g * MAXK + a] = acc;
    if (g == G - 1 && dc < wv.k)
      B[dc * wv.k + a] = acc;
  }
  __syncthreads();
  // invRow_g = Ainv[r_g] - V^T w_g with FP64 accumulation; the rows two at a
  // time, so that each V element loaded serves both
  for (int q = tid; q < nvec; q += NT)
    for (int g0 = 0; g0 < G; g0 += 2)
    {
      const bool two = g0 + 1 < G;
      double acc0[VW], acc1[VW];
#pragma unroll
      for (int e = 0; e < VW; ++e)
        acc0[e] = acc1[e] = 0.0;
#pragma unroll 4
      for (int d = 0; d < dc; ++d)
      {
        Vt vv            = reinterpret_cast<const Vt*>(V + (size_t)d * wv.npad)[q];
        const double wd0 = Wg[g0 * MAXK + d];
        const double wd1 = two ? Wg[(g0 + 1) * MAXK + d] : 0.0;
#pragma unroll
        for (int e = 0; e < VW; ++e)
        {
          acc0[e] += (double)reinterpret_cast<T*>(&vv)[e] * wd0;
          acc1[e] += (double)reinterpret_cast<T*>(&vv)[e] * wd1;
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h)
      {
        if (h == 1 && !two)
          break;
        const int g = g0 + h;
        Vt a        = arow[g][q];
        T* ap       = reinterpret_cast<T*>(&a);
#pragma unroll
        for (int e = 0; e < VW; ++e)
          ap[e] = (T)((double)ap[e] - (h ? acc1[e] : acc0[e]));
        reinterpret_cast<Vt*>(wv.invRow + (size_t)g * wv.npad)[q] = a;
      }
    }
  __syncthreads(); // the callers' reductions reuse m.red
}

// One epoch of the fused sweep: the moves iel0 .. iel0+G-1 of one spin
// (G <= min(max_moves, lim - iel0)), ending at the first accepted one; the
// same arithmetic per move as do_move (without the three-body Jastrow).
// Returns G (read from shared memory after the set-up barrier).  esp: the
// moves' stencil weights (epoch_smem_bytes, in the dynamic shared memory
// after the J2 candidate lists).  Block-wide.
template <typename T>
__device__ int do_epoch(const SysSmem<T>& ss, const DevSystem* __restrict__ sys, const WV<T>& wv, MoveSmem& m,
                        SplineSmem<T>* esp, const T* __restrict__ ions, int iel0, int lim, int max_moves,
                        double accept_thr, const double* urp, const double* dlt, double* trace, T* smem,
                        bool prefetch_next)
{
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  const bool DET = ss.comp & QMC_WF_DET, J1 = ss.comp & QMC_WF_J1, J2 = ss.comp & QMC_WF_J2;
  const int s = iel0 < ss.n_up ? 0 : 1, rbase = s ? ss.n_up : 0;
  const int npad = wv.npad, nvec = npad / VW, N = wv.N;
  // epoch positions in m.sums: old [0, 12), new [12, 24)
  double* epos_old = m.sums;
  double* epos_new = m.sums + 3 * EPOCH_MAX;
  if (tid < 32)
  {
    // warp 0 finds the epoch (the first accepted move among the next
    // navail) and sets up each of its moves: lanes 3g..3g+2 the three
    // dimensions of move g's proposed position and stencil; lanes 12-14 the
    // move after the epoch when its stencil is prefetched
    const int navail = min(min(max_moves, EPOCH_MAX), lim - iel0);
    const bool acc_l = lane < navail && urp[lane] < accept_thr;
    const unsigned ab = __ballot_sync(0xffffffffu, acc_l);
    const int G       = ab ? __ffs(ab) : navail;
    const int g = lane / 3, d = lane % 3, inext = iel0 + G;
    const bool cur = lane < 3 * G;
    const bool nxt = lane >= 12 && lane < 15 && prefetch_next && inext < N;
    double r = 0.0, pn = 0.0;
    if (cur)
    {
      r  = wv.R[3 * (iel0 + g) + d];
      pn = r + dlt[3 * g + d];
    }
    else if (nxt)
    {
      r  = wv.R[3 * inext + d];
      pn = r + dlt[3 * G + d];
    }
    const int g0    = cur ? 3 * g : 12;
    const double p0 = __shfl_sync(0xffffffffu, pn, g0), p1 = __shfl_sync(0xffffffffu, pn, g0 + 1),
                 p2 = __shfl_sync(0xffffffffu, pn, g0 + 2);
    const double u  = p0 * ss.spoG[d] + p1 * ss.spoG[3 + d] + p2 * ss.spoG[6 + d];
    long long b     = 0;
    if (DET && (cur || nxt))
      b = spline_dim<T>(u, ss.sdinv[d], ss.sgrid[d], ss.sstride[d], cur ? esp[g].a[d] : nullptr,
                        cur ? esp[g].da[d] : nullptr, cur ? esp[g].d2a[d] : nullptr);
    const int gb       = cur ? 3 * g : 12;
    const long long bs = __shfl_sync(0xffffffffu, b, gb) + __shfl_sync(0xffffffffu, b, gb + 1) +
        __shfl_sync(0xffffffffu, b, gb + 2);
    if (cur)
    {
      epos_old[3 * g + d] = r;
      epos_new[3 * g + d] = pn;
      if (g == G - 1)
      {
        m.pos_old[d] = r;
        m.pos_new[d] = pn;
      }
      if (d == 0 && DET)
        esp[g].base = bs;
    }
    if (lane == 12 && nxt && DET)
      m.next_base = bs;
    if (lane == 0)
    {
      m.eG     = G;
      m.accept = ab ? 1 : 0;
      m.dc     = DET ? wv.dcount[s] : 0;
    }
  }
  __syncthreads();
  phase_mark(m, PH_SETUP);
  const int G = m.eG;
  // the first move's stencil starts towards L2 now (16 rows), so that its
  // HBM latency overlaps getInvRow; each later move's starts when the move
  // before it has read its own (all of them at once, or two per walker at a
  // time, would not stay in the L2 with hundreds of walkers)
  if (DET && tid >= 32 && tid < 48)
    prefetch_l2((const T*)sys->coefs + esp[0].base + ((tid - 32) >> 2) * sys->xs + ((tid - 32) & 3) * sys->ys,
                (unsigned)(4 * sys->zs * sizeof(T)));
  if (DET && prefetch_next && iel0 + G < N && tid < 18)
  {
    const int i2 = iel0 + G, s2 = i2 < ss.n_up ? 0 : 1, r2 = i2 - (s2 ? ss.n_up : 0);
    if (tid < 16)
      prefetch_l2((const T*)sys->coefs + m.next_base + (tid >> 2) * sys->xs + (tid & 3) * sys->ys,
                  (unsigned)(4 * sys->zs * sizeof(T)));
    else if (tid == 16)
      prefetch_l2(wv.ainv(s2) + (size_t)r2 * npad, (unsigned)(npad * sizeof(T)));
    else
      prefetch_l2(wv.dpsi(s2) + (size_t)r2 * 3 * npad, (unsigned)(3 * npad * sizeof(T)));
  }
  phase_mark(m, PH_REDUCE);
  int rows[EPOCH_MAX];
#pragma unroll
  for (int g = 0; g < EPOCH_MAX; ++g)
    rows[g] = iel0 + (g < G ? g : 0) - rbase;
  const int dc = m.dc;
  if (DET && dc > 0)
    get_inv_rows(wv, m, s, rows, G, dc);
  phase_mark(m, PH_INVROW);
  const T* coefs       = (const T*)sys->coefs;
  const long long xs = sys->xs, ys = sys->ys, zs = sys->zs;
  const double dinv[3] = {sys->dinv[0], sys->dinv[1], sys->dinv[2]};
  const bool trace_lap = ss.lap_mode == QMC_LAP_TRACE;
  const uint64_t dpol  = l2_evict_first();
  for (int g = 0; g < G; ++g)
  {
    const bool last = g == G - 1;
    T part[16];
#pragma unroll
    for (int i = 0; i < 16; ++i)
      part[i] = T(0);
    if (DET)
    {
      const int r    = rows[g];
      const T* irow  = dc > 0 ? wv.invRow + (size_t)g * npad : wv.ainv(s) + (size_t)r * npad;
      const T* dprow = wv.dpsi(s) + (size_t)r * 3 * npad;
      for (int q = tid; q < nvec; q += NT)
      {
        Vt iv        = reinterpret_cast<const Vt*>(irow)[q];
        const T* ivp = reinterpret_cast<const T*>(&iv);
        for (int c = 0; c < 3; ++c)
        {
          Vt gr = ld_stream_rw(reinterpret_cast<const Vt*>(dprow + (size_t)c * npad) + q, dpol);
#pragma unroll
          for (int e = 0; e < VW; ++e)
            part[4 + c] += ivp[e] * reinterpret_cast<T*>(&gr)[e];
        }
        SplineOut<T> o;
        spline_eval<T, false>(coefs, xs, ys, zs, esp[g], dinv, q * VW, o);
        Vt pv, gxv, gyv, gzv, lv;
#pragma unroll
        for (int e = 0; e < VW; ++e)
        {
          reinterpret_cast<T*>(&pv)[e]  = o.v[e];
          reinterpret_cast<T*>(&gxv)[e] = o.gx[e];
          reinterpret_cast<T*>(&gyv)[e] = o.gy[e];
          reinterpret_cast<T*>(&gzv)[e] = o.gz[e];
          reinterpret_cast<T*>(&lv)[e]  = trace_lap ? o.hxx[e] + o.hyy[e] + o.hzz[e] : o.hxx[e];
          part[0] += ivp[e] * o.v[e];
          part[1] += ivp[e] * o.gx[e];
          part[2] += ivp[e] * o.gy[e];
          part[3] += ivp[e] * o.gz[e];
        }
        if (last) // the only move of the epoch whose rows acceptMove may need
        {
          reinterpret_cast<Vt*>(wv.psiV)[q]             = pv;
          reinterpret_cast<Vt*>(wv.dpsiV)[q]            = gxv;
          reinterpret_cast<Vt*>(wv.dpsiV + npad)[q]     = gyv;
          reinterpret_cast<Vt*>(wv.dpsiV + 2 * npad)[q] = gzv;
          reinterpret_cast<Vt*>(wv.d2psiV)[q]           = lv;
        }
      }
      phase_mark(m, PH_SPO);
    }
    // the next move's stencil starts towards L2 once this move's has been
    // read, so that its latency overlaps this move's Jastrow sums
    if (DET && g + 1 < G && tid >= 32 && tid < 48)
      prefetch_l2((const T*)sys->coefs + esp[g + 1].base + ((tid - 32) >> 2) * xs + ((tid - 32) & 3) * ys,
                  (unsigned)(4 * zs * sizeof(T)));
    if (J1)
      j1_partials(ss, ions, epos_new + 3 * g, part + 7);
    if (J2)
      j2_partials(ss, wv.Rs, wv.Npad, iel0 + g, epos_new + 3 * g, part + 12, true, reinterpret_cast<int*>(smem));
    phase_mark(m, PH_JASTROW);
    // the first half of block_sum<16>: warp sums into this move's slice
#pragma unroll
    for (int i = 0; i < 16; ++i)
    {
      const double sw = warp_sum((double)part[i]);
      if (lane == 0)
        m.red[(g * nw + wid) * 16 + i] = sw;
    }
  }
  __syncthreads();
  // the second half: warp g (mod the warp count) sums move g's slices over
  // the warps
  double* esum = m.col; // [EPOCH_MAX][16]
  for (int g = wid; g < G; g += nw)
  {
#pragma unroll
    for (int i = 0; i < 16; ++i)
    {
      double sw = lane < nw ? m.red[(g * nw + lane) * 16 + i] : 0.0;
      sw        = warp_sum(sw);
      if (lane == 0)
        esum[g * 16 + i] = sw;
    }
  }
  __syncthreads();
  if (tid < G)
  {
    // ratio and gradients of move g = tid (do_move's assembly)
    const int g = tid, iel = iel0 + g;
    const double* S = esum + 16 * g;
    const double rdet = DET ? S[0] : 1.0;
    double ratio      = rdet;
    double gn[3], gq[3];
    for (int c = 0; c < 3; ++c)
    {
      gn[c] = DET ? (1.0 / rdet) * S[1 + c] : 0.0;
      gq[c] = DET ? S[4 + c] : 0.0;
    }
    if (J1)
    {
      for (int c = 0; c < 3; ++c)
      {
        gn[c] += S[8 + c];
        gq[c] += (double)wv.Grad[c * wv.N + iel];
      }
      ratio *= exp((double)wv.Vat[iel] - S[7]);
    }
    if (J2)
    {
      for (int c = 0; c < 3; ++c)
      {
        gn[c] += S[13 + c];
        gq[c] += (double)wv.dUat[c * wv.N + iel];
      }
      ratio *= exp((double)wv.Uat[iel] - S[12]);
    }
    if (!isfinite(ratio))
      atomicOr(wv.status, DEV_ERR_NONFINITE);
    const bool acc_g = g == G - 1 && m.accept;
    if (trace)
    {
      double* tr = trace + (size_t)g * 8;
      tr[0]      = ratio;
      tr[1] = gn[0], tr[2] = gn[1], tr[3] = gn[2];
      tr[4] = gq[0], tr[5] = gq[1], tr[6] = gq[2];
      tr[7] = acc_g ? 1.0 : 0.0;
    }
    if (g == G - 1)
    {
      m.ratio_det = rdet;
      if (J1)
      {
        m.curAt  = S[7];
        m.curLap = S[11];
        for (int c = 0; c < 3; ++c)
          m.curGrad[c] = S[8 + c];
      }
      if (J2)
        m.curUat = S[12];
    }
  }
  __syncthreads();
  phase_mark(m, PH_REDUCE);
  if (m.accept)
  {
    const int iel = iel0 + G - 1, r = iel - rbase;
    if (DET)
      det_accept(wv, m, s, r, m.ratio_det, true, true, smem);
    phase_mark(m, PH_DET_ACCEPT);
    if (J1 && tid == 0)
    {
      wv.jlog[0] += (double)wv.Vat[iel] - m.curAt;
      wv.Vat[iel] = (T)m.curAt;
      for (int c = 0; c < 3; ++c)
        wv.Grad[c * wv.N + iel] = (T)m.curGrad[c];
      wv.Lap[iel] = (T)m.curLap;
    }
    if (J2)
      j2_accept(ss, wv, m, iel, reinterpret_cast<int*>(smem));
    __syncthreads();
    phase_mark(m, PH_J2_ACCEPT);
    if (tid == 0)
      for (int c = 0; c < 3; ++c)
      {
        wv.R[3 * iel + c]        = m.pos_new[c];
        wv.Rs[c * wv.Npad + iel] = (T)m.pos_new[c];
      }
    __syncthreads();
    phase_mark(m, PH_POSITION);
  }
  return G;
}

} // namespace qmc
