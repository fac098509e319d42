// others.cu -- drop-in verb kernels, the evaluateLog pipeline (SPO matrix,
// FP64 Gauss-Jordan inverse, Jastrow recompute, evaluateGL), SPO evaluation
// at arbitrary points and the DelayedUpdate engine kernel.
#include "device.cuh"

namespace qmc
{
// ------------------------------------------------------------- verbs ----
// One CTA per walker.  The per-move scalars live in MoveState between calls.
template <typename T>
__global__ void __launch_bounds__(256) verb_kernel(const DevSystem* __restrict__ sys, DevWalkers dw, VerbArgs a)
{
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  __shared__ SysSmem<T> ss;
  __shared__ MoveSmem m;
  __shared__ SplineSmem<T> sp;
  __shared__ int s_invrow, s_partial, s_jpartial, s_active, s_flag;
  extern __shared__ __align__(16) unsigned char dyn[];
  // the walker's view in shared memory rather than registers (as in the
  // fused sweep)
  __shared__ WV<T> wv;
  T* smem     = reinterpret_cast<T*>(dyn);
  const int w = blockIdx.x, tid = threadIdx.x, NT = blockDim.x;
  if (tid == 0)
    wv = make_wv<T>(dw, w);
  load_sys(sys, ss); // ends with a barrier
  MoveState* ms  = wv.ms;
  const bool DET = ss.comp & QMC_WF_DET, J1 = ss.comp & QMC_WF_J1, J2 = ss.comp & QMC_WF_J2;
  const bool J3 = ss.comp & QMC_WF_J3;
  J3Smem<T>& J  = *reinterpret_cast<J3Smem<T>*>(dyn);
  const int iat = a.iat;
  const int s = iat < ss.n_up ? 0 : 1, r = iat - (s ? ss.n_up : 0);
  const int npad = wv.npad, nvec = npad / VW, N = wv.N;
  const T* ions = (const T*)sys->ion_soa;
  if (tid == 0)
  {
    m.tc_on    = 0;
    m.tc_abort = 0;
    m.timing   = 0;
    s_invrow   = ms->invrow_id[s];
    s_partial  = ms->partial[s];
    s_jpartial = ms->j_partial;
    s_active   = ms->active;
    s_flag     = a.flags ? a.flags[w] : 1;
    for (int c = 0; c < 3; ++c)
    {
      m.pos_new[c] = ms->pos[c];
      m.pos_old[c] = wv.R[3 * iat + c];
    }
  }
  __syncthreads();
  switch (a.op)
  {
  case VERB_SET_ACTIVE:
    break;
  case VERB_MAKE_MOVE:
    if (tid == 0)
    {
      ms->active = iat;
      for (int c = 0; c < 3; ++c)
        ms->pos[c] = wv.R[3 * iat + c] + a.displ[3 * w + c];
    }
    break;
  case VERB_EVAL_GRAD:
  {
    double part[3] = {0.0, 0.0, 0.0};
    if (DET)
    {
      get_inv_row(wv, m, s, r, wv.dcount[s]);
      const T* dprow = wv.dpsi(s) + (size_t)r * 3 * npad;
      for (int q = tid; q < nvec; q += NT)
      {
        Vt iv = reinterpret_cast<const Vt*>(wv.invRow)[q];
        for (int c = 0; c < 3; ++c)
        {
          Vt g = reinterpret_cast<const Vt*>(dprow + (size_t)c * npad)[q];
#pragma unroll
          for (int e = 0; e < VW; ++e)
            part[c] += (double)(reinterpret_cast<T*>(&iv)[e] * reinterpret_cast<T*>(&g)[e]);
        }
      }
    }
    block_sum<3>(part, m.red, m.sums);
    if (tid == 0)
    {
      if (DET)
        ms->invrow_id[s] = r;
      for (int c = 0; c < 3; ++c)
      {
        double g = m.sums[c];
        if (J1)
          g += (double)wv.Grad[c * N + iat];
        if (J2)
          g += (double)wv.dUat[c * N + iat];
        if (J3)
          g += (double)wv.j3dUat[c * N + iat];
        dw.out_grad[3 * w + c] = g;
      }
    }
    break;
  }
  case VERB_RATIO_GRAD:
  case VERB_RATIO:
  {
    const bool grads = a.op == VERB_RATIO_GRAD;
    if (s_active != iat)
    {
      if (tid == 0)
        atomicOr(wv.status, DEV_ERR_STATE);
      break;
    }
    double part[16];
#pragma unroll
    for (int i = 0; i < 16; ++i)
      part[i] = 0.0;
    if (DET)
    {
      if (tid == 0)
        spline_locate(sys, m.pos_new, sp);
      if (s_invrow != r)
        get_inv_row(wv, m, s, r, wv.dcount[s]);
      __syncthreads();
      const T* coefs = (const T*)sys->coefs;
      const double dinv[3] = {sys->dinv[0], sys->dinv[1], sys->dinv[2]};
      for (int q = tid; q < nvec; q += NT)
      {
        Vt iv        = reinterpret_cast<const Vt*>(wv.invRow)[q];
        const T* ivp = reinterpret_cast<const T*>(&iv);
        if (grads)
        {
          SplineOut<T> o;
          spline_eval<T, false>(coefs, sys->xs, sys->ys, sys->zs, sp, dinv, q * VW, o);
          for (int e = 0; e < VW; ++e)
          {
            const int j = q * VW + e;
            wv.psiV[j]            = o.v[e];
            wv.dpsiV[j]           = o.gx[e];
            wv.dpsiV[npad + j]    = o.gy[e];
            wv.dpsiV[2 * npad + j] = o.gz[e];
            wv.d2psiV[j] = ss.lap_mode == QMC_LAP_TRACE ? o.hxx[e] + o.hyy[e] + o.hzz[e] : o.hxx[e];
            part[0] += (double)(ivp[e] * o.v[e]);
            part[1] += (double)(ivp[e] * o.gx[e]);
            part[2] += (double)(ivp[e] * o.gy[e]);
            part[3] += (double)(ivp[e] * o.gz[e]);
          }
        }
        else
        {
          T v[VW];
          spline_eval_v(coefs, sys->xs, sys->ys, sys->zs, sp, q * VW, v);
          for (int e = 0; e < VW; ++e)
          {
            wv.psiV[q * VW + e] = v[e];
            part[0] += (double)(ivp[e] * v[e]);
          }
        }
      }
    }
    if (J1)
    {
      if (grads)
        j1_partials(ss, ions, m.pos_new, part + 7);
      else
        j1_value(ss, ions, m.pos_new, part + 7);
    }
    if (J2)
      j2_partials(ss, wv.Rs, wv.Npad, iat, m.pos_new, part + 12, grads, reinterpret_cast<int*>(dyn));
    if (J3)
    {
      double jp[4] = {0.0, 0.0, 0.0, 0.0};
      j3_partials(ss, sys, wv, ions, J, iat, m.pos_new, jp);
      block_sum<4>(jp, m.red, m.sums + 16);
    }
    block_sum<16>(part, m.red, m.sums);
    if (tid == 0)
    {
      const double* S = m.sums;
      const double rdet = DET ? S[0] : 1.0;
      double ratio      = rdet, gn[3] = {0.0, 0.0, 0.0};
      if (DET)
      {
        ms->cur_ratio[s] = rdet;
        ms->invrow_id[s] = r;
        ms->partial[s]   = grads ? 1 : 0;
        if (grads)
          for (int c = 0; c < 3; ++c)
            gn[c] = (1.0 / rdet) * S[1 + c];
      }
      ms->j_partial = grads ? 1 : 0;
      if (J1)
      {
        ms->j1_curAt = S[7];
        if (grads)
        {
          ms->j1_curLap = S[11];
          for (int c = 0; c < 3; ++c)
          {
            ms->j1_curGrad[c] = S[8 + c];
            gn[c] += S[8 + c];
          }
        }
        ratio *= exp((double)wv.Vat[iat] - S[7]);
      }
      if (J2)
      {
        ms->j2_curUat = S[12];
        if (grads)
          for (int c = 0; c < 3; ++c)
            gn[c] += S[13 + c];
        ratio *= exp((double)wv.Uat[iat] - S[12]);
      }
      if (J3)
      {
        ms->j3_curUat = S[16];
        for (int c = 0; c < 3; ++c)
        {
          ms->j3_curGrad[c] = S[17 + c];
          if (grads)
            gn[c] += S[17 + c];
        }
        ratio *= exp((double)wv.j3Uat[iat] - S[16]);
      }
      if (!isfinite(ratio))
        atomicOr(wv.status, DEV_ERR_NONFINITE);
      dw.out_ratio[w] = ratio;
      for (int c = 0; c < 3; ++c)
        dw.out_grad[3 * w + c] = gn[c];
    }
    break;
  }
  case VERB_WF_ACCEPT:
  {
    if (!s_flag)
      break;
    if (s_active != iat)
    {
      if (tid == 0)
        atomicOr(wv.status, DEV_ERR_STATE);
      break;
    }
    if (DET)
    {
      det_accept(wv, m, s, r, ms->cur_ratio[s], s_partial != 0, true, smem);
      if (tid == 0)
      {
        ms->invrow_id[s] = -1;
        ms->cur_ratio[s] = 1.0;
      }
    }
    if (J1)
    {
      if (!s_jpartial)
      {
        double part[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        j1_partials(ss, ions, m.pos_new, part);
        block_sum<5>(part, m.red, m.sums);
        if (tid == 0)
        {
          ms->j1_curLap = m.sums[4];
          for (int c = 0; c < 3; ++c)
            ms->j1_curGrad[c] = m.sums[1 + c];
        }
      }
      if (tid == 0)
      {
        wv.jlog[0] += (double)wv.Vat[iat] - ms->j1_curAt;
        wv.Vat[iat] = (T)ms->j1_curAt;
        for (int c = 0; c < 3; ++c)
          wv.Grad[c * N + iat] = (T)ms->j1_curGrad[c];
        wv.Lap[iat] = (T)ms->j1_curLap;
      }
    }
    if (J2)
    {
      if (tid == 0)
        m.curUat = ms->j2_curUat;
      __syncthreads();
      j2_accept(ss, wv, m, iat, reinterpret_cast<int*>(dyn));
    }
    if (J3)
      j3_accept(ss, sys, wv, m, J, ions, iat);
    break;
  }
  case VERB_PSET_ACCEPT:
    if (tid == 0)
    {
      if (s_flag)
      {
        if (s_active != iat)
          atomicOr(wv.status, DEV_ERR_STATE);
        else
          for (int c = 0; c < 3; ++c)
          {
            wv.R[3 * iat + c]        = ms->pos[c];
            wv.Rs[c * wv.Npad + iat] = (T)ms->pos[c];
          }
      }
      ms->active = -1;
    }
    break;
  case VERB_COMPLETE:
    if (DET)
    {
      flush(wv, m, 0, smem);
      flush(wv, m, 1, smem);
      if (tid == 0)
        ms->invrow_id[0] = ms->invrow_id[1] = -1;
    }
    break;
  case VERB_TEMP_ROWS:
  {
    const int act = s_active;
    const T px = (T)m.pos_new[0], py = (T)m.pos_new[1], pz = (T)m.pos_new[2];
    if (a.aa_r || a.aa_dr)
      for (int j = tid; j < N; j += NT)
      {
        const T flip = j < act ? T(1) : T(-1);
        T dx = (wv.Rs[j] - px) * flip, dy = (wv.Rs[wv.Npad + j] - py) * flip, dz = (wv.Rs[2 * wv.Npad + j] - pz) * flip;
        const T rr = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
        if (a.aa_r)
          a.aa_r[(size_t)w * N + j] = (double)rr;
        if (a.aa_dr)
        {
          a.aa_dr[((size_t)w * N + j) * 3]     = (double)(dx * flip);
          a.aa_dr[((size_t)w * N + j) * 3 + 1] = (double)(dy * flip);
          a.aa_dr[((size_t)w * N + j) * 3 + 2] = (double)(dz * flip);
        }
      }
    const int I = ss.n_ions;
    if (a.ab_r || a.ab_dr)
      for (int c = tid; c < I; c += NT)
      {
        T dx = (ions[c] - px) * T(-1), dy = (ions[I + c] - py) * T(-1), dz = (ions[2 * I + c] - pz) * T(-1);
        const T rr = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
        if (a.ab_r)
          a.ab_r[(size_t)w * I + c] = (double)rr;
        if (a.ab_dr)
        {
          a.ab_dr[((size_t)w * I + c) * 3]     = (double)(-dx);
          a.ab_dr[((size_t)w * I + c) * 3 + 1] = (double)(-dy);
          a.ab_dr[((size_t)w * I + c) * 3 + 2] = (double)(-dz);
        }
      }
    break;
  }
  }
}

// --------------------------------------------------- evaluateLog parts --
// SPOSet::evaluate_notranspose for every electron of every walker: the
// FP64 Slater matrices (for the inverse) and the derivative rows.
template <typename T>
__global__ void __launch_bounds__(256) spo_matrix_kernel(const DevSystem* __restrict__ sys, DevWalkers dw, int want_lu,
                                                         int ratio_mode_only)
{
  constexpr int VW = Vec16<T>::width;
  __shared__ SplineSmem<T> sp;
  __shared__ double pos[3];
  const int i = blockIdx.x, w = blockIdx.y;
  const WV<T> wv = make_wv<T>(dw, w);
  // DiracDeterminant::evaluateGL (DiracDeterminant.cpp:163-168) re-evaluates
  // the derivative rows only when the determinant's last move was a
  // ratio-only one (UpdateMode ORB_PBYP_RATIO); the test is uniform per block
  if (ratio_mode_only && wv.ms->partial[i < sys->n_up ? 0 : 1])
    return;
  if (threadIdx.x == 0)
  {
    for (int c = 0; c < 3; ++c)
      pos[c] = wv.R[3 * i + c];
    spline_locate(sys, pos, sp);
  }
  __syncthreads();
  const int s = i < sys->n_up ? 0 : 1, r = i - (s ? sys->n_up : 0);
  const int npad = wv.npad, nvec = npad / VW;
  const double dinv[3] = {sys->dinv[0], sys->dinv[1], sys->dinv[2]};
  const bool trace_lap = sys->lap_mode == QMC_LAP_TRACE;
  T* dp  = wv.dpsi(s) + (size_t)r * 3 * npad;
  T* d2p = wv.d2psi(s) + (size_t)r * npad;
  double* lrow = want_lu ? wv.lu + ((size_t)s * wv.n + r) * npad : nullptr;
  for (int q = threadIdx.x; q < nvec; q += blockDim.x)
  {
    SplineOut<T> o;
    spline_eval<T, false>((const T*)sys->coefs, sys->xs, sys->ys, sys->zs, sp, dinv, q * VW, o);
    for (int e = 0; e < VW; ++e)
    {
      const int j = q * VW + e;
      if (lrow)
        lrow[j] = (double)o.v[e];
      dp[j]            = o.gx[e];
      dp[npad + j]     = o.gy[e];
      dp[2 * npad + j] = o.gz[e];
      d2p[j]           = trace_lap ? o.hxx[e] + o.hyy[e] + o.hzz[e] : o.hxx[e];
    }
  }
}

// In-place Gauss-Jordan inverse with partial pivoting in FP64 of the Slater
// matrix A[i][j] = phi_j(r_i) of one walker and spin; writes
// psiM = (A^{-1})^T in the walker precision, log|det A| and its phase
// (DiracMatrix::invert_transpose + computeLogDet, DiracMatrix.h:25-38,
// 93-119: the pivots are LU's U diagonal, the pivot rows LU's ipiv).
template <typename T> __global__ void __launch_bounds__(512) gj_inverse_kernel(DevWalkers dw)
{
  extern __shared__ __align__(16) unsigned char dyn[];
  const int n = dw.n, npad = dw.npad;
  double* col = reinterpret_cast<double*>(dyn);      // [n]
  int* perm   = reinterpret_cast<int*>(col + n);     // [n]
  __shared__ double s_val[32];
  __shared__ int s_idx[32];
  __shared__ double s_logdet;
  __shared__ int s_sign, s_p, s_sing;
  const int s = blockIdx.x, w = blockIdx.y, tid = threadIdx.x, NT = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  const WV<T> wv = make_wv<T>(dw, w);
  double* M      = wv.lu + (size_t)s * n * npad;
  if (tid == 0)
  {
    s_logdet = 0.0;
    s_sign   = 1;
    s_sing   = 0;
  }
  __syncthreads();
  for (int k = 0; k < n; ++k)
  {
    // pivot: first row of maximal |M[i][k]|, i >= k
    double bv = -1.0;
    int bi    = n;
    for (int i = k + tid; i < n; i += NT)
    {
      // a NaN entry competes as 0: the pivot is then always a row < n
      const double v = fmax(fabs(M[(size_t)i * npad + k]), 0.0);
      if (v > bv)
        bv = v, bi = i;
    }
    for (int o = 16; o > 0; o >>= 1)
    {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
      const int oi    = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ov > bv || (ov == bv && oi < bi))
        bv = ov, bi = oi;
    }
    if (lane == 0)
      s_val[wid] = bv, s_idx[wid] = bi;
    __syncthreads();
    if (tid == 0)
    {
      double v = s_val[0];
      int p    = s_idx[0];
      for (int q = 1; q < nw; ++q)
        if (s_val[q] > v || (s_val[q] == v && s_idx[q] < p))
          v = s_val[q], p = s_idx[q];
      s_p     = p;
      perm[k] = p;
    }
    __syncthreads();
    const int p = s_p;
    if (p != k)
      for (int j = tid; j < n; j += NT)
      {
        const double t            = M[(size_t)k * npad + j];
        M[(size_t)k * npad + j] = M[(size_t)p * npad + j];
        M[(size_t)p * npad + j] = t;
      }
    __syncthreads();
    const double piv = M[(size_t)k * npad + k];
    const bool zero  = !(fabs(piv) > 0.0); // a NaN pivot counts as zero
    if (tid == 0)
    {
      if (p != k)
        s_sign = -s_sign;
      if (zero)
        s_sing = 1;
      else
      {
        s_logdet += log(fabs(piv));
        if (piv < 0)
          s_sign = -s_sign;
      }
    }
    if (zero)
    {
      __syncthreads();
      continue;
    }
    const double rp = 1.0 / piv;
    for (int i = tid; i < n; i += NT)
      col[i] = M[(size_t)i * npad + k];
    __syncthreads();
    for (int j = tid; j < n; j += NT)
      M[(size_t)k * npad + j] = (j == k) ? rp : M[(size_t)k * npad + j] * rp;
    __syncthreads();
    // eliminate every other row; warp per row, lanes over columns
    for (int i = wid; i < n; i += nw)
    {
      if (i == k)
        continue;
      const double f = col[i];
      double* mi       = M + (size_t)i * npad;
      const double* mk = M + (size_t)k * npad;
      for (int j = lane; j < n; j += 32)
        mi[j] = (j == k) ? -f * rp : mi[j] - f * mk[j];
    }
    __syncthreads();
  }
  // (P A)^{-1} -> A^{-1}: swap columns back in reverse pivot order
  for (int k = n - 1; k >= 0; --k)
  {
    const int p = perm[k];
    if (p != k)
      for (int i = tid; i < n; i += NT)
      {
        const double t            = M[(size_t)i * npad + k];
        M[(size_t)i * npad + k] = M[(size_t)i * npad + p];
        M[(size_t)i * npad + p] = t;
      }
    __syncthreads();
  }
  // psiM[i][j] = Ainv(j, i)
  T* out = wv.ainv(s);
  for (int i = wid; i < n; i += nw)
    for (int j = lane; j < n; j += 32)
      out[(size_t)i * npad + j] = (T)M[(size_t)j * npad + i];
  if (tid == 0)
  {
    wv.det_log[s]   = s_logdet;
    wv.det_phase[s] = s_sign > 0 ? 0.0 : kPi;
    wv.dcount[s]    = 0;
    if (s_sing)
      atomicOr(wv.status, DEV_ERR_SINGULAR);
  }
}

// Blocked form of the same inverse for n <= GJB_MAX_N: the sweep operator
// applied to 32-column panels.  Rows are never swapped; pivot rows are
// tracked (piv[c] = row that pivots column c).  For a panel C with pivot
// rows P the block exchange of (P, C) is
//     A[:, C]  <- F        (the panel after unblocked Gauss-Jordan on it)
//     A[i, J]  <- [i not in P] A[i, J] + sum_k F[i][k] A[P_k, J]   (J not in C)
// so each panel costs one pass over the matrix instead of 32.  The panel
// lives in shared memory.  A pivot of magnitude <= n eps max|A| counts as
// zero (numerically singular).  At the end A holds the exchanged matrix:
// A^{-1}[a][b] = M[piv[a]][pinv[b]], so psiM[i][j] = M[piv[j]][pinv[i]];
// the sign of det A is the pivots' sign times the parity of piv.
// the panel's rank-32 update on the FP64 tensor cores (mma.sync .f64)
// rather than as CUDA-core FMAs with a 4 x 4 register tile
#ifndef GJB_DMMA
#define GJB_DMMA 1
#endif
constexpr int GJB_B = 32;      // panel width
constexpr int GJB_FS = GJB_B + 1; // padded panel row (conflict-free row-per-thread access)
// padded row of a chunk's pivot rows: the update's B fragments (row k + lane % 4,
// column lane / 4 + 8 t) then fall in distinct banks across each half-warp
constexpr int GJB_RS = 36;
__host__ __device__ constexpr size_t gjb_smem_bytes(int n)
{
  return (((size_t)n * GJB_FS + 1) & ~(size_t)1) * sizeof(double) + (size_t)2 * GJB_B * GJB_RS * sizeof(double) +
      (size_t)2 * n * sizeof(int);
}
constexpr size_t GJB_MAX_SMEM = 226 * 1024;

template <typename T> __global__ void __launch_bounds__(512, 1) gj_blocked_kernel(DevWalkers dw)
{
  extern __shared__ __align__(16) unsigned char dyn[];
  const int n = dw.n, npad = dw.npad;
  double* F = reinterpret_cast<double*>(dyn);   // [n][GJB_FS] panel
  double* R = F + (((size_t)n * GJB_FS + 1) & ~(size_t)1); // [2][GJB_B][GJB_RS] pivot rows of a column chunk (16-byte aligned)
  int* piv  = reinterpret_cast<int*>(R + 2 * GJB_B * GJB_RS); // [n] pivot row of each column
  int* pinv = piv + n;                                 // [n] column pivoted by each row, -1 while free
  __shared__ double s_val[32];
  __shared__ int s_idx[32];
  __shared__ double s_logdet, s_tiny;
  __shared__ int s_neg, s_sing;
  const int s = blockIdx.x, w = blockIdx.y, tid = threadIdx.x, NT = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  const WV<T> wv = make_wv<T>(dw, w);
  double* M = wv.lu + (size_t)s * n * npad;

  // threshold for a zero pivot: n eps max|A| (warp per row, lanes along it)
  double mx = 0.0;
  for (int i = tid; i < n; i += NT)
    pinv[i] = -1;
  for (int i = wid; i < n; i += nw)
  {
    const double* row = M + (size_t)i * npad;
    for (int j = lane; j < n; j += 32)
      mx = fmax(mx, fabs(row[j]));
  }
  for (int o = 16; o > 0; o >>= 1)
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0)
    s_val[wid] = mx;
  __syncthreads();
  if (tid == 0)
  {
    double v = 0.0;
    for (int q = 0; q < nw; ++q)
      v = fmax(v, s_val[q]);
    s_tiny   = (double)n * DBL_EPSILON * v;
    s_logdet = 0.0;
    s_neg    = 0;
    s_sing   = 0;
  }
  __syncthreads();
  const double tiny = s_tiny;

  for (int c0 = 0; c0 < n; c0 += GJB_B)
  {
    const int bw = min(GJB_B, n - c0);
    for (int idx = tid; idx < n * GJB_B; idx += NT)
    {
      const int i = idx / GJB_B, kk = idx % GJB_B;
      F[i * GJB_FS + kk] = kk < bw ? M[(size_t)i * npad + c0 + kk] : 0.0;
    }
    __syncthreads();
    // ---- unblocked Gauss-Jordan on the panel, two barriers per pivot: every
    // thread reduces the warps' candidates itself (same order, same pivot);
    // the other rows are eliminated with the unscaled pivot row times 1/pv,
    // and the pivot row is scaled at the start of the next step (it is no
    // longer a candidate, and the next elimination reads it after the
    // barrier)
    int pp     = -1;  // pivot row of the previous step, still unscaled
    double prp = 0.0; // its reciprocal pivot
    int pk     = 0;   // its column
    for (int kk = 0; kk < bw; ++kk)
    {
      if (pp >= 0 && tid < bw)
        F[pp * GJB_FS + tid] = tid == pk ? prp : F[pp * GJB_FS + tid] * prp;
      double bv = -1.0;
      int bi    = n;
      for (int i = tid; i < n; i += NT)
        if (pinv[i] < 0)
        {
          // a NaN entry competes as 0: some free row is always taken, so
          // piv and pinv end as full permutations of 0..n-1
          const double v = fmax(fabs(F[i * GJB_FS + kk]), 0.0);
          if (v > bv)
            bv = v, bi = i;
        }
      for (int o = 16; o > 0; o >>= 1)
      {
        const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int oi    = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ov > bv || (ov == bv && oi < bi))
          bv = ov, bi = oi;
      }
      if (lane == 0)
        s_val[wid] = bv, s_idx[wid] = bi;
      __syncthreads();
      double v = s_val[0];
      int p    = s_idx[0];
      for (int q = 1; q < nw; ++q)
        if (s_val[q] > v || (s_val[q] == v && s_idx[q] < p))
          v = s_val[q], p = s_idx[q];
      const double pv = F[p * GJB_FS + kk];
      const bool ok   = fabs(pv) > tiny;
      if (tid == 0)
      {
        piv[c0 + kk] = p;
        pinv[p]      = c0 + kk;
        if (!ok)
          s_sing = 1; // zero pivot: reported, column left as is
        else
        {
          s_logdet += log(fabs(pv));
          if (pv < 0)
            s_neg ^= 1;
        }
      }
      pp = -1;
      if (ok)
      {
        const double rp = 1.0 / pv;
        for (int i = tid; i < n; i += NT)
          if (i != p)
          {
            double* fi     = F + i * GJB_FS;
            const double g = fi[kk] * rp;
            for (int q = 0; q < bw; ++q)
              fi[q] = q == kk ? -g : fi[q] - g * F[p * GJB_FS + q];
          }
        pp = p, prp = rp, pk = kk;
      }
      __syncthreads();
    }
    if (pp >= 0 && tid < bw)
      F[pp * GJB_FS + tid] = tid == pk ? prp : F[pp * GJB_FS + tid] * prp;
    __syncthreads();
    // ---- the other columns, in chunks of 32: A[:, J] <- [i not in P] A[:, J] + F A[P, J]
    // (the chunks' pivot rows alternate between two buffers: one barrier per
    // chunk; a buffer is refilled only after every thread has passed the
    // next chunk's barrier, i.e. finished with it)
    int rbuf = 0;
    for (int j0 = 0; j0 < n; j0 += 32)
    {
      if (j0 == c0)
        continue;
      const int jw = min(32, n - j0);
      double* Rb   = R + rbuf * GJB_B * GJB_RS;
      rbuf ^= 1;
      for (int idx = tid; idx < GJB_B * 32; idx += NT)
      {
        const int k = idx >> 5, jj = idx & 31;
        Rb[k * GJB_RS + jj] = (k < bw && jj < jw) ? M[(size_t)piv[c0 + k] * npad + j0 + jj] : 0.0;
      }
      __syncthreads();
#if GJB_DMMA
      // the rank-32 update on the FP64 tensor cores (mma.sync m8n8k4 .f64):
      // each warp takes three 8-row groups at a time and the chunk's four
      // 8-column tiles; fragments: A (8 x 4 of the panel) one element per
      // lane at (lane / 4, lane % 4), B (4 x 8 of the pivot rows) at
      // (lane % 4, lane / 4), C (8 x 8) two at (lane / 4, 2 (lane % 4) + e).
      // Group g holds rows 32 (g / 4) + g % 4 + 4 r (r = 0..7): with the
      // panel's row stride of 33 doubles the A fragments of a half-warp then
      // fall in distinct banks (consecutive rows put lane % 4 and lane / 4 on
      // the same banks)
      {
        const int qr = lane >> 2, qc = lane & 3;
        const int ngroups = (n + 31) / 32 * 4;
        auto grow = [&](int g) { return (g >> 2) * 32 + (g & 3) + 4 * qr; };
        for (int gb = wid * 3; gb < ngroups; gb += nw * 3)
        {
          double acc[3][4][2];
#pragma unroll
          for (int u = 0; u < 3; ++u)
          {
            const int i     = gb + u < ngroups ? grow(gb + u) : n;
            const int c     = i < n ? pinv[i] : c0;
            const bool zero = i >= n || (c >= c0 && c < c0 + bw);
            const double* mi = M + (size_t)(i < n ? i : 0) * npad + j0;
            // a lane's two columns of a tile are adjacent: one 16-byte load
#pragma unroll
            for (int t = 0; t < 4; ++t)
            {
              const int col = t * 8 + 2 * qc;
              if (!zero && col + 1 < jw)
              {
                const double2 v = *reinterpret_cast<const double2*>(mi + col);
                acc[u][t][0] = v.x, acc[u][t][1] = v.y;
              }
              else
              {
                acc[u][t][0] = (zero || col >= jw) ? 0.0 : mi[col];
                acc[u][t][1] = 0.0;
              }
            }
          }
#pragma unroll 2
          for (int k = 0; k < GJB_B; k += 4)
          {
            double b[4];
#pragma unroll
            for (int t = 0; t < 4; ++t)
              b[t] = Rb[(k + qc) * GJB_RS + t * 8 + qr];
#pragma unroll
            for (int u = 0; u < 3; ++u)
            {
              const double a = F[min(grow(gb + u), n - 1) * GJB_FS + k + qc];
#pragma unroll
              for (int t = 0; t < 4; ++t)
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                             : "+d"(acc[u][t][0]), "+d"(acc[u][t][1])
                             : "d"(a), "d"(b[t]));
            }
          }
#pragma unroll
          for (int u = 0; u < 3; ++u)
          {
            const int i = gb + u < ngroups ? grow(gb + u) : n;
            if (i >= n)
              continue;
            double* mi = M + (size_t)i * npad + j0;
#pragma unroll
            for (int t = 0; t < 4; ++t)
            {
              const int col = t * 8 + 2 * qc;
              if (col + 1 < jw)
                *reinterpret_cast<double2*>(mi + col) = make_double2(acc[u][t][0], acc[u][t][1]);
              else if (col < jw)
                mi[col] = acc[u][t][0];
            }
          }
        }
      }
#else
      // each thread updates a 4-row x 4-column tile: columns j0 + 2 cg + {0, 1}
      // and j0 + 16 + 2 cg + {0, 1} (cg = lane % 8: a row's 32 columns are
      // two 128-byte runs over 8 lanes), rows ib..ib+3 (rg = lane / 8), so
      // that one shared-memory load feeds several FMAs; each element's FMA
      // chain over the panel runs in the same order as a row-by-row update
      const int cg = lane & 7, rg = lane >> 3;
      const int ja = 2 * cg, jb = 16 + 2 * cg;
      const bool va = ja < jw, vb = jb < jw; // jw is even unless n is odd
      for (int ib = wid * 16 + rg * 4; ib < n; ib += nw * 16)
      {
        double acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
          const int i     = ib + u;
          const int c     = i < n ? pinv[i] : c0;
          const bool zero = i >= n || (c >= c0 && c < c0 + bw);
          const double* mi = M + (size_t)(i < n ? i : 0) * npad + j0;
#pragma unroll
          for (int e = 0; e < 2; ++e)
          {
            acc[u][e]     = (zero || ja + e >= jw) ? 0.0 : mi[ja + e];
            acc[u][2 + e] = (zero || jb + e >= jw) ? 0.0 : mi[jb + e];
          }
        }
#pragma unroll 4
        for (int k = 0; k < GJB_B; ++k)
        {
          const double2 ra = *reinterpret_cast<const double2*>(Rb + k * GJB_RS + ja);
          const double2 rb = *reinterpret_cast<const double2*>(Rb + k * GJB_RS + jb);
#pragma unroll
          for (int u = 0; u < 4; ++u)
          {
            const double f = F[min(ib + u, n - 1) * GJB_FS + k];
            acc[u][0]      = fma(f, ra.x, acc[u][0]);
            acc[u][1]      = fma(f, ra.y, acc[u][1]);
            acc[u][2]      = fma(f, rb.x, acc[u][2]);
            acc[u][3]      = fma(f, rb.y, acc[u][3]);
          }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
        {
          const int i = ib + u;
          if (i >= n)
            continue;
          double* mi = M + (size_t)i * npad + j0;
#pragma unroll
          for (int e = 0; e < 2; ++e)
          {
            if (va && ja + e < jw)
              mi[ja + e] = acc[u][e];
            if (vb && jb + e < jw)
              mi[jb + e] = acc[u][2 + e];
          }
        }
      }
#endif
    }
    for (int idx = tid; idx < n * bw; idx += NT)
    {
      const int i = idx / bw, kk = idx % bw;
      M[(size_t)i * npad + c0 + kk] = F[i * GJB_FS + kk];
    }
    __syncthreads();
  }
  // psiM[i][j] = A^{-1}[j][i] = M[piv[j]][pinv[i]], through the panel's
  // shared memory (free now): 32 rows M[piv[j]] at a time are read whole
  // and coalesced, then every row i of psiM takes its 32 columns from
  // column pinv[i] of them (an odd row stride keeps those reads on distinct
  // banks), so that neither side gathers single doubles from global memory
  T* out       = wv.ainv(s);
  double* S    = F;     // [32][SS] over the panel and the chunk buffers: 32 (n + 1) <= 33 n + 2304 doubles
  const int SS = n | 1; // >= n, odd
  for (int jb = 0; jb < n; jb += 32)
  {
    const int jw = min(32, n - jb);
    for (int idx = tid; idx < jw * n; idx += NT)
    {
      const int jj = idx / n, c = idx - jj * n;
      S[jj * SS + c] = M[(size_t)piv[jb + jj] * npad + c];
    }
    __syncthreads();
    for (int idx = tid; idx < n * 32; idx += NT)
    {
      const int i = idx >> 5, jj = idx & 31;
      if (jj < jw)
        out[(size_t)i * npad + jb + jj] = (T)S[jj * SS + pinv[i]];
    }
    __syncthreads();
  }
  if (tid == 0)
  {
    // parity of the permutation c -> piv[c] from its cycles
    int odd = 0;
    for (int c = 0; c < n; ++c)
    {
      if (piv[c] < 0)
        continue;
      int j = c, len = 0;
      while (piv[j] >= 0)
      {
        const int nx = piv[j];
        piv[j]       = -1;
        j            = nx;
        ++len;
      }
      odd ^= (len - 1) & 1;
    }
    wv.det_log[s]   = s_logdet;
    wv.det_phase[s] = (s_neg ^ odd) ? kPi : 0.0;
    wv.dcount[s]    = 0;
    if (s_sing)
      atomicOr(wv.status, DEV_ERR_SINGULAR);
  }
}

// J1 / J2 from scratch (OneBodyJastrow::recompute, TwoBodyJastrow::recompute):
// warp per electron over its full rows.
template <typename T>
__global__ void __launch_bounds__(256) jastrow_recompute_kernel(const DevSystem* __restrict__ sys, DevWalkers dw)
{
  __shared__ SysSmem<T> ss;
  load_sys(sys, ss);
  const int w = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const WV<T> wv = make_wv<T>(dw, w);
  const int N = wv.N, I = ss.n_ions, Npad = wv.Npad;
  const T* ions = (const T*)sys->ion_soa;
  const T* Rs   = wv.Rs;
  for (int i = wid; i < N; i += nw)
  {
    const T px = Rs[i], py = Rs[Npad + i], pz = Rs[2 * Npad + i];
    if (ss.comp & QMC_WF_J1)
    {
      double v = 0, g0 = 0, g1 = 0, g2 = 0, l = 0;
      for (int c = lane; c < I; c += 32)
      {
        T dx = (ions[c] - px) * T(-1), dy = (ions[I + c] - py) * T(-1), dz = (ions[2 * I + c] - pz) * T(-1);
        const T r = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
        const FunctorT<T>& f = ss.j1[ion_group(ss, c)];
        if (r < f.cutoff)
        {
          T u, du, d2u;
          functor_vgl(f, r, u, du, d2u);
          v += u;
          g0 += (double)(du * -dx);
          g1 += (double)(du * -dy);
          g2 += (double)(du * -dz);
          l += (double)(d2u + T(2) * du);
        }
      }
      v = warp_sum(v), g0 = warp_sum(g0), g1 = warp_sum(g1), g2 = warp_sum(g2), l = warp_sum(l);
      if (lane == 0)
      {
        wv.Vat[i]         = (T)v;
        wv.Grad[i]        = (T)g0;
        wv.Grad[N + i]    = (T)g1;
        wv.Grad[2 * N + i] = (T)g2;
        wv.Lap[i]         = (T)l;
      }
    }
    if (ss.comp & QMC_WF_J2)
    {
      const int gi = i < ss.n_up ? 0 : 1;
      double v = 0, g0 = 0, g1 = 0, g2 = 0, l = 0;
      for (int j = lane; j < N; j += 32)
      {
        if (j == i)
          continue;
        const T flip = j < i ? T(1) : T(-1);
        T dx = (Rs[j] - px) * flip, dy = (Rs[Npad + j] - py) * flip, dz = (Rs[2 * Npad + j] - pz) * flip;
        const T r = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
        const FunctorT<T>& f = (gi == (j < ss.n_up ? 0 : 1)) ? ss.j2uu : ss.j2ud;
        if (r < f.cutoff)
        {
          T u, du, d2u;
          functor_vgl(f, r, u, du, d2u);
          v += u;
          g0 += (double)(du * dx * flip);
          g1 += (double)(du * dy * flip);
          g2 += (double)(du * dz * flip);
          l += (double)(d2u + T(2) * du);
        }
      }
      v = warp_sum(v), g0 = warp_sum(g0), g1 = warp_sum(g1), g2 = warp_sum(g2), l = warp_sum(l);
      if (lane == 0)
      {
        wv.Uat[i]          = (T)v;
        wv.dUat[i]         = (T)g0;
        wv.dUat[N + i]     = (T)g1;
        wv.dUat[2 * N + i] = (T)g2;
        wv.d2Uat[i]        = (T)(-l);
      }
    }
  }
}

// ThreeBodyJastrow::recompute (ThreeBodyJastrow.h:222-243, 391-427): the
// per-ion electron lists in ascending electron order (build_compact_list),
// then for every electron the sums over all its triples.  The reference
// walks the triangle k < j and adds the k-side terms back; the functor is
// symmetric in its two electrons (gamma(l,m,n) = gamma(m,l,n)), so the full
// sums per electron are the same quantities.  Warp per list, then warp per
// electron.
constexpr int J3R_WARPS = 8;
template <typename T>
__global__ void __launch_bounds__(256) j3_recompute_kernel(const DevSystem* __restrict__ sys, DevWalkers dw)
{
  __shared__ SysSmem<T> ss;
  __shared__ int s_ion[J3R_WARPS][J3_NEAR];
  __shared__ T s_r[J3R_WARPS][J3_NEAR], s_d[J3R_WARPS][3][J3_NEAR];
  __shared__ int s_seg[J3R_WARPS][2 * J3_NEAR + 1];
  load_sys(sys, ss);
  const int w = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const WV<T> wv     = make_wv<T>(dw, w);
  const int N = wv.N, I = ss.n_ions, Np = wv.Npad, cap = wv.j3cap;
  const T* ions      = (const T*)sys->ion_soa;
  const T* gam       = (const T*)sys->j3_gamma;
  const unsigned below = (1u << lane) - 1u;
  for (int li = wid; li < 2 * I; li += nw)
  {
    const int kg = li / I, ion = li % I;
    const T cut  = ss.j3cut[ion_group(ss, ion)];
    const int e0 = kg ? ss.n_up : 0, e1 = kg ? N : ss.n_up;
    int* lst     = wv.j3list + (size_t)li * cap;
    int c        = 0;
    for (int j0 = e0; j0 < e1; j0 += 32)
    {
      const int j = j0 + lane;
      bool in     = false;
      if (j < e1)
      {
        T dx, dy, dz;
        in = j3_ion_dist(ss, ions, ion, wv.Rs[j], wv.Rs[Np + j], wv.Rs[2 * Np + j], cut, dx, dy, dz) < cut;
      }
      const unsigned b = __ballot_sync(0xffffffffu, in);
      const int at     = c + __popc(b & below);
      if (in)
      {
        if (at < cap)
          lst[at] = j;
        else
          atomicOr(wv.status, DEV_ERR_CAPACITY);
      }
      c += __popc(b);
    }
    if (lane == 0)
      wv.j3cnt[li] = c < cap ? c : cap;
  }
  __syncthreads();
  for (int j = wid; j < N; j += nw)
  {
    const T px = wv.Rs[j], py = wv.Rs[Np + j], pz = wv.Rs[2 * Np + j];
    int nn     = 0;
    for (int c0 = 0; c0 < I; c0 += 32)
    {
      const int c = c0 + lane;
      bool in     = false;
      T dx = 0, dy = 0, dz = 0, r = 0;
      if (c < I)
      {
        const T cut = ss.j3cut[ion_group(ss, c)];
        r           = j3_ion_dist(ss, ions, c, px, py, pz, cut, dx, dy, dz);
        in          = r < cut;
      }
      const unsigned b = __ballot_sync(0xffffffffu, in);
      const int at     = nn + __popc(b & below);
      if (in)
      {
        if (at < J3_NEAR)
        {
          s_ion[wid][at]  = c;
          s_r[wid][at]    = r;
          s_d[wid][0][at] = dx;
          s_d[wid][1][at] = dy;
          s_d[wid][2][at] = dz;
        }
        else
          atomicOr(wv.status, DEV_ERR_CAPACITY);
      }
      nn += __popc(b);
    }
    nn           = nn < J3_NEAR ? nn : J3_NEAR;
    const int ns = 2 * nn;
    __syncwarp();
    for (int s = lane; s < ns; s += 32)
      s_seg[wid][s + 1] = wv.j3cnt[(s / nn) * I + s_ion[wid][s % nn]];
    __syncwarp();
    if (lane == 0)
    {
      s_seg[wid][0] = 0;
      for (int s = 1; s <= ns; ++s)
        s_seg[wid][s] += s_seg[wid][s - 1];
    }
    __syncwarp();
    const J3Near<T> nv{nn, s_seg[wid], s_ion[wid], s_r[wid], s_d[wid][0], s_d[wid][1], s_d[wid][2]};
    const int P = s_seg[wid][ns];
    double u = 0, g0 = 0, g1 = 0, g2 = 0, l = 0;
    for (int p = lane; p < P; p += 32)
    {
      J3Terms<T> o;
      if (j3_triple(ss, gam, wv, ions, nv, p, j, px, py, pz, o))
      {
        u += (double)o.uj;
        g0 += (double)o.gj[0];
        g1 += (double)o.gj[1];
        g2 += (double)o.gj[2];
        l += (double)o.lj;
      }
    }
    u = warp_sum(u), g0 = warp_sum(g0), g1 = warp_sum(g1), g2 = warp_sum(g2), l = warp_sum(l);
    if (lane == 0)
    {
      wv.j3Uat[j]          = (T)u;
      wv.j3dUat[j]         = (T)g0;
      wv.j3dUat[N + j]     = (T)g1;
      wv.j3dUat[2 * N + j] = (T)g2;
      wv.j3d2Uat[j]        = (T)l;
    }
    __syncwarp(); // the warp's near-ion arrays are rewritten for its next electron
  }
}

template <typename T>
__global__ void __launch_bounds__(256) gl_kernel(const DevSystem* __restrict__ sys, DevWalkers dw)
{
  __shared__ SysSmem<T> ss;
  __shared__ MoveSmem m;
  load_sys(sys, ss);
  const WV<T> wv = make_wv<T>(dw, blockIdx.x);
  evaluate_gl(ss, wv, m, dw.logpsi + blockIdx.x);
}

template <typename T> __global__ void sync_rs_kernel(DevWalkers dw)
{
  const int w = blockIdx.x;
  T* Rs       = (T*)dw.Rs + (size_t)w * 3 * dw.Npad;
  for (int i = threadIdx.x; i < dw.Npad; i += blockDim.x)
    for (int c = 0; c < 3; ++c)
      Rs[c * dw.Npad + i] = i < dw.N ? (T)dw.R[((size_t)w * dw.N + i) * 3 + c] : T(0);
}

// SPOSet::evaluate (VGH, or values only) at arbitrary Cartesian points
template <typename T>
__global__ void __launch_bounds__(256) spo_points_kernel(const DevSystem* __restrict__ sys, const double* pos, double* v,
                                                         double* g, double* h, int values_only)
{
  constexpr int VW = Vec16<T>::width;
  __shared__ SplineSmem<T> sp;
  __shared__ double p[3];
  const int ip = blockIdx.x;
  if (threadIdx.x == 0)
  {
    for (int c = 0; c < 3; ++c)
      p[c] = pos[3 * ip + c];
    spline_locate(sys, p, sp);
  }
  __syncthreads();
  const int norb = sys->norb, nvec = sys->npad / VW;
  const double dinv[3] = {sys->dinv[0], sys->dinv[1], sys->dinv[2]};
  for (int q = threadIdx.x; q < nvec; q += blockDim.x)
  {
    if (values_only)
    {
      T out[VW];
      spline_eval_v((const T*)sys->coefs, sys->xs, sys->ys, sys->zs, sp, q * VW, out);
      for (int e = 0; e < VW; ++e)
        if (q * VW + e < norb && v)
          v[(size_t)ip * norb + q * VW + e] = (double)out[e];
      continue;
    }
    SplineOut<T> o;
    spline_eval<T, true>((const T*)sys->coefs, sys->xs, sys->ys, sys->zs, sp, dinv, q * VW, o);
    for (int e = 0; e < VW; ++e)
    {
      const int j = q * VW + e;
      if (j >= norb)
        continue;
      if (v)
        v[(size_t)ip * norb + j] = (double)o.v[e];
      if (g)
      {
        g[((size_t)ip * 3 + 0) * norb + j] = (double)o.gx[e];
        g[((size_t)ip * 3 + 1) * norb + j] = (double)o.gy[e];
        g[((size_t)ip * 3 + 2) * norb + j] = (double)o.gz[e];
      }
      if (h)
      {
        const T hv[6] = {o.hxx[e], o.hxy[e], o.hxz[e], o.hyy[e], o.hyz[e], o.hzz[e]};
        for (int c = 0; c < 6; ++c)
          h[((size_t)ip * 6 + c) * norb + j] = (double)hv[c];
      }
    }
  }
}

// DelayedUpdate engine on spin 0 of walker 0 of a batch view
template <typename T>
__global__ void __launch_bounds__(256) det_engine_kernel(DevWalkers dw, int op, int row, int tc)
{
  __shared__ MoveSmem m;
  extern __shared__ __align__(16) unsigned char dyn[];
  T* smem        = reinterpret_cast<T*>(dyn);
  const WV<T> wv = make_wv<T>(dw, 0);
  if (threadIdx.x == 0)
    m.timing = 0;
  if constexpr (sizeof(T) == 4)
    tc_begin(m, op == DETENG_GET_INV_ROW ? 0 : tc, dw.wait_cycles); // accept_row flushes when the delay fills
  else
    tc_none(m);
  if (op == DETENG_GET_INV_ROW)
    get_inv_row(wv, m, 0, row, wv.dcount[0]);
  else if (op == DETENG_ACCEPT_ROW)
  {
    get_inv_row(wv, m, 0, row, wv.dcount[0]); // fills row dc of Binv, as DiracDeterminant does via ratio
    __syncthreads();
    det_accept(wv, m, 0, row, 1.0, false, false, smem);
  }
  else
    flush(wv, m, 0, smem);
  if constexpr (sizeof(T) == 4)
    tc_end(m);
}

// ----------------------------------------------------------- launchers --
template <typename K> static void allow_smem(K kernel, size_t bytes)
{
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_verb(bool fp32, const DevSystem* sys, const DevWalkers& dw, const VerbArgs& a, int threads,
                        int max_k, cudaStream_t st)
{
  if (max_k > MAXK)
    return cudaErrorInvalidValue;
  // dynamic shared memory: the flush scratch, or the J3 move scratch
  const size_t b32 = std::max(flush_smem_bytes<float>(), sizeof(J3Smem<float>));
  const size_t b64 = std::max(flush_smem_bytes<double>(), sizeof(J3Smem<double>));
  if (fp32)
  {
    allow_smem(verb_kernel<float>, b32);
    verb_kernel<float><<<dw.W, threads, b32, st>>>(sys, dw, a);
  }
  else
  {
    allow_smem(verb_kernel<double>, b64);
    verb_kernel<double><<<dw.W, threads, b64, st>>>(sys, dw, a);
  }
  return cudaGetLastError();
}

cudaError_t launch_spo_matrix(bool fp32, const DevSystem* sys, const DevWalkers& dw, bool want_lu, cudaStream_t st,
                              bool ratio_mode_only)
{
  dim3 grid(dw.N, dw.W);
  const int vw      = fp32 ? 4 : 2;
  const int threads = min(256, round_up(dw.npad / vw, 32));
  if (fp32)
    spo_matrix_kernel<float><<<grid, threads, 0, st>>>(sys, dw, want_lu ? 1 : 0, ratio_mode_only ? 1 : 0);
  else
    spo_matrix_kernel<double><<<grid, threads, 0, st>>>(sys, dw, want_lu ? 1 : 0, ratio_mode_only ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_gj_inverse(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads, int n_spins,
                              cudaStream_t st)
{
  (void)sys;
  dim3 grid(n_spins, dw.W);
  const size_t bsm = gjb_smem_bytes(dw.n);
  if (bsm <= GJB_MAX_SMEM)
  {
    if (fp32)
    {
      allow_smem(gj_blocked_kernel<float>, bsm);
      gj_blocked_kernel<float><<<grid, 512, bsm, st>>>(dw);
    }
    else
    {
      allow_smem(gj_blocked_kernel<double>, bsm);
      gj_blocked_kernel<double><<<grid, 512, bsm, st>>>(dw);
    }
    return cudaGetLastError();
  }
  const size_t smem = (size_t)dw.n * (sizeof(double) + sizeof(int));
  if (fp32)
  {
    allow_smem(gj_inverse_kernel<float>, smem);
    gj_inverse_kernel<float><<<grid, threads, smem, st>>>(dw);
  }
  else
  {
    allow_smem(gj_inverse_kernel<double>, smem);
    gj_inverse_kernel<double><<<grid, threads, smem, st>>>(dw);
  }
  return cudaGetLastError();
}

cudaError_t launch_jastrow_recompute(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads,
                                     cudaStream_t st)
{
  if (fp32)
    jastrow_recompute_kernel<float><<<dw.W, threads, 0, st>>>(sys, dw);
  else
    jastrow_recompute_kernel<double><<<dw.W, threads, 0, st>>>(sys, dw);
  return cudaGetLastError();
}

cudaError_t launch_j3_recompute(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads,
                                cudaStream_t st)
{
  (void)threads; // one warp per list / electron, J3R_WARPS warps
  if (fp32)
    j3_recompute_kernel<float><<<dw.W, 32 * J3R_WARPS, 0, st>>>(sys, dw);
  else
    j3_recompute_kernel<double><<<dw.W, 32 * J3R_WARPS, 0, st>>>(sys, dw);
  return cudaGetLastError();
}

cudaError_t launch_gl(bool fp32, const DevSystem* sys, const DevWalkers& dw, int threads, cudaStream_t st)
{
  if (fp32)
    gl_kernel<float><<<dw.W, threads, 0, st>>>(sys, dw);
  else
    gl_kernel<double><<<dw.W, threads, 0, st>>>(sys, dw);
  return cudaGetLastError();
}

cudaError_t launch_sync_rs(bool fp32, const DevWalkers& dw, cudaStream_t st)
{
  if (fp32)
    sync_rs_kernel<float><<<dw.W, 256, 0, st>>>(dw);
  else
    sync_rs_kernel<double><<<dw.W, 256, 0, st>>>(dw);
  return cudaGetLastError();
}

// activeR(iat) (ParticleSet.h:222): the proposed position while iat is the
// active electron, else the current one
__global__ void active_pos_kernel(DevWalkers dw, int iat, double* pos)
{
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= dw.W)
    return;
  const MoveState& ms = dw.ms[w];
  for (int c = 0; c < 3; ++c)
    pos[3 * w + c] = ms.active == iat ? ms.pos[c] : dw.R[((size_t)w * dw.N + iat) * 3 + c];
}

cudaError_t launch_active_pos(const DevWalkers& dw, int iat, double* pos, cudaStream_t st)
{
  active_pos_kernel<<<(dw.W + 127) / 128, 128, 0, st>>>(dw, iat, pos);
  return cudaGetLastError();
}

cudaError_t launch_spo_points(bool fp32, const DevSystem* sys, int n_pos, const double* pos, double* v, double* g,
                              double* h, bool values_only, cudaStream_t st)
{
  if (n_pos <= 0)
    return cudaSuccess;
  if (fp32)
    spo_points_kernel<float><<<n_pos, 128, 0, st>>>(sys, pos, v, g, h, values_only ? 1 : 0);
  else
    spo_points_kernel<double><<<n_pos, 128, 0, st>>>(sys, pos, v, g, h, values_only ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_det_engine(bool fp32, int op, const DevWalkers& dw, int row, int max_k, cudaStream_t st, bool tc)
{
  if (max_k > MAXK)
    return cudaErrorInvalidValue;
  if (tc && (!fp32 || max_k > TC_KD))
    return cudaErrorInvalidValue;
  if (fp32)
  {
    const size_t bytes = tc && tc_flush_smem_bytes(max_k) > flush_smem_bytes<float>() ? tc_flush_smem_bytes(max_k)
                                                                                      : flush_smem_bytes<float>();
    allow_smem(det_engine_kernel<float>, bytes);
    det_engine_kernel<float><<<1, 256, bytes, st>>>(dw, op, row, tc ? 1 : 0);
  }
  else
  {
    allow_smem(det_engine_kernel<double>, flush_smem_bytes<double>());
    det_engine_kernel<double><<<1, 256, flush_smem_bytes<double>(), st>>>(dw, op, row, 0);
  }
  return cudaGetLastError();
}

} // namespace qmc
