// flush_tc.cuh -- the Woodbury flush of an FP32 walker on the tensor cores.
//
// Same algebra as flush() (DelayedUpdate::updateInvMat, DelayedUpdate.h:
// 184-191, row-major):  U2 = Binv V,  tm = Ainv U^T - E,  Ainv -= tm U2,
// with the two n x n x dc products on tcgen05 in 3xTF32: every operand x is
// split into hi = tf32(x) and lo = tf32(x - hi), and A B is accumulated in
// FP32 in TMEM as A_lo B_hi + A_hi B_lo + A_hi B_hi.  U2 is formed with FP64
// accumulation and stored, transposed and split, as an image of ready
// K-major tiles in per-walker global scratch (L2-resident).
//
// Per 128-row block of Ainv (M = 128):
//   GEMM1  TMEM[0:Kd) = Ainv[rows, :] U^T     K = npad in chunks of 16, two
//                                             shared-memory stages
//   tm  = TMEM - E  -> split into shared memory (A operand of GEMM2)
//   GEMM2  for each 32-column block: TMEM[32 (t&1)] = tm U2[:, cols]; two
//          accumulators and two B stages so the next block's MMA runs while
//          this block's columns of Ainv are read, updated and written back.
// Kd = dc rounded up to 16 (<= 64).  One thread issues the MMAs; warps 0-3
// read the accumulators (warp w owns TMEM lanes 32w..32w+31 = rows).
// GEMM1's result (Kd columns) is read out of TMEM before GEMM2's two
// 32-column accumulators reuse the same 64 columns.
// The tiles overlay the cached Binv of the fused sweep once U2 is formed.
// Included by flush.cuh inside namespace qmc.
#pragma once

constexpr int TC_BK1  = 16; // K chunk of GEMM1
constexpr int TC_BN2  = 32; // columns per GEMM2 block
constexpr int TC_COLS = 64; // TMEM columns per CTA

// padded delay of a flush of dc delayed rows: N of GEMM1, K of GEMM2
__host__ __device__ constexpr int tc_kd(int dc) { return (dc + 15) / 16 * 16; }
// the flush's tile layout is sized for the largest padded delay of the
// batch's rank, 32 (delay rank <= 32) or 64
__host__ __device__ constexpr int tc_kdm(int kmax) { return kmax <= 32 ? 32 : 64; }
// floats of one GEMM1 stage: A hi / lo (128 x 16) and B hi / lo (KDM x 16)
__host__ __device__ constexpr int tc_stage1(int KDM) { return 2 * 128 * TC_BK1 + 2 * KDM * TC_BK1; }

// shared-memory bytes of the tensor-core flush tiles for delay ranks up to
// kmax: two GEMM1 stages, or GEMM2's A operand (hi / lo, 128 x KDM) and two
// B stages (hi / lo, 32 x KDM), whichever is larger (48 KB up to delay 32,
// 96 KB up to 64)
__host__ __device__ constexpr size_t tc_flush_smem_bytes(int kmax)
{
  return (size_t)4 * (2 * 128 * tc_kdm(kmax) + 2 * 2 * TC_BN2 * tc_kdm(kmax)) >
          (size_t)4 * 2 * tc_stage1(tc_kdm(kmax))
      ? (size_t)4 * (2 * 128 * tc_kdm(kmax) + 2 * 2 * TC_BN2 * tc_kdm(kmax))
      : (size_t)4 * 2 * tc_stage1(tc_kdm(kmax));
}

// tensor-core state of a CTA whose kernel has no tensor-core code
__device__ __forceinline__ void tc_none(MoveSmem& m)
{
  if (threadIdx.x == 0)
  {
    m.tc_on    = 0;
    m.tc_abort = 0;
    m.tc_phase = 0;
  }
  __syncthreads();
}
// set-up / tear-down of the CTA's tensor-core state (all threads call); a
// CTA that does not use the tensor cores gives up its allocation right at
// once so that the SM keeps taking further CTAs.  `limit`: SM cycles after
// which each bounded wait of the flush gives up (DevWalkers::wait_cycles).
__device__ __forceinline__ void tc_begin(MoveSmem& m, int on, long long limit)
{
  if (threadIdx.x == 0)
  {
    m.tc_on    = on;
    m.tc_abort = 0;
    m.tc_phase = 0;
    m.tc_limit = limit;
  }
  if (!on && threadIdx.x < 32)
    tc_relinquish();
  if (on)
  {
    if (threadIdx.x < 32)
      tc_alloc(&m.tc_tmem, TC_COLS);
    if (threadIdx.x == 0)
    {
      for (int b = 0; b < 5; ++b)
        mbar_init(&m.tc_bar[b], 1);
      mbar_fence_init();
    }
    tc_fence_before();
  }
  __syncthreads();
  if (on)
    tc_fence_after();
}
// After a wait gave up, MMAs the CTA issued may still be writing its TMEM
// columns: the issuing thread (thread 0) commits once more to the drain
// barrier, which arrives when all of them have completed, and waits for it
// (bounded by the default limit, not the batch's, which may be tiny) before
// the columns are released to the next CTA on this SM.
__device__ __forceinline__ void tc_end(MoveSmem& m)
{
  __syncthreads();
  if (m.tc_on && m.tc_abort && threadIdx.x == 0)
  {
    tc_commit(&m.tc_bar[4]);
    mbar_wait(&m.tc_bar[4], 0u, kTcWaitCycles);
  }
  __syncthreads();
  if (m.tc_on && threadIdx.x < 32)
  {
    tc_fence_after();
    tc_dealloc(m.tc_tmem, TC_COLS);
  }
}

// all threads: bounded wait on commit barrier b; records a timeout
__device__ __forceinline__ void tc_wait(MoveSmem& m, int b, uint32_t& ph, const WV<float>& wv)
{
  if (!mbar_wait(&m.tc_bar[b], (ph >> b) & 1u, m.tc_limit))
  {
    m.tc_abort = 1;
    atomicOr(wv.status, DEV_ERR_TIMEOUT);
  }
  ph ^= 1u << b;
}

__device__ __forceinline__ void tc_split_store(float* hi, float* lo, int off, float4 x)
{
  float4 h, l;
  tf32_split(x.x, h.x, l.x);
  tf32_split(x.y, h.y, l.y);
  tf32_split(x.z, h.z, l.z);
  tf32_split(x.w, h.w, l.w);
  *reinterpret_cast<float4*>(hi + off) = h;
  *reinterpret_cast<float4*>(lo + off) = l;
}

// `smem`: at least tc_flush_smem_bytes(k) of dynamic shared memory when the
// walker view has no cached Binv (the tiles then start there).
// Out of line: the sweep calls the flush from four places, and one shared
// copy instead of four inlined ones leaves the move code fewer spills (the
// sweep measured 187 ms instead of 201 at NiO-128, 512 walkers).
// The layout for delay ranks up to KDM (64; the delay-32 form below is the
// same algorithm with its constants, kept apart because the move code ran
// 2% slower with a shared template).
template <int KDM>
static __device__ __noinline__ void flush_tc_body(const WV<float>& wv, MoveSmem& m, int s, float* smem)
{
  // the delayed rows' electrons, in the block-reduction scratch (free during
  // a flush): static shared memory here would count against every CTA of
  // the sweep, which sits at four walkers per SM with 128 bytes to spare
  int* dls = reinterpret_cast<int*>(m.red);
  static_assert(sizeof(MoveSmem::red) >= TC_KD * sizeof(int), "dls does not fit");
  const int tid = threadIdx.x, NT = blockDim.x, warp = tid >> 5, lane = tid & 31;
  const int dc = wv.dcount[s];
  __syncthreads();
  if (dc == 0 || m.tc_abort)
    return;
  phase_mark(m, PH_DET_ACCEPT);
  const int npad = wv.npad, n = wv.n, k = wv.k;
  const int Kd = tc_kd(dc);
  constexpr int STG1 = tc_stage1(KDM);
  constexpr int RB   = KDM * TC_BK1 / 4 > 128 ? 2 : 1; // float4 of a B chunk per thread (NT >= 128)
  const double* B = wv.binv(s);
  const float* U  = wv.u(s);
  const float* V  = wv.v(s);
  float* A        = wv.ainv(s);
  const int* dl   = wv.dl(s);
  float* img      = wv.tci;
  if (tid < KDM)
    dls[tid] = tid < dc ? dl[tid] : -1;

  // ---- image of U2^T = (Binv V)^T: tile t = rows 32t..32t+31 (columns of
  // U2), [hi (32 x Kd)][lo (32 x Kd)], FP64 accumulation over the delays ----
  for (int j = tid; j < npad; j += NT)
  {
    float* hi     = img + (size_t)(j >> 5) * 2 * 32 * Kd;
    float* lo     = hi + 32 * Kd;
    const int row = j & 31;
    for (int d0 = 0; d0 < Kd; d0 += 8)
    {
      double acc[8];
#pragma unroll
      for (int b = 0; b < 8; ++b)
        acc[b] = 0.0;
      if (d0 < dc)
        for (int e = 0; e < dc; ++e)
        {
          const double ve = (double)V[(size_t)e * npad + j];
#pragma unroll
          for (int b = 0; b < 8; ++b)
            acc[b] += B[(d0 + b < dc ? d0 + b : 0) * k + e] * ve;
        }
#pragma unroll
      for (int q = 0; q < 2; ++q)
      {
        float4 x;
        float* xp = reinterpret_cast<float*>(&x);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          xp[c] = d0 + 4 * q + c < dc ? (float)acc[4 * q + c] : 0.f;
        tc_split_store(hi, lo, canon(row, d0 + 4 * q, Kd), x);
      }
    }
  }
  // the tiles overlay the cached Binv: keep the other spin's copy if cached
  double* keep = (wv.bsm && wv.bsm_spin != s) ? wv.Binv + (size_t)wv.bsm_spin * k * k : nullptr;
  __syncthreads();
  phase_mark(m, PH_FLUSH_U2);
  if (keep)
  {
    for (int i = tid; i < k * k; i += NT)
      keep[i] = wv.bsm[i];
    __syncthreads();
  }
  float* tiles = wv.bsm ? reinterpret_cast<float*>(wv.bsm) : smem;

  const uint32_t tm0  = m.tc_tmem;
  uint32_t ph         = m.tc_phase;
  const uint32_t id1  = tc_idesc_tf32(128, Kd), id2 = tc_idesc_tf32(128, TC_BN2);
  const uint32_t sbo1 = (TC_BK1 / 4) * 128, sbo2 = (uint32_t)(Kd / 4) * 128;
  const int C1 = npad / TC_BK1, T2 = npad / TC_BN2;
  constexpr int NA = 128 * TC_BK1 / 4; // float4 of an A chunk
  const int NB     = Kd * TC_BK1 / 4;  // float4 of a B chunk
  float* a2        = tiles;                // GEMM2 A: [hi 128 x Kd][lo 128 x Kd]
  float* b2        = tiles + 2 * 128 * Kd; // GEMM2 B stages: [hi 32 x Kd][lo 32 x Kd] x 2

  for (int m0 = 0; m0 < n && !m.tc_abort; m0 += 128)
  {
    // ------------------------------- GEMM1: TMEM[0:Kd) = Ainv[m0:m0+128, :] U^T
    float4 ra[4], rb[RB];
    auto load1 = [&](int c) {
      const int k0 = c * TC_BK1;
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
        const int idx = u * NT + tid, row = m0 + (idx >> 2);
        ra[u] = (idx < NA && row < n) ? *reinterpret_cast<const float4*>(A + (size_t)row * npad + k0 + 4 * (idx & 3))
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < RB; ++u)
      {
        const int idx = u * NT + tid, d = idx >> 2; // NB <= RB NT
        rb[u] = (idx < NB && d < dc) ? *reinterpret_cast<const float4*>(U + (size_t)d * npad + k0 + 4 * (idx & 3))
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
      }
    };
    load1(0);
    for (int c = 0; c < C1; ++c)
    {
      const int st = c & 1;
      float* S     = tiles + st * STG1; // [A hi][A lo][B hi][B lo]
      if (c >= 2)
        tc_wait(m, st, ph, wv); // the MMAs of chunk c-2 have read this stage
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
        const int idx = u * NT + tid;
        if (idx < NA)
          tc_split_store(S, S + 128 * TC_BK1, canon(idx >> 2, 4 * (idx & 3), TC_BK1), ra[u]);
      }
#pragma unroll
      for (int u = 0; u < RB; ++u)
      {
        const int idx = u * NT + tid;
        if (idx < NB)
          tc_split_store(S + 2 * 128 * TC_BK1, S + 2 * 128 * TC_BK1 + KDM * TC_BK1,
                         canon(idx >> 2, 4 * (idx & 3), TC_BK1), rb[u]);
      }
      if (c + 1 < C1)
        load1(c + 1);
      fence_async_smem();
      __syncthreads();
      if (m.tc_abort)
        break;
      if (tid == 0)
      {
        tc_fence_after();
#pragma unroll
        for (int ks = 0; ks < TC_BK1 / 8; ++ks)
        {
          const uint64_t ah = tc_desc(S + ks * 64, 128, sbo1);
          const uint64_t al = tc_desc(S + 128 * TC_BK1 + ks * 64, 128, sbo1);
          const uint64_t bh = tc_desc(S + 2 * 128 * TC_BK1 + ks * 64, 128, sbo1);
          const uint64_t bl = tc_desc(S + 2 * 128 * TC_BK1 + KDM * TC_BK1 + ks * 64, 128, sbo1);
          tc_mma_tf32(tm0, al, bh, id1, (c > 0 || ks > 0) ? 1u : 0u);
          tc_mma_tf32(tm0, ah, bl, id1, 1u);
          tc_mma_tf32(tm0, ah, bh, id1, 1u);
        }
        tc_commit(&m.tc_bar[st]);
      }
    }
    if (m.tc_abort)
      break;
    for (int c = C1 >= 2 ? C1 - 2 : 0; c < C1; ++c)
      tc_wait(m, c & 1, ph, wv);
    __syncthreads();
    if (m.tc_abort)
      break;
    tc_fence_after();
    phase_mark(m, PH_FLUSH_G1);

    // ------------------------- tm = TMEM - E, split into the GEMM2 A operand
    if (warp < 4)
    {
      const int r = 32 * warp + lane, row = m0 + r;
      for (int h = 0; h < Kd; h += 16)
      {
        float v[16];
        tc_ld16(tm0 + ((uint32_t)(32 * warp) << 16) + (uint32_t)h, v);
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
          float4 x;
          float* xp = reinterpret_cast<float*>(&x);
#pragma unroll
          for (int c = 0; c < 4; ++c)
            xp[c] = v[4 * q + c] - (dls[h + 4 * q + c] == row ? 1.f : 0.f);
          tc_split_store(a2, a2 + 128 * Kd, canon(r, h + 4 * q, Kd), x);
        }
      }
    }
    tc_fence_before();

    // ------------------------------------------ GEMM2 and the Ainv update
    // B tile t (U2^T hi/lo, 8 KB of the per-walker image) into stage st:
    // 16-byte cp.async copies, no registers held while they land
    auto load2 = [&](int t, int st) {
      const uint4* src = reinterpret_cast<const uint4*>(img + (size_t)t * 2 * 32 * Kd);
      uint4* dst       = reinterpret_cast<uint4*>(b2 + st * 2 * TC_BN2 * Kd);
      for (int i = tid; i < 2 * TC_BN2 * Kd / 4; i += NT)
        tc_cp_async16(dst + i, src + i);
      tc_cp_async_commit();
    };
    auto mma2 = [&](int t) {
      float* Bs = b2 + (t & 1) * 2 * TC_BN2 * Kd;
      tc_fence_after();
      for (int ks = 0; ks < Kd / 8; ++ks)
      {
        const uint64_t ah = tc_desc(a2 + ks * 64, 128, sbo2);
        const uint64_t al = tc_desc(a2 + 128 * Kd + ks * 64, 128, sbo2);
        const uint64_t bh = tc_desc(Bs + ks * 64, 128, sbo2);
        const uint64_t bl = tc_desc(Bs + TC_BN2 * Kd + ks * 64, 128, sbo2);
        const uint32_t d  = tm0 + (uint32_t)(TC_BN2 * (t & 1));
        tc_mma_tf32(d, al, bh, id2, ks > 0 ? 1u : 0u);
        tc_mma_tf32(d, ah, bl, id2, 1u);
        tc_mma_tf32(d, ah, bh, id2, 1u);
      }
      tc_commit(&m.tc_bar[2 + (t & 1)]);
    };
    // Per column block t: the MMAs of block t+1 are issued first, then those
    // of block t are waited for, block t+2's B tile starts into the stage
    // they have just released, and the Ainv update of block t runs while
    // block t+1 multiplies.  B tiles are thus copied two blocks ahead.
    load2(0, 0);
    if (T2 > 1)
      load2(1, 1);
    for (int t = 0; t < T2; ++t)
    {
      tc_cp_async_wait_all(); // this thread's copies of block t+1's tile (and block 0's)
      fence_async_smem();
      __syncthreads();
      if (m.tc_abort)
        break;
      if (tid == 0)
      {
        if (t == 0)
          mma2(0);
        if (t + 1 < T2)
          mma2(t + 1);
      }
      tc_wait(m, 2 + (t & 1), ph, wv);
      tc_fence_after();
      if (t + 2 < T2)
        load2(t + 2, t & 1); // its stage was read by the MMAs of block t, now complete
      if (warp < 4)
      {
        const int row = m0 + 32 * warp + lane;
        float* p      = A + (size_t)row * npad + t * TC_BN2;
        for (int h = 0; h < TC_BN2; h += 16)
        {
          float v[16];
          tc_ld16(tm0 + ((uint32_t)(32 * warp) << 16) + (uint32_t)(TC_BN2 * (t & 1) + h), v);
          if (row < n)
          {
            float4 a[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
              a[q] = *reinterpret_cast<const float4*>(p + h + 4 * q);
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
              a[q].x -= v[4 * q];
              a[q].y -= v[4 * q + 1];
              a[q].z -= v[4 * q + 2];
              a[q].w -= v[4 * q + 3];
              *reinterpret_cast<float4*>(p + h + 4 * q) = a[q];
            }
          }
        }
      }
      tc_fence_before();
    }
    tc_cp_async_wait_all(); // nothing in flight if the loop was left early
    __syncthreads();
    phase_mark(m, PH_FLUSH);
  }
  if (tid == 0)
  {
    m.tc_phase   = ph;
    wv.dcount[s] = 0;
  }
  __syncthreads();
  if (keep)
  {
    for (int i = tid; i < k * k; i += NT)
      wv.bsm[i] = keep[i];
    __syncthreads();
  }
  phase_mark(m, PH_FLUSH);
}

constexpr int TC_KD32    = 32;                                   // padded delay of the 48 KB layout
constexpr int TC_STG1_32 = 2 * 128 * TC_BK1 + 2 * TC_KD32 * TC_BK1; // floats per GEMM1 stage

// `smem`: at least tc_flush_smem_bytes(k) of dynamic shared memory when the
// walker view has no cached Binv (the tiles then start there).
// Out of line: the sweep calls the flush from four places, and one shared
// copy instead of four inlined ones leaves the move code fewer spills (the
// sweep measured 187 ms instead of 201 at NiO-128, 512 walkers).
static __device__ __noinline__ void flush_tc(const WV<float>& wv, MoveSmem& m, int s, float* smem)
{
  if (wv.k > TC_KD32)
  {
    flush_tc_body<64>(wv, m, s, smem); // delay ranks 33-64: the 96 KB layout
    return;
  }
  __shared__ int dls[TC_KD32];
  const int tid = threadIdx.x, NT = blockDim.x, warp = tid >> 5, lane = tid & 31;
  const int dc = wv.dcount[s];
  __syncthreads();
  if (dc == 0 || m.tc_abort)
    return;
  phase_mark(m, PH_DET_ACCEPT);
  const int npad = wv.npad, n = wv.n, k = wv.k;
  const int Kd = dc <= 16 ? 16 : 32;
  const double* B = wv.binv(s);
  const float* U  = wv.u(s);
  const float* V  = wv.v(s);
  float* A        = wv.ainv(s);
  const int* dl   = wv.dl(s);
  float* img      = wv.tci;
  if (tid < TC_KD32)
    dls[tid] = tid < dc ? dl[tid] : -1;

  // ---- image of U2^T = (Binv V)^T: tile t = rows 32t..32t+31 (columns of
  // U2), [hi (32 x Kd)][lo (32 x Kd)], FP64 accumulation over the delays ----
  for (int j = tid; j < npad; j += NT)
  {
    float* hi     = img + (size_t)(j >> 5) * 2 * 32 * Kd;
    float* lo     = hi + 32 * Kd;
    const int row = j & 31;
    for (int d0 = 0; d0 < Kd; d0 += 8)
    {
      double acc[8];
#pragma unroll
      for (int b = 0; b < 8; ++b)
        acc[b] = 0.0;
      if (d0 < dc)
        for (int e = 0; e < dc; ++e)
        {
          const double ve = (double)V[(size_t)e * npad + j];
#pragma unroll
          for (int b = 0; b < 8; ++b)
            acc[b] += B[(d0 + b < dc ? d0 + b : 0) * k + e] * ve;
        }
#pragma unroll
      for (int q = 0; q < 2; ++q)
      {
        float4 x;
        float* xp = reinterpret_cast<float*>(&x);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          xp[c] = d0 + 4 * q + c < dc ? (float)acc[4 * q + c] : 0.f;
        tc_split_store(hi, lo, canon(row, d0 + 4 * q, Kd), x);
      }
    }
  }
  // the tiles overlay the cached Binv: keep the other spin's copy if cached
  double* keep = (wv.bsm && wv.bsm_spin != s) ? wv.Binv + (size_t)wv.bsm_spin * k * k : nullptr;
  __syncthreads();
  phase_mark(m, PH_FLUSH_U2);
  if (keep)
  {
    for (int i = tid; i < k * k; i += NT)
      keep[i] = wv.bsm[i];
    __syncthreads();
  }
  float* tiles = wv.bsm ? reinterpret_cast<float*>(wv.bsm) : smem;

  const uint32_t tm0  = m.tc_tmem;
  uint32_t ph         = m.tc_phase;
  const uint32_t id1  = tc_idesc_tf32(128, Kd), id2 = tc_idesc_tf32(128, TC_BN2);
  const uint32_t sbo1 = (TC_BK1 / 4) * 128, sbo2 = (uint32_t)(Kd / 4) * 128;
  const int C1 = npad / TC_BK1, T2 = npad / TC_BN2;
  constexpr int NA = 128 * TC_BK1 / 4; // float4 of an A chunk
  const int NB     = Kd * TC_BK1 / 4;  // float4 of a B chunk
  float* a2        = tiles;                // GEMM2 A: [hi 128 x Kd][lo 128 x Kd]
  float* b2        = tiles + 2 * 128 * Kd; // GEMM2 B stages: [hi 32 x Kd][lo 32 x Kd] x 2

  for (int m0 = 0; m0 < n && !m.tc_abort; m0 += 128)
  {
    // ------------------------------- GEMM1: TMEM[0:Kd) = Ainv[m0:m0+128, :] U^T
    float4 ra[4], rb;
    auto load1 = [&](int c) {
      const int k0 = c * TC_BK1;
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
        const int idx = u * NT + tid, row = m0 + (idx >> 2);
        ra[u] = (idx < NA && row < n) ? *reinterpret_cast<const float4*>(A + (size_t)row * npad + k0 + 4 * (idx & 3))
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
      }
      const int d = tid >> 2;
      rb = (tid < NB && d < dc) ? *reinterpret_cast<const float4*>(U + (size_t)d * npad + k0 + 4 * (tid & 3))
                                : make_float4(0.f, 0.f, 0.f, 0.f);
    };
    load1(0);
    for (int c = 0; c < C1; ++c)
    {
      const int st = c & 1;
      float* S     = tiles + st * TC_STG1_32; // [A hi][A lo][B hi][B lo]
      if (c >= 2)
        tc_wait(m, st, ph, wv); // the MMAs of chunk c-2 have read this stage
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
        const int idx = u * NT + tid;
        if (idx < NA)
          tc_split_store(S, S + 128 * TC_BK1, canon(idx >> 2, 4 * (idx & 3), TC_BK1), ra[u]);
      }
      if (tid < NB)
        tc_split_store(S + 2 * 128 * TC_BK1, S + 2 * 128 * TC_BK1 + TC_KD32 * TC_BK1,
                       canon(tid >> 2, 4 * (tid & 3), TC_BK1), rb);
      if (c + 1 < C1)
        load1(c + 1);
      fence_async_smem();
      __syncthreads();
      if (m.tc_abort)
        break;
      if (tid == 0)
      {
        tc_fence_after();
#pragma unroll
        for (int ks = 0; ks < TC_BK1 / 8; ++ks)
        {
          const uint64_t ah = tc_desc(S + ks * 64, 128, sbo1);
          const uint64_t al = tc_desc(S + 128 * TC_BK1 + ks * 64, 128, sbo1);
          const uint64_t bh = tc_desc(S + 2 * 128 * TC_BK1 + ks * 64, 128, sbo1);
          const uint64_t bl = tc_desc(S + 2 * 128 * TC_BK1 + TC_KD32 * TC_BK1 + ks * 64, 128, sbo1);
          tc_mma_tf32(tm0, al, bh, id1, (c > 0 || ks > 0) ? 1u : 0u);
          tc_mma_tf32(tm0, ah, bl, id1, 1u);
          tc_mma_tf32(tm0, ah, bh, id1, 1u);
        }
        tc_commit(&m.tc_bar[st]);
      }
    }
    if (m.tc_abort)
      break;
    for (int c = C1 >= 2 ? C1 - 2 : 0; c < C1; ++c)
      tc_wait(m, c & 1, ph, wv);
    __syncthreads();
    if (m.tc_abort)
      break;
    tc_fence_after();
    phase_mark(m, PH_FLUSH_G1);

    // ------------------------- tm = TMEM - E, split into the GEMM2 A operand
    if (warp < 4)
    {
      const int r = 32 * warp + lane, row = m0 + r;
      for (int h = 0; h < Kd; h += 16)
      {
        float v[16];
        tc_ld16(tm0 + ((uint32_t)(32 * warp) << 16) + (uint32_t)h, v);
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
          float4 x;
          float* xp = reinterpret_cast<float*>(&x);
#pragma unroll
          for (int c = 0; c < 4; ++c)
            xp[c] = v[4 * q + c] - (dls[h + 4 * q + c] == row ? 1.f : 0.f);
          tc_split_store(a2, a2 + 128 * Kd, canon(r, h + 4 * q, Kd), x);
        }
      }
    }
    tc_fence_before();

    // ------------------------------------------ GEMM2 and the Ainv update
    // B tile t (U2^T hi/lo, 8 KB of the per-walker image) into stage st:
    // 16-byte cp.async copies, no registers held while they land
    auto load2 = [&](int t, int st) {
      const uint4* src = reinterpret_cast<const uint4*>(img + (size_t)t * 2 * 32 * Kd);
      uint4* dst       = reinterpret_cast<uint4*>(b2 + st * 2 * TC_BN2 * Kd);
      for (int i = tid; i < 2 * TC_BN2 * Kd / 4; i += NT)
        tc_cp_async16(dst + i, src + i);
      tc_cp_async_commit();
    };
    auto mma2 = [&](int t) {
      float* Bs = b2 + (t & 1) * 2 * TC_BN2 * Kd;
      tc_fence_after();
      for (int ks = 0; ks < Kd / 8; ++ks)
      {
        const uint64_t ah = tc_desc(a2 + ks * 64, 128, sbo2);
        const uint64_t al = tc_desc(a2 + 128 * Kd + ks * 64, 128, sbo2);
        const uint64_t bh = tc_desc(Bs + ks * 64, 128, sbo2);
        const uint64_t bl = tc_desc(Bs + TC_BN2 * Kd + ks * 64, 128, sbo2);
        const uint32_t d  = tm0 + (uint32_t)(TC_BN2 * (t & 1));
        tc_mma_tf32(d, al, bh, id2, ks > 0 ? 1u : 0u);
        tc_mma_tf32(d, ah, bl, id2, 1u);
        tc_mma_tf32(d, ah, bh, id2, 1u);
      }
      tc_commit(&m.tc_bar[2 + (t & 1)]);
    };
    // Per column block t: the MMAs of block t+1 are issued first, then those
    // of block t are waited for, block t+2's B tile starts into the stage
    // they have just released, and the Ainv update of block t runs while
    // block t+1 multiplies.  B tiles are thus copied two blocks ahead.
    load2(0, 0);
    if (T2 > 1)
      load2(1, 1);
    for (int t = 0; t < T2; ++t)
    {
      tc_cp_async_wait_all(); // this thread's copies of block t+1's tile (and block 0's)
      fence_async_smem();
      __syncthreads();
      if (m.tc_abort)
        break;
      if (tid == 0)
      {
        if (t == 0)
          mma2(0);
        if (t + 1 < T2)
          mma2(t + 1);
      }
      tc_wait(m, 2 + (t & 1), ph, wv);
      tc_fence_after();
      if (t + 2 < T2)
        load2(t + 2, t & 1); // its stage was read by the MMAs of block t, now complete
      if (warp < 4)
      {
        const int row = m0 + 32 * warp + lane;
        float* p      = A + (size_t)row * npad + t * TC_BN2;
        for (int h = 0; h < TC_BN2; h += 16)
        {
          float v[16];
          tc_ld16(tm0 + ((uint32_t)(32 * warp) << 16) + (uint32_t)(TC_BN2 * (t & 1) + h), v);
          if (row < n)
          {
            float4 a[4];
#pragma unroll
            for (int q = 0; q < 4; ++q)
              a[q] = *reinterpret_cast<const float4*>(p + h + 4 * q);
#pragma unroll
            for (int q = 0; q < 4; ++q)
            {
              a[q].x -= v[4 * q];
              a[q].y -= v[4 * q + 1];
              a[q].z -= v[4 * q + 2];
              a[q].w -= v[4 * q + 3];
              *reinterpret_cast<float4*>(p + h + 4 * q) = a[q];
            }
          }
        }
      }
      tc_fence_before();
    }
    tc_cp_async_wait_all(); // nothing in flight if the loop was left early
    __syncthreads();
    phase_mark(m, PH_FLUSH);
  }
  if (tid == 0)
  {
    m.tc_phase   = ph;
    wv.dcount[s] = 0;
  }
  __syncthreads();
  if (keep)
  {
    for (int i = tid; i < k * k; i += NT)
      wv.bsm[i] = keep[i];
    __syncthreads();
  }
  phase_mark(m, PH_FLUSH);
}
