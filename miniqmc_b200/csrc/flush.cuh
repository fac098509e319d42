// flush.cuh -- the Woodbury flush of the delayed update, per walker in its CTA.
//
// DelayedUpdate::updateInvMat (DelayedUpdate.h:155-231) in row-major terms:
//   U2 = Binv V                     (dc x n)
//   tm = Ainv U^T - E               (n x dc), E[i][d] = [i == delay_list[d]]
//   Ainv <- Ainv - tm U2            (n x n, rank-dc update)
// Binv is staged in shared memory (FP64); tm and U2 live in per-walker
// scratch (L2-resident); both GEMMs are register-tiled SIMT loops with 4x4
// outputs per thread over shared-memory tiles.  Tile loads are issued in
// batches of 16-byte vectors so that several loads per thread are in flight.
// Included by device.cuh inside namespace qmc.
#pragma once

template <typename T> struct FlushCfg
{
  static constexpr int BK = sizeof(T) == 4 ? 32 : 16; // K chunk of tm = Ainv U^T
  static constexpr int KC = sizeof(T) == 4 ? 32 : 16; // K chunk of Ainv -= tm U2
  static constexpr int BN = 64;                       // output columns per tile
};

// dynamic shared memory the flush needs for a block of `threads` threads
template <typename T> __host__ __device__ constexpr size_t flush_smem_bytes_for(int threads, int kmax)
{
  const size_t bm1 = (size_t)(threads / 8) * 4;  // rows per tm tile
  const size_t bm2 = (size_t)(threads / 16) * 4; // rows per update tile
  const size_t a   = sizeof(T) * ((size_t)FlushCfg<T>::BK * (bm1 + 1) + (size_t)FlushCfg<T>::BK * 36);
  const size_t b   = sizeof(T) * ((size_t)FlushCfg<T>::KC * (bm2 + 1) + (size_t)FlushCfg<T>::KC * (FlushCfg<T>::BN + 4));
  const size_t c   = sizeof(double) * (size_t)kmax * kmax;
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}
template <typename T> __host__ __device__ constexpr size_t flush_smem_bytes()
{
  return flush_smem_bytes_for<T>(256, 64);
}
// shared-memory bytes of the active spin's k x k Binv in the fused sweep
__host__ __device__ constexpr size_t bsm_bytes(int k)
{
  return ((size_t)k * k * sizeof(double) + 15) / 16 * 16;
}

#include "flush_tc.cuh"

template <typename T> __device__ void flush(const WV<T>& wv, MoveSmem& m, int s, T* smem)
{
  if constexpr (sizeof(T) == 4)
    if (m.tc_on)
    {
      flush_tc(wv, m, s, smem);
      return;
    }
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  constexpr int BK = FlushCfg<T>::BK, KC = FlushCfg<T>::KC, BN = FlushCfg<T>::BN;
  const int tid = threadIdx.x, NT = blockDim.x;
  const int dc = wv.dcount[s];
  __syncthreads();
  if (dc == 0)
    return;
  phase_mark(m, PH_DET_ACCEPT);
  const int npad = wv.npad, n = wv.n, k = wv.k;
  const double* B = wv.binv(s);
  const T* U      = wv.u(s);
  const T* V      = wv.v(s);
  T* A            = wv.ainv(s);
  const int* dl   = wv.dl(s);
  T* tm           = wv.tm;
  T* U2           = wv.U2;
  Vt zero;
#pragma unroll
  for (int e = 0; e < VW; ++e)
    reinterpret_cast<T*>(&zero)[e] = T(0);

  // ---- U2 = Binv V (FP64 accumulation, Binv staged in shared memory) ----
  double* Bs = reinterpret_cast<double*>(smem);
  for (int i = tid; i < dc * dc; i += NT)
    Bs[i] = B[(i / dc) * k + (i % dc)];
  __syncthreads();
  for (int j = tid; j < npad; j += NT)
    for (int bb = 0; bb < dc; bb += 8)
    {
      double acc[8];
#pragma unroll
      for (int b = 0; b < 8; ++b)
        acc[b] = 0.0;
      int a = 0;
      for (; a + 4 <= dc; a += 4)
      {
        T va[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          va[u] = V[(size_t)(a + u) * npad + j];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int b = 0; b < 8; ++b)
            acc[b] += Bs[(bb + b < dc ? bb + b : 0) * dc + a + u] * (double)va[u];
      }
      for (; a < dc; ++a)
      {
        const double va = (double)V[(size_t)a * npad + j];
#pragma unroll
        for (int b = 0; b < 8; ++b)
          acc[b] += Bs[(bb + b < dc ? bb + b : 0) * dc + a] * va;
      }
#pragma unroll
      for (int b = 0; b < 8; ++b)
        if (bb + b < dc)
          U2[(size_t)(bb + b) * npad + j] = (T)acc[b];
    }
  __syncthreads();

  // ---- tm = Ainv U^T - E: tiles of BM1 rows x 32 delayed rows ----------
  {
    const int tx = tid & 7, ty = tid >> 3;
    const int BM1 = (NT >> 3) * 4;
    constexpr int VPR = BK / VW; // vectors per tile row
    T* As = smem;                  // [BK][BM1+1]
    T* Us = smem + BK * (BM1 + 1); // [BK][36]
    const int nva = BM1 * VPR;     // == 4 * NT
    for (int d0 = 0; d0 < dc; d0 += 32)
      for (int i0 = 0; i0 < n; i0 += BM1)
      {
        T acc[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c)
            acc[r][c] = T(0);
        for (int k0 = 0; k0 < npad; k0 += BK)
        {
          {
            Vt buf[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
            {
              const int idx = u * NT + tid, ii = idx / VPR, vv = idx % VPR, row = i0 + ii;
              buf[u] = (idx < nva && row < n)
                  ? *reinterpret_cast<const Vt*>(A + (size_t)row * npad + k0 + vv * VW)
                  : zero;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
            {
              const int idx = u * NT + tid, ii = idx / VPR, vv = idx % VPR;
              if (idx < nva)
#pragma unroll
                for (int e = 0; e < VW; ++e)
                  As[(vv * VW + e) * (BM1 + 1) + ii] = reinterpret_cast<const T*>(&buf[u])[e];
            }
          }
          for (int base = 0; base < 32 * VPR; base += 2 * NT)
          {
            Vt buf[2];
#pragma unroll
            for (int u = 0; u < 2; ++u)
            {
              const int idx = base + u * NT + tid, dd = idx / VPR, vv = idx % VPR, d = d0 + dd;
              buf[u] = (idx < 32 * VPR && d < dc)
                  ? *reinterpret_cast<const Vt*>(U + (size_t)d * npad + k0 + vv * VW)
                  : zero;
            }
#pragma unroll
            for (int u = 0; u < 2; ++u)
            {
              const int idx = base + u * NT + tid, dd = idx / VPR, vv = idx % VPR;
              if (idx < 32 * VPR)
#pragma unroll
                for (int e = 0; e < VW; ++e)
                  Us[(vv * VW + e) * 36 + dd] = reinterpret_cast<const T*>(&buf[u])[e];
            }
          }
          __syncthreads();
#pragma unroll 8
          for (int kk = 0; kk < BK; ++kk)
          {
            T a[4], u[4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
              a[r] = As[kk * (BM1 + 1) + ty * 4 + r];
#pragma unroll
            for (int c = 0; c < 4; ++c)
              u[c] = Us[kk * 36 + tx * 4 + c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
              for (int c = 0; c < 4; ++c)
                acc[r][c] += a[r] * u[c];
          }
          __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < 4; ++r)
        {
          const int row = i0 + ty * 4 + r;
#pragma unroll
          for (int c = 0; c < 4; ++c)
          {
            const int d = d0 + tx * 4 + c;
            if (row < n && d < dc)
              tm[(size_t)row * k + d] = acc[r][c] - (dl[d] == row ? T(1) : T(0));
          }
        }
      }
  }
  __syncthreads();

  // ---- Ainv -= tm U2: tiles of BM2 rows x BN columns -------------------
  {
    const int tx = tid & 15, ty = tid >> 4;
    const int BM2 = (NT >> 4) * 4;
    constexpr int VPRB = BN / VW;  // vectors per U2 tile row
    T* Ts = smem;                  // [KC][BM2+1]
    T* Vs = smem + KC * (BM2 + 1); // [KC][BN+4]
    for (int i0 = 0; i0 < n; i0 += BM2)
      for (int j0 = 0; j0 < npad; j0 += BN)
      {
        const int col = j0 + tx * 4;
        // issue the loads of this thread's 4x4 block of Ainv first
        T cur[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
        {
          const int row = i0 + ty * 4 + r;
#pragma unroll
          for (int c = 0; c < 4; ++c)
            cur[r][c] = (row < n && col < npad) ? A[(size_t)row * npad + col + c] : T(0);
        }
        T acc[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c)
            acc[r][c] = T(0);
        for (int k0 = 0; k0 < dc; k0 += KC)
        {
          const int kc = min(KC, dc - k0);
          // tm rows: BM2 x KC scalars, KC/4 per thread
          for (int base = 0; base < BM2 * KC; base += 8 * NT)
          {
            T buf[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
            {
              const int idx = base + u * NT + tid, ii = idx / KC, kk = idx % KC, row = i0 + ii;
              buf[u] = (idx < BM2 * KC && row < n && kk < kc) ? tm[(size_t)row * k + k0 + kk] : T(0);
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
            {
              const int idx = base + u * NT + tid, ii = idx / KC, kk = idx % KC;
              if (idx < BM2 * KC)
                Ts[kk * (BM2 + 1) + ii] = buf[u];
            }
          }
          for (int base = 0; base < KC * VPRB; base += 4 * NT)
          {
            Vt buf[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
            {
              const int idx = base + u * NT + tid, kk = idx / VPRB, vv = idx % VPRB, cc = j0 + vv * VW;
              buf[u] = (idx < KC * VPRB && kk < kc && cc < npad)
                  ? *reinterpret_cast<const Vt*>(U2 + (size_t)(k0 + kk) * npad + cc)
                  : zero;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
            {
              const int idx = base + u * NT + tid, kk = idx / VPRB, vv = idx % VPRB;
              if (idx < KC * VPRB)
                *reinterpret_cast<Vt*>(&Vs[kk * (BN + 4) + vv * VW]) = buf[u];
            }
          }
          __syncthreads();
#pragma unroll 8
          for (int kk = 0; kk < kc; ++kk)
          {
            T t[4], v[4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
              t[r] = Ts[kk * (BM2 + 1) + ty * 4 + r];
#pragma unroll
            for (int c = 0; c < 4; ++c)
              v[c] = Vs[kk * (BN + 4) + tx * 4 + c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
              for (int c = 0; c < 4; ++c)
                acc[r][c] += t[r] * v[c];
          }
          __syncthreads();
        }
        if (col < npad)
#pragma unroll
          for (int r = 0; r < 4; ++r)
          {
            const int row = i0 + ty * 4 + r;
            if (row < n)
            {
              T* p = A + (size_t)row * npad + col;
#pragma unroll
              for (int c = 0; c < 4; ++c)
                p[c] = cur[r][c] - acc[r][c];
            }
          }
      }
  }
  if (tid == 0)
    wv.dcount[s] = 0;
  __syncthreads();
  phase_mark(m, PH_FLUSH);
}
