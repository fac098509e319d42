// j3.cuh -- the three-body (electron-electron-ion) Jastrow on the device
// (ThreeBodyJastrow.h:30-677, PolynomialFunctor3D.h:443-560).
//
// State of a walker: Uat, dUat, d2Uat per electron and, per ion and electron
// spin, the list of the electrons within the ion's cutoff
// (ThreeBodyJastrow::elecs_inside), kept in the reference's order: appended
// when an electron enters, the last entry moved into the hole when one
// leaves.  The distances and displacements of listed electrons are
// recomputed from the positions (the same arithmetic on the same values the
// reference stores them from).
//
// A move of electron j touches the triples (j, k, I) with ion I within its
// cutoff of j and k in I's lists: a few tens in the NiO cells.  They are
// enumerated as (near ion, spin) segments in shared memory and evaluated one
// triple per thread.  acceptMove evaluates the triples of the old and the
// new position together and adds each electron k's new - old contributions
// in triple order (the first triple of k sums them), so the update is
// deterministic.
#pragma once

namespace qmc
{
constexpr int J3_NEAR = 64;  // ions within the cutoff of one position
constexpr int J3_PMAX = 1024; // triples of one acceptMove (old + new position)

// shared-memory scratch of the J3 move code (carved from the dynamic shared
// memory; side 0 = proposed position, side 1 = current position)
template <typename T> struct J3Smem
{
  T near_r[2][J3_NEAR];
  T near_d[2][3][J3_NEAR]; // ion - electron
  T pv[J3_PMAX], pl[J3_PMAX], pg[3][J3_PMAX];
  int near_ion[2][J3_NEAR];
  int seg[2][2 * J3_NEAR + 1];
  int pk[J3_PMAX];
  int n_near[2];
  int wcnt[32];
};

// value and derivatives of one PolynomialFunctor3D term set
template <typename T> struct J3Val
{
  T v, g0, g1, g2, h00, h11, h22, h01, h02;
};

// r^p, d/dr r^p, d2/dr2 r^p for p = 0..3
template <typename T> __device__ __forceinline__ void j3_powers(T r, T* p, T* p1, T* p2)
{
  p[0] = T(1), p[1] = r, p[2] = r * r, p[3] = r * r * r;
  p1[0] = T(0), p1[1] = T(1), p1[2] = T(2) * r, p1[3] = T(3) * r * r;
  p2[0] = T(0), p2[1] = T(0), p2[2] = T(2), p2[3] = T(6) * r;
}

// PolynomialFunctor3D::evaluateVGL for one triple inside both ion cutoffs
// (N_eI = N_ee = 3, C = 3): the value, the gradients along r12, r1I, r2I
// divided by those distances, the Hessian diagonal, and the (12,1I) and
// (12,2I) entries divided by the distance products.  gam = gamma[l][m][n]
// (l: r1I power, m: r2I power, n: r12 power); L = the ion cutoff.
template <typename T>
__device__ __forceinline__ J3Val<T> j3_vgl(const T* __restrict__ gam, T L, T r12, T r1I, T r2I)
{
  T pl[4], pl1[4], pl2[4], pm[4], pm1[4], pm2[4], pn[4], pn1[4], pn2[4];
  j3_powers(r1I, pl, pl1, pl2);
  j3_powers(r2I, pm, pm1, pm2);
  j3_powers(r12, pn, pn1, pn2);
  T val = 0, g0 = 0, g1 = 0, g2 = 0, h00 = 0, h11 = 0, h22 = 0, h01 = 0, h02 = 0;
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int m = 0; m < 4; ++m)
    {
      T s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
      for (int n = 0; n < 4; ++n)
      {
        const T g = __ldg(gam + 16 * l + 4 * m + n);
        s0 += g * pn[n];
        s1 += g * pn1[n];
        s2 += g * pn2[n];
      }
      const T lm = pl[l] * pm[m], l1m = pl1[l] * pm[m], lm1 = pl[l] * pm1[m];
      val += lm * s0;
      g0 += lm * s1;
      h00 += lm * s2;
      g1 += l1m * s0;
      h01 += l1m * s1;
      g2 += lm1 * s0;
      h02 += lm1 * s1;
      h11 += pl2[l] * pm[m] * s0;
      h22 += pl[l] * pm2[m] * s0;
    }
  // times ((r1I - L)(r2I - L))^C, product rule applied C times
  const T a = r2I - L, b = r1I - L, ab = a * b;
#pragma unroll
  for (int i = 0; i < 3; ++i)
  {
    h00 = ab * h00;
    h01 = ab * h01 + a * g0;
    h02 = ab * h02 + b * g0;
    h11 = ab * h11 + T(2) * a * g1;
    h22 = ab * h22 + T(2) * b * g2;
    g0  = ab * g0;
    g1  = ab * g1 + a * val;
    g2  = ab * g2 + b * val;
    val *= ab;
  }
  J3Val<T> o;
  o.v   = val;
  o.g0  = g0 / r12;
  o.g1  = g1 / r1I;
  o.g2  = g2 / r2I;
  o.h00 = h00;
  o.h11 = h11;
  o.h22 = h22;
  o.h01 = h01 / (r12 * r1I);
  o.h02 = h02 / (r12 * r2I);
  return o;
}

// PolynomialFunctor3D::evaluateV for one triple inside both ion cutoffs:
// the value only
template <typename T> __device__ __forceinline__ T j3_v(const T* __restrict__ gam, T L, T r12, T r1I, T r2I)
{
  const T pl[4] = {T(1), r1I, r1I * r1I, r1I * r1I * r1I};
  const T pm[4] = {T(1), r2I, r2I * r2I, r2I * r2I * r2I};
  const T pn[4] = {T(1), r12, r12 * r12, r12 * r12 * r12};
  T val = 0;
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int m = 0; m < 4; ++m)
    {
      T s0 = 0;
#pragma unroll
      for (int n = 0; n < 4; ++n)
        s0 += __ldg(gam + 16 * l + 4 * m + n) * pn[n];
      val += pl[l] * pm[m] * s0;
    }
  const T ab = (r2I - L) * (r1I - L);
  return val * ab * ab * ab;
}

// the minimum-image e-I distance of ion c from (px, py, pz) and the
// displacement ion - electron (DistanceTableBA, every entry flipped), or a
// value not below `cut` when every image is beyond it.  Every membership
// decision of the electron lists goes through here.
template <typename T>
__device__ __forceinline__ T j3_ion_dist(const SysSmem<T>& ss, const T* __restrict__ ions, int c, T px, T py, T pz,
                                         T cut, T& dx, T& dy, T& dz)
{
  const int I = ss.n_ions;
  dx = (ions[c] - px) * T(-1), dy = (ions[I + c] - py) * T(-1), dz = (ions[2 * I + c] - pz) * T(-1);
  if (beyond_cutoff(dx, dy, dz, ss.gb, ss.mi_scale2, cut * cut))
    return cut;
  const T r = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
  dx *= T(-1), dy *= T(-1), dz *= T(-1);
  return r;
}

// the ions within their cutoff of pos, in ascending order, into side `side`
// (ions_nearby of ThreeBodyJastrow::computeU3).  Block-wide.
template <typename T>
__device__ void j3_near(const SysSmem<T>& ss, const T* __restrict__ ions, const double* pos, J3Smem<T>& J, int side,
                        unsigned* status)
{
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = (NT + 31) >> 5;
  const int I = ss.n_ions;
  const T px = (T)pos[0], py = (T)pos[1], pz = (T)pos[2];
  int base = 0;
  for (int c0 = 0; c0 < I; c0 += NT)
  {
    const int c = c0 + tid;
    bool in     = false;
    T dx = 0, dy = 0, dz = 0, r = 0;
    if (c < I)
    {
      const T cut = ss.j3cut[ion_group(ss, c)];
      r           = j3_ion_dist(ss, ions, c, px, py, pz, cut, dx, dy, dz);
      in          = r < cut;
    }
    const unsigned b = __ballot_sync(0xffffffffu, in);
    if (lane == 0)
      J.wcnt[wid] = __popc(b);
    __syncthreads();
    int at = base, tot = 0;
    for (int q = 0; q < nw; ++q)
    {
      at += q < wid ? J.wcnt[q] : 0;
      tot += J.wcnt[q];
    }
    at += __popc(b & ((1u << lane) - 1u));
    if (in)
    {
      if (at < J3_NEAR)
      {
        J.near_ion[side][at]  = c;
        J.near_r[side][at]    = r;
        J.near_d[side][0][at] = dx;
        J.near_d[side][1][at] = dy;
        J.near_d[side][2][at] = dz;
      }
      else
        atomicOr(status, DEV_ERR_CAPACITY);
    }
    base += tot;
    __syncthreads(); // wcnt is rewritten by the next chunk
  }
  if (tid == 0)
    J.n_near[side] = base < J3_NEAR ? base : J3_NEAR;
  __syncthreads();
}

// triple offsets of side `side`: segment s = kg * n_near + slot holds the
// electrons of spin kg listed at near ion `slot`; returns the triple count.
// Block-wide.
template <typename T> __device__ int j3_segments(const WV<T>& wv, J3Smem<T>& J, int side)
{
  const int nn = J.n_near[side], ns = 2 * nn;
  for (int s = threadIdx.x; s < ns; s += blockDim.x)
  {
    const int kg = s / nn, ion = J.near_ion[side][s % nn];
    J.seg[side][s + 1] = wv.j3cnt[kg * wv.I + ion];
  }
  __syncthreads();
  if (threadIdx.x == 0)
  {
    J.seg[side][0] = 0;
    for (int s = 1; s <= ns; ++s)
      J.seg[side][s] += J.seg[side][s - 1];
  }
  __syncthreads();
  return J.seg[side][ns];
}

// the near ions of one position with their triple segments
template <typename T> struct J3Near
{
  int nn;
  const int* seg;
  const int* ion;
  const T* r;
  const T* dx;
  const T* dy;
  const T* dz;
};
template <typename T> __device__ __forceinline__ J3Near<T> j3_view(const J3Smem<T>& J, int side)
{
  return J3Near<T>{J.n_near[side], J.seg[side], J.near_ion[side], J.near_r[side], J.near_d[side][0],
                   J.near_d[side][1], J.near_d[side][2]};
}

// triple p of the near ions `nv` of electron jel at (px, py, pz): the terms of
// ThreeBodyJastrow::computeU3_engine for jel (Uj, dUj, d2Uj) and for the
// listed electron k (Uk, dUk, d2Uk).  False when k is jel itself.
template <typename T> struct J3Terms
{
  int k;
  T uj, gj[3], lj, uk, gk[3], lk;
};
template <typename T>
__device__ __forceinline__ bool j3_triple(const SysSmem<T>& ss, const T* __restrict__ gamma, const WV<T>& wv,
                                          const T* __restrict__ ions, const J3Near<T>& nv, int p, int jel, T px,
                                          T py, T pz, J3Terms<T>& o)
{
  const int nn = nv.nn;
  int s        = 0;
  while (nv.seg[s + 1] <= p)
    ++s;
  const int kg = s / nn, slot = s % nn, ion = nv.ion[slot];
  const int k  = wv.j3list[((size_t)kg * wv.I + ion) * wv.j3cap + (p - nv.seg[s])];
  o.k          = k;
  if (k == jel)
    return false;
  const int Np = wv.Npad, I = ss.n_ions;
  const T kx = wv.Rs[k], ky = wv.Rs[Np + k], kz = wv.Rs[2 * Np + k];
  // k - I: ion - R_k
  T kIx = (ions[ion] - kx) * T(-1), kIy = (ions[I + ion] - ky) * T(-1), kIz = (ions[2 * I + ion] - kz) * T(-1);
  const T rkI = min_image(kIx, kIy, kIz, ss.rb, ss.gb, ss.cn);
  kIx *= T(-1), kIy *= T(-1), kIz *= T(-1);
  // j - k: R_k - r_j with the AA table's flip (TwoBodyJastrow rows)
  const T flip = k < jel ? T(1) : T(-1);
  T jkx = (kx - px) * flip, jky = (ky - py) * flip, jkz = (kz - pz) * flip;
  const T rjk = min_image(jkx, jky, jkz, ss.rb, ss.gb, ss.cn);
  jkx *= flip, jky *= flip, jkz *= flip;
  const T rjI = nv.r[slot];
  const T jIx = nv.dx[slot], jIy = nv.dy[slot], jIz = nv.dz[slot];
  const int ig = ion_group(ss, ion), jg = jel < ss.n_up ? 0 : 1;
  const J3Val<T> f = j3_vgl(gamma + (size_t)(2 * ig + (jg == kg ? 0 : 1)) * 64, ss.j3cut[ig], rjk, rjI, rkI);
  const T jk_jI = jkx * jIx + jky * jIy + jkz * jIz;
  const T kI_jk = kIx * jkx + kIy * jky + kIz * jkz;
  o.uj    = f.v;
  o.gj[0] = f.g1 * jIx + jkx * f.g0;
  o.gj[1] = f.g1 * jIy + jky * f.g0;
  o.gj[2] = f.g1 * jIz + jkz * f.g0;
  o.lj    = -(f.h00 + f.h11 + T(2) * (f.g0 + f.g1) + T(2) * f.h01 * jk_jI);
  o.uk    = f.v;
  o.gk[0] = kIx * f.g2 - jkx * f.g0;
  o.gk[1] = kIy * f.g2 - jky * f.g0;
  o.gk[2] = kIz * f.g2 - jkz * f.g0;
  o.lk    = -(f.h00 + f.h22 + T(2) * (f.g0 + f.g2) - T(2) * f.h02 * kI_jk);
  return true;
}

// ratioGrad / ratio of electron iel at pos: adds sum Uj and sum dUj of its
// triples to part[0..3] (per-thread partials).  Block-wide.
template <typename T, typename A>
__device__ void j3_partials(const SysSmem<T>& ss, const DevSystem* __restrict__ sys, const WV<T>& wv,
                            const T* __restrict__ ions, J3Smem<T>& J, int iel, const double* pos, A* part)
{
  j3_near(ss, ions, pos, J, 0, wv.status);
  const int P   = j3_segments(wv, J, 0);
  const T* gam  = (const T*)sys->j3_gamma;
  const T px = (T)pos[0], py = (T)pos[1], pz = (T)pos[2];
  const J3Near<T> nv = j3_view(J, 0);
  for (int p = threadIdx.x; p < P; p += blockDim.x)
  {
    J3Terms<T> o;
    if (j3_triple(ss, gam, wv, ions, nv, p, iel, px, py, pz, o))
    {
      part[0] += (A)o.uj;
      part[1] += (A)o.gj[0];
      part[2] += (A)o.gj[1];
      part[3] += (A)o.gj[2];
    }
  }
}

// ThreeBodyJastrow::acceptMove of electron iel from m.pos_old to m.pos_new:
// every listed electron's Uat, dUat, d2Uat gains its new - old triple terms,
// iel's own values become those of the new position, logJ3 changes by
// Uat_old(iel) - Uat_new(iel), and iel enters or leaves the lists of the
// ions whose cutoff it crossed.  Block-wide.
template <typename T>
__device__ void j3_accept(const SysSmem<T>& ss, const DevSystem* __restrict__ sys, const WV<T>& wv, MoveSmem& m,
                          J3Smem<T>& J, const T* __restrict__ ions, int iel)
{
  const int tid = threadIdx.x, NT = blockDim.x, N = wv.N, I = ss.n_ions;
  j3_near(ss, ions, m.pos_new, J, 0, wv.status);
  j3_near(ss, ions, m.pos_old, J, 1, wv.status);
  const int P0 = j3_segments(wv, J, 0);
  const int P1 = j3_segments(wv, J, 1);
  const int P  = P0 + P1;
  if (P > J3_PMAX)
  {
    if (tid == 0)
      atomicOr(wv.status, DEV_ERR_CAPACITY);
    __syncthreads();
    return;
  }
  const T* gam = (const T*)sys->j3_gamma;
  const J3Near<T> nv[2] = {j3_view(J, 0), j3_view(J, 1)};
  double part[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0}; // new: U, dU[3], d2U; old: U
  for (int p = tid; p < P; p += NT)
  {
    const int side  = p < P0 ? 0 : 1;
    const double* q = side ? m.pos_old : m.pos_new;
    J3Terms<T> o;
    if (j3_triple(ss, gam, wv, ions, nv[side], side ? p - P0 : p, iel, (T)q[0], (T)q[1], (T)q[2], o))
    {
      if (side == 0)
      {
        part[0] += (double)o.uj;
        part[1] += (double)o.gj[0];
        part[2] += (double)o.gj[1];
        part[3] += (double)o.gj[2];
        part[4] += (double)o.lj;
      }
      else
        part[5] += (double)o.uj;
      J.pk[p]    = o.k;
      J.pv[p]    = o.uk;
      J.pl[p]    = o.lk;
      J.pg[0][p] = o.gk[0];
      J.pg[1][p] = o.gk[1];
      J.pg[2][p] = o.gk[2];
    }
    else
      J.pk[p] = -1;
  }
  block_sum<6>(part, m.red, m.sums);
  // Uat[k] += newUk[k] - oldUk[k] (ThreeBodyJastrow.h:325-333), each k by its
  // first triple
  for (int p = tid; p < P; p += NT)
  {
    const int k = J.pk[p];
    if (k < 0)
      continue;
    bool first = true;
    for (int q = 0; q < p && first; ++q)
      first = J.pk[q] != k;
    if (!first)
      continue;
    T nv = 0, nl = 0, ov = 0, ol = 0, ng[3] = {0, 0, 0}, og[3] = {0, 0, 0};
    for (int q = p; q < P; ++q)
      if (J.pk[q] == k)
      {
        if (q < P0)
        {
          nv += J.pv[q], nl += J.pl[q];
          ng[0] += J.pg[0][q], ng[1] += J.pg[1][q], ng[2] += J.pg[2][q];
        }
        else
        {
          ov += J.pv[q], ol += J.pl[q];
          og[0] += J.pg[0][q], og[1] += J.pg[1][q], og[2] += J.pg[2][q];
        }
      }
    wv.j3Uat[k] += nv - ov;
    wv.j3d2Uat[k] += nl - ol;
    wv.j3dUat[k] += ng[0] - og[0];
    wv.j3dUat[N + k] += ng[1] - og[1];
    wv.j3dUat[2 * N + k] += ng[2] - og[2];
  }
  if (tid == 0)
  {
    wv.jlog[2] += m.sums[5] - m.sums[0];
    wv.j3Uat[iel]         = (T)m.sums[0];
    wv.j3dUat[iel]        = (T)m.sums[1];
    wv.j3dUat[N + iel]    = (T)m.sums[2];
    wv.j3dUat[2 * N + iel] = (T)m.sums[3];
    wv.j3d2Uat[iel]       = (T)m.sums[4];
  }
  // list membership (ThreeBodyJastrow.h:350-388): ions near only the new
  // position gain iel, ions near only the old one lose it
  const int jg = iel < ss.n_up ? 0 : 1, n0 = J.n_near[0], n1 = J.n_near[1];
  for (int t = tid; t < n0 + n1; t += NT)
  {
    const int side = t < n0 ? 0 : 1, ion = J.near_ion[side][side ? t - n0 : t];
    const int no = side ? n0 : n1;
    bool both    = false;
    for (int q = 0; q < no && !both; ++q)
      both = J.near_ion[1 - side][q] == ion;
    if (both)
      continue;
    int* cnt = wv.j3cnt + jg * I + ion;
    int* lst = wv.j3list + ((size_t)jg * I + ion) * wv.j3cap;
    const int c = *cnt;
    if (side == 0)
    {
      if (c < wv.j3cap)
      {
        lst[c] = iel;
        *cnt   = c + 1;
      }
      else
        atomicOr(wv.status, DEV_ERR_CAPACITY);
    }
    else
      for (int q = 0; q < c; ++q)
        if (lst[q] == iel)
        {
          lst[q] = lst[c - 1];
          *cnt   = c - 1;
          break;
        }
  }
  __syncthreads();
}

} // namespace qmc
