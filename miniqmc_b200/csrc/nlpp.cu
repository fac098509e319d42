// nlpp.cu -- non-local pseudopotential ratios (NonLocalPP, the step after
// the diffusion in miniqmc's loop).
//
// For every electron jel and every ion iat whose minimum-image distance d is
// below rmax, the wavefunction ratio psi(r') / psi(R) is evaluated at the 12
// quadrature points of a sphere rotated at random once per call:
//   QMC_NLPP_SPHERE  r' = R_jel + displ + d rot_k          (NonLocalPP::
//                    evaluate, NonLocalPP.hpp:115-134: a sphere around the ion)
//   QMC_NLPP_DRIVER  r' = R_jel + d rot_k - displ          (the miniqmc driver's
//                    makeMove, miniqmc.cpp:472-495)
// with displ the e-I displacement of DistanceTableBA (ion - electron through
// DTD_BConds with every entry flipped, ParticleBConds.h:154-217).  The ratio
// is WaveFunction::ratio (WaveFunction.cpp): the SPO values at r' dotted
// with the electron's inverse row (DiracDeterminant::ratio; no delayed rows
// are pending after completeUpdates), times exp(Vat - J1(r')),
// exp(Uat - J2(r')) and exp(Uat3 - J3(r')) (OneBodyJastrow / TwoBodyJastrow
// ratio, ThreeBodyJastrow::evaluateRatios through computeU).
//
// One CTA per walker.  Per electron the ions within rmax are gathered in
// ascending order by a warp-ballot compaction; per ion the 12 knots are
// evaluated together: every thread walks its 16-byte orbital vectors for all
// 12 stencils (det partials in registers, warp-reduced), and the J1 / J2
// pairs (ion or electron, knot) within the cutoff add into per-knot sums in
// shared memory; the J3 value of each knot is one warp's: its ions within
// the J3 cutoff by ballot, then the (ion, listed electron) triples over the
// lanes.
#include "device.cuh"
#include "host_api.hpp"

#include <cmath>
#include <random>

namespace qmc
{
constexpr int NLPP_K     = 12; // quadrature points (NonLocalPP.hpp:61)
constexpr int NLPP_MAXIN = 32; // ions within rmax of one electron

struct NlppArgs
{
  double rot[NLPP_K][3]; // rotated unit vectors of this call
  double rmax;
  int form;
  double* wsum;      // [W] sum of weight x ratio
  long long* count;  // [W] points evaluated
  double* ratios;    // walker 0: every ratio in (electron, ion, knot) order, or null
  int max_ratios;
  // the points form (WaveFunction::evaluateRatios): one CTA, walker
  // `walker`, electron `pts_iat` (>= 0) at the n_pts positions `pts`
  // ([n][3], absolute), ratios into pts_out ([n]); the ion search, wsum and
  // count are not used
  int walker;
  int pts_iat;
  int n_pts;
  const double* pts;
  double* pts_out;
};

template <typename T>
__global__ void __launch_bounds__(256, 3) nlpp_kernel(const DevSystem* __restrict__ sys, DevWalkers dw, NlppArgs a)
{
  using Vt         = typename Vec16<T>::type;
  constexpr int VW = Vec16<T>::width;
  __shared__ SysSmem<T> ss;
  __shared__ SplineSmem<T> sk[NLPP_K];
  __shared__ double vpos[NLPP_K][3];
  __shared__ double sums[4 * NLPP_K];
  __shared__ int s_n, wcnt[8], in_iat[NLPP_MAXIN];
  __shared__ double in_d[NLPP_MAXIN], in_dx[NLPP_MAXIN][3];
  __shared__ int j3_ion[8][J3_NEAR], j3_seg[8][2 * J3_NEAR + 1];
  __shared__ T j3_r[8][J3_NEAR];
  __shared__ int spin_used[2];
  // per-warp J2 candidate lists: warp w's electrons (chunks of 32, w mod nw)
  // that can be within the J2 cutoff of any of the 12 points
  extern __shared__ int cand[];
  const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = NT >> 5;
  load_sys(sys, ss);
  const bool PTS = a.pts_iat >= 0;
  const int w    = PTS ? a.walker : blockIdx.x;
  const WV<T> wv = make_wv<T>(dw, w);
  const bool DET = ss.comp & QMC_WF_DET, J1 = ss.comp & QMC_WF_J1, J2 = ss.comp & QMC_WF_J2;
  const bool J3  = ss.comp & QMC_WF_J3;
  if (tid < 2)
    spin_used[tid] = 0;
  const int N = wv.N, I = ss.n_ions, npad = wv.npad, nvec = npad / VW;
  const T* ions  = (const T*)sys->ion_soa;
  const T* coefs = (const T*)sys->coefs;
  if (DET && (wv.dcount[0] != 0 || wv.dcount[1] != 0))
  {
    if (tid == 0)
      atomicOr(wv.status, DEV_ERR_STATE); // delayed rows pending: completeUpdates first
    return;
  }
  double wsum     = 0.0;
  long long cnt   = 0;
  int n_out       = 0;
  const double wk = 1.0 / NLPP_K;
  for (int jel = PTS ? a.pts_iat : 0; jel < (PTS ? a.pts_iat + 1 : N); ++jel)
  {
    const int s = jel < ss.n_up ? 0 : 1, r = jel - (s ? ss.n_up : 0);
    const double ex = wv.R[3 * jel], ey = wv.R[3 * jel + 1], ez = wv.R[3 * jel + 2];
    // ---- ions within rmax, in ascending order
    if (tid == 0)
      s_n = 0;
    __syncthreads();
    for (int c0 = 0; c0 < (PTS ? 0 : I); c0 += NT)
    {
      const int c = c0 + tid;
      bool in     = false;
      T dx = 0, dy = 0, dz = 0, rr = 0;
      if (c < I)
      {
        dx = (ions[c] - (T)ex) * T(-1), dy = (ions[I + c] - (T)ey) * T(-1), dz = (ions[2 * I + c] - (T)ez) * T(-1);
        rr = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
        dx *= T(-1), dy *= T(-1), dz *= T(-1);
        in = rr < (T)a.rmax;
      }
      const unsigned b = __ballot_sync(0xffffffffu, in);
      if (lane == 0)
        wcnt[wid] = __popc(b);
      __syncthreads();
      int base = s_n;
      for (int q = 0; q < wid; ++q)
        base += wcnt[q];
      const int pos = base + __popc(b & ((1u << lane) - 1u));
      if (in)
      {
        if (pos < NLPP_MAXIN)
        {
          in_iat[pos]   = c;
          in_d[pos]     = (double)rr;
          in_dx[pos][0] = (double)dx, in_dx[pos][1] = (double)dy, in_dx[pos][2] = (double)dz;
        }
        else
          atomicOr(wv.status, DEV_ERR_INDEX);
      }
      __syncthreads();
      if (tid == 0)
      {
        int t = 0;
        for (int q = 0; q < nw; ++q)
          t += wcnt[q];
        s_n += t;
      }
      __syncthreads();
    }
    // the points form takes its positions in groups of 12 (the last group's
    // unused slots repeat its last point and are not reported)
    const int n_in = PTS ? (a.n_pts + NLPP_K - 1) / NLPP_K : min(s_n, NLPP_MAXIN);
    for (int li = 0; li < n_in; ++li)
    {
      // ---- the 12 virtual positions and their stencils
      if (tid < NLPP_K)
      {
        const int k = tid;
        if (PTS)
        {
          const int q = min(li * NLPP_K + k, a.n_pts - 1);
          for (int c = 0; c < 3; ++c)
            vpos[k][c] = a.pts[3 * q + c];
        }
        else
        {
          const double d  = in_d[li];
          const double sg = a.form == 0 ? 1.0 : -1.0;
          vpos[k][0]      = ex + sg * in_dx[li][0] + d * a.rot[k][0];
          vpos[k][1]      = ey + sg * in_dx[li][1] + d * a.rot[k][1];
          vpos[k][2]      = ez + sg * in_dx[li][2] + d * a.rot[k][2];
        }
        if (DET)
          spline_locate(sys, vpos[k], sk[k]);
      }
      if (tid < 4 * NLPP_K)
        sums[tid] = 0.0;
      __syncthreads();
      // ---- determinant: SPO values at the 12 points . inverse row
      if (DET)
      {
        T acc[NLPP_K];
#pragma unroll
        for (int k = 0; k < NLPP_K; ++k)
          acc[k] = T(0);
        const T* arow = wv.ainv(s) + (size_t)r * npad;
        for (int q = tid; q < nvec; q += NT)
        {
          const Vt iv = reinterpret_cast<const Vt*>(arow)[q];
#pragma unroll 1
          for (int k = 0; k < NLPP_K; ++k)
          {
            T v[VW];
            spline_eval_v<T>(coefs, sys->xs, sys->ys, sys->zs, sk[k], q * VW, v);
#pragma unroll
            for (int e = 0; e < VW; ++e)
              acc[k] += reinterpret_cast<const T*>(&iv)[e] * v[e];
          }
        }
#pragma unroll
        for (int k = 0; k < NLPP_K; ++k)
        {
          const double sk2 = warp_sum((double)acc[k]);
          if (lane == 0)
            atomicAdd(&sums[k], sk2);
        }
      }
      // ---- J1: ions within the cutoff of each point (AB row, flipped)
      if (J1)
        for (int idx = tid; idx < I * NLPP_K; idx += NT)
        {
          const int c = idx % I, k = idx / I;
          T dx = (ions[c] - (T)vpos[k][0]) * T(-1), dy = (ions[I + c] - (T)vpos[k][1]) * T(-1),
            dz = (ions[2 * I + c] - (T)vpos[k][2]) * T(-1);
          const FunctorT<T>& f = ss.j1[ion_group(ss, c)];
          if (beyond_cutoff(dx, dy, dz, ss.gb, ss.mi_scale2, f.cutoff * f.cutoff))
            continue;
          const T rr = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
          if (rr < f.cutoff)
            atomicAdd(&sums[NLPP_K + k], (double)functor_v(f, rr));
        }
      // ---- J2: the other electrons within the cutoff of each point (AA row,
      // flip at jel).  The 12 points lie at distance d from the centre C of
      // their sphere, so an electron whose every image is at least rc + d
      // from C (the exact cutoff test, widened) adds to no point: each warp
      // lists its remaining electrons once, then all lanes work through
      // (candidate, point) pairs.
      if (J2)
      {
        const int gi = jel < ss.n_up ? 0 : 1;
        // the sphere's centre and radius; for the points form the first
        // point and the largest distance of the others from it
        double gc[3], grad = 0.0;
        if (PTS)
        {
          for (int c = 0; c < 3; ++c)
            gc[c] = vpos[0][c];
          for (int k = 1; k < NLPP_K; ++k)
          {
            const double qx = vpos[k][0] - gc[0], qy = vpos[k][1] - gc[1], qz = vpos[k][2] - gc[2];
            grad = fmax(grad, sqrt(qx * qx + qy * qy + qz * qz));
          }
          grad *= 1.0 + 1e-6; // covers the rounding of the test below
        }
        else
        {
          const double sg = a.form == 0 ? 1.0 : -1.0;
          for (int c = 0; c < 3; ++c)
            gc[c] = (c == 0 ? ex : c == 1 ? ey : ez) + sg * in_dx[li][c];
          grad = in_d[li];
        }
        const T cx = (T)gc[0], cy = (T)gc[1], cz = (T)gc[2];
        const T reach  = (T)grad + (ss.j2uu.cutoff > ss.j2ud.cutoff ? ss.j2uu.cutoff : ss.j2ud.cutoff);
        const int per  = ((((N + 31) >> 5) + nw - 1) / nw) << 5;
        int* lst       = cand + wid * per;
        int cnt        = 0;
        const unsigned below = (1u << lane) - 1u;
        for (int c0 = wid; (c0 << 5) < N; c0 += nw)
        {
          const int j = (c0 << 5) + lane;
          bool in     = false;
          if (j < N && j != jel)
            in = !beyond_cutoff(wv.Rs[j] - cx, wv.Rs[wv.Npad + j] - cy, wv.Rs[2 * wv.Npad + j] - cz, ss.gb,
                                ss.mi_scale2, reach * reach);
          const unsigned b = __ballot_sync(0xffffffffu, in);
          if (in)
            lst[cnt + __popc(b & below)] = j;
          cnt += __popc(b);
        }
        __syncwarp();
        for (int idx = lane; idx < cnt * NLPP_K; idx += 32)
        {
          const int j = lst[idx % cnt], k = idx / cnt;
          const T flip = j < jel ? T(1) : T(-1);
          T dx = (wv.Rs[j] - (T)vpos[k][0]) * flip, dy = (wv.Rs[wv.Npad + j] - (T)vpos[k][1]) * flip,
            dz = (wv.Rs[2 * wv.Npad + j] - (T)vpos[k][2]) * flip;
          const FunctorT<T>& f = (gi == (j < ss.n_up ? 0 : 1)) ? ss.j2uu : ss.j2ud;
          if (beyond_cutoff(dx, dy, dz, ss.gb, ss.mi_scale2, f.cutoff * f.cutoff))
            continue;
          const T rr = min_image(dx, dy, dz, ss.rb, ss.gb, ss.cn);
          if (rr < f.cutoff)
            atomicAdd(&sums[2 * NLPP_K + k], (double)functor_v(f, rr));
        }
      }
      // ---- J3: warp per point
      if (J3)
      {
        const unsigned below = (1u << lane) - 1u;
        const T* gam         = (const T*)sys->j3_gamma;
        const int jg         = jel < ss.n_up ? 0 : 1;
        for (int k = wid; k < NLPP_K; k += nw)
        {
          const T px = (T)vpos[k][0], py = (T)vpos[k][1], pz = (T)vpos[k][2];
          int nn     = 0;
          for (int c0 = 0; c0 < I; c0 += 32)
          {
            const int c = c0 + lane;
            bool in     = false;
            T rr        = 0;
            if (c < I)
            {
              const T cut = ss.j3cut[ion_group(ss, c)];
              T dx, dy, dz;
              rr = j3_ion_dist(ss, ions, c, px, py, pz, cut, dx, dy, dz);
              in = rr < cut;
            }
            const unsigned b = __ballot_sync(0xffffffffu, in);
            const int at     = nn + __popc(b & below);
            if (in)
            {
              if (at < J3_NEAR)
                j3_ion[wid][at] = c, j3_r[wid][at] = rr;
              else
                atomicOr(wv.status, DEV_ERR_CAPACITY);
            }
            nn += __popc(b);
          }
          nn           = nn < J3_NEAR ? nn : J3_NEAR;
          const int ns = 2 * nn;
          __syncwarp();
          for (int q = lane; q < ns; q += 32)
            j3_seg[wid][q + 1] = wv.j3cnt[(q / nn) * I + j3_ion[wid][q % nn]];
          __syncwarp();
          if (lane == 0)
          {
            j3_seg[wid][0] = 0;
            for (int q = 1; q <= ns; ++q)
              j3_seg[wid][q] += j3_seg[wid][q - 1];
          }
          __syncwarp();
          const int P = j3_seg[wid][ns];
          double u    = 0.0;
          for (int p = lane; p < P; p += 32)
          {
            int q = 0;
            while (j3_seg[wid][q + 1] <= p)
              ++q;
            const int kg = q / nn, slot = q % nn, ion = j3_ion[wid][slot];
            const int k2 = wv.j3list[((size_t)kg * I + ion) * wv.j3cap + (p - j3_seg[wid][q])];
            if (k2 == jel)
              continue;
            const T kx = wv.Rs[k2], ky = wv.Rs[wv.Npad + k2], kz = wv.Rs[2 * wv.Npad + k2];
            T ix = (ions[ion] - kx) * T(-1), iy = (ions[I + ion] - ky) * T(-1), iz = (ions[2 * I + ion] - kz) * T(-1);
            const T rkI  = min_image(ix, iy, iz, ss.rb, ss.gb, ss.cn);
            const T flip = k2 < jel ? T(1) : T(-1);
            T ex = (kx - px) * flip, ey = (ky - py) * flip, ez = (kz - pz) * flip;
            const T rjk = min_image(ex, ey, ez, ss.rb, ss.gb, ss.cn);
            const int ig = ion_group(ss, ion);
            u += (double)j3_v(gam + (size_t)(2 * ig + (jg == kg ? 0 : 1)) * 64, ss.j3cut[ig], rjk,
                              j3_r[wid][slot], rkI);
          }
          u = warp_sum(u);
          if (lane == 0)
            sums[3 * NLPP_K + k] = u;
          __syncwarp(); // this warp's near-ion arrays are rewritten for its next point
        }
      }
      __syncthreads();
      if (tid == 0)
      {
        spin_used[s] = 1;
        const double vat = J1 ? (double)wv.Vat[jel] : 0.0, uat = J2 ? (double)wv.Uat[jel] : 0.0;
        const double u3  = J3 ? (double)wv.j3Uat[jel] : 0.0;
        for (int k = 0; k < NLPP_K; ++k)
        {
          double ratio = DET ? sums[k] : 1.0;
          if (J1)
            ratio *= exp(vat - sums[NLPP_K + k]);
          if (J2)
            ratio *= exp(uat - sums[2 * NLPP_K + k]);
          if (J3)
            ratio *= exp(u3 - sums[3 * NLPP_K + k]);
          wsum += wk * ratio;
          ++cnt;
          if (PTS)
          {
            if (li * NLPP_K + k < a.n_pts)
              a.pts_out[li * NLPP_K + k] = ratio;
          }
          else if (w == 0 && a.ratios && n_out < a.max_ratios)
            a.ratios[n_out++] = ratio;
        }
      }
      __syncthreads();
    }
  }
  // DiracDeterminant::evaluateRatios leaves the update mode as it was
  // (DiracDeterminant.cpp:216-224)
  if (PTS)
    return;
  if (tid == 0)
  {
    a.wsum[w]  = wsum;
    a.count[w] = cnt;
    // DiracDeterminant::ratio leaves a determinant it evaluated in the
    // ratio-only update mode (its next evaluateGL re-evaluates dpsiM)
    for (int q = 0; q < 2; ++q)
      if (DET && spin_used[q])
        wv.ms->partial[q] = 0;
  }
}

cudaError_t launch_nlpp(bool fp32, const DevSystem* sys, const DevWalkers& dw, const NlppArgs& a, int threads,
                        cudaStream_t st)
{
  // the per-warp J2 candidate lists: up to ceil(chunks / warps) chunks of 32
  // electrons per warp
  const int nw = threads / 32, per = ((((dw.N + 31) / 32) + nw - 1) / nw) * 32;
  const size_t bytes = (size_t)nw * per * sizeof(int);
  if (fp32)
  {
    cudaFuncSetAttribute(nlpp_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    nlpp_kernel<float><<<a.pts_iat >= 0 ? 1 : dw.W, threads, bytes, st>>>(sys, dw, a);
  }
  else
  {
    cudaFuncSetAttribute(nlpp_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    nlpp_kernel<double><<<a.pts_iat >= 0 ? 1 : dw.W, threads, bytes, st>>>(sys, dw, a);
  }
  return cudaGetLastError();
}

// NonLocalPP::randomize (NonLocalPP.hpp:98-110) on the 12-point sphere of
// NonLocalPP's constructor (:61-80), call `call` (0-based) of a stream that
// every mover seeds with 11 (:58, StdRandom::init): three uniforms per call
void nlpp_sphere(int call, double out[NLPP_K][3])
{
  static const double g[NLPP_K][3] = {
      {1.0, 0.0, 0.0},
      {-1.0, 0.0, 0.0},
      {0.4472135955, 0.894427191, 0.0},
      {-0.4472135955, 0.7236067977, 0.5257311121},
      {0.4472135955, 0.2763932023, 0.8506508084},
      {-0.4472135955, -0.2763932023, 0.8506508084},
      {0.4472135955, -0.7236067977, 0.5257311121},
      {-0.4472135955, -0.894427191, 0.0},
      {0.4472135955, -0.7236067977, -0.5257311121},
      {-0.4472135955, -0.2763932023, -0.8506508084},
      {0.4472135955, 0.2763932023, -0.8506508084},
      {-0.4472135955, 0.7236067977, -0.5257311121}};
  std::mt19937 gen(11u);
  std::uniform_real_distribution<double> uni(0.0, 1.0);
  double u[3] = {0, 0, 0};
  for (int c = 0; c <= call; ++c)
    for (int i = 0; i < 3; ++i)
      u[i] = uni(gen);
  const double twopi = 2 * M_PI;
  const double phi = twopi * u[0], psi = twopi * u[1], cth = u[2] - 0.5;
  const double sph = std::sin(phi), cph = std::cos(phi), sth = std::sqrt(1.0 - cth * cth), sps = std::sin(psi),
               cps = std::cos(psi);
  const double m[9] = {cph * cth * cps - sph * sps,  sph * cth * cps + cph * sps,  -sth * cps,
                       -cph * cth * sps - sph * cps, -sph * cth * sps + cph * cps, sth * sps,
                       cph * sth,                    sph * sth,                    cth};
  for (int k = 0; k < NLPP_K; ++k)
    for (int i = 0; i < 3; ++i)
      out[k][i] = m[3 * i] * g[k][0] + m[3 * i + 1] * g[k][1] + m[3 * i + 2] * g[k][2];
}

} // namespace qmc

using namespace qmc;

extern "C" {

int qmc_nlpp_sphere(int n_calls, double* out)
{
  if (n_calls < 1 || !out)
    return fail(QMC_ERR_ARG, "bad arguments");
  for (int c = 0; c < n_calls; ++c)
    nlpp_sphere(c, reinterpret_cast<double(*)[3]>(out + (size_t)c * NLPP_K * 3));
  return QMC_OK;
}

int qmc_nlpp_evaluate(qmc_walkers* w, double rmax, int form, int64_t* n_points, double* wsum, double* ratios,
                      int max_ratios)
{
  if (!w || rmax <= 0 || (form != QMC_NLPP_SPHERE && form != QMC_NLPP_DRIVER) || (ratios && max_ratios < 0))
    return fail(QMC_ERR_ARG, "bad NLPP arguments");
  const size_t W = w->dw.W;
  NlppArgs a{};
  a.pts_iat = -1;
  nlpp_sphere((int)w->nlpp_calls, a.rot);
  a.rmax       = rmax;
  a.form       = form;
  a.max_ratios = ratios ? max_ratios : 0;
  double* d_w  = nullptr;
  CK(cudaMallocAsync(&d_w, W * (sizeof(double) + sizeof(long long)) + (size_t)a.max_ratios * sizeof(double) + 8,
                     w->stream));
  a.wsum   = d_w;
  a.count  = reinterpret_cast<long long*>(d_w + W);
  a.ratios = a.max_ratios ? d_w + 2 * W : nullptr;
  int threads = std::max(64, std::min(256, w->threads));
  CK(launch_nlpp(w->fp32, w->sys->d, w->dw, a, threads, w->stream));
  w->launches++;
  w->nlpp_calls++;
  w->ratio_moves = true; // the determinants it evaluated are in ratio-only mode
  std::vector<double> hw(W);
  std::vector<long long> hc(W);
  CK(cudaMemcpyAsync(hw.data(), a.wsum, W * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaMemcpyAsync(hc.data(), a.count, W * sizeof(long long), cudaMemcpyDeviceToHost, w->stream));
  if (a.max_ratios)
    CK(cudaMemcpyAsync(ratios, a.ratios, (size_t)a.max_ratios * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaFreeAsync(d_w, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  for (size_t i = 0; i < W; ++i)
  {
    if (wsum)
      wsum[i] = hw[i];
    if (n_points)
      n_points[i] = hc[i];
  }
  return device_status(w);
}

int qmc_wf_evaluate_ratios(qmc_walkers* w, int walker, int iat, int n_pos, const double* pos, double* ratios)
{
  if (!w || walker < 0 || walker >= w->dw.W || iat < 0 || iat >= w->dw.N || n_pos < 0 || (n_pos && (!pos || !ratios)))
    return fail(QMC_ERR_ARG, "bad evaluateRatios arguments");
  if (n_pos == 0)
    return QMC_OK;
  NlppArgs a{};
  a.walker   = walker;
  a.pts_iat  = iat;
  a.n_pts    = n_pos;
  double* d  = nullptr;
  CK(cudaMallocAsync(&d, (size_t)n_pos * 4 * sizeof(double), w->stream));
  CK(cudaMemcpyAsync(d, pos, (size_t)n_pos * 3 * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  a.pts     = d;
  a.pts_out = d + (size_t)n_pos * 3;
  int threads = std::max(64, std::min(256, w->threads));
  CK(launch_nlpp(w->fp32, w->sys->d, w->dw, a, threads, w->stream));
  w->launches++;
  CK(cudaMemcpyAsync(ratios, a.pts_out, (size_t)n_pos * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CK(cudaFreeAsync(d, w->stream));
  CK(cudaStreamSynchronize(w->stream));
  return device_status(w);
}

} // extern "C"
