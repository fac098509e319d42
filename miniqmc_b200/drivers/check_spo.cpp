// check_spo -- the reference's SPO checker (check_spo.cpp) on the C ABI.
//
// The reference checks its optimized einspline SPO against a plain
// implementation.  Here the SPO of the arithmetic form under test (-p,
// default mixed: the FP32 table) is checked against the FP64 table, both
// evaluated on the device at the same points: every proposed position of
// a random walk of the electrons (VGH; N normals per step, accept
// ur < 0.5), then NonLocalPP-style sphere points around each ion (values).
// Errors are sums of |difference| over the orbitals averaged per call, with
// the reference's tolerances (epsilon x 1e4, 3e6, 6e8 for V, G, H).
#include "driver_common.hpp"

#include <cstdlib>
#include <limits>
#include <string>
#include <unistd.h>

using drv::check;

namespace
{
void print_help()
{
  std::printf("usage:\n"
              "  check_spo [-hvV] [-g \"n0 n1 n2\"] [-m meshfactor]\n"
              "            [-n steps] [-r rmax] [-s seed] [-p mixed|fp64]\n"
              "options:\n"
              "  -a  size of each spline tile       default: num of orbs (ignored)\n"
              "  -c  number of members per team     default: 1 (ignored)\n"
              "  -g  set the 3D tiling.             default: 1 1 1\n"
              "  -h  print help and exit\n"
              "  -m  meshfactor                     default: 1.0\n"
              "  -n  number of MC steps             default: 5\n"
              "  -r  set the Rmax.                  default: 1.7\n"
              "  -s  set the random seed.           default: 11\n"
              "  -v  verbose output\n"
              "  -V  print version information and exit\n"
              "  -p  arithmetic form under test     default: mixed\n");
}
} // namespace

int main(int argc, char** argv)
{
  int na = 1, nb = 1, nc = 1, nsteps = 5, iseed = 11, nx = 37, ny = 37, nz = 37;
  double rmax = 1.7;
  bool fp64 = false;
  int opt;
  while (optind < argc)
  {
    if ((opt = getopt(argc, argv, "hvVa:c:f:g:m:n:r:s:p:")) != -1)
    {
      switch (opt)
      {
      case 'a':
      case 'c':
      case 'f':
      case 'v': break;
      case 'g':
        if (std::sscanf(optarg, "%d %d %d", &na, &nb, &nc) != 3)
        {
          print_help();
          return 1;
        }
        break;
      case 'h': print_help(); return 1;
      case 'm':
      {
        const double f = std::atof(optarg);
        nx = (int)(nx * f), ny = (int)(ny * f), nz = (int)(nz * f);
      }
      break;
      case 'n': nsteps = std::atoi(optarg); break;
      case 'r': rmax = std::atof(optarg); break;
      case 's': iseed = std::atoi(optarg); break;
      case 'V': std::printf("check_spo on libqmcgpu (sm_100a)\n"); return 1;
      case 'p': fp64 = std::string(optarg) == "fp64"; break;
      default: print_help(); return 1;
      }
    }
    else
    {
      std::fprintf(stderr, "Non-option arguments not allowed\n");
      print_help();
      return 1;
    }
  }
  if (nsteps < 1 || nx < 1 || ny < 1 || nz < 1)
  {
    print_help();
    return 1;
  }
  if (check(qmc_init(0), "qmc_init"))
    return 1;
  drv::NioSystem nio;
  if (nio.build(na, nb, nc, nx, ny, nz, false, iseed, QMC_WF_DET))
    return 1;
  const int nels = nio.nels, norb = nio.norb, nions = nio.n_ions;
  std::printf("Number of orbitals/splines = %d\nNumber of electrons = %d\nGrid = %d %d %d\n", norb, nels, nx, ny, nz);
  qmc_system *st_sys = nullptr, *rf_sys = nullptr;
  if (check(qmc_system_create(&nio.d, fp64 ? QMC_PREC_FP64 : QMC_PREC_MIXED, &st_sys), "qmc_system_create") ||
      check(qmc_system_create(&nio.d, QMC_PREC_FP64, &rf_sys), "qmc_system_create"))
    return 1;
  // the electrons of one mover (build_els from its stream) as the start
  qmc_walkers* w = nullptr;
  const uint32_t seed = drv::primes(1)[0];
  std::vector<double> R(3 * (size_t)nels);
  if (check(qmc_walkers_create(rf_sys, 1, 1, &w), "qmc_walkers_create") ||
      check(qmc_walkers_init_random(w, &seed), "init_random") ||
      check(qmc_walkers_get_positions(w, R.data()), "get_positions"))
    return 1;
  qmc_walkers_destroy(w);
  drv::HostRng rng(seed);
  {
    std::vector<double> skip(3 * (size_t)nels);
    rng.uniform(skip.data(), 3 * nels);
  }
  std::vector<double> ur(nels), delta(3 * (size_t)nels);
  rng.uniform(ur.data(), nels);

  std::vector<double> vt((size_t)nels * norb), vr((size_t)nels * norb), gt(3 * vt.size()), gr(3 * vt.size()),
      ht(6 * vt.size()), hr(6 * vt.size());
  double evgh_v = 0, evgh_g = 0, evgh_h = 0, ev_v = 0;
  long long nvgh = 0, nv = 0, accepted = 0;
  std::vector<double> sphere(12 * 3);
  const double zval = (double)nels / nions;
  for (int mc = 0; mc < nsteps; ++mc)
  {
    rng.normal(delta.data(), 3 * nels);
    rng.uniform(ur.data(), nels);
    // the proposed positions of the walk, electron by electron
    std::vector<double> P(3 * (size_t)nels);
    for (int iel = 0; iel < nels; ++iel)
    {
      for (int c = 0; c < 3; ++c)
        P[3 * iel + c] = R[3 * iel + c] + delta[3 * iel + c];
      if (ur[iel] < 0.5)
      {
        for (int c = 0; c < 3; ++c)
          R[3 * iel + c] = P[3 * iel + c];
        ++accepted;
      }
    }
    if (check(qmc_spo_evaluate_vgh(st_sys, nels, P.data(), vt.data(), gt.data(), ht.data()), "spo_evaluate_vgh") ||
        check(qmc_spo_evaluate_vgh(rf_sys, nels, P.data(), vr.data(), gr.data(), hr.data()), "spo_evaluate_vgh"))
      return 1;
    for (size_t i = 0; i < vt.size(); ++i)
      evgh_v += std::fabs(vt[i] - vr[i]);
    for (size_t i = 0; i < gt.size(); ++i)
      evgh_g += std::fabs(gt[i] - gr[i]);
    for (size_t i = 0; i < ht.size(); ++i)
      evgh_h += std::fabs(ht[i] - hr[i]);
    nvgh += nels;
    // sphere points around each ion (NonLocalPP's rotated knots of this step)
    rng.uniform(ur.data(), nels);
    std::vector<double> all(12 * 3 * (size_t)(mc + 1));
    if (check(qmc_nlpp_sphere(mc + 1, all.data()), "qmc_nlpp_sphere"))
      return 1;
    std::copy(all.end() - 36, all.end(), sphere.begin());
    std::vector<double> Q;
    for (int iat = 0, kat = 0; iat < nions && kat + 1 < nels; ++iat)
    {
      const int nnF  = (int)(ur[kat++] * zval);
      const double r = rmax * ur[kat++];
      for (int nn = 0; nn < nnF; ++nn)
        for (int k = 0; k < 12; ++k)
          for (int c = 0; c < 3; ++c)
            Q.push_back(nio.ion_pos[3 * iat + c] + r * sphere[3 * k + c]);
    }
    const int nq = (int)(Q.size() / 3);
    if (nq > 0)
    {
      std::vector<double> qt((size_t)nq * norb), qr((size_t)nq * norb);
      if (check(qmc_spo_evaluate_v(st_sys, nq, Q.data(), qt.data()), "spo_evaluate_v") ||
          check(qmc_spo_evaluate_v(rf_sys, nq, Q.data(), qr.data()), "spo_evaluate_v"))
        return 1;
      for (size_t i = 0; i < qt.size(); ++i)
        ev_v += std::fabs(qt[i] - qr[i]);
      nv += nq;
    }
  }
  // per call, as the reference averages (sphere moves per step)
  const double spheremoves = (double)nv / nsteps;
  ev_v /= spheremoves > 0 ? spheremoves : 1.0;
  evgh_v /= nvgh, evgh_g /= nvgh, evgh_h /= nvgh;
  const double eps = fp64 ? std::numeric_limits<double>::epsilon() : std::numeric_limits<float>::epsilon();
  const double small_v = eps * 1e4, small_g = eps * 3e6, small_h = eps * 6e8;
  std::printf("Accepted moves = %lld of %lld\nevaluate_v errors    V %g\nevaluate_vgh errors  V %g G %g H %g\n\n",
              accepted, (long long)nels * nsteps, ev_v, evgh_v, evgh_g, evgh_h);
  int nfail = 0;
  if (!(ev_v <= small_v))
    std::printf("Fail in evaluate_v, V error =%g\n", ev_v), ++nfail;
  if (!(evgh_v <= small_v))
    std::printf("Fail in evaluate_vgh, V error =%g\n", evgh_v), ++nfail;
  if (!(evgh_g <= small_g))
    std::printf("Fail in evaluate_vgh, G error =%g\n", evgh_g), ++nfail;
  if (!(evgh_h <= small_h))
    std::printf("Fail in evaluate_vgh, H error =%g\n", evgh_h), ++nfail;
  if (nfail == 0)
    std::printf("All checks passed for spo\n");
  qmc_system_destroy(st_sys);
  qmc_system_destroy(rf_sys);
  return 0;
}
