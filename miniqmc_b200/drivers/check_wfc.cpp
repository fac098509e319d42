// check_wfc -- the reference's wavefunction-component checker
// (check_wfc.cpp) on the C ABI.
//
// The reference checks each optimized component against its plain
// reference implementation.  Here the component in the arithmetic form
// under test (-p, default mixed) is checked against the same component in
// the plain FP64 form, both on the device, through the same verbs and on
// the same electrons: evaluateLog (value, G, L), then one sweep of evalGrad
// / makeMove / ratioGrad with the accept rule ur < ratio_ref, evaluateGL,
// and ratio-only moves (12 uniform displacements per electron-ion pair
// within -r).  Errors are averaged as the reference does (relative for Det,
// absolute otherwise), and the tolerance is the tested precision's epsilon
// times 1e6 (Det) or 1e4.
//
// -f J1 | J2 | J3 | JeeI | Det.  The Det check uses both spin determinants
// of the NiO cell with the well-conditioned uniform orbital fill on a 40^3
// grid (the reference's fill makes rank-1 matrices).
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
              "  check_wfc [-hvV] [-f wfc_component] [-g \"n0 n1 n2\"]\n"
              "            [-r rmax] [-s seed] [-p mixed|fp64]\n"
              "options:\n"
              "  -f  specify wavefunction component to check\n"
              "      one of: J1, J2, J3, Det.       default: J2\n"
              "  -g  set the 3D tiling.             default: 1 1 1\n"
              "  -h  print help and exit\n"
              "  -r  set the Rmax.                  default: 1.7\n"
              "  -s  set the random seed.           default: 11\n"
              "  -v  verbose output\n"
              "  -V  print version information and exit\n"
              "  -p  arithmetic form under test     default: mixed\n");
}

double grad_err(const double* g, const double* r, bool rel)
{
  const double d0 = g[0] - r[0], d1 = g[1] - r[1], d2 = g[2] - r[2];
  const double dd = d0 * d0 + d1 * d1 + d2 * d2;
  return rel ? std::sqrt(dd / (g[0] * r[0] + g[1] * r[1] + g[2] * r[2])) : std::sqrt(dd);
}
double val_err(double v, double r, bool rel) { return rel ? std::fabs((v - r) / r) : std::fabs(v - r); }
} // namespace

int main(int argc, char** argv)
{
  int na = 1, nb = 1, nc = 1, iseed = 11;
  double rmax = 1.7;
  bool fp64 = false;
  std::string wfc_name = "J2";
  int opt;
  while (optind < argc)
  {
    if ((opt = getopt(argc, argv, "hvVf:g:r:s:p:")) != -1)
    {
      switch (opt)
      {
      case 'f': wfc_name = optarg; break;
      case 'g':
        if (std::sscanf(optarg, "%d %d %d", &na, &nb, &nc) != 3)
        {
          print_help();
          return 1;
        }
        break;
      case 'h': print_help(); return 1;
      case 'r': rmax = std::atof(optarg); break;
      case 's': iseed = std::atoi(optarg); break;
      case 'v': break;
      case 'V': std::printf("check_wfc on libqmcgpu (sm_100a)\n"); return 1;
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
  int comp = 0;
  if (wfc_name == "J1")
    comp = QMC_WF_J1;
  else if (wfc_name == "J2")
    comp = QMC_WF_J2;
  else if (wfc_name == "J3" || wfc_name == "JeeI")
    comp = QMC_WF_J3;
  else if (wfc_name == "Det")
    comp = QMC_WF_DET;
  else
  {
    std::fprintf(stderr, "Uknown wave funciton component:  %s\n\n", wfc_name.c_str());
    print_help();
    return 1;
  }
  const bool det = comp == QMC_WF_DET;
  if (check(qmc_init(0), "qmc_init"))
    return 1;
  drv::NioSystem nio;
  const int grid = det ? 40 : 8;
  if (nio.build(na, nb, nc, grid, grid, grid, false, iseed, comp))
    return 1;
  const int nels = nio.nels, nions = nio.n_ions;
  qmc_system *st_sys = nullptr, *rf_sys = nullptr;
  if (check(qmc_system_create(&nio.d, fp64 ? QMC_PREC_FP64 : QMC_PREC_MIXED, &st_sys), "qmc_system_create") ||
      check(qmc_system_create(&nio.d, QMC_PREC_FP64, &rf_sys), "qmc_system_create"))
    return 1;
  qmc_walkers *wt = nullptr, *wr = nullptr;
  if (check(qmc_walkers_create(st_sys, 1, 1, &wt), "qmc_walkers_create") ||
      check(qmc_walkers_create(rf_sys, 1, 1, &wr), "qmc_walkers_create"))
    return 1;
  // one mover, seeded as the reference's first thread (PrimeNumberSet[0])
  const uint32_t seed = drv::primes(1)[0];
  if (check(qmc_walkers_init_random(wt, &seed), "init_random") ||
      check(qmc_walkers_init_random(wr, &seed), "init_random"))
    return 1;
  drv::HostRng rng(seed);
  std::vector<double> tmp(3 * (size_t)nels);
  rng.uniform(tmp.data(), 3 * nels); // build_els
  std::vector<double> ur(nels);
  rng.uniform(ur.data(), nels);
  std::printf("Built %s\nBuilt %s_ref\n", wfc_name.c_str(), wfc_name.c_str());

  double lt = 0, lr = 0;
  int s1 = qmc_wf_evaluate_log(wt, &lt), s2 = qmc_wf_evaluate_log(wr, &lr);
  if (check(s1, "qmc_wf_evaluate_log") || check(s2, "qmc_wf_evaluate_log"))
    return 1;
  std::vector<double> Gt(3 * (size_t)nels), Gr(3 * (size_t)nels), Lt(nels), Lr(nels);
  auto gl = [&](double* log_t, double* log_r) {
    return check(qmc_wf_evaluate_gl(wt, Gt.data(), Lt.data(), log_t), "qmc_wf_evaluate_gl") ||
        check(qmc_wf_evaluate_gl(wr, Gr.data(), Lr.data(), log_r), "qmc_wf_evaluate_gl");
  };
  if (gl(&lt, &lr))
    return 1;
  const int i12 = 12 < nels ? 12 : 0;
  std::printf("Check values %.10g {%.10g, %.10g, %.10g} %.10g\n", lt, Gt[3 * i12], Gt[3 * i12 + 1], Gt[3 * i12 + 2],
              Lt[i12]);
  std::printf("Check values ref %.10g {%.10g, %.10g, %.10g} %.10g\n\n", lr, Gr[3 * i12], Gr[3 * i12 + 1],
              Gr[3 * i12 + 2], Lr[i12]);
  double elog_v = std::fabs((lt - lr) / nels), elog_g = 0, elog_l = 0;
  for (int i = 0; i < nels; ++i)
  {
    elog_g += grad_err(&Gt[3 * i], &Gr[3 * i], det);
    elog_l += val_err(Lt[i], Lr[i], det);
  }
  elog_g /= nels, elog_l /= nels;
  std::printf("evaluateLog::V Error = %g\nevaluateLog::G Error = %g\nevaluateLog::L Error = %g\n", (lt - lr) / nels,
              elog_g, elog_l);

  // one sweep: evalGrad, makeMove, ratioGrad, accept if ur < ratio_ref
  std::vector<double> delta(3 * (size_t)nels);
  rng.normal(delta.data(), 3 * nels);
  double g_eval = 0, g_ratio = 0, r_ratio = 0;
  int naccepted = 0;
  for (int iel = 0; iel < nels; ++iel)
  {
    double gt[3] = {0, 0, 0}, gr[3] = {0, 0, 0};
    if (check(qmc_pset_set_active(wt, iel), "set_active") || check(qmc_pset_set_active(wr, iel), "set_active") ||
        check(qmc_wf_eval_grad(wt, iel, gt), "eval_grad") || check(qmc_wf_eval_grad(wr, iel, gr), "eval_grad"))
      return 1;
    g_eval += grad_err(gt, gr, det);
    if (check(qmc_pset_make_move(wt, iel, &delta[3 * iel]), "make_move") ||
        check(qmc_pset_make_move(wr, iel, &delta[3 * iel]), "make_move"))
      return 1;
    double rt = 0, rr = 0;
    gt[0] = gt[1] = gt[2] = gr[0] = gr[1] = gr[2] = 0;
    if (check(qmc_wf_ratio_grad(wt, iel, &rt, gt), "ratio_grad") ||
        check(qmc_wf_ratio_grad(wr, iel, &rr, gr), "ratio_grad"))
      return 1;
    g_ratio += grad_err(gt, gr, det);
    r_ratio += std::fabs(rt / rr - 1);
    const int acc = ur[iel] < rr ? 1 : 0;
    naccepted += acc;
    if (check(qmc_wf_accept_restore(wt, iel, &acc), "accept_restore") ||
        check(qmc_wf_accept_restore(wr, iel, &acc), "accept_restore") ||
        check(qmc_pset_accept_reject(wt, iel, &acc), "accept_reject") ||
        check(qmc_pset_accept_reject(wr, iel, &acc), "accept_reject"))
      return 1;
  }
  if (check(qmc_wf_complete_updates(wt), "complete_updates") || check(qmc_wf_complete_updates(wr), "complete_updates") ||
      check(qmc_pset_done(wt), "done") || check(qmc_pset_done(wr), "done"))
    return 1;
  g_eval /= nels, g_ratio /= nels, r_ratio /= nels;
  std::printf("Accepted %d/%d\nevalGrad::G      Error = %g\nratioGrad::G     Error = %g\nratioGrad::Ratio Error = %g\n",
              naccepted, nels, g_eval, g_ratio, r_ratio);
  if (gl(nullptr, nullptr))
    return 1;
  double egl_g = 0, egl_l = 0;
  for (int i = 0; i < nels; ++i)
  {
    egl_g += grad_err(&Gt[3 * i], &Gr[3 * i], det);
    egl_l += val_err(Lt[i], Lr[i], det);
  }
  egl_g /= nels, egl_l /= nels;
  std::printf("evaluteGL::G Error = %g\nevaluteGL::L Error = %g\n", egl_g, egl_l);

  // ratio only: 12 uniform displacements per (electron, ion within rmax)
  constexpr int nknots = 12;
  std::vector<double> ab_r(nions), kd(3 * nknots);
  double r_sphere = 0;
  int nsphere     = 0;
  const double zero[3] = {0, 0, 0};
  const int rej        = 0;
  for (int jel = 0; jel < nels; ++jel)
  {
    if (check(qmc_pset_make_move(wr, jel, zero), "make_move") ||
        check(qmc_pset_get_temp_rows(wr, nullptr, nullptr, ab_r.data(), nullptr), "get_temp_rows") ||
        check(qmc_pset_accept_reject(wr, jel, &rej), "accept_reject"))
      return 1;
    for (int iat = 0; iat < nions; ++iat)
      if (ab_r[iat] < rmax)
      {
        ++nsphere;
        rng.uniform(kd.data(), 3 * nknots);
        for (int k = 0; k < nknots; ++k)
        {
          double rt = 0, rr = 0;
          if (check(qmc_pset_make_move(wt, jel, &kd[3 * k]), "make_move") ||
              check(qmc_wf_ratio(wt, jel, &rt), "ratio") || check(qmc_pset_accept_reject(wt, jel, &rej), "reject") ||
              check(qmc_pset_make_move(wr, jel, &kd[3 * k]), "make_move") ||
              check(qmc_wf_ratio(wr, jel, &rr), "ratio") || check(qmc_pset_accept_reject(wr, jel, &rej), "reject"))
            return 1;
          r_sphere += std::fabs(rt / rr - 1);
        }
      }
  }
  std::printf("ratio with SphereMove  Error = %g # of moves =%d\n", nsphere ? r_sphere / nsphere : 0.0, nsphere);
  const double ratio_err = r_sphere / ((double)nels * nknots);

  const double eps   = fp64 ? std::numeric_limits<double>::epsilon() : std::numeric_limits<float>::epsilon();
  const double small = eps * (det ? 1e6 : 1e4);
  std::printf("Passing Tolerance %g\n\n", small);
  struct
  {
    const char* what;
    double err;
  } checks[] = {{"evaluateLog, V", elog_v}, {"evaluateLog, G", elog_g}, {"evaluateLog, L", elog_l},
                {"evalGrad, G", g_eval},    {"ratioGrad, ratio", r_ratio}, {"ratioGrad, G", g_ratio},
                {"evaluateGL, G", egl_g},   {"evaluateGL, L", egl_l},   {"ratio, ratio", ratio_err}};
  bool fail = false;
  for (auto& c : checks)
    if (!(c.err <= small))
    {
      std::printf("Fail in %s error =%g for %s\n", c.what, c.err, wfc_name.c_str());
      fail = true;
    }
  if (!fail)
    std::printf("All checks passed for %s\n", wfc_name.c_str());
  qmc_walkers_destroy(wt);
  qmc_walkers_destroy(wr);
  qmc_system_destroy(st_sys);
  qmc_system_destroy(rf_sys);
  return 0;
}
