// miniqmc.cpp -- the miniqmc VMC driver on the B200 library.
//
// Same command line and output shape as the reference driver
// (src/Drivers/miniqmc.cpp:149-175 options, :300-396 setup, :406-468 the
// PbyP loop, :500-521 throughput), with the walkers advanced by the fused
// sweep of libqmcgpu.so through the C ABI (include/qmcgpu.h):
//
//   miniqmc [-bhjvV] [-g "n0 n1 n2"] [-m meshfactor] [-n steps] [-N substeps]
//           [-x rmax] [-r AcceptanceRatio] [-s seed] [-w walkers]
//           [-a tile_size] [-t timer_level] [-k delay_rank]
//           [-F reference|uniform] [-P mixed|fp64] [-R refresh_every]
//
// -g tiles the reference's 32-atom NiO cell (nio.hpp).  The reference's own
// orbital fill (-F reference) makes every Slater matrix rank 1 (one field
// times cos(2 pi n / N) per orbital), so its determinants are round-off; the
// library reports that as QMC_ERR_SINGULAR, and the default here is the
// well-conditioned SplitMix64 fill (-F uniform, seed -s).  -P picks the
// arithmetic form and -R the FP64 refresh interval of the inverses (0 = off).
// -a (spline tiles) is accepted and ignored: the table is one tile per
// walker CTA here.  -j adds the three-body Jastrow with buildJeeI's
// functors (WaveFunction.cpp:97-100, nio.hpp:171-245).  -b (the reference
// implementations) is not part of this library and stops the driver with a
// message.
// After the steps, the pseudopotential ratios of the reference's loop
// (miniqmc.cpp:472-495) run once per step through qmc_nlpp_evaluate, with
// -x as rmax and the driver's form of the virtual moves.
#include "driver_common.hpp"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unistd.h>
#include <vector>

using drv::check;
using drv::now_s;

namespace
{
void print_help()
{
  std::printf("usage:\n"
              "  miniqmc   [-bhjvV] [-g \"n0 n1 n2\"] [-m meshfactor]\n"
              "            [-n steps] [-N substeps] [-x rmax]\n"
              "            [-r AcceptanceRatio] [-s seed] [-w walkers]\n"
              "            [-a tile_size] [-t timer_level] [-k delay_rank]\n"
              "            [-F reference|uniform] [-P mixed|fp64] [-R refresh_every]\n"
              "options:\n"
              "  -a  size of each spline tile       default: num of orbs (ignored)\n"
              "  -b  use reference implementations  (not available)\n"
              "  -g  set the 3D tiling.             default: 1 1 1\n"
              "  -h  print help and exit\n"
              "  -j  enable three body Jastrow      default: off\n"
              "  -m  meshfactor                     default: 1.0\n"
              "  -n  number of MC steps             default: 5\n"
              "  -N  number of MC substeps          default: 1\n"
              "  -r  set the acceptance ratio.      default: 0.5\n"
              "  -s  set the random seed.           default: 11\n"
              "  -t  timer level: coarse or fine    default: fine\n"
              "  -k  matrix delayed update rank     default: 32\n"
              "  -v  verbose output\n"
              "  -V  print version information and exit\n"
              "  -w  number of walker(movers)       default: 512\n"
              "  -x  set the Rmax.                  default: 1.7\n"
              "  -F  orbital fill                   default: uniform\n"
              "  -P  arithmetic form                default: mixed\n"
              "  -R  FP64 refresh every R steps     default: 8\n");
}

} // namespace

int main(int argc, char** argv)
{
  int na = 1, nb = 1, nc = 1, nsteps = 5, nsubsteps = 1, iseed = 11, nmovers = 512, delay_rank = 32;
  int nx = 37, ny = 37, nz = 37, refresh = 8;
  double accept = 0.5, rmax = 1.7;
  bool verbose = false, fill_reference = false, fp64 = false, enable_j3 = false;
  std::string timer_level = "fine";
  int opt;
  while (optind < argc)
  {
    if ((opt = getopt(argc, argv, "bhjvVa:c:g:m:n:N:r:s:t:k:w:x:F:P:R:")) != -1)
    {
      switch (opt)
      {
      case 'a': break; // spline tiles: one tile per walker CTA here
      case 'c': break; // team size of the OpenMP driver: no counterpart
      case 'b':
        std::fprintf(stderr, "miniqmc: the reference implementations (-b) are not part of this library\n");
        return 1;
      case 'j': enable_j3 = true; break;
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
      case 'N': nsubsteps = std::atoi(optarg); break;
      case 'r': accept = std::atof(optarg); break;
      case 's': iseed = std::atoi(optarg); break;
      case 't': timer_level = optarg; break;
      case 'k': delay_rank = std::atoi(optarg); break;
      case 'v': verbose = true; break;
      case 'V': std::printf("miniqmc on libqmcgpu (sm_100a)\n"); return 1;
      case 'w': nmovers = std::atoi(optarg); break;
      case 'x': rmax = std::atof(optarg); break;
      case 'F': fill_reference = std::string(optarg) == "reference"; break;
      case 'P': fp64 = std::string(optarg) == "fp64"; break;
      case 'R': refresh = std::atoi(optarg); break;
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
  if (timer_level != "fine" && timer_level != "coarse")
  {
    std::fprintf(stderr, "Timer level should be 'coarse' or 'fine', name given: %s\n", timer_level.c_str());
    return 1;
  }
  if (na < 1 || nb < 1 || nc < 1 || nsteps < 0 || nsubsteps < 1 || nmovers < 1 || nx < 1 || ny < 1 || nz < 1)
  {
    print_help();
    return 1;
  }
  if (check(qmc_init(0), "qmc_init"))
    return 1;

  // ---- ions and electrons (build_ions + count_electrons, nio.hpp)
  drv::NioSystem nio;
  if (nio.build(na, nb, nc, nx, ny, nz, fill_reference, iseed, QMC_WF_ALL | (enable_j3 ? QMC_WF_J3 : 0)))
    return 1;
  const qmc_system_desc& d = nio.d;
  const int nels = nio.nels, norb = nio.norb;

  const size_t coef_bytes = (size_t)norb * (nx + 3) * (ny + 3) * (nz + 3) * (fp64 ? 8 : 4);
  std::printf("Number of orbitals/splines = %d\nTile size = %d\nNumber of tiles = 1\nNumber of electrons = %d\n"
              "Rmax = %g\nAcceptanceRatio = %g\nIterations = %d\nNumber of walkers per rank = %d\n\n"
              "SPO coefficients size = %zu bytes (%g MB)\ndelayed update rank = %d\n",
              norb, norb, nels, rmax, accept, nsteps, nmovers, coef_bytes, coef_bytes / 1048576.0, delay_rank);
  std::printf("Using the fused B200 sweep (%s form, %s orbital fill, FP64 refresh every %d steps).\n",
              fp64 ? "FP64" : "mixed-precision", fill_reference ? "reference" : "uniform", refresh);

  const double t_total0 = now_s();
  double t_setup = now_s();
  qmc_system* sys = nullptr;
  if (check(qmc_system_create(&d, fp64 ? QMC_PREC_FP64 : QMC_PREC_MIXED, &sys), "qmc_system_create"))
    return 1;
  t_setup = now_s() - t_setup;

  // ---- movers (Mover + build_WaveFunction + evaluateLog)
  double t_init   = now_s();
  qmc_walkers* w  = nullptr;
  if (check(qmc_walkers_create(sys, nmovers, delay_rank, &w), "qmc_walkers_create"))
    return 1;
  std::vector<uint32_t> seeds = drv::primes(nmovers);
  if (check(qmc_walkers_init_random(w, seeds.data()), "qmc_walkers_init_random"))
    return 1;
  int st = qmc_wf_evaluate_log(w, nullptr);
  if (st == QMC_ERR_SINGULAR)
    std::printf("note: the Slater matrices are singular (log|det| is round-off), as with the reference fill\n");
  else if (check(st, "qmc_wf_evaluate_log"))
    return 1;
  t_init = now_s() - t_init;

  // ---- the PbyP loop: nsteps x (nsubsteps x nels moves + completeUpdates, evaluateGL)
  std::vector<int64_t> acc(nmovers);
  std::vector<double> logpsi(nmovers);
  qmc_sweep_opts o;
  std::memset(&o, 0, sizeof(o));
  o.n_steps         = nsteps;
  o.n_substeps      = nsubsteps;
  o.accept          = accept;
  o.rng_mode        = QMC_RNG_DEVICE;
  o.recompute_every = refresh;
  o.n_accepted      = acc.data();
  o.logpsi          = logpsi.data();
  // each MC step: the diffusion sweep, then the NLPP ratios of every walker
  double t_diff = 0, t_ecp = 0;
  int64_t nlpp_points = 0;
  std::vector<int64_t> npts(nmovers);
  std::vector<double> wsum(nmovers);
  o.n_steps = 1;
  std::vector<int64_t> acc_total(nmovers, 0);
  for (int step = 0; step < nsteps; ++step)
  {
    double t0 = now_s();
    st        = qmc_sweep(w, &o);
    t_diff += now_s() - t0;
    if (st != QMC_OK && st != QMC_ERR_SINGULAR && check(st, "qmc_sweep"))
      return 1;
    for (int i = 0; i < nmovers; ++i)
      acc_total[i] += acc[i];
    t0 = now_s();
    st = qmc_nlpp_evaluate(w, rmax, QMC_NLPP_DRIVER, npts.data(), wsum.data(), nullptr, 0);
    t_ecp += now_s() - t0;
    if (st != QMC_OK && st != QMC_ERR_SINGULAR && check(st, "qmc_nlpp_evaluate"))
      return 1;
    for (int64_t p : npts)
      nlpp_points += p;
  }
  acc = acc_total;
  const double t_total = now_s() - t_total0;

  int64_t accepted = 0;
  for (int64_t a : acc)
    accepted += a;
  const double moves = (double)nmovers * nsteps * nsubsteps * nels;
  std::printf("================================== \n");
  std::printf("Stack timer profile\n%-24s %12s %12s\n", "Timer", "Inclusive_time", "Exclusive_time");
  std::printf("%-24s %12.5f %12.5f\n", "Total", t_total, t_total - t_setup - t_init - t_diff);
  std::printf("%-24s %12.5f %12.5f\n", "  Setup", t_setup, t_setup);
  std::printf("%-24s %12.5f %12.5f\n", "  Initialization", t_init, t_init);
  std::printf("%-24s %12.5f %12.5f\n", "  Diffusion", t_diff, t_diff);
  std::printf("%-24s %12.5f %12.5f\n", "  Pseudopotential", t_ecp, t_ecp);
  if (verbose)
  {
    double lp = 0;
    for (double x : logpsi)
      lp += x / nmovers;
    std::printf("accepted moves = %lld of %.0f (%.4f)\nmean log|psi| = %.15g\n", (long long)accepted, moves,
                accepted / moves, lp);
  }
  std::printf("\n========== Throughput ============ \n\n");
  std::printf("Total throughput ( N_walkers * N_elec^3 / Total time ) = %g\n",
              nmovers * std::pow((double)nels, 3) / t_total);
  std::printf("Diffusion throughput ( N_walkers * N_elec^3 / Diffusion time ) = %g\n",
              nmovers * std::pow((double)nels, 3) / t_diff);
  std::printf("Pseudopotential throughput ( N_walkers * N_elec^2 / Pseudopotential time ) = %g\n",
              nmovers * std::pow((double)nels, 2) / t_ecp);
  std::printf("Electron-moves/s ( N_walkers * steps * substeps * N_elec / Diffusion time ) = %g\n", moves / t_diff);
  std::printf("NLPP ratios/s ( points / Pseudopotential time ) = %g\n", nlpp_points / t_ecp);
  std::printf("Accepted moves = %lld\n\n", (long long)accepted);
  qmc_walkers_destroy(w);
  qmc_system_destroy(sys);
  return 0;
}
