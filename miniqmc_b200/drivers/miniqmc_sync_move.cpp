// miniqmc_sync_move -- the reference's batched driver
// (miniqmc_sync_move.cpp:432-521) on the C ABI's per-call verbs.
//
// The movers are split into batches of -c walkers (one qmc_walkers handle
// per batch).  Per substep and electron, a batch runs the flex_ sequence
// verb by verb: setActive, evalGrad, the trial move from the batch's first
// mover's random stream (nw uniforms, then 3 nw normals), ratioGrad, the
// threshold accept ur < -r, acceptMove/restore and the position update;
// then completeUpdates, donePbyP and evaluateGL, and the NonLocalPP ratios
// unless -P.  The random streams are the reference's: mt19937 seeded from
// PrimeNumberSet, libstdc++ uniforms and BoxMuller2 normals, so the accepted
// count equals the reference's for the same options.
//
// Options as the reference's; -c defaults to all movers in one batch (one
// launch per verb covers the batch on the device).  Own options: -p the
// arithmetic form (mixed | fp64), -F the orbital fill (uniform | reference).
#include "driver_common.hpp"

#include <cstdlib>
#include <string>
#include <unistd.h>

using drv::check;
using drv::now_s;

namespace
{
void print_help()
{
  std::printf("usage:\n"
              "  miniqmc_sync_move [-bhjPvV] [-g \"n0 n1 n2\"] [-m meshfactor]\n"
              "            [-n steps] [-N substeps] [-x rmax]\n"
              "            [-r AcceptanceRatio] [-s seed] [-w walkers]\n"
              "            [-a tile_size] [-t timer_level] [-c nw_b]\n"
              "            [-k delay_rank] [-p mixed|fp64] [-F uniform|reference]\n"
              "options:\n"
              "  -a  size of each spline tile       default: num of orbs (ignored)\n"
              "  -b  use reference implementations  (not available)\n"
              "  -c  number of walkers per batch    default: all walkers\n"
              "  -g  set the 3D tiling.             default: 1 1 1\n"
              "  -h  print help and exit\n"
              "  -j  enable three body Jastrow      default: off\n"
              "  -m  meshfactor                     default: 1.0\n"
              "  -n  number of MC steps             default: 5\n"
              "  -N  number of MC substeps          default: 1\n"
              "  -P  not running pseudo potential   default: off\n"
              "  -r  set the acceptance ratio.      default: 0.5\n"
              "  -s  set the random seed.           default: 11\n"
              "  -t  timer level: coarse or fine    default: fine\n"
              "  -k  matrix delayed update rank     default: 32\n"
              "  -v  verbose output\n"
              "  -V  print version information and exit\n"
              "  -w  number of walker(movers)       default: 512\n"
              "  -x  set the Rmax.                  default: 1.7\n"
              "  -p  arithmetic form                default: mixed\n"
              "  -F  orbital fill                   default: uniform\n");
}
} // namespace

int main(int argc, char** argv)
{
  int na = 1, nb = 1, nc = 1, nsteps = 5, nsubsteps = 1, iseed = 11, nmovers = 512, delay_rank = 32, nw_b = 0;
  int nx = 37, ny = 37, nz = 37;
  double accept = 0.5, rmax = 1.7;
  bool verbose = false, fill_reference = false, fp64 = false, enable_j3 = false, run_pseudo = true;
  std::string timer_level = "fine";
  int opt;
  while (optind < argc)
  {
    if ((opt = getopt(argc, argv, "bhjPvVa:c:g:m:n:N:r:s:t:k:w:x:p:F:")) != -1)
    {
      switch (opt)
      {
      case 'a': break;
      case 'b':
        std::fprintf(stderr, "miniqmc_sync_move: the reference implementations (-b) are not part of this library\n");
        return 1;
      case 'c': nw_b = std::atoi(optarg); break;
      case 'g':
        if (std::sscanf(optarg, "%d %d %d", &na, &nb, &nc) != 3)
        {
          print_help();
          return 1;
        }
        break;
      case 'h': print_help(); return 1;
      case 'j': enable_j3 = true; break;
      case 'm':
      {
        const double f = std::atof(optarg);
        nx = (int)(nx * f), ny = (int)(ny * f), nz = (int)(nz * f);
      }
      break;
      case 'n': nsteps = std::atoi(optarg); break;
      case 'N': nsubsteps = std::atoi(optarg); break;
      case 'P': run_pseudo = false; break;
      case 'r': accept = std::atof(optarg); break;
      case 's': iseed = std::atoi(optarg); break;
      case 't': timer_level = optarg; break;
      case 'k': delay_rank = std::atoi(optarg); break;
      case 'v': verbose = true; break;
      case 'V': std::printf("miniqmc_sync_move on libqmcgpu (sm_100a)\n"); return 1;
      case 'w': nmovers = std::atoi(optarg); break;
      case 'x': rmax = std::atof(optarg); break;
      case 'p': fp64 = std::string(optarg) == "fp64"; break;
      case 'F': fill_reference = std::string(optarg) == "reference"; break;
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
  if (nw_b <= 0 || nw_b > nmovers)
    nw_b = nmovers;
  if (na < 1 || nb < 1 || nc < 1 || nsteps < 0 || nsubsteps < 1 || nmovers < 1 || nx < 1 || ny < 1 || nz < 1)
  {
    print_help();
    return 1;
  }
  if (check(qmc_init(0), "qmc_init"))
    return 1;
  drv::NioSystem nio;
  if (nio.build(na, nb, nc, nx, ny, nz, fill_reference, iseed, QMC_WF_ALL | (enable_j3 ? QMC_WF_J3 : 0)))
    return 1;
  const int nels = nio.nels, norb = nio.norb;
  const int nbatches = (nmovers + nw_b - 1) / nw_b;
  std::printf("Number of orbitals/splines = %d\nNumber of electrons = %d\nRmax = %g\nAcceptanceRatio = %g\n"
              "Iterations = %d\nNumber of walkers per rank = %d\nNumber of batches = %d\ndelayed update rank = %d\n",
              norb, nels, rmax, accept, nsteps, nmovers, nbatches, delay_rank);
  std::printf("Using the per-call verbs of libqmcgpu (%s form).\n", fp64 ? "FP64" : "mixed-precision");

  const double t_total0 = now_s();
  qmc_system* sys       = nullptr;
  if (check(qmc_system_create(&nio.d, fp64 ? QMC_PREC_FP64 : QMC_PREC_MIXED, &sys), "qmc_system_create"))
    return 1;
  // movers: batch b holds movers [first, last) (FairDivideLow with equal
  // shares); each mover draws its electrons from its own stream on the device
  const std::vector<uint32_t> seeds = drv::primes(nmovers);
  struct Batch
  {
    qmc_walkers* w = nullptr;
    int first = 0, nw = 0;
    drv::HostRng* rng = nullptr;
  };
  std::vector<Batch> batches(nbatches);
  double t_init = now_s();
  for (int b = 0; b < nbatches; ++b)
  {
    Batch& B = batches[b];
    B.first  = b * nmovers / nbatches;
    B.nw     = (b + 1) * nmovers / nbatches - B.first;
    if (check(qmc_walkers_create(sys, B.nw, delay_rank, &B.w), "qmc_walkers_create"))
      return 1;
    if (check(qmc_walkers_init_random(B.w, seeds.data() + B.first), "qmc_walkers_init_random"))
      return 1;
    // the first mover's stream on the host, past its build_els draws (3N)
    B.rng = new drv::HostRng(seeds[B.first]);
    std::vector<double> skip(3 * (size_t)nels);
    B.rng->uniform(skip.data(), 3 * nels);
    const int st = qmc_wf_evaluate_log(B.w, nullptr);
    if (st != QMC_OK && st != QMC_ERR_SINGULAR && check(st, "qmc_wf_evaluate_log"))
      return 1;
  }
  t_init = now_s() - t_init;

  double t_diff = 0, t_ecp = 0, t_eval = 0, t_ratio = 0, t_update = 0;
  long long accepted = 0, nlpp_points = 0;
  double logpsi_sum = 0;
  for (int mc = 0; mc < nsteps; ++mc)
    for (Batch& B : batches)
    {
      const int nw = B.nw;
      std::vector<double> grad_now(3 * nw), grad_new(3 * nw), ratios(nw), delta(3 * nw), ur(nw), logpsi(nw);
      std::vector<int> is_acc(nw);
      double t0 = now_s();
      for (int l = 0; l < nsubsteps; ++l)
      {
        for (int iel = 0; iel < nels; ++iel)
        {
          if (check(qmc_pset_set_active(B.w, iel), "qmc_pset_set_active"))
            return 1;
          double t1 = now_s();
          std::fill(grad_now.begin(), grad_now.end(), 0.0);
          if (check(qmc_wf_eval_grad(B.w, iel, grad_now.data()), "qmc_wf_eval_grad"))
            return 1;
          t_eval += now_s() - t1;
          B.rng->uniform(ur.data(), nw);
          B.rng->normal(delta.data(), 3 * nw);
          if (check(qmc_pset_make_move(B.w, iel, delta.data()), "qmc_pset_make_move"))
            return 1;
          t1 = now_s();
          std::fill(grad_new.begin(), grad_new.end(), 0.0);
          if (check(qmc_wf_ratio_grad(B.w, iel, ratios.data(), grad_new.data()), "qmc_wf_ratio_grad"))
            return 1;
          t_ratio += now_s() - t1;
          for (int iw = 0; iw < nw; ++iw)
          {
            is_acc[iw] = ur[iw] < accept;
            accepted += is_acc[iw];
          }
          t1 = now_s();
          if (check(qmc_wf_accept_restore(B.w, iel, is_acc.data()), "qmc_wf_accept_restore"))
            return 1;
          t_update += now_s() - t1;
          if (check(qmc_pset_accept_reject(B.w, iel, is_acc.data()), "qmc_pset_accept_reject"))
            return 1;
        }
        if (check(qmc_wf_complete_updates(B.w), "qmc_wf_complete_updates"))
          return 1;
      }
      if (check(qmc_pset_done(B.w), "qmc_pset_done"))
        return 1;
      const int st = qmc_wf_evaluate_gl(B.w, nullptr, nullptr, logpsi.data());
      if (st != QMC_OK && st != QMC_ERR_SINGULAR && check(st, "qmc_wf_evaluate_gl"))
        return 1;
      t_diff += now_s() - t0;
      if (mc + 1 == nsteps)
        for (double x : logpsi)
          logpsi_sum += x;
      if (!run_pseudo)
        continue;
      t0 = now_s();
      std::vector<int64_t> npts(nw);
      std::vector<double> wsum(nw);
      const int se = qmc_nlpp_evaluate(B.w, rmax, QMC_NLPP_SPHERE, npts.data(), wsum.data(), nullptr, 0);
      if (se != QMC_OK && se != QMC_ERR_SINGULAR && check(se, "qmc_nlpp_evaluate"))
        return 1;
      t_ecp += now_s() - t0;
      for (int64_t p : npts)
        nlpp_points += p;
    }
  const double t_total = now_s() - t_total0;

  const double moves = (double)nmovers * nsteps * nsubsteps * nels;
  std::printf("================================== \n");
  std::printf("Stack timer profile\n%-24s %12s %12s\n", "Timer", "Inclusive_time", "Exclusive_time");
  std::printf("%-24s %12.5f %12.5f\n", "Total", t_total, t_total - t_init - t_diff - t_ecp);
  std::printf("%-24s %12.5f %12.5f\n", "  Initialization", t_init, t_init);
  std::printf("%-24s %12.5f %12.5f\n", "  Diffusion", t_diff, t_diff - t_eval - t_ratio - t_update);
  if (timer_level == "fine")
  {
    std::printf("%-24s %12.5f %12.5f\n", "    Current Gradient", t_eval, t_eval);
    std::printf("%-24s %12.5f %12.5f\n", "    New Gradient", t_ratio, t_ratio);
    std::printf("%-24s %12.5f %12.5f\n", "    Update", t_update, t_update);
  }
  std::printf("%-24s %12.5f %12.5f\n", "  Pseudopotential", t_ecp, t_ecp);
  if (verbose)
    std::printf("accepted moves = %lld of %.0f (%.4f)\nmean log|psi| = %.15g\n", accepted, moves, accepted / moves,
                logpsi_sum / nmovers);
  std::printf("\n========== Throughput ============ \n\n");
  std::printf("Total throughput ( N_walkers * N_elec^3 / Total time ) = %g\n",
              nmovers * std::pow((double)nels, 3) / t_total);
  std::printf("Diffusion throughput ( N_walkers * N_elec^3 / Diffusion time ) = %g\n",
              nmovers * std::pow((double)nels, 3) / t_diff);
  if (run_pseudo)
    std::printf("Pseudopotential throughput ( N_walkers * N_elec^2 / Pseudopotential time ) = %g\n",
                nmovers * std::pow((double)nels, 2) / t_ecp);
  std::printf("Electron-moves/s ( N_walkers * steps * substeps * N_elec / Diffusion time ) = %g\n", moves / t_diff);
  std::printf("Accepted moves = %lld\n\n", accepted);
  for (Batch& B : batches)
  {
    qmc_walkers_destroy(B.w);
    delete B.rng;
  }
  qmc_system_destroy(sys);
  return 0;
}
