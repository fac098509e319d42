// check_spo_gpu.cpp -- the reference's own SPO set (einspline_spo as its
// build_SPOSet makes it: its fill, its tiles) against SPOSetGpu, the SPOSet
// adapter over the device copy of the same table, at random points of the
// reference's NiO cell.  Values, gradients and the reference's Laplacian
// (hess.xx, einspline_spo.hpp:218) are compared per orbital; the tiles are
// read block by block from the reference (einspline_spo::evaluate_vgh), not
// through its tile-concatenating evaluate().
//
//   check_spo_gpu [-g "n0 n1 n2"] [-m meshfactor] [-a tile_size] [-n points]
//
// Exit code 0 and "All checks passed for spo on the device" when every
// relative error (against the largest magnitude of the quantity) is below
// 1e-10 in FP64 (QMCGPU_PRECISION=mixed: 1e-5).
#include <Utilities/Configuration.h>
#include <Utilities/PrimeNumberSet.h>
#include <Utilities/RandomGenerator.h>
#include <Particle/ParticleSet.h>
#include <Particle/ParticleSet_builder.hpp>
#include <Input/Input.hpp>
#include <QMCWaveFunctions/SPOSet_builder.h>
#include <QMCWaveFunctions/einspline_spo.hpp>

#include "qmcgpu_adapter.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <getopt.h>

using namespace qmcplusplus;

int main(int argc, char** argv)
{
  int na = 1, nb = 1, nc = 1, nx = 37, ny = 37, nz = 37, tile = -1, npoints = 16;
  int opt;
  while ((opt = getopt(argc, argv, "g:m:a:n:")) != -1)
  {
    switch (opt)
    {
    case 'g':
      if (std::sscanf(optarg, "%d %d %d", &na, &nb, &nc) != 3)
        return 1;
      break;
    case 'm':
    {
      const double f = std::atof(optarg);
      nx *= f, ny *= f, nz *= f;
      break;
    }
    case 'a':
      tile = std::atoi(optarg);
      break;
    case 'n':
      npoints = std::atoi(optarg);
      break;
    default:
      std::fprintf(stderr, "usage: check_spo_gpu [-g \"n0 n1 n2\"] [-m meshfactor] [-a tile_size] [-n points]\n");
      return 1;
    }
  }
  Tensor<int, 3> tmat(na, 0, 0, 0, nb, 0, 0, 0, nc);
  ParticleSet ions;
  Tensor<OHMMS_PRECISION, 3> lattice_b;
  build_ions(ions, tmat, lattice_b);
  const int nels = count_electrons(ions, 1), norb = nels / 2;
  tile           = tile > 0 ? tile : norb;
  const int nTiles = norb / tile;
  if (nTiles * tile != norb)
  {
    std::fprintf(stderr, "the tile size must divide %d orbitals\n", norb);
    return 1;
  }
  SPOSet* spo_main = build_SPOSet(false, nx, ny, nz, norb, nTiles, lattice_b);
  auto* ref        = dynamic_cast<einspline_spo<OHMMS_PRECISION>*>(spo_main);
  PrimeNumberSet<uint32_t> primes;
  RandomGenerator<QMCTraits::RealType> rng(primes[0]);
  ParticleSet els;
  build_els(els, ions, rng);
  auto sys = qmcgpu::device_system(spo_main, ions, els, false);
  qmcgpu::SPOSetGpu gpu(sys);
  SPOSet::ValueVector_t v(norb), l(norb);
  SPOSet::GradVector_t g(norb);
  double ev = 0, eg = 0, el = 0, mv = 0, mg = 0, ml = 0;
  for (int p = 0; p < npoints; ++p)
  {
    const int iel = p % nels;
    for (int c = 0; c < 3; ++c)
      els.R[iel][c] = 20.0 * rng() - 10.0; // any point: the orbitals are periodic
    ref->evaluate_vgh(els, iel);
    gpu.evaluate(els, iel, v, g, l);
    for (int b = 0; b < ref->nBlocks; ++b)
      for (int j = 0; j < ref->nSplinesPerBlock; ++j)
      {
        const int o = b * ref->nSplinesPerBlock + j;
        ev          = std::max(ev, std::fabs(v[o] - ref->psi[b][j]));
        mv          = std::max(mv, std::fabs((double)ref->psi[b][j]));
        for (int c = 0; c < 3; ++c)
        {
          eg = std::max(eg, std::fabs(g[o][c] - ref->grad[b].data(c)[j]));
          mg = std::max(mg, std::fabs((double)ref->grad[b].data(c)[j]));
        }
        el = std::max(el, std::fabs(l[o] - ref->hess[b].data(0)[j]));
        ml = std::max(ml, std::fabs((double)ref->hess[b].data(0)[j]));
      }
  }
  const double rv = ev / mv, rg = eg / mg, rl = el / ml;
  std::printf("orbitals %d in %d tiles, grid %d %d %d, %d points\n", norb, nTiles, nx, ny, nz, npoints);
  std::printf("value error %.3e, gradient error %.3e, laplacian error %.3e (relative to the largest)\n", rv, rg, rl);
  const double tol = std::getenv("QMCGPU_PRECISION") && std::strcmp(std::getenv("QMCGPU_PRECISION"), "mixed") == 0
      ? 1e-5
      : 1e-10;
  const bool ok = rv < tol && rg < tol && rl < tol;
  if (ok)
    std::printf("All checks passed for spo on the device\n");
  delete spo_main;
  return ok ? 0 : 2;
}
