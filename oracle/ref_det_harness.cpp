// ref_det_harness.cpp -- golden vectors of the determinant path from the
// reference's own code: DiracDeterminant<DelayedUpdate<double,double>> and
// DiracMatrix (LAPACK getrf/getri, BLAS gemv/ger/gemm) over its einspline
// SPO, on a well-conditioned orbital table.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/ref_harness.mk from the
// reference sources where they lie, linked against the image's OpenBLAS;
// output binary in oracle/_ref/.  tests/golden/make_golden.py stores the
// JSON it prints as tests/golden/reference_det_dump.json.
//
// The reference's own orbital fill (einspline_spo::set with init_random,
// BsplineAllocator::setCoefficientsForOrbitals) makes every orbital the same
// field times a scalar, so its Slater matrices are singular.  Here the table
// is allocated by einspline_spo::set without the fill, and every coefficient
// of every orbital is set independently to SplitMix64(11, index) - 0.5 in
// [-0.5, 0.5): the fill the product and the oracle call QMC_FILL_UNIFORM.
// System: the reference's NiO cell at -g "1 1 1" (32 ions, 384 electrons,
// 192 orbitals per spin), electrons from the driver's stream seeded with
// the first prime, a 16x16x16 grid; a determinant-only wavefunction (up and
// down), delay ranks 1 (Sherman-Morrison) and 32 (Woodbury GEMMs); one
// substep of the miniqmc move protocol with the threshold accept
// (miniqmc.cpp:424-460) on the same stream.
#include <Utilities/Configuration.h>
#include <Utilities/PrimeNumberSet.h>
#include <Utilities/RandomGenerator.h>
#include <Particle/ParticleSet.h>
#include <Particle/ParticleSet_builder.hpp>
#include <Input/Input.hpp>
#include <QMCWaveFunctions/einspline_spo.hpp>
#include <QMCWaveFunctions/DiracDeterminant.h>
#include <cstdint>
#include <cstdio>
#include <vector>

using namespace qmcplusplus;
typedef QMCTraits::RealType RealType;
typedef ParticleSet::ParticlePos_t ParticlePos_t;
typedef ParticleSet::PosType PosType;

static void arr(const char* key, const double* v, size_t n, bool comma = true)
{
  printf("\"%s\": [", key);
  for (size_t i = 0; i < n; ++i)
    printf("%s%.17g", i ? ", " : "", v[i]);
  printf("]%s\n", comma ? "," : "");
}
static void arri(const char* key, const int* v, size_t n, bool comma = true)
{
  printf("\"%s\": [", key);
  for (size_t i = 0; i < n; ++i)
    printf("%s%d", i ? ", " : "", v[i]);
  printf("]%s\n", comma ? "," : "");
}

// SplitMix64 (Steele, Lea and Flood 2014) of (seed, index), mapped to
// [0, 1) with 53 bits: the uniform fill's generator
static double splitmix_uniform(uint64_t seed, uint64_t index)
{
  uint64_t z = seed + (index + 1) * 0x9E3779B97F4A7C15ull;
  z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z          = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static void run(int delay, int nx, int ny, int nz)
{
  PrimeNumberSet<uint32_t> myPrimes;
  Tensor<int, 3> tmat(1, 0, 0, 0, 1, 0, 0, 0, 1);
  ParticleSet ions;
  Tensor<OHMMS_PRECISION, 3> lattice_b;
  build_ions(ions, tmat, lattice_b);
  RandomGenerator<RealType> rng(myPrimes[0]);
  ParticleSet els;
  build_els(els, ions, rng);
  const int N = els.getTotalNum(), nup = N / 2, norb = nup;
  els.update();

  einspline_spo<RealType> spo;
  spo.set(nx, ny, nz, norb, 1, false);
  spo.Lattice.set(lattice_b);
  auto* sp = spo.einsplines[0];
  for (int ix = 0; ix < nx + 3; ++ix)
    for (int iy = 0; iy < ny + 3; ++iy)
      for (int iz = 0; iz < nz + 3; ++iz)
      {
        const uint64_t g = ((uint64_t)ix * (ny + 3) + iy) * (nz + 3) + iz;
        for (int j = 0; j < norb; ++j)
          sp->coefs[ix * sp->x_stride + iy * sp->y_stride + iz * sp->z_stride + j] =
              splitmix_uniform(11, g * norb + j) - 0.5;
      }

  DiracDeterminant<> up(&spo, 0, delay), dn(&spo, nup, delay);
  ParticleSet::ParticleGradient_t G(N);
  ParticleSet::ParticleLaplacian_t L(N);
  G = 0.0;
  L = 0.0;
  const double l0u = up.evaluateLog(els, G, L), l0d = dn.evaluateLog(els, G, L);
  char key[64];
  printf("\"det_k%d\": {\n", delay);
  printf("\"grid\": [%d, %d, %d],\n\"delay\": %d,\n", nx, ny, nz, delay);
  printf("\"log_init\": [%.17g, %.17g],\n\"phase_init\": [%.17g, %.17g],\n", l0u, l0d, up.PhaseValue,
         dn.PhaseValue);
  {
    std::vector<double> g, l;
    for (int i = 0; i < N; ++i)
    {
      for (int d = 0; d < 3; ++d)
        g.push_back(G[i][d]);
      l.push_back(L[i]);
    }
    arr("G_init", g.data(), g.size());
    arr("L_init", l.data(), l.size());
  }
  std::vector<double> ur(N);
  ParticlePos_t delta(N);
  rng.generate_uniform(ur.data(), N);
  rng.generate_normal(&delta[0][0], 3 * N);
  std::vector<double> ratios, gnew, gnow;
  std::vector<int> acc;
  for (int iel = 0; iel < N; ++iel)
  {
    DiracDeterminant<>& det = iel < nup ? up : dn;
    els.setActive(iel);
    PosType g0 = det.evalGrad(els, iel);
    els.makeMove(iel, delta[iel]);
    PosType g(0.0);
    const double ratio = det.ratioGrad(els, iel, g);
    ratios.push_back(ratio);
    for (int d = 0; d < 3; ++d)
      gnew.push_back(g[d]), gnow.push_back(g0[d]);
    if (ur[iel] < 0.5)
    {
      det.acceptMove(els, iel);
      els.acceptMove(iel);
      acc.push_back(1);
    }
    else
    {
      els.rejectMove(iel);
      acc.push_back(0);
    }
  }
  up.completeUpdates();
  dn.completeUpdates();
  els.donePbyP();
  arr("ratio", ratios.data(), ratios.size());
  arr("grad_new", gnew.data(), gnew.size());
  arr("grad_now", gnow.data(), gnow.size());
  arri("accept", acc.data(), acc.size());
  printf("\"log_after\": [%.17g, %.17g],\n", up.LogValue, dn.LogValue);
  // rows of the updated inverse (psiM = (A^-1)^T) after completeUpdates
  const int rows[3] = {0, norb / 2, norb - 1};
  for (int s = 0; s < 2; ++s)
    for (int q = 0; q < 3; ++q)
    {
      const DiracDeterminant<>& det = s ? dn : up;
      std::vector<double> r(det.psiM[rows[q]], det.psiM[rows[q]] + norb);
      snprintf(key, sizeof key, "psiM_%s_row%d", s ? "dn" : "up", rows[q]);
      arr(key, r.data(), r.size());
    }
  // a fresh evaluation at the final positions
  G = 0.0;
  L = 0.0;
  const double l1u = up.evaluateLog(els, G, L), l1d = dn.evaluateLog(els, G, L);
  printf("\"log_fresh\": [%.17g, %.17g]\n", l1u, l1d);
  printf("},\n");
}

int main()
{
  printf("{\n");
  run(1, 16, 16, 16);
  run(32, 16, 16, 16);
  printf("\"_generator\": \"oracle/ref_det_harness.cpp compiled from the reference sources\"\n}\n");
  return 0;
}
