// ref_harness.cpp -- golden-vector dump from the reference's own code.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/ref_harness.mk from the
// reference sources where they lie (ParticleSet, distance tables, lattice,
// B-spline SPO, BsplineFunctor, One/TwoBodyJastrow, StdRandom, NiO input);
// output binary goes to oracle/_ref/.  The determinant needs an external
// BLAS/LAPACK and is not built here; its parity is pinned by the reference's
// unit-test known answers instead.  tests/golden/make_golden.py runs this
// binary and stores the JSON it prints as tests/golden/reference_dump.json.
#include <Utilities/Configuration.h>
#include <Utilities/PrimeNumberSet.h>
#include <Utilities/RandomGenerator.h>
#include <Particle/ParticleSet.h>
#include <Particle/ParticleSet_builder.hpp>
#include <Particle/DistanceTable.h>
#include <Input/Input.hpp>
#include <QMCWaveFunctions/einspline_spo.hpp>
#include <QMCWaveFunctions/Jastrow/BsplineFunctor.h>
#include <QMCWaveFunctions/Jastrow/OneBodyJastrow.h>
#include <QMCWaveFunctions/Jastrow/TwoBodyJastrow.h>
#include <QMCWaveFunctions/Jastrow/PolynomialFunctor3D.h>
#include <QMCWaveFunctions/Jastrow/ThreeBodyJastrow.h>
#include <Drivers/NonLocalPP.hpp>
#include <array>
#include <cstdio>
#include <random>
#include <string>
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
static std::vector<double> flat(const ParticlePos_t& R)
{
  std::vector<double> v;
  for (size_t i = 0; i < R.size(); ++i)
    for (int d = 0; d < 3; ++d)
      v.push_back(R[i][d]);
  return v;
}

static void dump_ions(const char* name, int na, int nb, int nc)
{
  Tensor<int, 3> tmat(na, 0, 0, 0, nb, 0, 0, 0, nc);
  ParticleSet ions;
  Tensor<OHMMS_PRECISION, 3> lattice_b;
  build_ions(ions, tmat, lattice_b);
  printf("\"%s\": {\n", name);
  std::vector<double> lat(9);
  for (int i = 0; i < 9; ++i)
    lat[i] = ions.Lattice.R[i];
  arr("lattice", lat.data(), 9);
  printf("\"ws\": %.17g,\n", ions.Lattice.WignerSeitzRadius);
  auto p = flat(ions.R);
  arr("ions", p.data(), p.size());
  std::vector<int> g(ions.getTotalNum());
  for (int i = 0; i < ions.getTotalNum(); ++i)
    g[i] = ions.GroupID[i];
  arri("groups", g.data(), g.size(), false);
  printf("},\n");
}

int main(int argc, char** argv)
{
  PrimeNumberSet<uint32_t> myPrimes;
  printf("{\n");
  {
    std::vector<int> p(12);
    for (int i = 0; i < 12; ++i)
      p[i] = (int)myPrimes[i];
    arri("primes", p.data(), p.size());
  }
  { // StdRandom<double> seeded with primes[0]
    RandomGenerator<RealType> r(myPrimes[0]);
    std::vector<double> u(16), nrm(15);
    r.generate_uniform(u.data(), 16);
    r.generate_normal(nrm.data(), 15);
    arr("rng_uniform_p0", u.data(), u.size());
    arr("rng_normal_p0_after16", nrm.data(), nrm.size());
    std::mt19937 mt(myPrimes[0]);
    std::vector<double> w(8);
    for (auto& x : w)
      x = (double)mt();
    arr("mt_words_p0", w.data(), w.size());
  }
  dump_ions("nio_111", 1, 1, 1);
  dump_ions("nio_112", 1, 1, 2);
  dump_ions("nio_211", 2, 1, 1);

  // ---- electrons, distance rows, Jastrows at -g "1 1 1" (check_wfc setup) ----
  Tensor<int, 3> tmat(1, 0, 0, 0, 1, 0, 0, 0, 1);
  ParticleSet ions;
  Tensor<OHMMS_PRECISION, 3> lattice_b;
  build_ions(ions, tmat, lattice_b);
  RandomGenerator<RealType> rng(myPrimes[0]);
  ParticleSet els;
  build_els(els, ions, rng);
  const int N = els.getTotalNum(), I = ions.getTotalNum();
  {
    auto p = flat(els.R);
    arr("els_111_p0", p.data(), p.size());
  }
  els.addTable(els, DT_SOA);
  const int ei = els.addTable(ions, DT_SOA);
  els.update();
  {
    els.setActive(5);
    const auto* aa = els.DistTables[0];
    std::vector<double> r(aa->Distances[5], aa->Distances[5] + N), dr;
    for (int j = 0; j < N; ++j)
      for (int d = 0; d < 3; ++d)
        dr.push_back(aa->Displacements[5].data(d)[j]);
    r[5] = -1.0; // the reference stores numeric max on the diagonal
    arr("aa_row5_r", r.data(), N);
    arr("aa_row5_dr", dr.data(), dr.size());
    PosType d(0.3, -0.7, 1.1);
    els.makeMove(7, d);
    std::vector<double> tr(aa->Temp_r.data(), aa->Temp_r.data() + N), tdr;
    for (int j = 0; j < N; ++j)
      for (int k = 0; k < 3; ++k)
        tdr.push_back(aa->Temp_dr.data(k)[j]);
    arr("aa_move7_r", tr.data(), N);
    arr("aa_move7_dr", tdr.data(), tdr.size());
    const auto* ab = els.DistTables[ei];
    std::vector<double> ar(ab->Temp_r.data(), ab->Temp_r.data() + I), adr;
    for (int j = 0; j < I; ++j)
      for (int k = 0; k < 3; ++k)
        adr.push_back(ab->Temp_dr.data(k)[j]);
    arr("ab_move7_r", ar.data(), I);
    arr("ab_move7_dr", adr.data(), adr.size());
    els.rejectMove(7);
  }
  // J1 / J2 exactly as check_wfc builds them (check_wfc.cpp:222-245)
  OneBodyJastrow<BsplineFunctor<RealType>> J1(ions, els);
  buildJ1(J1, els.Lattice.WignerSeitzRadius);
  TwoBodyJastrow<BsplineFunctor<RealType>> J2(els);
  buildJ2(J2, els.Lattice.WignerSeitzRadius);
  {
    std::vector<double> c(J2.F[0]->SplineCoefs.begin(), J2.F[0]->SplineCoefs.end());
    arr("j2_uu_coefs", c.data(), c.size());
    printf("\"j2_rcut\": %.17g,\n\"j2_dinv\": %.17g,\n", J2.F[0]->cutoff_radius, J2.F[0]->DeltaRInv);
    std::vector<double> c1(J1.F[0]->SplineCoefs.begin(), J1.F[0]->SplineCoefs.end());
    arr("j1_O_coefs", c1.data(), c1.size());
    printf("\"j1_rcut\": %.17g,\n", J1.F[0]->cutoff_radius);
    double dudr, d2u;
    std::vector<double> fv;
    for (double r : {0.05, 0.7, 1.3, 2.2, 3.3, 4.1})
    {
      double u = J2.F[1]->evaluate(r, dudr, d2u);
      fv.push_back(u), fv.push_back(dudr), fv.push_back(d2u);
    }
    arr("j2_ud_eval_at_0.05_0.7_1.3_2.2_3.3_4.1", fv.data(), fv.size());
  }
  {
    // fresh tables, as check_wfc does before evaluateLog (check_wfc.cpp:266-268):
    // setActive above wrote a full row into the triangular displacement pool
    els.update();
    els.G = 0.0;
    els.L = 0.0;
    double l1 = J1.evaluateLog(els, els.G, els.L);
    ParticleSet::ParticleGradient_t G1(els.G);
    ParticleSet::ParticleLaplacian_t L1(els.L);
    els.G = 0.0;
    els.L = 0.0;
    double l2 = J2.evaluateLog(els, els.G, els.L);
    printf("\"j1_log\": %.17g,\n\"j2_log\": %.17g,\n", l1, l2);
    std::vector<double> g1, g2, lap1, lap2;
    for (int i = 0; i < N; ++i)
    {
      for (int d = 0; d < 3; ++d)
        g1.push_back(G1[i][d]), g2.push_back(els.G[i][d]);
      lap1.push_back(L1[i]), lap2.push_back(els.L[i]);
    }
    arr("j1_G", g1.data(), g1.size());
    arr("j1_L", lap1.data(), lap1.size());
    arr("j2_G", g2.data(), g2.size());
    arr("j2_L", lap2.data(), lap2.size());
  }
  // one substep of the miniqmc move protocol with J1*J2 only and the
  // threshold accept (miniqmc.cpp:424-460), continuing the same stream
  {
    std::vector<double> ur(N);
    ParticlePos_t delta(N);
    rng.generate_uniform(ur.data(), N);
    rng.generate_normal(&delta[0][0], 3 * N);
    std::vector<double> ratios, gnew, gnow;
    std::vector<int> acc;
    for (int iel = 0; iel < N; ++iel)
    {
      els.setActive(iel);
      PosType g0 = J1.evalGrad(els, iel);
      g0 += J2.evalGrad(els, iel);
      els.makeMove(iel, delta[iel]);
      PosType g(0.0);
      double ratio = J1.ratioGrad(els, iel, g);
      ratio *= J2.ratioGrad(els, iel, g);
      ratios.push_back(ratio);
      for (int d = 0; d < 3; ++d)
        gnew.push_back(g[d]), gnow.push_back(g0[d]);
      if (ur[iel] < 0.5)
      {
        J1.acceptMove(els, iel);
        J2.acceptMove(els, iel);
        els.acceptMove(iel);
        acc.push_back(1);
      }
      else
      {
        els.rejectMove(iel);
        acc.push_back(0);
      }
    }
    els.donePbyP();
    els.G = 0.0;
    els.L = 0.0;
    J1.evaluateGL(els, els.G, els.L);
    J2.evaluateGL(els, els.G, els.L);
    arr("jsweep_ratio", ratios.data(), ratios.size());
    arr("jsweep_grad_new", gnew.data(), gnew.size());
    arr("jsweep_grad_now", gnow.data(), gnow.size());
    arri("jsweep_accept", acc.data(), acc.size());
    printf("\"jsweep_j1_log\": %.17g,\n\"jsweep_j2_log\": %.17g,\n", J1.LogValue, J2.LogValue);
    auto p = flat(els.R);
    arr("jsweep_R", p.data(), p.size());
    std::vector<double> g, l;
    for (int i = 0; i < N; ++i)
    {
      for (int d = 0; d < 3; ++d)
        g.push_back(els.G[i][d]);
      l.push_back(els.L[i]);
    }
    arr("jsweep_G", g.data(), g.size());
    arr("jsweep_L", l.data(), l.size());
  }
  // ---- SPO: einspline_spo::set (reference fill, seed 11) on an anisotropic grid ----
  {
    const int nx = 12, ny = 11, nz = 10, norb = 16;
    einspline_spo<RealType> spo;
    spo.set(nx, ny, nz, norb, 1);
    spo.Lattice.set(lattice_b);
    printf("\"spo_grid\": [%d, %d, %d],\n\"spo_norb\": %d,\n", nx, ny, nz, norb);
    std::vector<double> pos, v, g, h;
    for (int iel = 0; iel < 6; ++iel)
    {
      PosType p = els.R[iel * 11];
      if (iel == 5)
        p = PosType(-3.2, 40.1, -0.01); // outside the cell: exercises toUnit_floor
      for (int d = 0; d < 3; ++d)
        pos.push_back(p[d]);
      els.makeMove(iel * 11, p - els.R[iel * 11]);
      spo.evaluate_vgh(els, iel * 11);
      for (int n = 0; n < norb; ++n)
        v.push_back(spo.psi[0][n]);
      for (int d = 0; d < 3; ++d)
        for (int n = 0; n < norb; ++n)
          g.push_back(spo.grad[0].data(d)[n]);
      for (int d = 0; d < 6; ++d)
        for (int n = 0; n < norb; ++n)
          h.push_back(spo.hess[0].data(d)[n]);
      els.rejectMove(iel * 11);
    }
    arr("spo_pos", pos.data(), pos.size());
    arr("spo_v", v.data(), v.size());
    arr("spo_g", g.data(), g.size());
    arr("spo_h", h.data(), h.size());
  }
  // ---- the three-body (eeI) Jastrow, built as WaveFunction does with -j
  // (WaveFunction.cpp:97-100, nio.hpp buildJeeI): variant "q" on the
  // reference's own ions (every ion in group 0), variant "g" with the ions
  // split into their species (0-15 group 0, 16-31 group 1)
  for (int variant = 0; variant < 2; ++variant)
  {
    const char* tag = variant == 0 ? "q" : "g";
    std::vector<int> saved(ions.GroupID.begin(), ions.GroupID.end());
    if (variant == 1)
      for (int i = 0; i < I; ++i)
        ions.GroupID[i] = i < 16 ? 0 : 1;
    RandomGenerator<RealType> rng3(myPrimes[1]);
    ParticleSet e3;
    build_els(e3, ions, rng3);
    e3.addTable(e3, DT_SOA);
    ThreeBodyJastrow<PolynomialFunctor3D> J3(ions, e3);
    buildJeeI(J3, e3.Lattice.WignerSeitzRadius);
    e3.update();
    char key[64];
    if (variant == 0)
    {
      // buildJeeI's functors, captured through its addFunc interface
      struct Capture
      {
        using FuncType = PolynomialFunctor3D;
        PolynomialFunctor3D* f[2][2][2] = {};
        void addFunc(int i, int a, int b, PolynomialFunctor3D* p) { f[i][a][b] = p; }
      } cap;
      buildJeeI(cap, e3.Lattice.WignerSeitzRadius);
      printf("\"j3_rcut\": %.17g,\n", cap.f[0][0][0]->cutoff_radius);
      const char* names[4] = {"j3_gamma_uu0", "j3_gamma_ud0", "j3_gamma_uu1", "j3_gamma_ud1"};
      for (int q = 0; q < 4; ++q)
      {
        const PolynomialFunctor3D* f = cap.f[q / 2][0][q % 2];
        std::vector<double> gm;
        for (int l = 0; l < 4; ++l)
          for (int m = 0; m < 4; ++m)
            for (int n = 0; n < 4; ++n)
              gm.push_back(f->gamma(l, m, n));
        arr(names[q], gm.data(), gm.size());
      }
      std::vector<double> ev;
      for (auto pt : std::vector<std::array<double, 3>>{{1.1, 0.7, 1.3}, {0.4, 2.0, 0.9}, {2.5, 1.6, 1.7}})
      {
        TinyVector<RealType, 3> g;
        Tensor<RealType, 3> h;
        const double v = cap.f[0][0][1]->evaluate(pt[0], pt[1], pt[2], g, h);
        ev.push_back(v);
        for (int d = 0; d < 3; ++d)
          ev.push_back(g[d]);
        ev.push_back(h(0, 0)), ev.push_back(h(0, 1)), ev.push_back(h(0, 2));
        ev.push_back(h(1, 1)), ev.push_back(h(1, 2)), ev.push_back(h(2, 2));
      }
      arr("j3_ud0_eval_val_grad3_hess6", ev.data(), ev.size());
    }
    auto p0 = flat(e3.R);
    snprintf(key, sizeof(key), "j3%s_R0", tag);
    arr(key, p0.data(), p0.size());
    e3.G = 0.0;
    e3.L = 0.0;
    const double l3 = J3.evaluateLog(e3, e3.G, e3.L);
    printf("\"j3%s_log\": %.17g,\n", tag, l3);
    std::vector<double> g, l;
    for (int i = 0; i < N; ++i)
    {
      for (int d = 0; d < 3; ++d)
        g.push_back(e3.G[i][d]);
      l.push_back(e3.L[i]);
    }
    snprintf(key, sizeof(key), "j3%s_G", tag);
    arr(key, g.data(), g.size());
    snprintf(key, sizeof(key), "j3%s_L", tag);
    arr(key, l.data(), l.size());
    // one substep of the move protocol with J3 only, continuing the stream
    std::vector<double> ur(N);
    ParticlePos_t delta(N);
    rng3.generate_uniform(ur.data(), N);
    rng3.generate_normal(&delta[0][0], 3 * N);
    std::vector<double> ratios, gnew, gnow;
    std::vector<int> acc;
    for (int iel = 0; iel < N; ++iel)
    {
      e3.setActive(iel);
      PosType g0 = J3.evalGrad(e3, iel);
      e3.makeMove(iel, delta[iel]);
      PosType gn(0.0);
      ratios.push_back(J3.ratioGrad(e3, iel, gn));
      for (int d = 0; d < 3; ++d)
        gnew.push_back(gn[d]), gnow.push_back(g0[d]);
      if (ur[iel] < 0.5)
      {
        J3.acceptMove(e3, iel);
        e3.acceptMove(iel);
        acc.push_back(1);
      }
      else
      {
        e3.rejectMove(iel);
        acc.push_back(0);
      }
    }
    e3.donePbyP();
    e3.G = 0.0;
    e3.L = 0.0;
    J3.evaluateGL(e3, e3.G, e3.L);
    snprintf(key, sizeof(key), "j3%s_sweep_ratio", tag);
    arr(key, ratios.data(), ratios.size());
    snprintf(key, sizeof(key), "j3%s_sweep_grad_new", tag);
    arr(key, gnew.data(), gnew.size());
    snprintf(key, sizeof(key), "j3%s_sweep_grad_now", tag);
    arr(key, gnow.data(), gnow.size());
    snprintf(key, sizeof(key), "j3%s_sweep_accept", tag);
    arri(key, acc.data(), acc.size());
    printf("\"j3%s_sweep_log\": %.17g,\n", tag, J3.LogValue);
    g.clear(), l.clear();
    for (int i = 0; i < N; ++i)
    {
      for (int d = 0; d < 3; ++d)
        g.push_back(e3.G[i][d]);
      l.push_back(e3.L[i]);
    }
    snprintf(key, sizeof(key), "j3%s_sweep_G", tag);
    arr(key, g.data(), g.size());
    snprintf(key, sizeof(key), "j3%s_sweep_L", tag);
    arr(key, l.data(), l.size());
    for (int i = 0; i < I; ++i)
      ions.GroupID[i] = saved[i];
  }
  {
    // NonLocalPP's rotated quadrature spheres of its first three randomize
    // calls (its constructor reseeds its own stream with 11)
    RandomGenerator<double> rng(7);
    NonLocalPP<double> ecp(rng, ions);
    ParticleSet::ParticlePos_t rot(ecp.size());
    std::vector<double> v;
    for (int c = 0; c < 3; ++c)
    {
      ecp.randomize(rot);
      for (int k = 0; k < ecp.size(); ++k)
        for (int d = 0; d < 3; ++d)
          v.push_back(rot[k][d]);
    }
    arr("nlpp_spheres", v.data(), v.size(), false);
  }
  printf("}\n");
  return 0;
}
