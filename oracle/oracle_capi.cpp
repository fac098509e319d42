// oracle_capi.cpp -- extern "C" surface of the CPU FP64 oracle.
//
// TEST INFRASTRUCTURE ONLY (the checker).  The functions mirror the product's
// qmc_* C ABI (include/qmcgpu.h) one to one, prefixed oracle_, so a parity
// test drives both sides with identical calls.  Built into oracle/liboracle.so
// by oracle/Makefile; the product never links it.
#include "qmc_oracle.hpp"
#include "../include/qmcgpu.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace oracle;

struct oracle_system
{
  System sys;
};
struct oracle_walkers
{
  oracle_system* s;
  int W, k;
  std::vector<Walker> w;
  int nlpp_calls = 0;
};

static Functor to_functor(const qmc_functor& f)
{
  Functor F;
  F.SplineCoefs.assign(f.coefs, f.coefs + f.n_coefs);
  F.cutoff_radius = f.cutoff;
  F.DeltaRInv     = f.delta_r_inv;
  F.DeltaR        = 1.0 / f.delta_r_inv;
  return F;
}

extern "C" {

// ------------------------------------------------------------- helpers --
int oracle_rng_uniform(uint32_t seed, int n, double* out)
{
  Rng r(seed);
  r.uniform(out, n);
  return 0;
}
int oracle_rng_normal(uint32_t seed, int n_skip_uniform, int n, double* out)
{
  Rng r(seed);
  for (int i = 0; i < n_skip_uniform; ++i)
    r();
  r.normal(out, n);
  return 0;
}
int oracle_rng_words(uint32_t seed, int n, uint32_t* out)
{
  std::mt19937 mt(seed);
  for (int i = 0; i < n; ++i)
    out[i] = mt();
  return 0;
}
int oracle_primes(int n, uint32_t* out)
{
  auto p = primes(n);
  std::copy(p.begin(), p.end(), out);
  return 0;
}
double oracle_splitmix_uniform(uint64_t seed, uint64_t index) { return splitmix_uniform(seed, index); }

int oracle_lattice_ws_radius(const double* lattice, double* ws)
{
  Lattice L(lattice);
  *ws = L.WignerSeitzRadius;
  return 0;
}
// one row of DTD_BConds::computeDistances; dr is [n][3]
int oracle_distance_row(const double* lattice, const double* pos, const double* P, int n, int flip_ind,
                        double* r, double* dr)
{
  Lattice L(lattice);
  std::vector<double> dx(n), dy(n), dz(n);
  L.computeDistances(Vec3{pos[0], pos[1], pos[2]}, P, r, dx.data(), dy.data(), dz.data(), 0, n,
                     flip_ind);
  for (int i = 0; i < n; ++i)
    dr[3 * i] = dx[i], dr[3 * i + 1] = dy[i], dr[3 * i + 2] = dz[i];
  return 0;
}

int oracle_functor_setup(int n_params, double rcut, double cusp, const double* params, qmc_functor* out)
{
  if (n_params + 4 > QMC_MAX_FUNCTOR_COEFS || n_params < 2)
    return QMC_ERR_ARG;
  Functor F;
  F.setup(n_params, rcut, cusp, params);
  std::memset(out, 0, sizeof(*out));
  out->n_coefs     = (int)F.SplineCoefs.size();
  out->cutoff      = F.cutoff_radius;
  out->delta_r_inv = F.DeltaRInv;
  std::copy(F.SplineCoefs.begin(), F.SplineCoefs.end(), out->coefs);
  return 0;
}
// u, du/dr, d2u/dr2 (BsplineFunctor::evaluate)
int oracle_functor_eval(const qmc_functor* f, double r, double* out3)
{
  Functor F = to_functor(*f);
  out3[0]   = F.evaluate(r, out3[1], out3[2]);
  return 0;
}

int oracle_nio_count(int cell, int na, int nb, int nc, int* n_ions)
{
  *n_ions = (cell == QMC_NIO_REF32 ? 32 : 4) * na * nb * nc;
  return 0;
}
int oracle_nio_build(int cell, int na, int nb, int nc, int quirks, double* lattice, double* ion_pos,
                     int* ion_group, int* n_groups, double* spo_lattice)
{
  IonSet s = cell == QMC_NIO_REF32 ? build_nio_ref32(na, nb, nc, quirks) : build_nio_prim4(na, nb, nc);
  std::memcpy(lattice, s.lattice, sizeof(s.lattice));
  std::memcpy(spo_lattice, s.spo_lattice, sizeof(s.spo_lattice));
  std::copy(s.pos.begin(), s.pos.end(), ion_pos);
  std::copy(s.group.begin(), s.group.end(), ion_group);
  *n_groups = s.n_groups;
  return (int)s.group.size();
}
// buildJ1 / buildJ2 (nio.hpp:81-168)
int oracle_nio_jastrows(const double* lattice, qmc_functor* j1_O, qmc_functor* j1_Ni, qmc_functor* j2_uu,
                        qmc_functor* j2_ud)
{
  Lattice L(lattice);
  const double ws  = L.WignerSeitzRadius;
  const double Yuu[10] = {0.3062333936, 0.2068358231, 0.1324267459, 0.08673342451, 0.05641590391,
                          0.03626533946, 0.02269217959, 0.01331043612, 0.006750919735, 0.002827476478};
  const double Yud[10] = {0.4397856796, 0.2589475889, 0.1516634434, 0.08962897215, 0.05676614496,
                          0.03675758961, 0.02294244601, 0.01343860721, 0.00681803725, 0.002864695148};
  const double YO[10]  = {-1.060468469,  -0.9741652012, -0.8785027166, -0.6350075366, -0.3276892194,
                          -0.08646817952, -0.07340983171, -0.0377479213, -0.01507835571, -0.001101691898};
  const double YNi[10] = {-3.058259288, -3.077898004, -2.51188807,  -1.570208063,  -0.6204423266,
                          0.06272826611, 0.06228214399, 0.06665099211, 0.03230352443, 0.009254036239};
  const double rc2 = std::min(ws, 5.5727792532);
  const double rc1 = std::min(ws, 4.8261684030);
  oracle_functor_setup(10, rc2, 0.0, Yuu, j2_uu);
  oracle_functor_setup(10, rc2, 0.0, Yud, j2_ud);
  oracle_functor_setup(10, rc1, -0.25, YO, j1_O);
  oracle_functor_setup(10, rc1, -0.25, YNi, j1_Ni);
  return 0;
}

// PolynomialFunctor3D::reset_gamma (PolynomialFunctor3D.h:113-250)
int oracle_j3_functor_setup(double rcut, const double* params, qmc_j3_functor* out)
{
  J3Func f;
  f.setup(rcut, params);
  out->cutoff = f.cutoff_radius;
  for (int l = 0; l < 4; ++l)
    for (int m = 0; m < 4; ++m)
      for (int n = 0; n < 4; ++n)
        out->gamma[16 * l + 4 * m + n] = f.gamma[l][m][n];
  return 0;
}
static J3Func to_j3(const qmc_j3_functor& q)
{
  J3Func f;
  f.cutoff_radius = q.cutoff;
  for (int l = 0; l < 4; ++l)
    for (int m = 0; m < 4; ++m)
      for (int n = 0; n < 4; ++n)
        f.gamma[l][m][n] = q.gamma[16 * l + 4 * m + n];
  return f;
}
// PolynomialFunctor3D::evaluate(r12, r1I, r2I, grad, hess): out = value,
// grad[3], hess 00 01 02 11 12 22
int oracle_j3_functor_eval(const qmc_j3_functor* q, double r12, double r1I, double r2I, double* out10)
{
  const J3Func f = to_j3(*q);
  out10[0]       = f.eval(r12, r1I, r2I, out10 + 1, out10 + 4);
  return 0;
}
// buildJeeI (nio.hpp:171-245)
int oracle_nio_j3(const double* lattice, qmc_j3_functor* same, qmc_j3_functor* diff)
{
  Lattice L(lattice);
  const double rcut = std::min(L.WignerSeitzRadius, 4.8261684030);
  static const double Y[4][QMC_J3_PARAMS] = {
      {-0.003356164484, 0.002412623253, 0.01653623839, 0.0008341346169, -0.002808360734, 0.000710697475,
       0.01076942152, 0.0009228283355, 0.01576022161, -0.003585259096, 0.003323106938, -0.02282975998,
       -0.002246144403, -0.007196992871, -0.00404316239, 0.001465337212, 0.02026982926, -0.03528735393,
       0.04594087928, -0.008776410679, -0.001552528476, -0.005554407743, 0.001858594451, 0.002001634408,
       0.0009302256139, -0.0006304447229},
      {-0.006861627197, 0.003278047306, 0.03324006545, 0.003097361067, -0.004710623571, 9.652180317e-06,
       0.02212708787, -0.003718893286, 0.03390124932, -0.00710566395, 0.008807743592, -0.04281661568,
       -0.008463011294, -0.01269994613, -0.002005229447, 0.002186590944, 0.03350196472, -0.05677253817,
       0.07810604648, -0.009629896208, -0.006372643712, -0.01056861605, 0.002485188615, 0.008392442289,
       1.073423014e-05, -0.0004812466328},
      {-0.003775082438, -0.00169971229, 0.02162925441, 0.005674020544, -0.0008296047161, 0.00128057705,
       0.005487203215, 0.001637322446, 0.02976838198, -0.0003207100945, 0.01143855436, -0.05336741304,
       -0.00732359381, -0.01556942626, 0.0001149478453, 0.001838601199, 0.02570154203, -0.0675325214,
       0.1080671614, -0.01258358969, 0.001839834045, -0.02422400426, 0.005154953014, 0.003510582598,
       0.007464427016, -0.002454817757},
      {-0.009590393593, 0.002498010871, 0.04225872633, 0.00460311261, -0.01071033503, 0.001253155062,
       0.02934351285, -0.01823794726, 0.07224890393, -0.01020046849, 0.006310807929, -0.05655009412,
       -0.0363775247, 0.002062411388, 0.02037856173, 0.003372676617, 0.03915277249, -0.02680556816,
       0.08648136635, 0.01499088063, -0.02231984329, -0.02399792096, 0.001105720128, 0.02196005181,
       0.003162638982, -0.00119645772}};
  for (int s = 0; s < 2; ++s)
  {
    oracle_j3_functor_setup(rcut, Y[2 * s], same + s);
    oracle_j3_functor_setup(rcut, Y[2 * s + 1], diff + s);
  }
  return 0;
}

// -------------------------------------------------------------- system --
int oracle_system_create(const qmc_system_desc* d, int precision, oracle_system** out)
{
  const int comp0 = d && d->components ? d->components : QMC_WF_ALL;
  if (!d || !out || d->n_elec <= 0 || d->n_orb <= 0 ||
      ((comp0 & QMC_WF_DET) && (d->n_up != d->n_orb || d->n_elec - d->n_up != d->n_orb)))
    return QMC_ERR_ARG;
  auto* o  = new oracle_system;
  System& s = o->sys;
  s.lattice.set(d->lattice);
  s.spo_lattice.set(d->spo_lattice);
  s.n_ions   = d->n_ions;
  s.n_groups = d->n_ion_groups;
  s.n_elec   = d->n_elec;
  s.n_up     = d->n_up;
  s.norb     = d->n_orb;
  s.ion_pos.assign(d->ion_pos, d->ion_pos + 3 * (size_t)d->n_ions);
  s.ion_group.assign(d->ion_group, d->ion_group + d->n_ions);
  s.group_first.assign(s.n_groups, 0);
  s.group_last.assign(s.n_groups, 0);
  for (int g = 0; g < s.n_groups; ++g)
  {
    int f = -1, l = -1;
    for (int i = 0; i < s.n_ions; ++i)
      if (s.ion_group[i] == g)
      {
        if (f < 0)
          f = i;
        l = i + 1;
      }
    s.group_first[g] = f < 0 ? 0 : f;
    s.group_last[g]  = f < 0 ? 0 : l;
  }
  s.spline.allocate(d->grid[0], d->grid[1], d->grid[2], d->n_orb);
  if (d->spo_fill == QMC_FILL_REFERENCE)
    s.spline.fill_reference((uint32_t)d->spo_seed);
  else if (d->spo_fill == QMC_FILL_UNIFORM || d->spo_fill == QMC_FILL_UNIFORM_F32)
  {
    s.spline.fill_uniform(d->spo_seed);
    if (d->spo_fill == QMC_FILL_UNIFORM_F32)
      s.spline.round_to_float();
  }
  else
    std::copy(d->spo_user_coefs, d->spo_user_coefs + s.spline.coefs.size(), s.spline.coefs.begin());
  if (precision == QMC_PREC_MIXED)
    s.spline.round_to_float();
  s.lap_mode = d->lap_mode;
  const int comp = d->components ? d->components : QMC_WF_ALL;
  s.use_det  = (comp & QMC_WF_DET) != 0;
  s.use_j1   = (comp & QMC_WF_J1) != 0;
  s.use_j2   = (comp & QMC_WF_J2) != 0;
  s.use_j3   = (comp & QMC_WF_J3) != 0;
  if (s.use_j3)
    for (int g = 0; g < s.n_groups; ++g)
    {
      s.j3_same.push_back(to_j3(d->j3_same[g]));
      s.j3_diff.push_back(to_j3(d->j3_diff[g]));
    }
  for (int g = 0; g < s.n_groups; ++g)
    s.j1.push_back(to_functor(d->j1[g]));
  s.j2_uu = to_functor(d->j2_uu);
  s.j2_ud = to_functor(d->j2_ud);
  *out    = o;
  return 0;
}
int oracle_system_destroy(oracle_system* s)
{
  delete s;
  return 0;
}
int oracle_spo_evaluate_vgh(oracle_system* o, int n_pos, const double* pos, double* v, double* g, double* h)
{
  const System& s = o->sys;
  const int n     = s.norb;
  std::vector<double> vv(n), gg(3 * n), hh(6 * n);
  for (int p = 0; p < n_pos; ++p)
  {
    Vec3 u = s.spo_lattice.toUnit_floor(Vec3{pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]});
    s.spline.evaluate_vgh(u, vv.data(), gg.data(), hh.data());
    if (v)
      std::copy(vv.begin(), vv.end(), v + (size_t)p * n);
    if (g)
      std::copy(gg.begin(), gg.end(), g + (size_t)p * 3 * n);
    if (h)
      std::copy(hh.begin(), hh.end(), h + (size_t)p * 6 * n);
  }
  return 0;
}
int oracle_spo_evaluate_v(oracle_system* o, int n_pos, const double* pos, double* v)
{
  const System& s = o->sys;
  for (int p = 0; p < n_pos; ++p)
  {
    Vec3 u = s.spo_lattice.toUnit_floor(Vec3{pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]});
    s.spline.evaluate_v(u, v + (size_t)p * s.norb);
  }
  return 0;
}

// ------------------------------------------------------------- walkers --
// Oracle only: the arithmetic of the orbital and determinant path of the
// walkers created afterwards on this system (each walker keeps the flags it
// was created with; ARITH_* of qmc_oracle.hpp, 0 = FP64).  ARITH_SPO32 |
// ARITH_DET32 | ARITH_LOG32 restates the reference's mixed-precision build
// of that path.
int oracle_system_set_arith(oracle_system* s, int flags)
{
  if (!s || flags < 0 || flags > (ARITH_SPO32 | ARITH_DET32 | ARITH_LOG32))
    return QMC_ERR_ARG;
  s->sys.arith = flags;
  return 0;
}

int oracle_walkers_create(oracle_system* s, int W, int k, oracle_walkers** out)
{
  if (!s || W <= 0 || k <= 0 || k > s->sys.norb)
    return QMC_ERR_ARG;
  auto* o = new oracle_walkers{s, W, k, std::vector<Walker>(W)};
  for (auto& w : o->w)
    w.init(&s->sys, k);
  *out = o;
  return 0;
}
int oracle_walkers_destroy(oracle_walkers* w)
{
  delete w;
  return 0;
}
int oracle_walkers_init_random(oracle_walkers* o, const uint32_t* seeds)
{
  for (int i = 0; i < o->W; ++i)
    o->w[i].init_random(seeds[i]);
  return 0;
}
int oracle_walkers_set_positions(oracle_walkers* o, const double* R)
{
  const size_t N3 = 3 * (size_t)o->s->sys.n_elec;
  for (int i = 0; i < o->W; ++i)
    std::copy(R + i * N3, R + (i + 1) * N3, o->w[i].R.begin());
  return 0;
}
int oracle_walkers_get_positions(oracle_walkers* o, double* R)
{
  const size_t N3 = 3 * (size_t)o->s->sys.n_elec;
  for (int i = 0; i < o->W; ++i)
    std::copy(o->w[i].R.begin(), o->w[i].R.end(), R + i * N3);
  return 0;
}
// skip n uniform draws on every walker stream (keeps host/device streams aligned)
int oracle_walkers_skip(oracle_walkers* o, int n)
{
  for (auto& w : o->w)
    for (int i = 0; i < n; ++i)
      w.rng();
  return 0;
}

int oracle_pset_make_move(oracle_walkers* o, int iat, const double* displ)
{
  for (int i = 0; i < o->W; ++i)
    o->w[i].makeMove(iat, Vec3{displ[3 * i], displ[3 * i + 1], displ[3 * i + 2]});
  return 0;
}
int oracle_pset_accept_reject(oracle_walkers* o, int iat, const int* accept)
{
  for (int i = 0; i < o->W; ++i)
  {
    if (accept[i])
    {
      if (!o->w[i].acceptMove_pset(iat))
        return QMC_ERR_STATE;
    }
    else
      o->w[i].rejectMove_pset(iat);
  }
  return 0;
}
int oracle_pset_get_temp_rows(oracle_walkers* o, double* aa_r, double* aa_dr, double* ab_r, double* ab_dr)
{
  const int N = o->s->sys.n_elec, I = o->s->sys.n_ions;
  for (int i = 0; i < o->W; ++i)
  {
    const Walker& w = o->w[i];
    for (int j = 0; j < N; ++j)
    {
      if (aa_r)
        aa_r[(size_t)i * N + j] = w.aa_r[j];
      if (aa_dr)
      {
        aa_dr[((size_t)i * N + j) * 3]     = w.aa_dx[j];
        aa_dr[((size_t)i * N + j) * 3 + 1] = w.aa_dy[j];
        aa_dr[((size_t)i * N + j) * 3 + 2] = w.aa_dz[j];
      }
    }
    for (int j = 0; j < I; ++j)
    {
      if (ab_r)
        ab_r[(size_t)i * I + j] = w.ab_r[j];
      if (ab_dr)
      {
        ab_dr[((size_t)i * I + j) * 3]     = w.ab_dx[j];
        ab_dr[((size_t)i * I + j) * 3 + 1] = w.ab_dy[j];
        ab_dr[((size_t)i * I + j) * 3 + 2] = w.ab_dz[j];
      }
    }
  }
  return 0;
}

int oracle_wf_evaluate_log(oracle_walkers* o, double* logpsi)
{
  int st = 0;
  for (int i = 0; i < o->W; ++i)
  {
    if (!o->w[i].evaluateLog())
      st = QMC_ERR_SINGULAR;
    if (logpsi)
      logpsi[i] = o->w[i].LogValue;
  }
  return st;
}
int oracle_wf_eval_grad(oracle_walkers* o, int iat, double* grad)
{
  for (int i = 0; i < o->W; ++i)
  {
    Vec3 g = o->w[i].evalGrad(iat);
    for (int c = 0; c < 3; ++c)
      grad[3 * i + c] = g[c];
  }
  return 0;
}
int oracle_wf_ratio_grad(oracle_walkers* o, int iat, double* ratio, double* grad)
{
  for (int i = 0; i < o->W; ++i)
  {
    Vec3 g;
    ratio[i] = o->w[i].ratioGrad(iat, g);
    for (int c = 0; c < 3; ++c)
      grad[3 * i + c] = g[c];
  }
  return 0;
}
int oracle_wf_ratio(oracle_walkers* o, int iat, double* ratio)
{
  for (int i = 0; i < o->W; ++i)
    ratio[i] = o->w[i].ratio(iat);
  return 0;
}
int oracle_wf_evaluate_ratios(oracle_walkers* o, int walker, int iat, int n_pos, const double* pos, double* ratios)
{
  if (!o || walker < 0 || walker >= o->W || iat < 0 || iat >= o->w[walker].sys->n_elec || n_pos < 0)
    return 1;
  o->w[walker].evaluateRatios(iat, n_pos, pos, ratios);
  return 0;
}
int oracle_wf_accept_restore(oracle_walkers* o, int iat, const int* accept)
{
  for (int i = 0; i < o->W; ++i)
    if (accept[i])
      o->w[i].acceptMove(iat);
  return 0;
}
int oracle_wf_complete_updates(oracle_walkers* o)
{
  for (auto& w : o->w)
    w.completeUpdates();
  return 0;
}
int oracle_wf_evaluate_gl(oracle_walkers* o, double* G, double* L, double* logpsi)
{
  const int N = o->s->sys.n_elec;
  for (int i = 0; i < o->W; ++i)
  {
    Walker& w = o->w[i];
    w.evaluateGL();
    if (G)
      std::copy(w.G.begin(), w.G.end(), G + (size_t)i * 3 * N);
    if (L)
      std::copy(w.L.begin(), w.L.end(), L + (size_t)i * N);
    if (logpsi)
      logpsi[i] = w.LogValue;
  }
  return 0;
}
int oracle_wf_components(oracle_walkers* o, double* comp)
{
  for (int i = 0; i < o->W; ++i)
  {
    const Walker& w = o->w[i];
    comp[7 * i + 0] = w.det[0].LogValue;
    comp[7 * i + 1] = w.det[1].LogValue;
    comp[7 * i + 2] = w.det[0].PhaseValue;
    comp[7 * i + 3] = w.det[1].PhaseValue;
    comp[7 * i + 4] = w.j1_LogValue;
    comp[7 * i + 5] = w.j2_LogValue;
    comp[7 * i + 6] = w.j3_LogValue;
  }
  return 0;
}
int oracle_wf_get_inverse(oracle_walkers* o, int walker, int spin, double* psiM)
{
  Walker& w = o->w[walker];
  // apply pending delayed rows on a copy (the state itself is untouched)
  Walker::Det d = w.det[spin];
  if (w.arith & ARITH_DET32)
  {
    d.eng32.updateInvMat(d.psiM32.data());
    std::copy(d.psiM32.begin(), d.psiM32.end(), psiM);
    return 0;
  }
  d.eng.updateInvMat(d.psiM.data());
  std::copy(d.psiM.begin(), d.psiM.end(), psiM);
  return 0;
}

// The fused PbyP sweep (miniqmc.cpp:406-468) over every walker, OpenMP
// parallel over walkers (one walker per thread, as the reference driver).
int oracle_sweep(oracle_walkers* o, const qmc_sweep_opts* opt)
{
  const System& s = o->s->sys;
  const int N = s.n_elec, W = o->W, nsub = opt->n_substeps;
  int status  = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(| : status)
  for (int iw = 0; iw < W; ++iw)
  {
    Walker& w = o->w[iw];
    std::vector<double> ur(N), delta((size_t)3 * N);
    int64_t acc = 0;
    for (int mc = 0; mc < opt->n_steps; ++mc)
    {
      for (int l = 0; l < nsub; ++l)
      {
        const size_t blk = (((size_t)mc * W + iw) * nsub + l);
        if (opt->rng_mode == QMC_RNG_HOST)
        {
          std::copy_n(opt->ur + blk * N, N, ur.data());
          std::copy_n(opt->delta + blk * 3 * N, 3 * N, delta.data());
        }
        else
        {
          w.rng.uniform(ur.data(), N);
          w.rng.normal(delta.data(), 3 * N);
        }
        for (int iel = 0; iel < N; ++iel)
        {
          Vec3 grad_now = w.evalGrad(iel);
          w.makeMove(iel, Vec3{delta[3 * iel], delta[3 * iel + 1], delta[3 * iel + 2]});
          Vec3 grad_new;
          double ratio   = w.ratioGrad(iel, grad_new);
          const bool acc_move = ur[iel] < opt->accept;
          if (acc_move)
          {
            w.acceptMove(iel);
            w.acceptMove_pset(iel);
            acc++;
          }
          else
            w.rejectMove_pset(iel);
          if (opt->trace)
          {
            double* t = opt->trace + (blk * N + iel) * 8;
            t[0]      = ratio;
            t[1] = grad_new[0], t[2] = grad_new[1], t[3] = grad_new[2];
            t[4] = grad_now[0], t[5] = grad_now[1], t[6] = grad_now[2];
            t[7] = acc_move ? 1.0 : 0.0;
          }
        }
        w.completeUpdates();
      }
      w.activePtcl = -1; // donePbyP
      w.evaluateGL();
      if (opt->recompute_every > 0 && (mc + 1) % opt->recompute_every == 0)
      {
        for (int sp = 0; sp < 2; ++sp)
          if (!w.det_recompute(sp))
            status |= 1;
        w.evaluateGL();
      }
    }
    if (opt->n_accepted)
      opt->n_accepted[iw] = acc;
    if (opt->logpsi)
      opt->logpsi[iw] = w.LogValue;
  }
  return status ? QMC_ERR_SINGULAR : 0;
}

int oracle_num_threads()
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// ---------------------------------------------- DelayedUpdate engine ---
struct oracle_detengine
{
  int n, k;
  std::vector<double> psiM;
  DelayedUpdate eng;
};
int oracle_detengine_create(int n, int k, oracle_detengine** out)
{
  auto* e = new oracle_detengine{n, k, std::vector<double>((size_t)n * n), DelayedUpdate()};
  e->eng.resize(n, k);
  *out = e;
  return 0;
}
int oracle_detengine_destroy(oracle_detengine* e)
{
  delete e;
  return 0;
}
// invert_transpose(logdetT = a) -> psiM (DiracMatrix.h:93-119)
int oracle_detengine_invert_transpose(oracle_detengine* e, const double* a, double* logdet, double* phase)
{
  bool ok             = invert_transpose(e->n, a, e->psiM.data(), *logdet, *phase);
  e->eng.delay_count  = 0;
  return ok ? 0 : QMC_ERR_SINGULAR;
}
int oracle_detengine_get_inv_row(oracle_detengine* e, int row, double* invRow)
{
  e->eng.getInvRow(e->psiM.data(), row, invRow);
  return 0;
}
int oracle_detengine_accept_row(oracle_detengine* e, int row, const double* psiV)
{
  e->eng.acceptRow(e->psiM.data(), row, psiV);
  return 0;
}
int oracle_detengine_update_inv_mat(oracle_detengine* e)
{
  e->eng.updateInvMat(e->psiM.data());
  return 0;
}
int oracle_detengine_get_ainv(oracle_detengine* e, double* ainv)
{
  std::copy(e->psiM.begin(), e->psiM.end(), ainv);
  return 0;
}
int oracle_detengine_delay_count(oracle_detengine* e) { return e->eng.delay_count; }

int oracle_nlpp_sphere(int n_calls, double* out)
{
  for (int c = 0; c < n_calls; ++c)
    nlpp_sphere(c, reinterpret_cast<double(*)[3]>(out + (size_t)c * 36));
  return 0;
}

int oracle_nlpp_evaluate(oracle_walkers* o, double rmax, int form, int64_t* n_points, double* wsum, double* ratios,
                         int max_ratios)
{
  double rot[12][3];
  nlpp_sphere(o->nlpp_calls++, rot);
  std::vector<double> out;
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < o->W; ++i)
  {
    long long cnt = 0;
    const double s = o->w[i].nlpp(rmax, form, rot, cnt, (i == 0 && ratios) ? &out : nullptr);
    if (wsum)
      wsum[i] = s;
    if (n_points)
      n_points[i] = cnt;
  }
  if (ratios)
    for (int j = 0; j < max_ratios && j < (int)out.size(); ++j)
      ratios[j] = out[j];
  return 0;
}

} // extern "C"
