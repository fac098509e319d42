// qmc_oracle.hpp -- CPU FP64 restatement of miniqmc's VMC walker hot path.
//
// TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, the smoke check and
// the CPU-baseline leg of bench.py may call it; the product (libqmcgpu.so)
// never links, loads or calls it.
//
// Every routine restates the reference algorithm (QMCPACK/miniqmc, CPU
// branch) in plain loops, in the reference's order of operations, and cites
// the file:line it follows.  Differences are deliberate and listed:
//   * distance-table rows are computed on demand instead of stored (the
//     values are the ones the reference's setActive / move rows hold);
//   * BLAS gemv/ger/gemm and LAPACK getrf/getri are written out as loops
//     (same mathematics, row-major reading of the reference's column-major
//     calls -- DelayedUpdate.h:96-231, DiracMatrix.h:93-119).
// Third-party arithmetic: libstdc++ (GCC 13) std::mt19937 and
// std::uniform_real_distribution<double> (generate_canonical, 2 words per
// double), exactly what StdRandom.h:19-110 uses, plus glibc log/cos/sin for
// BoxMuller2 (RandomGenerator.h:46-79).
//
// Pinned by: the reference unit tests' known answers
// (test_dirac_matrix.cpp:44-162, test_dirac_det.cpp:196-515,
// test_particle.cpp:31-61, test_PrimeNumberSet.cpp), the values printed by
// the reference check_wfc driver, and golden dumps produced by compiling the
// reference's own headers (oracle/ref_harness.cpp) -- see tests/golden.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

namespace oracle
{
using Vec3 = std::array<double, 3>;
constexpr double kPi = 3.14159265358979323846;

// ---------------------------------------------------------------- RNG ----
// StdRandom<double, std::mt19937> (StdRandom.h:19-110)
struct Rng
{
  std::mt19937 mt;
  std::uniform_real_distribution<double> uni; // default [0,1)
  explicit Rng(uint32_t seed = 5489u) : mt(seed) {}
  double operator()() { return uni(mt); }
  void uniform(double* d, int n)
  {
    for (int i = 0; i < n; ++i)
      d[i] = uni(mt);
  }
  // BoxMuller2::generate(double) (RandomGenerator.h:49-62)
  void normal(double* a, int n)
  {
    for (int i = 0; i + 1 < n; i += 2)
    {
      double temp1 = 1.0 - 0.9999999999 * (*this)(), temp2 = (*this)();
      a[i]     = std::sqrt(-2.0 * std::log(temp1)) * std::cos(6.283185306 * temp2);
      a[i + 1] = std::sqrt(-2.0 * std::log(temp1)) * std::sin(6.283185306 * temp2);
    }
    if (n % 2 == 1)
    {
      double temp1 = 1 - 0.9999999999 * (*this)(), temp2 = (*this)();
      a[n - 1]     = std::sqrt(-2.0 * std::log(temp1)) * std::cos(6.283185306 * temp2);
    }
  }
};

// PrimeNumberSet<uint32_t>() (PrimeNumberSet.h:62-90): odd primes from 3
inline std::vector<uint32_t> primes(int count)
{
  std::vector<uint32_t> p;
  p.push_back(3);
  uint32_t largest = 3;
  while ((int)p.size() < count)
  {
    largest += 2;
    bool is_prime = true;
    for (size_t j = 0; j < p.size(); j++)
    {
      if (largest % p[j] == 0)
      {
        is_prime = false;
        break;
      }
      else if (p[j] * p[j] > largest)
        break;
    }
    if (is_prime)
      p.push_back(largest);
  }
  p.resize(count);
  return p;
}

// SplitMix64 (Steele, Lea & Flood 2014): the counter-based stream behind
// QMC_FILL_UNIFORM.  value(seed, i) = mix(seed + (i+1) * golden).
inline uint64_t splitmix64(uint64_t seed, uint64_t index)
{
  uint64_t z = seed + (index + 1) * 0x9E3779B97F4A7C15ull;
  z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline double splitmix_uniform(uint64_t seed, uint64_t index)
{
  return (double)(splitmix64(seed, index) >> 11) * (1.0 / 9007199254740992.0);
}

// ------------------------------------------------------------ Lattice ----
// 3x3 helpers with the reference's formulas (TensorOps.h:123-176)
inline double det3(const double* a)
{
  return (a[0] * (a[4] * a[8] - a[5] * a[7]) + a[1] * (a[5] * a[6] - a[3] * a[8]) +
          a[2] * (a[3] * a[7] - a[4] * a[6]));
}
inline void inverse3(const double* a, double* g)
{
  double vinv = 1 / det3(a);
  g[0]        = vinv * (a[4] * a[8] - a[5] * a[7]);
  g[1]        = vinv * (a[7] * a[2] - a[8] * a[1]);
  g[2]        = vinv * (a[1] * a[5] - a[2] * a[4]);
  g[3]        = vinv * (a[5] * a[6] - a[3] * a[8]);
  g[4]        = vinv * (a[8] * a[0] - a[6] * a[2]);
  g[5]        = vinv * (a[2] * a[3] - a[0] * a[5]);
  g[6]        = vinv * (a[3] * a[7] - a[4] * a[6]);
  g[7]        = vinv * (a[6] * a[1] - a[7] * a[0]);
  g[8]        = vinv * (a[0] * a[4] - a[1] * a[3]);
}
inline double dot3(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// found_shorter_base / find_reduced_basis (LatticeAnalyzer.h:134-183)
inline bool found_shorter_base(Vec3 rb[3])
{
  const double eps = 10.0 * std::numeric_limits<float>::epsilon();
  int imax         = 0;
  double r2max     = dot3(rb[0], rb[0]);
  for (int i = 1; i < 3; i++)
  {
    double r2 = dot3(rb[i], rb[i]);
    if ((r2 - r2max) > eps)
    {
      r2max = r2;
      imax  = i;
    }
  }
  Vec3 rb_new[4];
  for (int d = 0; d < 3; ++d)
  {
    rb_new[0][d] = rb[0][d] + rb[1][d] - rb[2][d];
    rb_new[1][d] = rb[0][d] + rb[2][d] - rb[1][d];
    rb_new[2][d] = rb[1][d] + rb[2][d] - rb[0][d];
    rb_new[3][d] = rb[0][d] + rb[1][d] + rb[2][d];
  }
  for (int i = 0; i < 4; ++i)
  {
    double r2 = dot3(rb_new[i], rb_new[i]);
    if ((r2 - r2max) < -eps)
    {
      rb[imax] = rb_new[i];
      return true;
    }
  }
  return false;
}
inline void find_reduced_basis(Vec3 rb[3])
{
  do
  {
    Vec3 saved[3] = {rb[0], rb[1], rb[2]};
    bool changed  = false;
    for (int i = 0; i < 3; ++i)
    {
      rb[i]   = Vec3{0.0, 0.0, 0.0};
      changed = found_shorter_base(rb);
      rb[i]   = saved[i];
      if (changed)
        break;
    }
    if (!changed && !found_shorter_base(rb))
      return;
  } while (1);
}

// CrystalLattice<double,3> (CrystalLattice.h:168-205, CrystalLattice.cpp:88-127)
// plus DTD_BConds<double,3,PPPG+SOA_OFFSET> (ParticleBConds.h:99-217)
struct Lattice
{
  double R[9];  // rows = lattice vectors
  double G[9];  // inverse(R)
  double WignerSeitzRadius;
  double SimulationCellRadius;
  // DTD_BConds state
  double r[9], g[9]; // reduced basis (rows) and its inverse
  double corners[8][3];

  Lattice() {}
  explicit Lattice(const double* R9) { set(R9); }

  void set(const double* R9)
  {
    std::memcpy(R, R9, sizeof(R));
    inverse3(R, G);
    Vec3 a[3];
    for (int i = 0; i < 3; ++i)
      a[i] = Vec3{R[3 * i], R[3 * i + 1], R[3 * i + 2]};
    // calcWignerSeitzRadius, bulk (LatticeAnalyzer.h:86-116)
    double rMin = 0.5 * std::numeric_limits<double>::max();
    for (int i = -1; i <= 1; i++)
      for (int j = -1; j <= 1; j++)
        for (int k = -1; k <= 1; k++)
          if (i || j || k)
          {
            Vec3 L;
            for (int d = 0; d < 3; ++d)
              L[d] = (double)i * a[0][d] + (double)j * a[1][d] + (double)k * a[2][d];
            rMin = std::min(rMin, dot3(L, L));
          }
    WignerSeitzRadius = 0.5 * std::sqrt(rMin);
    // calcSimulationCellRadius (LatticeAnalyzer.h:118-131)
    double scr = 0.5 * std::numeric_limits<double>::max();
    for (int i = 0; i < 3; ++i)
    {
      const Vec3& A = a[i];
      const Vec3& B = a[(i + 1) % 3];
      const Vec3& C = a[(i + 2) % 3];
      Vec3 BxC{B[1] * C[2] - B[2] * C[1], B[2] * C[0] - B[0] * C[2], B[0] * C[1] - B[1] * C[0]};
      double dist = 0.5 * std::abs(dot3(A, BxC)) / std::sqrt(dot3(BxC, BxC));
      scr         = std::min(scr, dist);
    }
    SimulationCellRadius = scr;
    if (WignerSeitzRadius > SimulationCellRadius &&
        WignerSeitzRadius - SimulationCellRadius <=
            WignerSeitzRadius * std::numeric_limits<float>::epsilon() * 2)
      WignerSeitzRadius = SimulationCellRadius;
    // DTD_BConds ctor
    Vec3 rb[3] = {a[0], a[1], a[2]};
    find_reduced_basis(rb);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        r[3 * i + j] = rb[i][j];
    inverse3(r, g);
    for (int d = 0; d < 3; ++d)
    {
      corners[0][d] = 0.0;
      corners[1][d] = -1.0 * rb[0][d];
      corners[2][d] = -1.0 * rb[1][d];
      corners[3][d] = -1.0 * rb[2][d];
      corners[4][d] = -1.0 * (rb[0][d] + rb[1][d]);
      corners[5][d] = -1.0 * (rb[0][d] + rb[2][d]);
      corners[6][d] = -1.0 * (rb[1][d] + rb[2][d]);
      corners[7][d] = -1.0 * (rb[0][d] + rb[1][d] + rb[2][d]);
    }
  }

  // toUnit = dot(r, G) (CrystalLattice.h:180-183, TinyVectorTensorOps.h:145-154)
  Vec3 toUnit(const Vec3& x) const
  {
    return Vec3{x[0] * G[0] + x[1] * G[3] + x[2] * G[6], x[0] * G[1] + x[1] * G[4] + x[2] * G[7],
                x[0] * G[2] + x[1] * G[5] + x[2] * G[8]};
  }
  // toUnit_floor (CrystalLattice.h:185-196)
  Vec3 toUnit_floor(const Vec3& x) const
  {
    Vec3 v = toUnit(x);
    for (int i = 0; i < 3; i++)
      if (-std::numeric_limits<double>::epsilon() < v[i] && v[i] < 0)
        v[i] = 0.0;
      else
        v[i] -= std::floor(v[i]);
    return v;
  }
  // toCart = dot(u, R) (CrystalLattice.h:201-205); ConvertPosUnit order
  // (FastParticleOperators.h:44-56)
  Vec3 toCart(const Vec3& u) const
  {
    return Vec3{u[0] * R[0] + u[1] * R[3] + u[2] * R[6], u[0] * R[1] + u[1] * R[4] + u[2] * R[7],
                u[0] * R[2] + u[1] * R[5] + u[2] * R[8]};
  }

  // DTD_BConds::computeDistances (ParticleBConds.h:153-217) for one source
  // point `pos` against points P[first,last) (AoS [n][3]).
  void computeDistances(const Vec3& pos, const double* P, double* temp_r, double* dx, double* dy,
                        double* dz, int first, int last, int flip_ind = 0) const
  {
    const double x0 = pos[0], y0 = pos[1], z0 = pos[2];
    const double g00 = g[0], g01 = g[1], g02 = g[2], g10 = g[3], g11 = g[4], g12 = g[5],
                 g20 = g[6], g21 = g[7], g22 = g[8];
    const double r00 = r[0], r01 = r[1], r02 = r[2], r10 = r[3], r11 = r[4], r12 = r[5],
                 r20 = r[6], r21 = r[7], r22 = r[8];
    for (int iat = first; iat < last; ++iat)
    {
      const double flip    = iat < flip_ind ? 1.0 : -1.0;
      const double displ_0 = (P[3 * iat + 0] - x0) * flip;
      const double displ_1 = (P[3 * iat + 1] - y0) * flip;
      const double displ_2 = (P[3 * iat + 2] - z0) * flip;
      const double ar_0    = -std::floor(displ_0 * g00 + displ_1 * g10 + displ_2 * g20);
      const double ar_1    = -std::floor(displ_0 * g01 + displ_1 * g11 + displ_2 * g21);
      const double ar_2    = -std::floor(displ_0 * g02 + displ_1 * g12 + displ_2 * g22);
      const double delx    = displ_0 + ar_0 * r00 + ar_1 * r10 + ar_2 * r20;
      const double dely    = displ_1 + ar_0 * r01 + ar_1 * r11 + ar_2 * r21;
      const double delz    = displ_2 + ar_0 * r02 + ar_1 * r12 + ar_2 * r22;
      double rmin          = delx * delx + dely * dely + delz * delz;
      int ic               = 0;
      for (int c = 1; c < 8; ++c)
      {
        const double x  = delx + corners[c][0];
        const double y  = dely + corners[c][1];
        const double z  = delz + corners[c][2];
        const double r2 = x * x + y * y + z * z;
        ic              = (r2 < rmin) ? c : ic;
        rmin            = (r2 < rmin) ? r2 : rmin;
      }
      temp_r[iat] = std::sqrt(rmin);
      dx[iat]     = flip * (delx + corners[ic][0]);
      dy[iat]     = flip * (dely + corners[ic][1]);
      dz[iat]     = flip * (delz + corners[ic][2]);
    }
  }
};

// ------------------------------------------------------------- NiO ------
// nio.hpp:23-79 (32-atom cell, O then Ni in lattice units)
static const double kNioCell[9] = {7.8811, 7.8811, 0.0, -7.8811, 7.8811, 0.0, 0.0, 0.0, 15.7622};
static const double kNio32[32][3] = {
    {0.5, 0.0, 0.25},  {0.0, 0.0, 0.75},  {0.25, 0.25, 0.5},  {0.5, 0.5, 0.25},
    {0.75, 0.25, 0.0}, {0.0, 0.5, 0.75},  {0.25, 0.75, 0.5},  {0.75, 0.75, 0.0},
    {0.0, 0.0, 0.25},  {0.25, 0.25, 0.0}, {0.5, 0.0, 0.75},   {0.75, 0.25, 0.5},
    {0.0, 0.5, 0.25},  {0.25, 0.75, 0.0}, {0.5, 0.5, 0.75},   {0.75, 0.75, 0.5},
    {0.0, 0.0, 0.0},   {0.0, 0.5, 0.0},   {0.25, 0.25, 0.75}, {0.5, 0.0, 0.5},
    {0.5, 0.5, 0.5},   {0.75, 0.25, 0.25}, {0.25, 0.75, 0.75}, {0.75, 0.75, 0.25},
    {0.5, 0.0, 0.0},   {0.0, 0.0, 0.5},   {0.25, 0.25, 0.25}, {0.5, 0.5, 0.0},
    {0.75, 0.25, 0.75}, {0.0, 0.5, 0.5},  {0.25, 0.75, 0.25}, {0.75, 0.75, 0.75}};

struct IonSet
{
  double lattice[9];
  double spo_lattice[9];
  std::vector<double> pos; // [n][3]
  std::vector<int> group;
  int n_groups = 2;
};

// tile_cell + expandSuperCell (nio.hpp:23-79, ParticleIOUtility.h:29-117)
// quirks: bit0 = keep lattice units at identity tiling, bit1 = all group 0
inline IonSet build_nio_ref32(int na, int nb, int nc, int quirks)
{
  IonSet s;
  std::memcpy(s.spo_lattice, kNioCell, sizeof(kNioCell));
  const bool one_group = quirks & 2;
  std::vector<int> primTypes(32);
  for (int i = 0; i < 32; ++i)
    primTypes[i] = one_group ? 0 : (i < 16 ? 0 : 1);
  s.n_groups = 2;
  if (na == 1 && nb == 1 && nc == 1)
  {
    std::memcpy(s.lattice, kNioCell, sizeof(kNioCell));
    Lattice prim(kNioCell);
    for (int i = 0; i < 32; ++i)
    {
      Vec3 u{kNio32[i][0], kNio32[i][1], kNio32[i][2]};
      Vec3 r = (quirks & 1) ? u : prim.toCart(u);
      s.pos.insert(s.pos.end(), r.begin(), r.end());
      s.group.push_back(primTypes[i]);
    }
    return s;
  }
  // PrimCell = nio_cell; supercell = dot(tmat, PrimCell.R) (ParticleIOUtility.h:64-65)
  Lattice prim(kNioCell);
  const int t[3] = {na, nb, nc};
  double sup[9];
  // the generic Tensor dot sums k = 0,1,2 in order; off-diagonal tmat are 0
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
    {
      double sum = 0.0;
      for (int k = 0; k < 3; ++k)
        sum += (double)(i == k ? t[i] : 0) * kNioCell[3 * k + j];
      sup[3 * i + j] = sum;
    }
  std::memcpy(s.lattice, sup, sizeof(sup));
  Lattice super(sup);
  const int maxCopies = 10;
  for (int ns = 0; ns < 2; ++ns)
    for (int i0 = -maxCopies; i0 <= maxCopies; i0++)
      for (int i1 = -maxCopies; i1 <= maxCopies; i1++)
        for (int i2 = -maxCopies; i2 <= maxCopies; i2++)
          for (int iat = 0; iat < 32; iat++)
          {
            if (primTypes[iat] != ns)
              continue;
            Vec3 uPrim{kNio32[iat][0], kNio32[iat][1], kNio32[iat][2]};
            for (int i = 0; i < 3; i++)
              uPrim[i] -= std::floor(uPrim[i]);
            Vec3 c = prim.toCart(uPrim);
            Vec3 r;
            for (int d = 0; d < 3; ++d)
              r[d] = c[d] + (double)i0 * kNioCell[d] + (double)i1 * kNioCell[3 + d] +
                  (double)i2 * kNioCell[6 + d];
            Vec3 u = super.toUnit(r);
            if ((u[0] >= -1.0e-6) && (u[0] < 0.9999) && (u[1] >= -1.0e-6) && (u[1] < 0.9999) &&
                (u[2] >= -1.0e-6) && (u[2] < 0.9999))
            {
              s.pos.insert(s.pos.end(), r.begin(), r.end());
              s.group.push_back(ns);
            }
          }
  return s;
}

// 4-atom NiO cell tiled (na,nb,nc); orbitals periodic on the supercell.
inline IonSet build_nio_prim4(int na, int nb, int nc)
{
  IonSet s;
  double prim[9];
  for (int i = 0; i < 9; ++i)
    prim[i] = 0.5 * kNioCell[i];
  const int t[3] = {na, nb, nc};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      s.lattice[3 * i + j] = (double)t[i] * prim[3 * i + j];
  std::memcpy(s.spo_lattice, s.lattice, sizeof(s.lattice));
  Lattice P(prim);
  const double basis[4][3] = {{0.0, 0.0, 0.5}, {0.5, 0.5, 0.0}, {0.0, 0.0, 0.0}, {0.5, 0.5, 0.5}};
  const int species[4]     = {0, 0, 1, 1};
  for (int ns = 0; ns < 2; ++ns)
    for (int i0 = 0; i0 < na; ++i0)
      for (int i1 = 0; i1 < nb; ++i1)
        for (int i2 = 0; i2 < nc; ++i2)
          for (int b = 0; b < 4; ++b)
          {
            if (species[b] != ns)
              continue;
            Vec3 u{basis[b][0] + i0, basis[b][1] + i1, basis[b][2] + i2};
            Vec3 r = P.toCart(u);
            s.pos.insert(s.pos.end(), r.begin(), r.end());
            s.group.push_back(ns);
          }
  s.n_groups = 2;
  return s;
}

// ------------------------------------------------------- BsplineFunctor --
// BsplineFunctor<double> (BsplineFunctor.h:43-339)
struct Functor
{
  std::vector<double> SplineCoefs;
  double cutoff_radius = 0.0, DeltaR = 0.0, DeltaRInv = 0.0;
  static constexpr double A[16] = {-1.0 / 6.0, 3.0 / 6.0, -3.0 / 6.0, 1.0 / 6.0, 3.0 / 6.0, -6.0 / 6.0,
                                   0.0 / 6.0,  4.0 / 6.0, -3.0 / 6.0, 3.0 / 6.0, 3.0 / 6.0, 1.0 / 6.0,
                                   1.0 / 6.0,  0.0 / 6.0, 0.0 / 6.0,  0.0 / 6.0};
  static constexpr double dA[16]  = {0.0, -0.5, 1.0, -0.5, 0.0, 1.5, -2.0, 0.0,
                                     0.0, -1.5, 1.0, 0.5,  0.0, 0.5, 0.0,  0.0};
  static constexpr double d2A[16] = {0.0, 0.0, -1.0, 1.0, 0.0, 0.0, 3.0, -2.0,
                                     0.0, 0.0, -3.0, 1.0, 0.0, 0.0, 1.0, 0.0};

  // setupParameters + resize + reset (BsplineFunctor.h:93-130)
  void setup(int n, double rcut, double cusp, const double* params)
  {
    cutoff_radius = rcut;
    int numCoefs  = n + 4;
    int numKnots  = numCoefs - 2;
    DeltaR        = cutoff_radius / (double)(numKnots - 1);
    DeltaRInv     = 1.0 / DeltaR;
    SplineCoefs.assign(numCoefs, 0.0);
    SplineCoefs[1] = params[0];
    SplineCoefs[2] = params[1];
    SplineCoefs[0] = params[1] - 2.0 * DeltaR * cusp;
    for (int i = 2; i < n; i++)
      SplineCoefs[i + 1] = params[i];
  }
  // evaluate(r, dudr, d2udr2) (BsplineFunctor.h:186-219)
  double evaluate(double r, double& dudr, double& d2udr2) const
  {
    if (r >= cutoff_radius)
    {
      dudr = d2udr2 = 0.0;
      return 0.0;
    }
    r *= DeltaRInv;
    double ipart, t;
    t     = std::modf(r, &ipart);
    int i = (int)ipart;
    double tp[4] = {t * t * t, t * t, t, 1.0};
    const double* c = SplineCoefs.data();
    d2udr2          = DeltaRInv * DeltaRInv *
        (c[i + 0] * (d2A[0] * tp[0] + d2A[1] * tp[1] + d2A[2] * tp[2] + d2A[3] * tp[3]) +
         c[i + 1] * (d2A[4] * tp[0] + d2A[5] * tp[1] + d2A[6] * tp[2] + d2A[7] * tp[3]) +
         c[i + 2] * (d2A[8] * tp[0] + d2A[9] * tp[1] + d2A[10] * tp[2] + d2A[11] * tp[3]) +
         c[i + 3] * (d2A[12] * tp[0] + d2A[13] * tp[1] + d2A[14] * tp[2] + d2A[15] * tp[3]));
    dudr = DeltaRInv *
        (c[i + 0] * (dA[0] * tp[0] + dA[1] * tp[1] + dA[2] * tp[2] + dA[3] * tp[3]) +
         c[i + 1] * (dA[4] * tp[0] + dA[5] * tp[1] + dA[6] * tp[2] + dA[7] * tp[3]) +
         c[i + 2] * (dA[8] * tp[0] + dA[9] * tp[1] + dA[10] * tp[2] + dA[11] * tp[3]) +
         c[i + 3] * (dA[12] * tp[0] + dA[13] * tp[1] + dA[14] * tp[2] + dA[15] * tp[3]));
    return (c[i + 0] * (A[0] * tp[0] + A[1] * tp[1] + A[2] * tp[2] + A[3] * tp[3]) +
            c[i + 1] * (A[4] * tp[0] + A[5] * tp[1] + A[6] * tp[2] + A[7] * tp[3]) +
            c[i + 2] * (A[8] * tp[0] + A[9] * tp[1] + A[10] * tp[2] + A[11] * tp[3]) +
            c[i + 3] * (A[12] * tp[0] + A[13] * tp[1] + A[14] * tp[2] + A[15] * tp[3]));
  }
  // evaluateV (BsplineFunctor.h:222-263): sum over [iStart,iEnd), skipping iat
  double evaluateV(int iat, int iStart, int iEnd, const double* dist) const
  {
    double d        = 0.0;
    const double* c = SplineCoefs.data();
    for (int jat = iStart; jat < iEnd; ++jat)
    {
      double r = dist[jat];
      if (!(r < cutoff_radius && jat != iat))
        continue;
      r *= DeltaRInv;
      int i      = (int)r;
      double t   = r - double(i);
      double tp0 = t * t * t, tp1 = t * t, tp2 = t;
      double d1  = c[i + 0] * (A[0] * tp0 + A[1] * tp1 + A[2] * tp2 + A[3]);
      double d2  = c[i + 1] * (A[4] * tp0 + A[5] * tp1 + A[6] * tp2 + A[7]);
      double d3  = c[i + 2] * (A[8] * tp0 + A[9] * tp1 + A[10] * tp2 + A[11]);
      double d4  = c[i + 3] * (A[12] * tp0 + A[13] * tp1 + A[14] * tp2 + A[15]);
      d += (d1 + d2 + d3 + d4);
    }
    return d;
  }
  // evaluateVGL (BsplineFunctor.h:265-339): writes only pairs inside the cutoff
  void evaluateVGL(int iat, int iStart, int iEnd, const double* dist, double* val, double* grad,
                   double* lapl) const
  {
    const double dSquareDeltaRinv = DeltaRInv * DeltaRInv;
    const double* c               = SplineCoefs.data();
    for (int jat = iStart; jat < iEnd; ++jat)
    {
      double r = dist[jat];
      if (!(r < cutoff_radius && jat != iat))
        continue;
      double rinv   = 1.0 / r;
      r *= DeltaRInv;
      int iGather   = (int)r;
      double t      = r - double(iGather);
      double tp0    = t * t * t, tp1 = t * t, tp2 = t;
      double s0 = c[iGather], s1 = c[iGather + 1], s2 = c[iGather + 2], s3 = c[iGather + 3];
      lapl[jat] = dSquareDeltaRinv *
          (s0 * (d2A[2] * tp2 + d2A[3]) + s1 * (d2A[6] * tp2 + d2A[7]) + s2 * (d2A[10] * tp2 + d2A[11]) +
           s3 * (d2A[14] * tp2 + d2A[15]));
      grad[jat] = DeltaRInv * rinv *
          (s0 * (dA[1] * tp1 + dA[2] * tp2 + dA[3]) + s1 * (dA[5] * tp1 + dA[6] * tp2 + dA[7]) +
           s2 * (dA[9] * tp1 + dA[10] * tp2 + dA[11]) + s3 * (dA[13] * tp1 + dA[14] * tp2 + dA[15]));
      val[jat] = (s0 * (A[0] * tp0 + A[1] * tp1 + A[2] * tp2 + A[3]) +
                  s1 * (A[4] * tp0 + A[5] * tp1 + A[6] * tp2 + A[7]) +
                  s2 * (A[8] * tp0 + A[9] * tp1 + A[10] * tp2 + A[11]) +
                  s3 * (A[12] * tp0 + A[13] * tp1 + A[14] * tp2 + A[15]));
    }
  }
};

// --------------------------------------------------------- Spline SPO ---
// multi_UBspline_3d_d as created by BsplineAllocator::allocateMultiBspline
// (BsplineAllocator.hpp:84-136) on [0,1)^3 with PERIODIC ends, evaluated by
// MultiBsplineEval (MultiBspline.hpp:34-280).
struct Spline
{
  int nx = 0, ny = 0, nz = 0, norb = 0;
  double delta_inv[3];
  std::vector<double> coefs; // [(nx+3)][(ny+3)][(nz+3)][norb]
  size_t zs = 0, ys = 0, xs = 0;

  void allocate(int nx_, int ny_, int nz_, int norb_)
  {
    nx = nx_, ny = ny_, nz = nz_, norb = norb_;
    const int ng[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d)
    {
      double delta = (1.0 - 0.0) / (double)(ng[d] + 3 - 3);
      delta_inv[d] = 1.0 / delta;
    }
    zs = norb;
    ys = (size_t)(nz + 3) * zs;
    xs = (size_t)(ny + 3) * ys;
    coefs.assign((size_t)(nx + 3) * xs, 0.0);
  }
  // einspline_spo::set with init_random (einspline_spo.hpp:128-160) +
  // setCoefficientsForOrbitals (BsplineAllocator.hpp:160-182)
  void fill_reference(uint32_t seed)
  {
    Rng myrandom(seed);
    std::vector<double> coef_data((size_t)(nx + 3) * (ny + 3) * (nz + 3));
    myrandom.uniform(coef_data.data(), (int)coef_data.size());
    std::vector<double> prefactor(norb);
    for (int ind = 0; ind < norb; ind++)
      prefactor[ind] = std::cos(2 * M_PI * ind / norb);
    for (int ix = 0; ix < nx + 3; ix++)
      for (int iy = 0; iy < ny + 3; iy++)
        for (int iz = 0; iz < nz + 3; iz++)
          for (int ind = 0; ind < norb; ind++)
            coefs[ix * xs + iy * ys + iz * zs + ind] =
                coef_data[((size_t)ix * (ny + 3) + iy) * (nz + 3) + iz] * prefactor[ind];
  }
  void fill_uniform(uint64_t seed)
  {
    for (size_t i = 0; i < coefs.size(); ++i)
      coefs[i] = splitmix_uniform(seed, i) - 0.5;
  }
  void round_to_float()
  {
    for (auto& c : coefs)
      c = (double)(float)c;
  }

  // getSplineBound (MultiBsplineEvalHelper.hpp:43-64), in the evaluation
  // type T (double, or float for the reference's mixed build)
  template <typename T> static void bound(T x, T& dx, int& ind, int nmax)
  {
    if (x < 0)
    {
      ind = 0;
      dx  = T(0);
    }
    else
    {
      T ipart;
      dx  = std::modf(x, &ipart);
      ind = static_cast<int>(ipart);
      if (ind > nmax)
      {
        ind = nmax;
        dx  = T(1) - std::numeric_limits<T>::epsilon();
      }
    }
  }
  // MultiBsplineData<T>::compute_prefactors (MultiBsplineData.hpp:52-80)
  template <typename T> static void prefactors(T a[4], T da[4], T d2a[4], T tx)
  {
    const T A00 = -1.0 / 6.0, A01 = 3.0 / 6.0, A02 = -3.0 / 6.0, A03 = 1.0 / 6.0;
    const T A10 = 3.0 / 6.0, A11 = -6.0 / 6.0, A12 = 0.0 / 6.0, A13 = 4.0 / 6.0;
    const T A20 = -3.0 / 6.0, A21 = 3.0 / 6.0, A22 = 3.0 / 6.0, A23 = 1.0 / 6.0;
    const T A30 = 1.0 / 6.0, A31 = 0.0 / 6.0, A32 = 0.0 / 6.0, A33 = 0.0 / 6.0;
    const T dA01 = -0.5, dA02 = 1.0, dA03 = -0.5;
    const T dA11 = 1.5, dA12 = -2.0, dA13 = 0.0;
    const T dA21 = -1.5, dA22 = 1.0, dA23 = 0.5;
    const T dA31 = 0.5, dA32 = 0.0, dA33 = 0.0;
    const T d2A02 = -1.0, d2A03 = 1.0;
    const T d2A12 = 3.0, d2A13 = -2.0;
    const T d2A22 = -3.0, d2A23 = 1.0;
    const T d2A32 = 1.0, d2A33 = 0.0;
    a[0]   = ((A00 * tx + A01) * tx + A02) * tx + A03;
    a[1]   = ((A10 * tx + A11) * tx + A12) * tx + A13;
    a[2]   = ((A20 * tx + A21) * tx + A22) * tx + A23;
    a[3]   = ((A30 * tx + A31) * tx + A32) * tx + A33;
    da[0]  = (dA01 * tx + dA02) * tx + dA03;
    da[1]  = (dA11 * tx + dA12) * tx + dA13;
    da[2]  = (dA21 * tx + dA22) * tx + dA23;
    da[3]  = (dA31 * tx + dA32) * tx + dA33;
    d2a[0] = d2A02 * tx + d2A03;
    d2a[1] = d2A12 * tx + d2A13;
    d2a[2] = d2A22 * tx + d2A23;
    d2a[3] = d2A32 * tx + d2A33;
  }
  template <typename T> void locate(const Vec3& u, int idx[3], T a[3][4], T da[3][4], T d2a[3][4]) const
  {
    const int ng[3] = {nx, ny, nz};
    for (int d = 0; d < 3; ++d)
    {
      T t;
      bound<T>((T)u[d] * (T)delta_inv[d], t, idx[d], ng[d] - 1);
      prefactors<T>(a[d], da[d], d2a[d], t);
    }
  }
  // evaluate_v (MultiBspline.hpp:34-63)
  void evaluate_v(const Vec3& u, double* vals) const
  {
    int id[3];
    double a[3][4], da[3][4], d2a[3][4];
    locate<double>(u, id, a, da, d2a);
    std::fill(vals, vals + norb, 0.0);
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++)
      {
        const double pre00 = a[0][i] * a[1][j];
        const double* c    = coefs.data() + ((id[0] + i) * xs + (id[1] + j) * ys + id[2] * zs);
        for (int n = 0; n < norb; n++)
          vals[n] += pre00 *
              (a[2][0] * c[n] + a[2][1] * c[n + zs] + a[2][2] * c[n + 2 * zs] + a[2][3] * c[n + 3 * zs]);
      }
  }
  // evaluate_vgh (MultiBspline.hpp:163-280): g[3][norb], h[6][norb]
  void evaluate_vgh(const Vec3& u, double* vals, double* g, double* h) const
  {
    evaluate_vgh_t<double>(u, vals, g, h);
  }
  // the same in the evaluation type T: T = float restates MultiBspline<float>
  // of the reference's mixed build (FP32 unit coordinates, prefactors and
  // accumulators over an FP32 table; the outputs are widened to double)
  template <typename T> void evaluate_vgh_t(const Vec3& u, double* vals, double* g, double* h) const
  {
    int id[3];
    T a[3][4], da[3][4], d2a[3][4];
    locate<T>(u, id, a, da, d2a);
    const size_t o = norb;
    std::vector<T> acc(10 * o, T(0));
    T *vv = acc.data(), *gx = vv + o, *gy = vv + 2 * o, *gz = vv + 3 * o;
    T *hxx = vv + 4 * o, *hxy = vv + 5 * o, *hxz = vv + 6 * o, *hyy = vv + 7 * o, *hyz = vv + 8 * o,
      *hzz = vv + 9 * o;
    const T *c0 = a[2], *dc = da[2], *d2c = d2a[2];
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++)
      {
        const double* coefs0 = coefs.data() + ((id[0] + i) * xs + (id[1] + j) * ys + id[2] * zs);
        const double* coefs1 = coefs0 + zs;
        const double* coefs2 = coefs0 + 2 * zs;
        const double* coefs3 = coefs0 + 3 * zs;
        const T pre20        = d2a[0][i] * a[1][j];
        const T pre10        = da[0][i] * a[1][j];
        const T pre00        = a[0][i] * a[1][j];
        const T pre11        = da[0][i] * da[1][j];
        const T pre01        = a[0][i] * da[1][j];
        const T pre02        = a[0][i] * d2a[1][j];
        for (int n = 0; n < norb; n++)
        {
          T v0 = (T)coefs0[n], v1 = (T)coefs1[n], v2 = (T)coefs2[n], v3 = (T)coefs3[n];
          T sum0 = c0[0] * v0 + c0[1] * v1 + c0[2] * v2 + c0[3] * v3;
          T sum1 = dc[0] * v0 + dc[1] * v1 + dc[2] * v2 + dc[3] * v3;
          T sum2 = d2c[0] * v0 + d2c[1] * v1 + d2c[2] * v2 + d2c[3] * v3;
          hxx[n] += pre20 * sum0;
          hxy[n] += pre11 * sum0;
          hxz[n] += pre10 * sum1;
          hyy[n] += pre02 * sum0;
          hyz[n] += pre01 * sum1;
          hzz[n] += pre00 * sum2;
          gx[n] += pre10 * sum0;
          gy[n] += pre01 * sum0;
          gz[n] += pre00 * sum1;
          vv[n] += pre00 * sum0;
        }
      }
    const T dxInv = (T)delta_inv[0], dyInv = (T)delta_inv[1], dzInv = (T)delta_inv[2];
    const T dxx = dxInv * dxInv, dyy = dyInv * dyInv, dzz = dzInv * dzInv;
    const T dxy = dxInv * dyInv, dxz = dxInv * dzInv, dyz = dyInv * dzInv;
    for (size_t n = 0; n < o; n++)
    {
      vals[n]      = vv[n];
      g[n]         = gx[n] * dxInv;
      g[o + n]     = gy[n] * dyInv;
      g[2 * o + n] = gz[n] * dzInv;
      h[n]         = hxx[n] * dxx;
      h[o + n]     = hxy[n] * dxy;
      h[2 * o + n] = hxz[n] * dxz;
      h[3 * o + n] = hyy[n] * dyy;
      h[4 * o + n] = hyz[n] * dyz;
      h[5 * o + n] = hzz[n] * dzz;
    }
  }
};

// ---------------------------------------------- DiracMatrix (FP64 LU) ---
// invert_transpose (DiracMatrix.h:93-119): psiM = (A^{-1})^T with
// A[i][j] = phi_j(r_i).  getrf = LU with partial pivoting (first |max|,
// reciprocal scaling as dgetf2); logdet and phase from the U diagonal and
// the pivots (computeLogDet, DiracMatrix.h:25-38); the inverse from the LU.
// Returns false on a zero pivot.
inline bool invert_transpose(int n, const double* A, double* psiM, double& logdet, double& phase)
{
  std::vector<double> M(A, A + (size_t)n * n);
  std::vector<int> piv(n);
  bool ok = true;
  for (int j = 0; j < n; ++j)
  {
    int p       = j;
    double amax = std::abs(M[(size_t)j * n + j]);
    for (int i = j + 1; i < n; ++i)
      if (std::abs(M[(size_t)i * n + j]) > amax)
      {
        amax = std::abs(M[(size_t)i * n + j]);
        p    = i;
      }
    piv[j] = p;
    if (p != j)
      for (int k = 0; k < n; ++k)
        std::swap(M[(size_t)j * n + k], M[(size_t)p * n + k]);
    const double pivot = M[(size_t)j * n + j];
    if (pivot == 0.0)
    {
      ok = false;
      continue;
    }
    const double rp = 1.0 / pivot;
    for (int i = j + 1; i < n; ++i)
      M[(size_t)i * n + j] *= rp;
    for (int i = j + 1; i < n; ++i)
    {
      const double lij = M[(size_t)i * n + j];
      double* mi       = &M[(size_t)i * n];
      const double* mj = &M[(size_t)j * n];
      for (int k = j + 1; k < n; ++k)
        mi[k] -= lij * mj[k];
    }
  }
  logdet       = 0.0;
  int sign_det = 1;
  for (int i = 0; i < n; i++)
  {
    sign_det *= (piv[i] == i) ? 1 : -1;
    sign_det *= (M[(size_t)i * n + i] > 0) ? 1 : -1;
    logdet += std::log(std::abs(M[(size_t)i * n + i]));
  }
  phase = (sign_det > 0) ? 0.0 : kPi;
  if (!ok)
    return false;
  // X = A^{-1}: solve A X = I column by column (P A = L U)
  std::vector<double> X((size_t)n * n, 0.0), col(n);
  for (int c = 0; c < n; ++c)
  {
    std::fill(col.begin(), col.end(), 0.0);
    col[c] = 1.0;
    for (int j = 0; j < n; ++j)
      if (piv[j] != j)
        std::swap(col[j], col[piv[j]]);
    for (int i = 0; i < n; ++i)
    {
      double s = col[i];
      for (int k = 0; k < i; ++k)
        s -= M[(size_t)i * n + k] * col[k];
      col[i] = s;
    }
    for (int i = n - 1; i >= 0; --i)
    {
      double s = col[i];
      for (int k = i + 1; k < n; ++k)
        s -= M[(size_t)i * n + k] * col[k];
      col[i] = s / M[(size_t)i * n + i];
    }
    for (int i = 0; i < n; ++i)
      X[(size_t)i * n + c] = col[i];
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j)
      psiM[(size_t)i * n + j] = X[(size_t)j * n + i];
  return true;
}

// ------------------------------------------------------ DelayedUpdate ---
// DelayedUpdate<T,T_FP> (DelayedUpdate.h:28-231), row-major.  T = double is
// the FP64 build; T = float restates the arithmetic of the reference's
// mixed-precision build (QMC_MIXED_PRECISION: ValueType float, so U, V,
// Binv, tempMat and every product and dot of the getInvRow / acceptRow /
// updateInvMat GEMVs and GEMMs are FP32; the inverse itself is the FP64
// DiracMatrix<T_FP>).
template <typename T> struct DelayedUpdateT
{
  int norb = 0, kmax = 0, delay_count = 0;
  std::vector<T> U, V, Binv, tempMat, p, temp;
  std::vector<int> delay_list;

  void resize(int n, int delay)
  {
    norb = n;
    kmax = delay;
    U.assign((size_t)delay * n, T(0));
    V.assign((size_t)delay * n, T(0));
    Binv.assign((size_t)delay * delay, T(0));
    tempMat.assign((size_t)n * delay, T(0));
    p.assign(delay, T(0));
    temp.assign(n, T(0));
    delay_list.assign(delay, 0);
    delay_count = 0;
  }
  // getInvRow (DelayedUpdate.h:95-114)
  void getInvRow(const T* Ainv, int rowchanged, T* invRow)
  {
    const int n = norb, k = kmax, dc = delay_count;
    std::copy_n(Ainv + (size_t)rowchanged * n, n, invRow);
    if (dc == 0)
      return;
    for (int d = 0; d < dc; ++d)
    {
      T s = T(0);
      for (int j = 0; j < n; ++j)
        s += U[(size_t)d * n + j] * invRow[j];
      p[d] = s;
    }
    T* w = &Binv[(size_t)dc * k]; // Binv[delay_count] holds the product
    if (dc < k)
      for (int a = 0; a < dc; ++a)
      {
        T s = T(0);
        for (int b = 0; b < dc; ++b)
          s += Binv[(size_t)b * k + a] * p[b];
        w[a] = s;
      }
    for (int j = 0; j < n; ++j)
    {
      T s = T(0);
      for (int d = 0; d < dc; ++d)
        s += V[(size_t)d * n + j] * w[d];
      invRow[j] -= s;
    }
  }
  // acceptRow (DelayedUpdate.h:123-153)
  void acceptRow(T* Ainv, int rowchanged, const T* psiV)
  {
    const int n = norb, k = kmax, dc = delay_count;
    std::copy_n(Ainv + (size_t)rowchanged * n, n, &V[(size_t)dc * n]);
    std::copy_n(psiV, n, &U[(size_t)dc * n]);
    delay_list[dc] = rowchanged;
    for (int d = 0; d <= dc; ++d)
    {
      T s = T(0);
      for (int j = 0; j < n; ++j)
        s += V[(size_t)d * n + j] * psiV[j];
      p[d] = -s;
    }
    T y = -p[dc];
    for (int i = 0; i < dc; i++)
      y += Binv[(size_t)dc * k + i] * p[i];
    Binv[(size_t)dc * k + dc] = y = T(1) / y;
    for (int b = 0; b < dc; ++b)
    {
      T s = T(0);
      for (int a = 0; a < dc; ++a)
        s += Binv[(size_t)b * k + a] * p[a];
      Binv[(size_t)b * k + dc] = y * s;
    }
    for (int b = 0; b < dc; ++b)
      for (int a = 0; a < dc; ++a)
        Binv[(size_t)b * k + a] -= Binv[(size_t)dc * k + a] * Binv[(size_t)b * k + dc];
    for (int i = 0; i < dc; i++)
      Binv[(size_t)dc * k + i] *= -y;
    delay_count++;
    if (delay_count == k)
      updateInvMat(Ainv);
  }
  // updateInvMat (DelayedUpdate.h:155-231)
  void updateInvMat(T* Ainv)
  {
    const int n = norb, k = kmax, dc = delay_count;
    if (dc == 0)
      return;
    if (dc == 1)
    {
      for (int i = 0; i < n; ++i)
      {
        T s = T(0);
        for (int j = 0; j < n; ++j)
          s += Ainv[(size_t)i * n + j] * U[j];
        temp[i] = s;
      }
      temp[delay_list[0]] -= T(1);
      const T b00 = Binv[0];
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
          Ainv[(size_t)i * n + j] += -b00 * V[j] * temp[i];
    }
    else
    {
      for (int i = 0; i < n; ++i)
        for (int d = 0; d < dc; ++d)
        {
          T s = T(0);
          for (int j = 0; j < n; ++j)
            s += U[(size_t)d * n + j] * Ainv[(size_t)i * n + j];
          tempMat[(size_t)i * k + d] = s;
        }
      for (int d = 0; d < dc; d++)
        tempMat[(size_t)delay_list[d] * k + d] -= T(1);
      std::vector<T> U2((size_t)dc * n, T(0));
      for (int b = 0; b < dc; ++b)
        for (int a = 0; a < dc; ++a)
        {
          const T bba = Binv[(size_t)b * k + a];
          for (int j = 0; j < n; ++j)
            U2[(size_t)b * n + j] += bba * V[(size_t)a * n + j];
        }
      std::copy(U2.begin(), U2.end(), U.begin());
      for (int i = 0; i < n; ++i)
        for (int d = 0; d < dc; ++d)
        {
          const T t = tempMat[(size_t)i * k + d];
          for (int j = 0; j < n; ++j)
            Ainv[(size_t)i * n + j] -= t * U2[(size_t)d * n + j];
        }
    }
    delay_count = 0;
  }
};
using DelayedUpdate = DelayedUpdateT<double>;

// -------------------------------------------------- PolynomialFunctor3D --
// The eeI functor of the three-body Jastrow (PolynomialFunctor3D.h:38-560)
// with N_eI = N_ee = 3 and C = 3: the gamma(l, m, n) coefficients follow
// from the free parameters through the e-e and e-I no-cusp constraints
// (resize: the constraint matrix and its row reduction; reset_gamma).
struct J3Func
{
  static constexpr int NeI = 3, Nee = 3, C = 3;
  double cutoff_radius = 0.0;
  double gamma[NeI + 1][NeI + 1][Nee + 1] = {};

  void setup(double rcut, const double* params)
  {
    cutoff_radius   = rcut;
    const double L  = 0.5 * rcut;
    const int NumGamma = (NeI + 1) * (NeI + 2) / 2 * (Nee + 1);
    const int NumC     = (2 * NeI + 1) + (NeI + Nee + 1);
    int index[NeI + 1][NeI + 1][Nee + 1];
    int num = 0;
    for (int m = 0; m <= NeI; m++)
      for (int l = m; l <= NeI; l++)
        for (int n = 0; n <= Nee; n++)
          index[l][m][n] = index[m][l][n] = num++;
    std::vector<double> A((size_t)NumC * NumGamma, 0.0);
    auto a = [&](int r, int c) -> double& { return A[(size_t)r * NumGamma + c]; };
    int k;
    for (k = 0; k <= 2 * NeI; k++)
      for (int m = 0; m <= k; m++)
      {
        const int l = k - m;
        if (l <= NeI && m <= NeI)
        {
          const int i = index[l][m][1];
          if (l > m)
            a(k, i) = 2.0;
          else if (l == m)
            a(k, i) = 1.0;
        }
      }
    for (int kp = 0; kp <= NeI + Nee; kp++)
    {
      if (kp <= Nee)
      {
        a(k + kp, index[0][0][kp]) = (double)C;
        a(k + kp, index[0][1][kp]) = -L;
      }
      for (int l = 1; l <= kp; l++)
      {
        const int n = kp - l;
        if (n >= 0 && n <= Nee && l <= NeI)
        {
          a(k + kp, index[l][0][n]) = (double)C;
          a(k + kp, index[l][1][n]) = -L;
        }
      }
    }
    // row reduction with the reference's column scan and row pivoting
    std::vector<bool> indep(NumGamma, false);
    int col = -1;
    for (int row = 0; row < NumC; row++)
    {
      int max_loc;
      double max_abs;
      do
      {
        col++;
        max_loc = row;
        max_abs = std::abs(a(row, col));
        for (int ri = row + 1; ri < NumC; ri++)
          if (std::abs(a(ri, col)) > max_abs)
          {
            max_loc = ri;
            max_abs = std::abs(a(ri, col));
          }
        if (max_abs < 1.0e-6)
          indep[col] = true;
      } while (max_abs < 1.0e-6);
      for (int c = 0; c < NumGamma; c++)
        std::swap(a(row, c), a(max_loc, c));
      const double lead_inv = 1.0 / a(row, col);
      for (int c = 0; c < NumGamma; c++)
        a(row, c) *= lead_inv;
      for (int ri = 0; ri < NumC; ri++)
        if (ri != row)
        {
          const double val = a(ri, col);
          for (int c = 0; c < NumGamma; c++)
            a(ri, c) -= val * a(row, c);
        }
    }
    for (int c = col + 1; c < NumGamma; c++)
      indep[c] = true;
    std::vector<double> g(NumGamma, 0.0);
    int var = 0;
    for (int i = 0; i < NumGamma; i++)
      if (indep[i])
        g[i] = params[var++];
    var = 0;
    for (int i = 0; i < NumGamma; i++)
      if (!indep[i])
      {
        for (int j = 0; j < NumGamma; j++)
          if (i != j)
            g[i] -= a(var, j) * g[j];
        var++;
      }
    num = 0;
    for (int m = 0; m <= NeI; m++)
      for (int l = m; l <= NeI; l++)
        for (int n = 0; n <= Nee; n++)
          gamma[m][l][n] = gamma[l][m][n] = g[num++];
  }
  // value, grad (d/dr_12, d/dr_1I, d/dr_2I) and the Hessian entries (00, 01,
  // 02, 11, 12, 22) (PolynomialFunctor3D::evaluate with derivatives)
  double eval(double r12, double r1I, double r2I, double* gr, double* h) const
  {
    const double L = 0.5 * cutoff_radius;
    for (int i = 0; i < 3; ++i)
      gr[i] = 0.0;
    for (int i = 0; i < 6; ++i)
      h[i] = 0.0;
    if (r1I >= L || r2I >= L)
      return 0.0;
    double val = 0.0, g0 = 0, g1 = 0, g2 = 0, h00 = 0, h01 = 0, h02 = 0, h11 = 0, h12 = 0, h22 = 0;
    double r2l = 1, r2l_1 = 0, r2l_2 = 0, lf = 0;
    for (int l = 0; l <= NeI; l++)
    {
      double r2m = 1, r2m_1 = 0, r2m_2 = 0, mf = 0;
      for (int m = 0; m <= NeI; m++)
      {
        double r2n = 1, r2n_1 = 0, r2n_2 = 0, nf = 0;
        for (int n = 0; n <= Nee; n++)
        {
          const double gg = gamma[l][m][n];
          const double g00x = gg * r2l * r2m, g10x = gg * r2l_1 * r2m, g01x = gg * r2l * r2m_1, gxx0 = gg * r2n;
          val += g00x * r2n;
          g0 += g00x * r2n_1;
          g1 += g10x * r2n;
          g2 += g01x * r2n;
          h00 += g00x * r2n_2;
          h01 += g10x * r2n_1;
          h02 += g01x * r2n_1;
          h11 += gxx0 * r2l_2 * r2m;
          h12 += gxx0 * r2l_1 * r2m_1;
          h22 += gxx0 * r2l * r2m_2;
          nf += 1;
          r2n_2 = r2n_1 * nf;
          r2n_1 = r2n * nf;
          r2n *= r12;
        }
        mf += 1;
        r2m_2 = r2m_1 * mf;
        r2m_1 = r2m * mf;
        r2m *= r2I;
      }
      lf += 1;
      r2l_2 = r2l_1 * lf;
      r2l_1 = r2l * lf;
      r2l *= r1I;
    }
    const double a2 = r2I - L, a1 = r1I - L, b = a2 * a1;
    for (int i = 0; i < C; i++)
    {
      h00 = b * h00;
      h01 = b * h01 + a2 * g0;
      h02 = b * h02 + a1 * g0;
      h11 = b * h11 + 2.0 * a2 * g1;
      h12 = b * h12 + a1 * g1 + a2 * g2 + val;
      h22 = b * h22 + 2.0 * a1 * g2;
      g0  = b * g0;
      g1  = b * g1 + a2 * val;
      g2  = b * g2 + a1 * val;
      val *= b;
    }
    gr[0] = g0, gr[1] = g1, gr[2] = g2;
    h[0] = h00, h[1] = h01, h[2] = h02, h[3] = h11, h[4] = h12, h[5] = h22;
    return val;
  }
};

// ------------------------------------------------------------ System ---
// ARITH_SPO32: the orbitals are evaluated in FP32 arithmetic (MultiBspline<
//   float>, the reference's mixed build; einspline_spo.hpp:172-223).
// ARITH_DET32: the determinant's inverse, delayed rows and every dot and
//   product of DiracDeterminant / DelayedUpdate in FP32 (ValueType float),
//   the LU inverse in FP64 and rounded to FP32 (DiracMatrix<double>::
//   invert_transpose of the mixed build, DiracMatrix.h:93-119 with
//   MIXED_PRECISION, DiracDeterminant.cpp:30-60).
// ARITH_LOG32: the log|det| accumulation of acceptMove in FP32 (LogValue is
//   RealType = float in the mixed build, DiracDeterminant.cpp:129-146).
enum
{
  ARITH_SPO32 = 1,
  ARITH_DET32 = 2,
  ARITH_LOG32 = 4
};

struct System
{
  Lattice lattice;     // simulation cell (electrons and ions)
  Lattice spo_lattice; // cell on which the orbitals are periodic
  int n_ions = 0, n_groups = 0, n_elec = 0, n_up = 0, norb = 0;
  std::vector<double> ion_pos;
  std::vector<int> ion_group;
  std::vector<int> group_first, group_last;
  Spline spline;
  int lap_mode = 0;
  // arithmetic of the orbital and determinant path of the walkers created
  // next (ARITH_* flags; 0 is FP64 throughout): restates the reference's
  // mixed-precision build piece by piece, so that each piece's share of the
  // error can be measured
  int arith = 0;
  bool use_det = true, use_j1 = true, use_j2 = true, use_j3 = false;
  std::vector<Functor> j1; // per ion group
  Functor j2_uu, j2_ud;
  std::vector<J3Func> j3_same, j3_diff; // per ion group: same-spin and opposite-spin electron pairs
};

// NonLocalPP's 12-point sphere (NonLocalPP.hpp:61-80) rotated by
// NonLocalPP::randomize (:98-110) for call `call` of the stream that
// NonLocalPP's constructor seeds with 11 (:58): three uniforms per call
inline void nlpp_sphere(int call, double out[12][3])
{
  static const double g[12][3] = {{1.0, 0.0, 0.0},
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
  double phi = 0, psi = 0, cth = 0;
  for (int c = 0; c <= call; ++c)
  {
    phi = 2 * M_PI * uni(gen);
    psi = 2 * M_PI * uni(gen);
    cth = uni(gen) - 0.5;
  }
  const double sph = std::sin(phi), cph = std::cos(phi), sth = std::sqrt(1.0 - cth * cth);
  const double sps = std::sin(psi), cps = std::cos(psi);
  const double m[3][3] = {{cph * cth * cps - sph * sps, sph * cth * cps + cph * sps, -sth * cps},
                          {-cph * cth * sps - sph * cps, -sph * cth * sps + cph * cps, sth * sps},
                          {cph * sth, sph * sth, cth}};
  for (int k = 0; k < 12; ++k)
    for (int i = 0; i < 3; ++i)
      out[k][i] = m[i][0] * g[k][0] + m[i][1] * g[k][1] + m[i][2] * g[k][2];
}

// --------------------------------------------------------- Walker state --
struct Walker
{
  const System* sys = nullptr;
  Rng rng;
  std::vector<double> R; // [N][3]
  // active move (ParticleSet::activePtcl / activePos, ParticleSet.cpp:316-324)
  int activePtcl = -1;
  Vec3 activePos{0, 0, 0};
  // temp rows of the active move
  std::vector<double> aa_r, aa_dx, aa_dy, aa_dz, ab_r, ab_dx, ab_dy, ab_dz;
  // scratch rows
  std::vector<double> row_r, row_dx, row_dy, row_dz;

  // Determinants (DiracDeterminant.cpp:30-280) per spin
  struct Det
  {
    int first = 0, n = 0;
    std::vector<double> psiM, psiM_temp, dpsiM, d2psiM; // dpsiM [n][n][3]
    std::vector<double> psiV, dpsiV, d2psiV, invRow;      // dpsiV [n][3]
    double LogValue = 0.0, PhaseValue = 0.0, curRatio = 1.0;
    int invRow_id = -1;
    bool partial  = false; // UpdateMode == ORB_PBYP_PARTIAL
    DelayedUpdate eng;
    // ARITH_DET32: the FP32 inverse and delayed rows (psiM above then holds
    // the same values widened, for evaluateGL and the inverse read-out)
    std::vector<float> psiM32, invRow32, psiV32;
    DelayedUpdateT<float> eng32;
  } det[2];

  // J1 (OneBodyJastrow.h:110-283)
  std::vector<double> j1_Vat, j1_Grad, j1_Lap; // Grad [N][3]
  std::vector<double> j1_U, j1_dU, j1_d2U;
  double j1_curAt = 0, j1_curLap = 0, j1_LogValue = 0;
  Vec3 j1_curGrad{0, 0, 0};
  bool j1_partial = false;
  // J2 (TwoBodyJastrow.h:121-430)
  std::vector<double> j2_Uat, j2_dUat, j2_d2Uat; // dUat [N][3]
  std::vector<double> cur_u, cur_du, cur_d2u, old_u, old_du, old_d2u;
  double j2_cur_Uat = 0, j2_LogValue = 0;
  bool j2_partial = false;
  // wavefunction (WaveFunction.cpp:178-279)
  std::vector<double> G, L; // [N][3], [N]
  double LogValue = 0.0;

  int arith = 0; // ARITH_* of the system when this walker was created
  void init(const System* s, int delay)
  {
    sys         = s;
    arith       = s->arith;
    const int N = s->n_elec, I = s->n_ions;
    R.assign((size_t)N * 3, 0.0);
    for (auto* v : {&aa_r, &aa_dx, &aa_dy, &aa_dz, &row_r, &row_dx, &row_dy, &row_dz})
      v->assign(std::max(N, I), 0.0);
    for (auto* v : {&ab_r, &ab_dx, &ab_dy, &ab_dz})
      v->assign(I, 0.0);
    for (int s2 = 0; s2 < 2; ++s2)
    {
      Det& d  = det[s2];
      d.first = s2 == 0 ? 0 : s->n_up;
      d.n     = s->norb;
      const size_t n = d.n;
      d.psiM.assign(n * n, 0.0);
      d.psiM_temp.assign(n * n, 0.0);
      d.dpsiM.assign(n * n * 3, 0.0);
      d.d2psiM.assign(n * n, 0.0);
      d.psiV.assign(n, 0.0);
      d.dpsiV.assign(n * 3, 0.0);
      d.d2psiV.assign(n, 0.0);
      d.invRow.assign(n, 0.0);
      d.eng.resize(d.n, delay);
      if (arith & ARITH_DET32)
      {
        d.psiM32.assign(n * n, 0.f);
        d.invRow32.assign(n, 0.f);
        d.psiV32.assign(n, 0.f);
        d.eng32.resize(d.n, delay);
      }
    }
    j1_Vat.assign(N, 0.0);
    j1_Grad.assign((size_t)N * 3, 0.0);
    j1_Lap.assign(N, 0.0);
    j1_U.assign(I, 0.0);
    j1_dU.assign(I, 0.0);
    j1_d2U.assign(I, 0.0);
    j2_Uat.assign(N, 0.0);
    j2_dUat.assign((size_t)N * 3, 0.0);
    j2_d2Uat.assign(N, 0.0);
    for (auto* v : {&cur_u, &cur_du, &cur_d2u, &old_u, &old_du, &old_d2u})
      v->assign(N, 0.0);
    G.assign((size_t)N * 3, 0.0);
    L.assign(N, 0.0);
    if (s->use_j3)
      j3_init();
  }

  // build_els (ParticleSet_builder.cpp:33-53): 3N uniforms in lattice units
  void init_random(uint32_t seed)
  {
    rng        = Rng(seed);
    const int N = sys->n_elec;
    std::vector<double> u((size_t)N * 3);
    rng.uniform(u.data(), 3 * N);
    for (int i = 0; i < N; ++i)
    {
      Vec3 r = sys->lattice.toCart(Vec3{u[3 * i], u[3 * i + 1], u[3 * i + 2]});
      R[3 * i] = r[0], R[3 * i + 1] = r[1], R[3 * i + 2] = r[2];
    }
  }

  Vec3 pos(int i) const { return Vec3{R[3 * i], R[3 * i + 1], R[3 * i + 2]}; }
  // ParticleSet::activeR (ParticleSet.h:222)
  Vec3 activeR(int iat) const { return (iat == activePtcl) ? activePos : pos(iat); }

  // AA row of electron iat at its current position (setActive; flip = iat,
  // self distance = max: DistanceTableAA.h:85-95)
  void aa_row_current(int iat)
  {
    sys->lattice.computeDistances(pos(iat), R.data(), row_r.data(), row_dx.data(), row_dy.data(),
                                  row_dz.data(), 0, sys->n_elec, iat);
    row_r[iat] = std::numeric_limits<double>::max();
  }
  // AB row (DistanceTableBA.h:83-97; flip_ind = 0 -> every entry flipped)
  void ab_row(const Vec3& p, double* r, double* dx, double* dy, double* dz) const
  {
    sys->lattice.computeDistances(p, sys->ion_pos.data(), r, dx, dy, dz, 0, sys->n_ions, 0);
  }

  // ---- SPO (einspline_spo::evaluate, einspline_spo.hpp:172-223) ----
  void spo_vgh(const Vec3& r, double* psi, double* dpsi /*[n][3]*/, double* d2psi) const
  {
    const int n = sys->norb;
    std::vector<double> v(n), g(3 * n), h(6 * n);
    Vec3 u = sys->spo_lattice.toUnit_floor(r);
    if (arith & ARITH_SPO32)
      sys->spline.evaluate_vgh_t<float>(u, v.data(), g.data(), h.data());
    else
      sys->spline.evaluate_vgh(u, v.data(), g.data(), h.data());
    for (int j = 0; j < n; ++j)
    {
      psi[j]          = v[j];
      dpsi[3 * j + 0] = g[j];
      dpsi[3 * j + 1] = g[n + j];
      dpsi[3 * j + 2] = g[2 * n + j];
      d2psi[j]        = sys->lap_mode == 0 ? h[j] : h[j] + h[3 * n + j] + h[5 * n + j];
    }
  }
  void spo_v(const Vec3& r, double* psi) const
  {
    Vec3 u = sys->spo_lattice.toUnit_floor(r);
    sys->spline.evaluate_v(u, psi);
  }

  // ---- determinant ----
  bool det32() const { return (arith & ARITH_DET32) != 0; }
  // ARITH_DET32: the FP32 inverse widened into psiM (after every change)
  void det_widen(Det& d)
  {
    for (size_t i = 0; i < d.psiM32.size(); ++i)
      d.psiM[i] = d.psiM32[i];
  }
  // FP32 storage of the orbital rows the FP32 determinant keeps
  void det_round_rows(double* p, size_t count) const
  {
    if (det32())
      for (size_t i = 0; i < count; ++i)
        p[i] = (double)(float)p[i];
  }
  bool det_recompute(int s)
  {
    Det& d      = det[s];
    const int n = d.n;
    for (int i = 0; i < n; ++i)
      spo_vgh(activeR(d.first + i), &d.psiM_temp[(size_t)i * n], &d.dpsiM[(size_t)i * n * 3],
              &d.d2psiM[(size_t)i * n]);
    det_round_rows(d.psiM_temp.data(), d.psiM_temp.size());
    det_round_rows(d.dpsiM.data(), d.dpsiM.size());
    det_round_rows(d.d2psiM.data(), d.d2psiM.size());
    bool ok = invert_transpose(n, d.psiM_temp.data(), d.psiM.data(), d.LogValue, d.PhaseValue);
    d.eng.delay_count = 0;
    if (det32())
    {
      for (size_t i = 0; i < d.psiM.size(); ++i)
        d.psiM32[i] = (float)d.psiM[i];
      det_widen(d);
      d.eng32.delay_count = 0;
      if (arith & ARITH_LOG32)
        d.LogValue = (double)(float)d.LogValue;
    }
    return ok;
  }
  Vec3 det_evalGrad(int s, int iat)
  {
    Det& d      = det[s];
    const int r = iat - d.first, n = d.n;
    d.invRow_id = r;
    if (det32())
    {
      d.eng32.getInvRow(d.psiM32.data(), r, d.invRow32.data());
      float gf[3] = {0.f, 0.f, 0.f};
      const double* dp = &d.dpsiM[(size_t)r * n * 3];
      for (int j = 0; j < n; ++j)
        for (int c = 0; c < 3; ++c)
          gf[c] += d.invRow32[j] * (float)dp[3 * j + c];
      for (int j = 0; j < n; ++j)
        d.invRow[j] = d.invRow32[j];
      return Vec3{gf[0], gf[1], gf[2]};
    }
    d.eng.getInvRow(d.psiM.data(), r, d.invRow.data());
    Vec3 g{0, 0, 0};
    const double* dp = &d.dpsiM[(size_t)r * n * 3];
    for (int j = 0; j < n; ++j)
      for (int c = 0; c < 3; ++c)
        g[c] += d.invRow[j] * dp[3 * j + c];
    return g;
  }
  double det_ratioGrad(int s, int iat, Vec3& grad)
  {
    Det& d      = det[s];
    const int r = iat - d.first, n = d.n;
    spo_vgh(activeR(iat), d.psiV.data(), d.dpsiV.data(), d.d2psiV.data());
    d.partial = true;
    if (det32())
    {
      // DiracDeterminant::ratioGrad in FP32 (DiracDeterminant.cpp:80-122)
      det_round_rows(d.psiV.data(), n);
      det_round_rows(d.dpsiV.data(), 3 * (size_t)n);
      det_round_rows(d.d2psiV.data(), n);
      for (int j = 0; j < n; ++j)
        d.psiV32[j] = (float)d.psiV[j];
      if (d.invRow_id != r)
      {
        d.invRow_id = r;
        d.eng32.getInvRow(d.psiM32.data(), r, d.invRow32.data());
      }
      float ratio = 0.f;
      for (int j = 0; j < n; ++j)
        ratio += d.invRow32[j] * d.psiV32[j];
      d.curRatio = ratio;
      float gf[3] = {0.f, 0.f, 0.f};
      for (int j = 0; j < n; ++j)
        for (int c = 0; c < 3; ++c)
          gf[c] += d.invRow32[j] * (float)d.dpsiV[3 * j + c];
      const float rinv = 1.f / ratio;
      for (int c = 0; c < 3; ++c)
        grad[c] += (double)(rinv * gf[c]);
      return ratio;
    }
    if (d.invRow_id != r)
    {
      d.invRow_id = r;
      d.eng.getInvRow(d.psiM.data(), r, d.invRow.data());
    }
    double ratio = 0.0;
    for (int j = 0; j < n; ++j)
      ratio += d.invRow[j] * d.psiV[j];
    d.curRatio = ratio;
    Vec3 g{0, 0, 0};
    for (int j = 0; j < n; ++j)
      for (int c = 0; c < 3; ++c)
        g[c] += d.invRow[j] * d.dpsiV[3 * j + c];
    const double rinv = 1.0 / ratio;
    for (int c = 0; c < 3; ++c)
      grad[c] += rinv * g[c];
    return ratio;
  }
  double det_ratio(int s, int iat)
  {
    Det& d      = det[s];
    const int r = iat - d.first, n = d.n;
    spo_v(activeR(iat), d.psiV.data());
    d.partial = false;
    if (det32())
    {
      det_round_rows(d.psiV.data(), n);
      for (int j = 0; j < n; ++j)
        d.psiV32[j] = (float)d.psiV[j];
      if (d.invRow_id != r)
      {
        d.invRow_id = r;
        d.eng32.getInvRow(d.psiM32.data(), r, d.invRow32.data());
      }
      float ratio = 0.f;
      for (int j = 0; j < n; ++j)
        ratio += d.invRow32[j] * d.psiV32[j];
      d.curRatio = ratio;
      return ratio;
    }
    if (d.invRow_id != r)
    {
      d.invRow_id = r;
      d.eng.getInvRow(d.psiM.data(), r, d.invRow.data());
    }
    double ratio = 0.0;
    for (int j = 0; j < n; ++j)
      ratio += d.invRow[j] * d.psiV[j];
    d.curRatio = ratio;
    return ratio;
  }
  void det_accept(int s, int iat)
  {
    Det& d      = det[s];
    const int r = iat - d.first, n = d.n;
    d.PhaseValue += (d.curRatio > 0) ? 0.0 : kPi;
    if (arith & ARITH_LOG32)
      d.LogValue = (double)((float)d.LogValue + std::log(std::abs((float)d.curRatio)));
    else
      d.LogValue += std::log(std::abs(d.curRatio));
    if (det32())
    {
      d.eng32.acceptRow(d.psiM32.data(), r, d.psiV32.data());
      if (d.eng32.delay_count == 0) // the delay was full: updateInvMat ran
        det_widen(d);
    }
    else
      d.eng.acceptRow(d.psiM.data(), r, d.psiV.data());
    d.invRow_id = -1;
    if (d.partial)
    {
      std::copy_n(d.dpsiV.data(), 3 * n, &d.dpsiM[(size_t)r * n * 3]);
      std::copy_n(d.d2psiV.data(), n, &d.d2psiM[(size_t)r * n]);
    }
    d.curRatio = 1.0;
  }
  void det_complete(int s)
  {
    det[s].invRow_id = -1;
    if (det32())
    {
      det[s].eng32.updateInvMat(det[s].psiM32.data());
      det_widen(det[s]);
    }
    else
      det[s].eng.updateInvMat(det[s].psiM.data());
  }
  void det_GL(int s)
  {
    Det& d      = det[s];
    const int n = d.n;
    // DiracDeterminant::evaluateGL (DiracDeterminant.cpp:157-187): after a
    // ratio-only move the orbital derivatives are re-evaluated (psiM kept)
    if (!d.partial)
      for (int i = 0; i < n; ++i)
        spo_vgh(activeR(d.first + i), &d.psiM_temp[(size_t)i * n], &d.dpsiM[(size_t)i * n * 3],
                &d.d2psiM[(size_t)i * n]);
    for (int i = 0; i < n; ++i)
    {
      const int iat = d.first + i;
      double dot_temp = 0.0;
      Vec3 rv{0, 0, 0};
      const double* pm = &d.psiM[(size_t)i * n];
      for (int j = 0; j < n; ++j)
        dot_temp += pm[j] * d.d2psiM[(size_t)i * n + j];
      for (int j = 0; j < n; ++j)
        for (int c = 0; c < 3; ++c)
          rv[c] += pm[j] * d.dpsiM[((size_t)i * n + j) * 3 + c];
      for (int c = 0; c < 3; ++c)
        G[3 * iat + c] += rv[c];
      L[iat] += dot_temp - (rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2]);
    }
  }

  // ---- J1 ----
  void j1_computeU3(const double* dist)
  {
    const int I = sys->n_ions;
    std::fill_n(j1_U.data(), I, 0.0);
    std::fill_n(j1_dU.data(), I, 0.0);
    std::fill_n(j1_d2U.data(), I, 0.0);
    for (int jg = 0; jg < sys->n_groups; ++jg)
      if (jg < (int)sys->j1.size() && sys->group_last[jg] > sys->group_first[jg])
        sys->j1[jg].evaluateVGL(-1, sys->group_first[jg], sys->group_last[jg], dist, j1_U.data(),
                                j1_dU.data(), j1_d2U.data());
  }
  double j1_accumulateGL(const double* dx, const double* dy, const double* dz, Vec3& grad) const
  {
    const int I     = sys->n_ions;
    double lap      = 0.0;
    const double lf = 3 - 1.0;
    for (int j = 0; j < I; ++j)
      lap += j1_d2U[j] + lf * j1_dU[j];
    const double* dX[3] = {dx, dy, dz};
    for (int c = 0; c < 3; ++c)
    {
      double s = 0.0;
      for (int j = 0; j < I; ++j)
        s += j1_dU[j] * dX[c][j];
      grad[c] = s;
    }
    return lap;
  }
  void j1_recompute()
  {
    const int N = sys->n_elec, I = sys->n_ions;
    for (int iat = 0; iat < N; ++iat)
    {
      ab_row(pos(iat), row_r.data(), row_dx.data(), row_dy.data(), row_dz.data());
      j1_computeU3(row_r.data());
      double s = 0.0;
      for (int j = 0; j < I; ++j)
        s += j1_U[j];
      j1_Vat[iat] = s;
      Vec3 g;
      j1_Lap[iat] = j1_accumulateGL(row_dx.data(), row_dy.data(), row_dz.data(), g);
      for (int c = 0; c < 3; ++c)
        j1_Grad[3 * iat + c] = g[c];
    }
  }
  double j1_ratioGrad(int iat, Vec3& grad)
  {
    j1_partial = true;
    j1_computeU3(ab_r.data());
    j1_curLap = j1_accumulateGL(ab_dx.data(), ab_dy.data(), ab_dz.data(), j1_curGrad);
    double s  = 0.0;
    for (int j = 0; j < sys->n_ions; ++j)
      s += j1_U[j];
    j1_curAt = s;
    for (int c = 0; c < 3; ++c)
      grad[c] += j1_curGrad[c];
    return std::exp(j1_Vat[iat] - j1_curAt);
  }
  double j1_ratio(int iat)
  {
    j1_partial  = false;
    double cur  = 0.0;
    for (int jg = 0; jg < sys->n_groups; ++jg)
      if (jg < (int)sys->j1.size())
        cur += sys->j1[jg].evaluateV(-1, sys->group_first[jg], sys->group_last[jg], ab_r.data());
    j1_curAt = cur;
    return std::exp(j1_Vat[iat] - j1_curAt);
  }
  void j1_accept(int iat)
  {
    if (!j1_partial)
    {
      j1_computeU3(ab_r.data());
      j1_curLap = j1_accumulateGL(ab_dx.data(), ab_dy.data(), ab_dz.data(), j1_curGrad);
    }
    j1_LogValue += j1_Vat[iat] - j1_curAt;
    j1_Vat[iat] = j1_curAt;
    for (int c = 0; c < 3; ++c)
      j1_Grad[3 * iat + c] = j1_curGrad[c];
    j1_Lap[iat] = j1_curLap;
  }
  void j1_GL()
  {
    const int N = sys->n_elec;
    for (int i = 0; i < N; ++i)
      for (int c = 0; c < 3; ++c)
        G[3 * i + c] += j1_Grad[3 * i + c];
    for (int i = 0; i < N; ++i)
      L[i] -= j1_Lap[i];
    double s = 0.0;
    for (int i = 0; i < N; ++i)
      s += j1_Vat[i];
    j1_LogValue = -s;
  }

  // ---- J2 ----
  const Functor& j2f(int gi, int gj) const { return (gi == gj) ? sys->j2_uu : sys->j2_ud; }
  int egroup(int i) const { return i < sys->n_up ? 0 : 1; }
  void j2_computeU3(int iat, const double* dist, double* u, double* du, double* d2u, bool triangle)
  {
    const int N      = sys->n_elec;
    const int jelmax = triangle ? iat : N;
    std::fill_n(u, jelmax, 0.0);
    std::fill_n(du, jelmax, 0.0);
    std::fill_n(d2u, jelmax, 0.0);
    const int gfirst[2] = {0, sys->n_up}, glast[2] = {sys->n_up, N};
    for (int jg = 0; jg < 2; ++jg)
    {
      int iStart = gfirst[jg];
      int iEnd   = std::min(jelmax, glast[jg]);
      j2f(egroup(iat), jg).evaluateVGL(iat, iStart, iEnd, dist, u, du, d2u);
    }
  }
  void j2_recompute()
  {
    const int N     = sys->n_elec;
    const double lf = 3 - 1.0;
    std::fill(j2_Uat.begin(), j2_Uat.end(), 0.0);
    std::fill(j2_dUat.begin(), j2_dUat.end(), 0.0);
    std::fill(j2_d2Uat.begin(), j2_d2Uat.end(), 0.0);
    for (int iat = 0; iat < N; ++iat)
    {
      aa_row_current(iat);
      j2_computeU3(iat, row_r.data(), cur_u.data(), cur_du.data(), cur_d2u.data(), true);
      double s = 0.0;
      for (int j = 0; j < iat; ++j)
        s += cur_u[j];
      j2_Uat[iat] = s;
      double lap  = 0.0;
      for (int j = 0; j < iat; ++j)
        lap += cur_d2u[j] + lf * cur_du[j];
      const double* dX[3] = {row_dx.data(), row_dy.data(), row_dz.data()};
      for (int c = 0; c < 3; ++c)
      {
        double g = 0.0;
        for (int j = 0; j < iat; ++j)
          g += cur_du[j] * dX[c][j];
        j2_dUat[3 * iat + c] = g;
      }
      j2_d2Uat[iat] = -lap;
      for (int j = 0; j < iat; j++)
      {
        j2_Uat[j] += cur_u[j];
        j2_d2Uat[j] -= cur_d2u[j] + lf * cur_du[j];
      }
      for (int c = 0; c < 3; ++c)
        for (int j = 0; j < iat; j++)
          j2_dUat[3 * j + c] -= cur_du[j] * dX[c][j];
    }
  }
  double j2_ratioGrad(int iat, Vec3& grad)
  {
    j2_partial = true;
    const int N = sys->n_elec;
    j2_computeU3(iat, aa_r.data(), cur_u.data(), cur_du.data(), cur_d2u.data(), false);
    double s = 0.0;
    for (int j = 0; j < N; ++j)
      s += cur_u[j];
    j2_cur_Uat            = s;
    const double DiffVal  = j2_Uat[iat] - j2_cur_Uat;
    const double* dX[3]   = {aa_dx.data(), aa_dy.data(), aa_dz.data()};
    for (int c = 0; c < 3; ++c)
    {
      double g = 0.0;
      for (int j = 0; j < N; ++j)
        g += cur_du[j] * dX[c][j];
      grad[c] += g;
    }
    return std::exp(DiffVal);
  }
  double j2_ratio(int iat)
  {
    j2_partial = false;
    double cur = 0.0;
    const int gfirst[2] = {0, sys->n_up}, glast[2] = {sys->n_up, sys->n_elec};
    for (int jg = 0; jg < 2; ++jg)
      cur += j2f(egroup(iat), jg).evaluateV(iat, gfirst[jg], glast[jg], aa_r.data());
    j2_cur_Uat = cur;
    return std::exp(j2_Uat[iat] - j2_cur_Uat);
  }
  void j2_accept(int iat)
  {
    const int N     = sys->n_elec;
    const double lf = 3 - 1.0;
    aa_row_current(iat); // Distances[iat] / Displacements[iat] of setActive
    j2_computeU3(iat, row_r.data(), old_u.data(), old_du.data(), old_d2u.data(), false);
    if (!j2_partial)
      j2_computeU3(iat, aa_r.data(), cur_u.data(), cur_du.data(), cur_d2u.data(), false);
    double cur_d2Uat = 0.0;
    for (int j = 0; j < N; j++)
    {
      const double du   = cur_u[j] - old_u[j];
      const double newl = cur_d2u[j] + lf * cur_du[j];
      const double dl   = old_d2u[j] + lf * old_du[j] - newl;
      j2_Uat[j] += du;
      j2_d2Uat[j] += dl;
      cur_d2Uat -= newl;
    }
    Vec3 cur_dUat{0, 0, 0};
    const double* new_dX[3] = {aa_dx.data(), aa_dy.data(), aa_dz.data()};
    const double* old_dX[3] = {row_dx.data(), row_dy.data(), row_dz.data()};
    for (int c = 0; c < 3; ++c)
    {
      double cur_g = cur_dUat[c];
      for (int j = 0; j < N; j++)
      {
        const double newg = cur_du[j] * new_dX[c][j];
        const double dg   = newg - old_du[j] * old_dX[c][j];
        j2_dUat[3 * j + c] -= dg;
        cur_g += newg;
      }
      cur_dUat[c] = cur_g;
    }
    j2_LogValue += j2_Uat[iat] - j2_cur_Uat;
    j2_Uat[iat] = j2_cur_Uat;
    for (int c = 0; c < 3; ++c)
      j2_dUat[3 * iat + c] = cur_dUat[c];
    j2_d2Uat[iat] = cur_d2Uat;
  }
  void j2_GL()
  {
    const int N = sys->n_elec;
    double s    = 0.0;
    for (int i = 0; i < N; ++i)
    {
      s += j2_Uat[i];
      for (int c = 0; c < 3; ++c)
        G[3 * i + c] += j2_dUat[3 * i + c];
      L[i] += j2_d2Uat[i];
    }
    j2_LogValue = -0.5 * s;
  }

  // ---- three-body Jastrow (ThreeBodyJastrow.h:30-677) ----
  std::vector<double> j3_Uat, j3_dUat, j3_d2Uat;                         // dUat [N][3]
  std::vector<double> j3_newUk, j3_newdUk, j3_newd2Uk, j3_oldUk, j3_olddUk, j3_oldd2Uk;
  double j3_cur_Uat = 0, j3_cur_d2Uat = 0, j3_LogValue = 0;
  Vec3 j3_cur_dUat{0, 0, 0};
  bool j3_partial = false;
  std::vector<double> j3_cut;                    // [I] half the functor cutoff
  std::vector<std::vector<int>> j3_in;           // [eg * I + ion] elecs_inside
  std::vector<std::vector<double>> j3_in_d;      // their e-I distances
  std::vector<std::vector<Vec3>> j3_in_dx;       // their e-I displacements
  std::vector<double> c_jk, c_jI, c_kI;          // compressed pair lists
  std::vector<Vec3> c_djk, c_djI, c_dkI;
  std::vector<int> c_idx;
  std::vector<double> j3_r, j3_dx, j3_dy, j3_dz; // e-I row scratch

  const J3Func& j3f(int ig, int jg, int kg) const { return jg == kg ? sys->j3_same[ig] : sys->j3_diff[ig]; }
  void j3_init()
  {
    const int N = sys->n_elec, I = sys->n_ions;
    for (auto* v : {&j3_Uat, &j3_d2Uat, &j3_newUk, &j3_newd2Uk, &j3_oldUk, &j3_oldd2Uk})
      v->assign(N, 0.0);
    for (auto* v : {&j3_dUat, &j3_newdUk, &j3_olddUk})
      v->assign((size_t)N * 3, 0.0);
    j3_cut.assign(I, 0.0);
    for (int i = 0; i < I; ++i)
      j3_cut[i] = 0.5 * sys->j3_same[sys->ion_group[i]].cutoff_radius;
    j3_in.assign(2 * I, {});
    j3_in_d.assign(2 * I, {});
    j3_in_dx.assign(2 * I, {});
    for (auto* v : {&c_jk, &c_jI, &c_kI})
      v->assign(N, 0.0);
    for (auto* v : {&c_djk, &c_djI, &c_dkI})
      v->assign(N, Vec3{0, 0, 0});
    c_idx.assign(N, 0);
    for (auto* v : {&j3_r, &j3_dx, &j3_dy, &j3_dz})
      v->assign(I, 0.0);
  }
  // build_compact_list (ThreeBodyJastrow.h:222-243)
  void j3_build_lists()
  {
    const int N = sys->n_elec, I = sys->n_ions;
    for (auto& v : j3_in)
      v.clear();
    for (auto& v : j3_in_d)
      v.clear();
    for (auto& v : j3_in_dx)
      v.clear();
    for (int jel = 0; jel < N; ++jel)
    {
      const int jg = egroup(jel);
      ab_row(pos(jel), j3_r.data(), j3_dx.data(), j3_dy.data(), j3_dz.data());
      for (int iat = 0; iat < I; ++iat)
        if (j3_r[iat] < j3_cut[iat])
        {
          j3_in[jg * I + iat].push_back(jel);
          j3_in_d[jg * I + iat].push_back(j3_r[iat]);
          j3_in_dx[jg * I + iat].push_back(Vec3{j3_dx[iat], j3_dy[iat], j3_dz[iat]});
        }
    }
  }
  // computeU3_engine (ThreeBodyJastrow.h:484-580): evaluateVGL of the
  // compressed pairs, then the contributions to jel and to every kel
  void j3_engine(const J3Func& f, int cnt, double& Uj, Vec3& dUj, double& d2Uj, double* Uk, double* dUk, double* d2Uk)
  {
    std::vector<double> val(cnt), g0(cnt), g1(cnt), g2(cnt), h00(cnt), h11(cnt), h22(cnt), h01(cnt), h02(cnt);
    for (int p = 0; p < cnt; ++p)
    {
      double gr[3], h[6];
      val[p] = f.eval(c_jk[p], c_jI[p], c_kI[p], gr, h);
      g0[p]  = gr[0] / c_jk[p];
      g1[p]  = gr[1] / c_jI[p];
      g2[p]  = gr[2] / c_kI[p];
      h00[p] = h[0];
      h11[p] = h[3];
      h22[p] = h[5];
      h01[p] = h[1] / (c_jk[p] * c_jI[p]);
      h02[p] = h[2] / (c_jk[p] * c_kI[p]);
    }
    double s_g0 = 0, s_g1 = 0, s_h00 = 0, s_h11 = 0;
    for (int p = 0; p < cnt; ++p)
      Uj += val[p];
    for (int p = 0; p < cnt; ++p)
      s_g0 += g0[p];
    for (int p = 0; p < cnt; ++p)
      s_g1 += g1[p];
    for (int p = 0; p < cnt; ++p)
      s_h00 += h00[p];
    for (int p = 0; p < cnt; ++p)
      s_h11 += h11[p];
    d2Uj -= s_h00 + s_h11 + 2.0 * (s_g0 + s_g1);
    std::fill(h11.begin(), h11.end(), 0.0);
    for (int d = 0; d < 3; ++d)
    {
      double dx = 0.0;
      for (int p = 0; p < cnt; ++p)
      {
        h11[p] += c_dkI[p][d] * c_djk[p][d];
        dx += g1[p] * c_djI[p][d];
        const double temp = c_djk[p][d] * g0[p];
        dx += temp;
        c_djk[p][d] *= c_djI[p][d];
        c_dkI[p][d] = c_dkI[p][d] * g2[p] - temp;
      }
      dUj[d] += dx;
      if (d > 0)
        for (int p = 0; p < cnt; ++p)
          c_djk[p][0] += c_djk[p][d];
      for (int p = 0; p < cnt; ++p)
        dUk[3 * c_idx[p] + d] += c_dkI[p][d];
    }
    double sum = 0.0;
    for (int p = 0; p < cnt; ++p)
      sum += h01[p] * c_djk[p][0];
    d2Uj -= 2.0 * sum;
    for (int p = 0; p < cnt; ++p)
      h00[p] = h00[p] + h22[p] + 2.0 * (g0[p] + g2[p]) - 2.0 * h02[p] * h11[p];
    for (int p = 0; p < cnt; ++p)
    {
      Uk[c_idx[p]] += val[p];
      d2Uk[c_idx[p]] -= h00[p];
    }
  }
  // computeU3 (ThreeBodyJastrow.h:582-654)
  void j3_computeU3(int jel, const double* rI, const double* dxI, const double* dyI, const double* dzI,
                    const double* rk, const double* dxk, const double* dyk, const double* dzk, double& Uj, Vec3& dUj,
                    double& d2Uj, double* Uk, double* dUk, double* d2Uk, bool triangle)
  {
    const int N = sys->n_elec, I = sys->n_ions;
    Uj = 0.0, dUj = Vec3{0, 0, 0}, d2Uj = 0.0;
    const int jg = egroup(jel), kelmax = triangle ? jel : N;
    std::fill_n(Uk, kelmax, 0.0);
    std::fill_n(d2Uk, kelmax, 0.0);
    std::fill_n(dUk, 3 * (size_t)kelmax, 0.0);
    std::vector<int> near;
    for (int iat = 0; iat < I; ++iat)
      if (rI[iat] < j3_cut[iat])
        near.push_back(iat);
    for (int kg = 0; kg < 2; ++kg)
    {
      int cnt = 0;
      for (size_t ii = 0; ii < near.size(); ++ii)
      {
        const int iat = near[ii], ig = sys->ion_group[iat];
        const Vec3 djI{dxI[iat], dyI[iat], dzI[iat]};
        const auto& lst = j3_in[kg * I + iat];
        for (size_t kk = 0; kk < lst.size(); ++kk)
        {
          const int kel = lst[kk];
          if (kel < kelmax && kel != jel)
          {
            c_kI[cnt]  = j3_in_d[kg * I + iat][kk];
            c_jI[cnt]  = rI[iat];
            c_jk[cnt]  = rk[kel];
            c_dkI[cnt] = j3_in_dx[kg * I + iat][kk];
            c_djI[cnt] = djI;
            c_djk[cnt] = Vec3{dxk[kel], dyk[kel], dzk[kel]};
            c_idx[cnt] = kel;
            if (++cnt == N)
            {
              j3_engine(j3f(ig, jg, kg), cnt, Uj, dUj, d2Uj, Uk, dUk, d2Uk);
              cnt = 0;
            }
          }
        }
        if ((ii + 1 == near.size() || ig != sys->ion_group[near[ii + 1]]) && cnt > 0)
        {
          j3_engine(j3f(ig, jg, kg), cnt, Uj, dUj, d2Uj, Uk, dUk, d2Uk);
          cnt = 0;
        }
      }
    }
  }
  // computeU (ThreeBodyJastrow.h:429-482): the value only
  double j3_computeU(int jel, const double* rI, const double* rk)
  {
    const int I = sys->n_ions, N = sys->n_elec, jg = egroup(jel);
    std::vector<int> near;
    for (int iat = 0; iat < I; ++iat)
      if (rI[iat] < j3_cut[iat])
        near.push_back(iat);
    double Uj = 0.0;
    auto evalV = [&](const J3Func& f, int cnt) {
      const double L = 0.5 * f.cutoff_radius;
      double tot     = 0.0;
      for (int p = 0; p < cnt; ++p)
      {
        double val = 0.0, r2l = 1.0;
        for (int l = 0; l <= J3Func::NeI; l++)
        {
          double r2m = r2l;
          for (int m = 0; m <= J3Func::NeI; m++)
          {
            double r2n = r2m;
            for (int n = 0; n <= J3Func::Nee; n++)
            {
              val += f.gamma[l][m][n] * r2n;
              r2n *= c_jk[p];
            }
            r2m *= c_kI[p];
          }
          r2l *= c_jI[p];
        }
        const double b = (c_kI[p] - L) * (c_jI[p] - L);
        for (int i = 0; i < J3Func::C; i++)
          val *= b;
        tot += val;
      }
      return tot;
    };
    for (int kg = 0; kg < 2; ++kg)
    {
      int cnt = 0;
      for (size_t ii = 0; ii < near.size(); ++ii)
      {
        const int iat = near[ii], ig = sys->ion_group[iat];
        const auto& lst = j3_in[kg * I + iat];
        for (size_t kk = 0; kk < lst.size(); ++kk)
        {
          const int kel = lst[kk];
          if (kel != jel)
          {
            c_kI[cnt] = j3_in_d[kg * I + iat][kk];
            c_jk[cnt] = rk[kel];
            c_jI[cnt] = rI[iat];
            if (++cnt == N)
            {
              Uj += evalV(j3f(ig, jg, kg), cnt);
              cnt = 0;
            }
          }
        }
        if ((ii + 1 == near.size() || ig != sys->ion_group[near[ii + 1]]) && cnt > 0)
        {
          Uj += evalV(j3f(ig, jg, kg), cnt);
          cnt = 0;
        }
      }
    }
    return Uj;
  }
  // recompute (ThreeBodyJastrow.h:391-427)
  void j3_recompute()
  {
    const int N = sys->n_elec;
    j3_build_lists();
    for (int jel = 0; jel < N; ++jel)
    {
      ab_row(pos(jel), j3_r.data(), j3_dx.data(), j3_dy.data(), j3_dz.data());
      aa_row_current(jel);
      Vec3 dU;
      j3_computeU3(jel, j3_r.data(), j3_dx.data(), j3_dy.data(), j3_dz.data(), row_r.data(), row_dx.data(),
                   row_dy.data(), row_dz.data(), j3_Uat[jel], dU, j3_d2Uat[jel], j3_newUk.data(), j3_newdUk.data(),
                   j3_newd2Uk.data(), true);
      for (int c = 0; c < 3; ++c)
        j3_dUat[3 * jel + c] = dU[c];
      for (int kel = 0; kel < jel; kel++)
      {
        j3_Uat[kel] += j3_newUk[kel];
        j3_d2Uat[kel] += j3_newd2Uk[kel];
      }
      for (int c = 0; c < 3; ++c)
        for (int kel = 0; kel < jel; kel++)
          j3_dUat[3 * kel + c] += j3_newdUk[3 * kel + c];
    }
  }
  void j3_GL()
  {
    const int N = sys->n_elec;
    double s    = 0.0;
    for (int i = 0; i < N; ++i)
    {
      s += j3_Uat[i];
      for (int c = 0; c < 3; ++c)
        G[3 * i + c] += j3_dUat[3 * i + c];
      L[i] += j3_d2Uat[i];
    }
    j3_LogValue = -0.5 * s;
  }
  double j3_ratioGrad(int iat, Vec3& grad)
  {
    j3_partial = true;
    j3_computeU3(iat, ab_r.data(), ab_dx.data(), ab_dy.data(), ab_dz.data(), aa_r.data(), aa_dx.data(), aa_dy.data(),
                 aa_dz.data(), j3_cur_Uat, j3_cur_dUat, j3_cur_d2Uat, j3_newUk.data(), j3_newdUk.data(),
                 j3_newd2Uk.data(), false);
    for (int c = 0; c < 3; ++c)
      grad[c] += j3_cur_dUat[c];
    return std::exp(j3_Uat[iat] - j3_cur_Uat);
  }
  double j3_ratio(int iat)
  {
    j3_partial = false;
    j3_cur_Uat = j3_computeU(iat, ab_r.data(), aa_r.data());
    return std::exp(j3_Uat[iat] - j3_cur_Uat);
  }
  // acceptMove (ThreeBodyJastrow.h:300-389)
  void j3_accept(int iat)
  {
    const int N = sys->n_elec, I = sys->n_ions;
    ab_row(pos(iat), j3_r.data(), j3_dx.data(), j3_dy.data(), j3_dz.data());
    aa_row_current(iat);
    Vec3 dtemp;
    j3_computeU3(iat, j3_r.data(), j3_dx.data(), j3_dy.data(), j3_dz.data(), row_r.data(), row_dx.data(),
                 row_dy.data(), row_dz.data(), j3_Uat[iat], dtemp, j3_d2Uat[iat], j3_oldUk.data(), j3_olddUk.data(),
                 j3_oldd2Uk.data(), false);
    if (!j3_partial)
      j3_computeU3(iat, ab_r.data(), ab_dx.data(), ab_dy.data(), ab_dz.data(), aa_r.data(), aa_dx.data(),
                   aa_dy.data(), aa_dz.data(), j3_cur_Uat, j3_cur_dUat, j3_cur_d2Uat, j3_newUk.data(),
                   j3_newdUk.data(), j3_newd2Uk.data(), false);
    for (int jel = 0; jel < N; jel++)
    {
      j3_Uat[jel] += j3_newUk[jel] - j3_oldUk[jel];
      j3_d2Uat[jel] += j3_newd2Uk[jel] - j3_oldd2Uk[jel];
    }
    for (int c = 0; c < 3; ++c)
      for (int jel = 0; jel < N; jel++)
        j3_dUat[3 * jel + c] += j3_newdUk[3 * jel + c] - j3_olddUk[3 * jel + c];
    j3_LogValue += j3_Uat[iat] - j3_cur_Uat;
    j3_Uat[iat] = j3_cur_Uat;
    for (int c = 0; c < 3; ++c)
      j3_dUat[3 * iat + c] = j3_cur_dUat[c];
    j3_d2Uat[iat] = j3_cur_d2Uat;
    const int ig = egroup(iat);
    for (int jat = 0; jat < I; jat++)
    {
      auto& lst      = j3_in[ig * I + jat];
      auto& ld       = j3_in_d[ig * I + jat];
      auto& lx       = j3_in_dx[ig * I + jat];
      const bool in  = ab_r[jat] < j3_cut[jat];
      const auto it  = std::find(lst.begin(), lst.end(), iat);
      const size_t k = it - lst.begin();
      if (in)
      {
        if (it == lst.end())
        {
          lst.push_back(iat);
          ld.push_back(ab_r[jat]);
          lx.push_back(Vec3{ab_dx[jat], ab_dy[jat], ab_dz[jat]});
        }
        else
        {
          ld[k] = ab_r[jat];
          lx[k] = Vec3{ab_dx[jat], ab_dy[jat], ab_dz[jat]};
        }
      }
      else if (it != lst.end())
      {
        lst[k] = lst.back();
        lst.pop_back();
        ld[k] = ld.back();
        ld.pop_back();
        lx[k] = lx.back();
        lx.pop_back();
      }
    }
  }

  // ---- ParticleSet protocol (ParticleSet.cpp:280-378) ----
  void makeMove(int iat, const Vec3& displ)
  {
    activePtcl = iat;
    for (int c = 0; c < 3; ++c)
      activePos[c] = R[3 * iat + c] + displ[c];
    sys->lattice.computeDistances(activePos, R.data(), aa_r.data(), aa_dx.data(), aa_dy.data(),
                                  aa_dz.data(), 0, sys->n_elec, iat);
    ab_row(activePos, ab_r.data(), ab_dx.data(), ab_dy.data(), ab_dz.data());
  }
  bool acceptMove_pset(int iat)
  {
    if (iat != activePtcl)
      return false;
    for (int c = 0; c < 3; ++c)
      R[3 * iat + c] = activePos[c];
    activePtcl = -1;
    return true;
  }
  void rejectMove_pset(int) { activePtcl = -1; }

  // ---- NonLocalPP ratios (miniqmc.cpp:472-495, NonLocalPP.hpp:115-134) ----
  // For every electron and every ion within rmax (the e-I row of
  // DistanceTableBA: r and ion - electron), WaveFunction::ratio at the 12
  // points of `rot`: form 0 puts them at R + displ + r rot_k
  // (NonLocalPP::evaluate), form 1 at R + r rot_k - displ (the driver's
  // makeMove).  Returns the sum of ratio / 12; appends the ratios.
  double nlpp(double rmax, int form, const double (*rot)[3], long long& count, std::vector<double>* out)
  {
    const int N = sys->n_elec, I = sys->n_ions;
    std::vector<double> r(I), dx(I), dy(I), dz(I);
    double sum = 0.0;
    for (int jel = 0; jel < N; ++jel)
    {
      ab_row(pos(jel), r.data(), dx.data(), dy.data(), dz.data());
      for (int iat = 0; iat < I; ++iat)
        if (r[iat] < rmax)
          for (int k = 0; k < 12; ++k)
          {
            const double sg = form == 0 ? 1.0 : -1.0;
            const Vec3 d{sg * dx[iat] + r[iat] * rot[k][0], sg * dy[iat] + r[iat] * rot[k][1],
                         sg * dz[iat] + r[iat] * rot[k][2]};
            makeMove(jel, d);
            const double q = ratio(jel);
            rejectMove_pset(jel);
            sum += q / 12.0;
            ++count;
            if (out)
              out->push_back(q);
          }
    }
    return sum;
  }

  // ---- WaveFunction::evaluateRatios over a VirtualParticleSet
  // (NonLocalPP.hpp:115-134, DiracDeterminant.cpp:216-224): the ratio of
  // electron jel at each absolute position, the determinants' update mode
  // left as it was ----
  void evaluateRatios(int jel, int n, const double* p, double* out)
  {
    const int s     = jel < sys->n_up ? 0 : 1;
    const bool keep = det[s].partial;
    for (int k = 0; k < n; ++k)
    {
      activePtcl = jel;
      for (int c = 0; c < 3; ++c)
        activePos[c] = p[3 * k + c];
      sys->lattice.computeDistances(activePos, R.data(), aa_r.data(), aa_dx.data(), aa_dy.data(), aa_dz.data(), 0,
                                    sys->n_elec, jel);
      ab_row(activePos, ab_r.data(), ab_dx.data(), ab_dy.data(), ab_dz.data());
      out[k] = ratio(jel);
      rejectMove_pset(jel);
    }
    det[s].partial = keep;
  }

  // ---- WaveFunction (WaveFunction.cpp:178-279) ----
  bool evaluateLog()
  {
    std::fill(G.begin(), G.end(), 0.0);
    std::fill(L.begin(), L.end(), 0.0);
    activePtcl = -1;
    bool ok    = true;
    if (sys->use_det)
      for (int s = 0; s < 2; ++s)
      {
        ok &= det_recompute(s);
        det[s].partial = true;
        det_GL(s);
      }
    LogValue = det[0].LogValue + det[1].LogValue;
    if (sys->use_j1)
    {
      j1_recompute();
      j1_GL();
      LogValue += j1_LogValue;
    }
    if (sys->use_j2)
    {
      j2_recompute();
      j2_GL();
      LogValue += j2_LogValue;
    }
    if (sys->use_j3)
    {
      j3_recompute();
      j3_GL();
      LogValue += j3_LogValue;
    }
    return ok;
  }
  Vec3 evalGrad(int iat)
  {
    const int s = iat < sys->n_up ? 0 : 1;
    Vec3 g      = sys->use_det ? det_evalGrad(s, iat) : Vec3{0, 0, 0};
    if (sys->use_j1)
      for (int c = 0; c < 3; ++c)
        g[c] += j1_Grad[3 * iat + c];
    if (sys->use_j2)
      for (int c = 0; c < 3; ++c)
        g[c] += j2_dUat[3 * iat + c];
    if (sys->use_j3)
      for (int c = 0; c < 3; ++c)
        g[c] += j3_dUat[3 * iat + c];
    return g;
  }
  double ratioGrad(int iat, Vec3& grad)
  {
    grad         = Vec3{0, 0, 0};
    const int s  = iat < sys->n_up ? 0 : 1;
    double ratio = sys->use_det ? det_ratioGrad(s, iat, grad) : 1.0;
    if (sys->use_j1)
      ratio *= j1_ratioGrad(iat, grad);
    if (sys->use_j2)
      ratio *= j2_ratioGrad(iat, grad);
    if (sys->use_j3)
      ratio *= j3_ratioGrad(iat, grad);
    return ratio;
  }
  double ratio(int iat)
  {
    const int s = iat < sys->n_up ? 0 : 1;
    double r    = sys->use_det ? det_ratio(s, iat) : 1.0;
    if (sys->use_j1)
      r *= j1_ratio(iat);
    if (sys->use_j2)
      r *= j2_ratio(iat);
    if (sys->use_j3)
      r *= j3_ratio(iat);
    return r;
  }
  void acceptMove(int iat)
  {
    const int s = iat < sys->n_up ? 0 : 1;
    if (sys->use_det)
      det_accept(s, iat);
    if (sys->use_j1)
      j1_accept(iat);
    if (sys->use_j2)
      j2_accept(iat);
    if (sys->use_j3)
      j3_accept(iat);
  }
  void completeUpdates()
  {
    if (!sys->use_det)
      return;
    det_complete(0);
    det_complete(1);
  }
  void evaluateGL()
  {
    std::fill(G.begin(), G.end(), 0.0);
    std::fill(L.begin(), L.end(), 0.0);
    if (sys->use_det)
    {
      det_GL(0);
      det_GL(1);
    }
    LogValue = det[0].LogValue + det[1].LogValue;
    if (sys->use_j1)
    {
      j1_GL();
      LogValue += j1_LogValue;
    }
    if (sys->use_j2)
    {
      j2_GL();
      LogValue += j2_LogValue;
    }
    if (sys->use_j3)
    {
      j3_GL();
      LogValue += j3_LogValue;
    }
  }
};

} // namespace oracle
