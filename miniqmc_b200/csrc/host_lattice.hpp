// host_lattice.hpp -- host-side cell geometry and NiO input for the product.
//
// Restates, for the library's own use: CrystalLattice::reset (inverse,
// Wigner-Seitz radius; CrystalLattice.cpp:88-127, LatticeAnalyzer.h:86-131),
// find_reduced_basis and the DTD_BConds corners (LatticeAnalyzer.h:134-183,
// ParticleBConds.h:106-151), the NiO cell of nio.hpp:23-79 with
// expandSuperCell (ParticleIOUtility.h:29-117), the Jastrow tables of
// nio.hpp:81-168 and BsplineFunctor::setupParameters (BsplineFunctor.h:93-130).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

#include "../../include/qmcgpu.h"

namespace qmc_host
{
inline double det3(const double* a)
{
  return a[0] * (a[4] * a[8] - a[5] * a[7]) + a[1] * (a[5] * a[6] - a[3] * a[8]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}
inline void inverse3(const double* a, double* g)
{
  const double vinv = 1 / det3(a);
  g[0] = vinv * (a[4] * a[8] - a[5] * a[7]);
  g[1] = vinv * (a[7] * a[2] - a[8] * a[1]);
  g[2] = vinv * (a[1] * a[5] - a[2] * a[4]);
  g[3] = vinv * (a[5] * a[6] - a[3] * a[8]);
  g[4] = vinv * (a[8] * a[0] - a[6] * a[2]);
  g[5] = vinv * (a[2] * a[3] - a[0] * a[5]);
  g[6] = vinv * (a[3] * a[7] - a[4] * a[6]);
  g[7] = vinv * (a[6] * a[1] - a[7] * a[0]);
  g[8] = vinv * (a[0] * a[4] - a[1] * a[3]);
}
inline double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

inline double ws_radius(const double* R)
{
  double rmin = 0.5 * std::numeric_limits<double>::max();
  for (int i = -1; i <= 1; i++)
    for (int j = -1; j <= 1; j++)
      for (int k = -1; k <= 1; k++)
        if (i || j || k)
        {
          double L[3];
          for (int d = 0; d < 3; ++d)
            L[d] = (double)i * R[d] + (double)j * R[3 + d] + (double)k * R[6 + d];
          rmin = std::min(rmin, dot3(L, L));
        }
  double ws  = 0.5 * std::sqrt(rmin);
  double scr = 0.5 * std::numeric_limits<double>::max();
  for (int i = 0; i < 3; ++i)
  {
    const double* A = R + 3 * i;
    const double* B = R + 3 * ((i + 1) % 3);
    const double* C = R + 3 * ((i + 2) % 3);
    double BxC[3]   = {B[1] * C[2] - B[2] * C[1], B[2] * C[0] - B[0] * C[2], B[0] * C[1] - B[1] * C[0]};
    scr             = std::min(scr, 0.5 * std::abs(dot3(A, BxC)) / std::sqrt(dot3(BxC, BxC)));
  }
  if (ws > scr && ws - scr <= ws * std::numeric_limits<float>::epsilon() * 2)
    ws = scr;
  return ws;
}

inline bool shorter_base(double rb[3][3])
{
  const double eps = 10.0 * std::numeric_limits<float>::epsilon();
  int imax         = 0;
  double r2max     = dot3(rb[0], rb[0]);
  for (int i = 1; i < 3; i++)
  {
    const double r2 = dot3(rb[i], rb[i]);
    if ((r2 - r2max) > eps)
      r2max = r2, imax = i;
  }
  double cand[4][3];
  for (int d = 0; d < 3; ++d)
  {
    cand[0][d] = rb[0][d] + rb[1][d] - rb[2][d];
    cand[1][d] = rb[0][d] + rb[2][d] - rb[1][d];
    cand[2][d] = rb[1][d] + rb[2][d] - rb[0][d];
    cand[3][d] = rb[0][d] + rb[1][d] + rb[2][d];
  }
  for (int i = 0; i < 4; ++i)
    if ((dot3(cand[i], cand[i]) - r2max) < -eps)
    {
      std::memcpy(rb[imax], cand[i], sizeof(cand[i]));
      return true;
    }
  return false;
}
inline void reduced_basis(double rb[3][3])
{
  for (;;)
  {
    double saved[3][3];
    std::memcpy(saved, rb, sizeof(saved));
    bool changed = false;
    for (int i = 0; i < 3; ++i)
    {
      rb[i][0] = rb[i][1] = rb[i][2] = 0.0;
      changed = shorter_base(rb);
      std::memcpy(rb[i], saved[i], sizeof(saved[i]));
      if (changed)
        break;
    }
    if (!changed && !shorter_base(rb))
      return;
  }
}

// DTD_BConds state for a cell: reduced basis rows, inverse, 8 corners
inline void bconds(const double* R, double* rb9, double* gb9, double* corners24)
{
  double rb[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      rb[i][j] = R[3 * i + j];
  reduced_basis(rb);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      rb9[3 * i + j] = rb[i][j];
  inverse3(rb9, gb9);
  for (int d = 0; d < 3; ++d)
  {
    corners24[0 * 3 + d] = 0.0;
    corners24[1 * 3 + d] = -1.0 * rb[0][d];
    corners24[2 * 3 + d] = -1.0 * rb[1][d];
    corners24[3 * 3 + d] = -1.0 * rb[2][d];
    corners24[4 * 3 + d] = -1.0 * (rb[0][d] + rb[1][d]);
    corners24[5 * 3 + d] = -1.0 * (rb[0][d] + rb[2][d]);
    corners24[6 * 3 + d] = -1.0 * (rb[1][d] + rb[2][d]);
    corners24[7 * 3 + d] = -1.0 * (rb[0][d] + rb[1][d] + rb[2][d]);
  }
}

// smallest eigenvalue of the symmetric 3x3 matrix rb rb^T (cyclic Jacobi)
inline double min_metric_eigenvalue(const double* rb)
{
  double a[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      a[i][j] = rb[3 * i] * rb[3 * j] + rb[3 * i + 1] * rb[3 * j + 1] + rb[3 * i + 2] * rb[3 * j + 2];
  for (int sweep = 0; sweep < 60; ++sweep)
  {
    double off = std::abs(a[0][1]) + std::abs(a[0][2]) + std::abs(a[1][2]);
    if (off < 1e-300)
      break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q)
      {
        if (std::abs(a[p][q]) < 1e-300)
          continue;
        const double theta = (a[q][q] - a[p][p]) / (2 * a[p][q]);
        const double t     = (theta >= 0 ? 1.0 : -1.0) / (std::abs(theta) + std::sqrt(theta * theta + 1));
        const double c = 1 / std::sqrt(t * t + 1), s = t * c;
        for (int k = 0; k < 3; ++k)
        {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p]          = c * akp - s * akq;
          a[k][q]          = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k)
        {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k]          = c * apk - s * aqk;
          a[q][k]          = s * apk + c * aqk;
        }
      }
  }
  return std::min(a[0][0], std::min(a[1][1], a[2][2]));
}

// r = dot(u, R) (ConvertPosUnit, FastParticleOperators.h:44-56)
inline void to_cart(const double* R, const double* u, double* r)
{
  r[0] = u[0] * R[0] + u[1] * R[3] + u[2] * R[6];
  r[1] = u[0] * R[1] + u[1] * R[4] + u[2] * R[7];
  r[2] = u[0] * R[2] + u[1] * R[5] + u[2] * R[8];
}
inline void to_unit(const double* G, const double* r, double* u)
{
  u[0] = r[0] * G[0] + r[1] * G[3] + r[2] * G[6];
  u[1] = r[0] * G[1] + r[1] * G[4] + r[2] * G[7];
  u[2] = r[0] * G[2] + r[1] * G[5] + r[2] * G[8];
}

static const double kNioCell[9] = {7.8811, 7.8811, 0.0, -7.8811, 7.8811, 0.0, 0.0, 0.0, 15.7622};
// the 32 sites of nio.hpp:37-68 in lattice units: 16 O then 16 Ni
static const double kNio32[32][3] = {
    {0.5, 0.0, 0.25},   {0.0, 0.0, 0.75},   {0.25, 0.25, 0.5},  {0.5, 0.5, 0.25},   {0.75, 0.25, 0.0},
    {0.0, 0.5, 0.75},   {0.25, 0.75, 0.5},  {0.75, 0.75, 0.0},  {0.0, 0.0, 0.25},   {0.25, 0.25, 0.0},
    {0.5, 0.0, 0.75},   {0.75, 0.25, 0.5},  {0.0, 0.5, 0.25},   {0.25, 0.75, 0.0},  {0.5, 0.5, 0.75},
    {0.75, 0.75, 0.5},  {0.0, 0.0, 0.0},    {0.0, 0.5, 0.0},    {0.25, 0.25, 0.75}, {0.5, 0.0, 0.5},
    {0.5, 0.5, 0.5},    {0.75, 0.25, 0.25}, {0.25, 0.75, 0.75}, {0.75, 0.75, 0.25}, {0.5, 0.0, 0.0},
    {0.0, 0.0, 0.5},    {0.25, 0.25, 0.25}, {0.5, 0.5, 0.0},    {0.75, 0.25, 0.75}, {0.0, 0.5, 0.5},
    {0.25, 0.75, 0.25}, {0.75, 0.75, 0.75}};

struct Ions
{
  double lattice[9], spo_lattice[9];
  std::vector<double> pos;
  std::vector<int> group;
  int n_groups = 2;
};

inline Ions nio_ref32(int na, int nb, int nc, int quirks)
{
  Ions s;
  std::memcpy(s.spo_lattice, kNioCell, sizeof(kNioCell));
  std::vector<int> types(32);
  for (int i = 0; i < 32; ++i)
    types[i] = (quirks & QMC_NIO_QUIRK_ONE_GROUP) ? 0 : (i < 16 ? 0 : 1);
  if (na == 1 && nb == 1 && nc == 1)
  {
    std::memcpy(s.lattice, kNioCell, sizeof(kNioCell));
    for (int i = 0; i < 32; ++i)
    {
      double r[3];
      if (quirks & QMC_NIO_QUIRK_UNIT_IONS)
        std::memcpy(r, kNio32[i], sizeof(r));
      else
        to_cart(kNioCell, kNio32[i], r);
      s.pos.insert(s.pos.end(), r, r + 3);
      s.group.push_back(types[i]);
    }
    return s;
  }
  const int t[3] = {na, nb, nc};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
    {
      double sum = 0.0;
      for (int k = 0; k < 3; ++k)
        sum += (double)(i == k ? t[i] : 0) * kNioCell[3 * k + j];
      s.lattice[3 * i + j] = sum;
    }
  double G[9];
  inverse3(s.lattice, G);
  for (int ns = 0; ns < 2; ++ns)
    for (int i0 = -10; i0 <= 10; i0++)
      for (int i1 = -10; i1 <= 10; i1++)
        for (int i2 = -10; i2 <= 10; i2++)
          for (int iat = 0; iat < 32; iat++)
          {
            if (types[iat] != ns)
              continue;
            double up[3], c[3], r[3], u[3];
            for (int d = 0; d < 3; ++d)
              up[d] = kNio32[iat][d] - std::floor(kNio32[iat][d]);
            to_cart(kNioCell, up, c);
            for (int d = 0; d < 3; ++d)
              r[d] = c[d] + (double)i0 * kNioCell[d] + (double)i1 * kNioCell[3 + d] + (double)i2 * kNioCell[6 + d];
            to_unit(G, r, u);
            if (u[0] >= -1.0e-6 && u[0] < 0.9999 && u[1] >= -1.0e-6 && u[1] < 0.9999 && u[2] >= -1.0e-6 &&
                u[2] < 0.9999)
            {
              s.pos.insert(s.pos.end(), r, r + 3);
              s.group.push_back(ns);
            }
          }
  return s;
}

inline Ions nio_prim4(int na, int nb, int nc)
{
  Ions s;
  double prim[9];
  for (int i = 0; i < 9; ++i)
    prim[i] = 0.5 * kNioCell[i];
  const int t[3] = {na, nb, nc};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      s.lattice[3 * i + j] = (double)t[i] * prim[3 * i + j];
  std::memcpy(s.spo_lattice, s.lattice, sizeof(s.lattice));
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
            const double u[3] = {basis[b][0] + i0, basis[b][1] + i1, basis[b][2] + i2};
            double r[3];
            to_cart(prim, u, r);
            s.pos.insert(s.pos.end(), r, r + 3);
            s.group.push_back(ns);
          }
  return s;
}

inline int functor_setup(int n, double rcut, double cusp, const double* params, qmc_functor* out)
{
  if (n < 2 || n + 4 > QMC_MAX_FUNCTOR_COEFS || !params || !out || !(rcut > 0))
    return QMC_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  const int numCoefs = n + 4, numKnots = numCoefs - 2;
  const double DeltaR = rcut / (double)(numKnots - 1);
  out->n_coefs        = numCoefs;
  out->cutoff         = rcut;
  out->delta_r_inv    = 1.0 / DeltaR;
  out->coefs[1]       = params[0];
  out->coefs[2]       = params[1];
  out->coefs[0]       = params[1] - 2.0 * DeltaR * cusp;
  for (int i = 2; i < n; i++)
    out->coefs[i + 1] = params[i];
  return QMC_OK;
}

// PolynomialFunctor3D::reset_gamma (PolynomialFunctor3D.h:113-250) for
// N_eI = N_ee = 3, C = 3.  The 40 distinct gammas (gamma(l,m,n) =
// gamma(m,l,n)) obey 14 linear constraints: for every total e-I power k the
// e-e cusp sum over l + m = k of gamma(l,m,1) vanishes, and for every power
// k' the e-I no-cusp combination C gamma(l,0,n) - L gamma(l,1,n) over
// l + n = k' vanishes.  Reduced row echelon form (largest pivot in the
// column, columns whose remaining entries are all below 1e-6 skipped) splits
// the columns into 14 pivot columns and 26 free ones; the free ones take the
// parameters in column order and each pivot column follows from its row.
inline int j3_functor_setup(double rcut, const double* params, qmc_j3_functor* out)
{
  constexpr int NEI = 3, NEE = 3, CEXP = 3;
  constexpr int NG = (NEI + 1) * (NEI + 2) / 2 * (NEE + 1);
  constexpr int NC = 2 * NEI + 1 + NEI + NEE + 1;
  if (!params || !out || !(rcut > 0))
    return QMC_ERR_ARG;
  const double L = 0.5 * rcut;
  // column of gamma(l, m, n): m outer, then l >= m, then n
  int colof[NEI + 1][NEI + 1][NEE + 1];
  int nc = 0;
  for (int m = 0; m <= NEI; m++)
    for (int l = m; l <= NEI; l++)
      for (int n = 0; n <= NEE; n++)
        colof[l][m][n] = colof[m][l][n] = nc++;
  double A[NC][NG] = {};
  for (int k = 0; k <= 2 * NEI; k++)
    for (int m = 0; m <= k && m <= NEI; m++)
    {
      const int l = k - m;
      if (l <= NEI)
        A[k][colof[l][m][1]] = l > m ? 2.0 : (l == m ? 1.0 : A[k][colof[l][m][1]]);
    }
  for (int kp = 0; kp <= NEI + NEE; kp++)
  {
    double* row = A[2 * NEI + 1 + kp];
    for (int l = 0; l <= std::min(kp, NEI); l++)
    {
      const int n = kp - l;
      if (n > NEE)
        continue;
      row[colof[l][0][n]] = (double)CEXP;
      row[colof[l][1][n]] = -L;
    }
  }
  int pivot_col[NC];
  bool is_free[NG];
  for (int c = 0; c < NG; ++c)
    is_free[c] = true;
  int col = 0;
  for (int r = 0; r < NC; ++r)
  {
    int best = -1;
    for (; col < NG; ++col)
    {
      best      = r;
      double mx = std::fabs(A[r][col]);
      for (int q = r + 1; q < NC; ++q)
        if (std::fabs(A[q][col]) > mx)
          mx = std::fabs(A[q][col]), best = q;
      if (mx >= 1.0e-6)
        break;
    }
    if (col == NG)
      return QMC_ERR_ARG;
    for (int c = 0; c < NG; ++c)
      std::swap(A[r][c], A[best][c]);
    const double inv = 1.0 / A[r][col];
    for (int c = 0; c < NG; ++c)
      A[r][c] *= inv;
    for (int q = 0; q < NC; ++q)
      if (q != r)
      {
        const double f = A[q][col];
        for (int c = 0; c < NG; ++c)
          A[q][c] -= f * A[r][c];
      }
    pivot_col[r] = col;
    is_free[col] = false;
    ++col;
  }
  double g[NG] = {};
  for (int c = 0, p = 0; c < NG; ++c)
    if (is_free[c])
      g[c] = params[p++];
  for (int r = 0; r < NC; ++r)
  {
    const int pc = pivot_col[r];
    for (int c = 0; c < NG; ++c)
      if (c != pc)
        g[pc] -= A[r][c] * g[c];
  }
  out->cutoff = rcut;
  for (int l = 0; l <= NEI; l++)
    for (int m = 0; m <= NEI; m++)
      for (int n = 0; n <= NEE; n++)
        out->gamma[16 * l + 4 * m + n] = g[colof[l][m][n]];
  return QMC_OK;
}

} // namespace qmc_host
