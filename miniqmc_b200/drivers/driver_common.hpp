// driver_common.hpp -- pieces shared by the command-line drivers over the C
// ABI: the reference's seeds and host random streams, its NiO system, timers.
#pragma once

#include "qmcgpu.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

namespace drv
{
// PrimeNumberSet<uint32_t> (PrimeNumberSet.h): the primes from 3 upwards
inline std::vector<uint32_t> primes(int n)
{
  std::vector<uint32_t> p;
  for (uint32_t c = 3; (int)p.size() < n; c += 2)
  {
    bool ok = true;
    for (uint32_t q : p)
    {
      if (q * q > c)
        break;
      if (c % q == 0)
      {
        ok = false;
        break;
      }
    }
    if (ok)
      p.push_back(c);
  }
  return p;
}

inline double now_s()
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

inline int check(int st, const char* what)
{
  if (st != QMC_OK)
    std::fprintf(stderr, "%s failed: %s (%s)\n", what, qmc_status_string(st), qmc_last_error());
  return st;
}

// A mover's host random stream as the reference draws it: StdRandom's
// mt19937 with libstdc++'s uniform_real_distribution<double> (StdRandom.h),
// normals by BoxMuller2 (RandomGenerator.h:46-79)
struct HostRng
{
  std::mt19937 mt;
  std::uniform_real_distribution<double> uni;
  explicit HostRng(uint32_t seed) : mt(seed) {}
  double uniform() { return uni(mt); }
  void uniform(double* d, int n)
  {
    for (int i = 0; i < n; ++i)
      d[i] = uni(mt);
  }
  void normal(double* a, int n)
  {
    auto pair = [&](double& c, double* s) {
      const double t1 = 1.0 - 0.9999999999 * uni(mt), t2 = uni(mt);
      const double r  = std::sqrt(-2.0 * std::log(t1));
      c               = r * std::cos(6.283185306 * t2);
      if (s)
        *s = r * std::sin(6.283185306 * t2);
    };
    int i = 0;
    for (; i + 1 < n; i += 2)
      pair(a[i], a + i + 1);
    if (i < n)
      pair(a[i], nullptr);
  }
};

// The reference's NiO input (nio.hpp:23-79, build_ions + count_electrons)
// on a tiling of its 32-atom cell, with its spline grid and Jastrows; the
// arrays the description points to live here.
struct NioSystem
{
  qmc_system_desc d;
  std::vector<double> ion_pos;
  std::vector<int> ion_group;
  int n_ions = 0, nels = 0, norb = 0;

  int build(int na, int nb, int nc, int nx, int ny, int nz, bool fill_reference, int seed, int components)
  {
    std::memset(&d, 0, sizeof(d));
    if (check(qmc_nio_count(QMC_NIO_REF32, na, nb, nc, &n_ions), "qmc_nio_count"))
      return 1;
    ion_pos.assign(3 * (size_t)n_ions, 0.0);
    ion_group.assign(n_ions, 0);
    if (check(qmc_nio_build(QMC_NIO_REF32, na, nb, nc, 0, d.lattice, ion_pos.data(), ion_group.data(),
                            &d.n_ion_groups, d.spo_lattice),
              "qmc_nio_build"))
      return 1;
    nels = 0;
    for (int g : ion_group)
      nels += g == 0 ? 6 : 18; // valence electrons of O and Ni
    norb     = nels / 2;
    d.n_ions = n_ions, d.ion_pos = ion_pos.data(), d.ion_group = ion_group.data();
    d.n_elec = nels, d.n_up = norb, d.n_orb = norb;
    d.grid[0] = nx, d.grid[1] = ny, d.grid[2] = nz;
    d.spo_fill   = fill_reference ? QMC_FILL_REFERENCE : QMC_FILL_UNIFORM;
    d.spo_seed   = (uint64_t)seed;
    d.lap_mode   = QMC_LAP_HXX;
    d.components = components;
    if (check(qmc_nio_jastrows(d.lattice, &d.j1[0], &d.j1[1], &d.j2_uu, &d.j2_ud), "qmc_nio_jastrows"))
      return 1;
    if (components & QMC_WF_J3)
    {
      qmc_j3_functor same[2], diff[2];
      if (check(qmc_nio_j3(d.lattice, same, diff), "qmc_nio_j3"))
        return 1;
      for (int g = 0; g < d.n_ion_groups; ++g)
        d.j3_same[g] = same[g < 2 ? g : 1], d.j3_diff[g] = diff[g < 2 ? g : 1];
    }
    return 0;
  }
};

} // namespace drv
