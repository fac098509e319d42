// qmcgpu_adapter.cpp -- SPOSetGpu, the device system and walker batches,
// and WaveFunctionComponentGpu over the C ABI (qmcgpu_adapter.hpp).
#include "qmcgpu_adapter.hpp"

#include <Utilities/RandomGenerator.h>
#include <QMCWaveFunctions/einspline_spo.hpp>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>

namespace qmcplusplus
{
namespace qmcgpu
{
namespace
{
std::mutex g_mu, g_warn_mu;

const char* env(const char* name) { return std::getenv(name); }

bool env_is(const char* name, const char* value)
{
  const char* v = env(name);
  return v && std::strcmp(v, value) == 0;
}

// qmc_init on the calling thread (the device is per host thread)
void ensure_device()
{
  thread_local bool done = false;
  if (done)
    return;
  const char* d = env("QMCGPU_DEVICE");
  check(qmc_init(d ? std::atoi(d) : 0), "qmc_init");
  done = true;
}

// The displacement d with r + d == a in double arithmetic, so that the
// device's R + d (one double add) lands exactly on the host's proposed
// position a.  a - r is exact unless the two differ widely in magnitude;
// then a step of an ulp or two closes the gap.
double exact_displ(double r, double a)
{
  volatile double d = a - r;
  for (int i = 0; i < 8; ++i)
  {
    volatile double s = r + d;
    if (s == a)
      break;
    d = s < a ? std::nextafter((double)d, HUGE_VAL) : std::nextafter((double)d, -HUGE_VAL);
  }
  return d;
}

template <typename PS>
void displacements(const PS& P, int iat, double* d)
{
  for (int c = 0; c < 3; ++c)
    d[c] = exact_displ((double)P.R[iat][c], (double)P.activePos[c]);
}
} // namespace

int check(int status, const char* what)
{
  if (status == QMC_OK)
    return status;
  if (status == QMC_ERR_SINGULAR || status == QMC_ERR_NONFINITE)
  {
    static std::set<std::string> seen;
    std::lock_guard<std::mutex> g(g_warn_mu);
    const std::string key = std::string(what) + qmc_status_string(status);
    if (seen.insert(key).second)
      std::fprintf(stderr, "qmcgpu: %s reported %s (%s)%s\n", what, qmc_status_string(status), qmc_last_error(),
                   status == QMC_ERR_SINGULAR ? "; the reference's own orbital table is singular, "
                                                "QMCGPU_SPO_FILL=uniform gives a well-conditioned one"
                                              : "");
    return status;
  }
  std::fprintf(stderr, "qmcgpu: %s failed: %s (%s)\n", what, qmc_status_string(status), qmc_last_error());
  std::exit(1);
}

void fail(const char* what)
{
  std::fprintf(stderr, "qmcgpu: %s\n", what);
  std::exit(1);
}

DeviceSystem::~DeviceSystem()
{
  if (sys)
    qmc_system_destroy(sys);
}

std::shared_ptr<DeviceSystem> device_system(const SPOSet* spo, const ParticleSet& ions, const ParticleSet& els,
                                            bool j3)
{
  static std::map<const SPOSet*, std::weak_ptr<DeviceSystem>> registry;
  std::lock_guard<std::mutex> g(g_mu);
  ensure_device();
  const int comp = QMC_WF_ALL | (j3 ? QMC_WF_J3 : 0);
  auto it        = registry.find(spo);
  if (it != registry.end())
    if (auto s = it->second.lock())
    {
      if (s->components != comp || s->n_elec != els.getTotalNum())
        fail("one SPO set was given two different wavefunctions");
      return s;
    }
  using spo_t    = einspline_spo<OHMMS_PRECISION>;
  const spo_t* e = dynamic_cast<const spo_t*>(spo);
  if (!e || e->einsplines.empty())
    fail("the SPO set is not the reference's einspline_spo (the -b reference implementation is not offered)");
  auto s        = std::make_shared<DeviceSystem>();
  s->components = comp;
  s->n_elec     = els.getTotalNum();
  s->n_orb      = e->size();
  s->precision  = env_is("QMCGPU_PRECISION", "mixed") ? QMC_PREC_MIXED : QMC_PREC_FP64;
  if (s->n_elec != 2 * s->n_orb)
    fail("the determinants need as many orbitals as electrons of each spin");

  qmc_system_desc d;
  std::memset(&d, 0, sizeof(d));
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
    {
      d.lattice[3 * i + j]     = els.Lattice.R(i, j);
      d.spo_lattice[3 * i + j] = e->Lattice.R(i, j);
    }
  // the ions, grouped by species (a stable sort; the species keep their
  // indices, which pick the Jastrow functors as nio.hpp's builders do)
  const int I = ions.getTotalNum();
  std::vector<int> order(I);
  for (int i = 0; i < I; ++i)
    order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ions.GroupID[a] < ions.GroupID[b]; });
  std::vector<double> ion_pos(3 * (size_t)I);
  std::vector<int> ion_group(I);
  for (int q = 0; q < I; ++q)
  {
    for (int c = 0; c < 3; ++c)
      ion_pos[3 * q + c] = ions.R[order[q]][c];
    ion_group[q] = ions.GroupID[order[q]];
  }
  d.n_ions       = I;
  d.n_ion_groups = ions.getSpeciesSet().getTotalNum();
  d.ion_pos      = ion_pos.data();
  d.ion_group    = ion_group.data();
  d.n_elec       = s->n_elec;
  d.n_up         = s->n_elec / 2;
  d.n_orb        = s->n_orb;
  const auto* sp = e->einsplines[0];
  d.grid[0] = sp->x_grid.num, d.grid[1] = sp->y_grid.num, d.grid[2] = sp->z_grid.num;
  d.lap_mode   = QMC_LAP_HXX; // einspline_spo.hpp:218 stores hess.xx as the Laplacian
  d.components = comp;
  // the orbital table: the SPO set's own, gathered from its tiles into one
  // [nx+3][ny+3][nz+3][n_orb] array, or the library's uniform fill
  std::vector<double> coefs;
  if (env_is("QMCGPU_SPO_FILL", "uniform"))
  {
    d.spo_fill       = QMC_FILL_UNIFORM;
    const char* seed = env("QMCGPU_SPO_SEED");
    d.spo_seed       = seed ? std::strtoull(seed, nullptr, 10) : 11;
  }
  else
  {
    const size_t nx = d.grid[0] + 3, ny = d.grid[1] + 3, nz = d.grid[2] + 3, n = s->n_orb;
    coefs.assign(nx * ny * nz * n, 0.0);
    for (int b = 0; b < e->nBlocks; ++b)
    {
      const auto* t = e->einsplines[b];
      for (size_t ix = 0; ix < nx; ++ix)
        for (size_t iy = 0; iy < ny; ++iy)
          for (size_t iz = 0; iz < nz; ++iz)
          {
            const auto* src = t->coefs + ix * t->x_stride + iy * t->y_stride + iz * t->z_stride;
            double* dst     = coefs.data() + ((ix * ny + iy) * nz + iz) * n;
            for (int j = 0; j < e->nSplinesPerBlock; ++j)
              if (b * e->nSplinesPerBlock + j < (int)n)
                dst[b * e->nSplinesPerBlock + j] = src[j];
          }
    }
    d.spo_fill       = QMC_FILL_USER;
    d.spo_user_coefs = coefs.data();
  }
  // the reference's NiO Jastrows (nio.hpp buildJ1 / buildJ2 / buildJeeI)
  // with the cutoffs of this cell
  check(qmc_nio_jastrows(d.lattice, &d.j1[0], &d.j1[1], &d.j2_uu, &d.j2_ud), "qmc_nio_jastrows");
  if (j3)
  {
    qmc_j3_functor same[2], diff[2];
    check(qmc_nio_j3(d.lattice, same, diff), "qmc_nio_j3");
    for (int gi = 0; gi < d.n_ion_groups; ++gi)
      d.j3_same[gi] = same[gi < 2 ? gi : 1], d.j3_diff[gi] = diff[gi < 2 ? gi : 1];
  }
  check(qmc_system_create(&d, s->precision, &s->sys), "qmc_system_create");
  registry[spo] = s;
  return s;
}

// ---------------------------------------------------------------- SPOSetGpu

SPOSetGpu::SPOSetGpu(std::shared_ptr<DeviceSystem> sys) : sys_(std::move(sys))
{
  OrbitalSetSize = sys_->n_orb;
  className      = "SPOSetGpu";
}

void SPOSetGpu::evaluate(const ParticleSet& P, int iat, ValueVector_t& psi_v)
{
  ensure_device();
  const int n = OrbitalSetSize;
  double r[3];
  for (int c = 0; c < 3; ++c)
    r[c] = P.activeR(iat)[c];
  v_.resize(n);
  check(qmc_spo_evaluate_v(sys_->sys, 1, r, v_.data()), "qmc_spo_evaluate_v");
  for (int j = 0; j < n; ++j)
    psi_v[j] = v_[j];
}

void SPOSetGpu::evaluate(const ParticleSet& P, int iat, ValueVector_t& psi_v, GradVector_t& dpsi_v,
                         ValueVector_t& d2psi_v)
{
  ensure_device();
  const int n = OrbitalSetSize;
  double r[3];
  for (int c = 0; c < 3; ++c)
    r[c] = P.activeR(iat)[c];
  v_.resize(n), g_.resize(3 * n), h_.resize(6 * n);
  check(qmc_spo_evaluate_vgh(sys_->sys, 1, r, v_.data(), g_.data(), h_.data()), "qmc_spo_evaluate_vgh");
  for (int j = 0; j < n; ++j)
  {
    psi_v[j] = v_[j];
    for (int c = 0; c < 3; ++c)
      dpsi_v[j][c] = g_[c * n + j];
    d2psi_v[j] = h_[j]; // H_xx (einspline_spo.hpp:218)
  }
}

// -------------------------------------------------------------------- Batch

Batch::Batch(std::shared_ptr<DeviceSystem> s, int n_walkers, int delay) : W(n_walkers), sys(std::move(s))
{
  ensure_device();
  // every batch runs on its own stream (the library's default), so movers
  // on different host threads overlap on the device
  check(qmc_walkers_create(sys->sys, W, delay, &h), "qmc_walkers_create");
  d3.resize(3 * W), r.resize(W), g3.resize(3 * W), flags.resize(W);
}

Batch::~Batch()
{
  if (h)
    qmc_walkers_destroy(h);
}

// ------------------------------------------------- WaveFunctionComponentGpu

WaveFunctionComponentGpu::WaveFunctionComponentGpu(std::shared_ptr<DeviceSystem> sys, int delay,
                                                   const ParticleSet& els)
    : sys_(std::move(sys)), delay_(delay)
{
  WaveFunctionComponentName = "SlaterJastrowGpu";
  for (int c = 0; c < 3; ++c)
    r0_[c] = els.R[0][c];
}

WaveFunctionComponentGpu::~WaveFunctionComponentGpu()
{
  const char* path = env("QMCGPU_ADAPTER_REPORT");
  if (!path)
    return;
  // JSON numbers, null where a value is not finite (a singular table)
  auto num = [](double x) {
    char b[40];
    if (std::isfinite(x))
      std::snprintf(b, sizeof b, "%.17g", x);
    else
      std::snprintf(b, sizeof b, "null");
    return std::string(b);
  };
  std::lock_guard<std::mutex> g(g_mu);
  if (FILE* f = std::fopen(path, "a"))
  {
    std::fprintf(f,
                 "{\"r0\": [%s, %s, %s], \"log\": %s, \"ratio_grad\": %lld, \"sum_log_ratio\": %s, "
                 "\"accepted\": %lld, \"virtual\": %lld, \"sum_virtual\": %s, \"status\": %d, \"batch\": %d}\n",
                 num(r0_[0]).c_str(), num(r0_[1]).c_str(), num(r0_[2]).c_str(), num(LogValue).c_str(), n_ratio_grad_,
                 num(sum_log_ratio_).c_str(), n_accepted_, n_virtual_, num(sum_virtual_).c_str(), first_status_,
                 batch_ ? batch_->W : 0);
    std::fclose(f);
  }
}

WaveFunctionComponentGpu* WaveFunctionComponentGpu::cast(WaveFunctionComponent* c)
{
  auto* g = dynamic_cast<WaveFunctionComponentGpu*>(c);
  if (!g)
    fail("a walker list mixes device and host wavefunction components");
  return g;
}

int WaveFunctionComponentGpu::note(int status, const char* what)
{
  if (status && !first_status_)
    first_status_ = status;
  return check(status, what);
}

Batch& WaveFunctionComponentGpu::batch_of(const std::vector<WaveFunctionComponent*>& list) const
{
  ensure_device(); // the drivers call from any OpenMP thread
  Batch* b = batch_.get();
  bool ok  = b && (int)list.size() == b->W;
  for (size_t i = 0; ok && i < list.size(); ++i)
    ok = list[i] == b->members[i];
  if (!ok)
    fail("a multi_ call must come with the walker list that multi_evaluateLog was given");
  return *b;
}

Batch& WaveFunctionComponentGpu::single(const char* verb)
{
  ensure_device(); // the drivers call from any OpenMP thread
  if (!batch_)
    fail("evaluateLog must come first");
  if (batch_->W != 1)
  {
    std::string m = std::string(verb) + " on one walker of a batch: use the multi_ form";
    fail(m.c_str());
  }
  return *batch_;
}

void WaveFunctionComponentGpu::make_batch(const std::vector<WaveFunctionComponent*>& list,
                                          const std::vector<ParticleSet*>& P_list)
{
  auto b     = std::make_shared<Batch>(sys_, (int)list.size(), delay_);
  b->members = list;
  const int N = sys_->n_elec;
  b->big.assign((size_t)b->W * N * 3, 0.0);
  for (int iw = 0; iw < b->W; ++iw)
  {
    auto* m    = cast(list[iw]);
    m->batch_  = b;
    m->slot_   = iw;
    const auto& R = P_list[iw]->R;
    for (int i = 0; i < N; ++i)
      for (int c = 0; c < 3; ++c)
        b->big[((size_t)iw * N + i) * 3 + c] = R[i][c];
  }
  note(qmc_walkers_set_positions(b->h, b->big.data()), "qmc_walkers_set_positions");
}

// ---- single-walker verbs (a batch of one)

WaveFunctionComponentGpu::RealType WaveFunctionComponentGpu::evaluateLog(ParticleSet& P,
                                                                         ParticleSet::ParticleGradient_t& G,
                                                                         ParticleSet::ParticleLaplacian_t& L)
{
  std::vector<WaveFunctionComponent*> list{this};
  std::vector<ParticleSet*> P_list{&P};
  std::vector<ParticleSet::ParticleGradient_t*> G_list{&G};
  std::vector<ParticleSet::ParticleLaplacian_t*> L_list{&L};
  ParticleSet::ParticleValue_t values(1);
  multi_evaluateLog(list, P_list, G_list, L_list, values);
  return values[0];
}

WaveFunctionComponentGpu::GradType WaveFunctionComponentGpu::evalGrad(ParticleSet& P, int iat)
{
  Batch& b = single("evalGrad");
  note(qmc_wf_eval_grad(b.h, iat, b.g3.data()), "qmc_wf_eval_grad");
  return GradType(b.g3[0], b.g3[1], b.g3[2]);
}

WaveFunctionComponentGpu::ValueType WaveFunctionComponentGpu::ratioGrad(ParticleSet& P, int iat, GradType& grad_iat)
{
  Batch& b = single("ratioGrad");
  displacements(P, iat, b.d3.data());
  note(qmc_pset_make_move(b.h, iat, b.d3.data()), "qmc_pset_make_move");
  note(qmc_wf_ratio_grad(b.h, iat, b.r.data(), b.g3.data()), "qmc_wf_ratio_grad");
  for (int c = 0; c < 3; ++c)
    grad_iat[c] += b.g3[c];
  ++n_ratio_grad_;
  sum_log_ratio_ += std::log(std::fabs(b.r[0]));
  return b.r[0];
}

void WaveFunctionComponentGpu::acceptMove(ParticleSet& P, int iat)
{
  Batch& b   = single("acceptMove");
  b.flags[0] = 1;
  note(qmc_wf_accept_restore(b.h, iat, b.flags.data()), "qmc_wf_accept_restore");
  note(qmc_pset_accept_reject(b.h, iat, b.flags.data()), "qmc_pset_accept_reject");
  ++n_accepted_;
}

void WaveFunctionComponentGpu::restore(int iat)
{
  Batch& b   = single("restore");
  b.flags[0] = 0;
  note(qmc_wf_accept_restore(b.h, iat, b.flags.data()), "qmc_wf_accept_restore");
  note(qmc_pset_accept_reject(b.h, iat, b.flags.data()), "qmc_pset_accept_reject");
}

WaveFunctionComponentGpu::ValueType WaveFunctionComponentGpu::ratio(ParticleSet& P, int iat)
{
  ensure_device();
  if (!batch_)
    fail("evaluateLog must come first");
  double q = 0.0;
  if (batch_->W == 1)
  {
    // DiracDeterminant::ratio (the update mode becomes ratio-only); the
    // proposed move stays pending on the device as it does on the host
    Batch& b = *batch_;
    displacements(P, iat, b.d3.data());
    note(qmc_pset_make_move(b.h, iat, b.d3.data()), "qmc_pset_make_move");
    note(qmc_wf_ratio(b.h, iat, b.r.data()), "qmc_wf_ratio");
    q = b.r[0];
  }
  else
  {
    // one walker of a batch: the ratio at the proposed position alone
    double pos[3];
    for (int c = 0; c < 3; ++c)
      pos[c] = P.activePos[c];
    note(qmc_wf_evaluate_ratios(batch_->h, slot_, iat, 1, pos, &q), "qmc_wf_evaluate_ratios");
  }
  ++n_virtual_;
  sum_virtual_ += q;
  return q;
}

void WaveFunctionComponentGpu::evaluateGL(ParticleSet& P, ParticleSet::ParticleGradient_t& G,
                                          ParticleSet::ParticleLaplacian_t& L, bool fromscratch)
{
  std::vector<WaveFunctionComponent*> list{this};
  std::vector<ParticleSet*> P_list{&P};
  std::vector<ParticleSet::ParticleGradient_t*> G_list{&G};
  std::vector<ParticleSet::ParticleLaplacian_t*> L_list{&L};
  single("evaluateGL");
  multi_evaluateGL(list, P_list, G_list, L_list, fromscratch);
}

void WaveFunctionComponentGpu::completeUpdates()
{
  Batch& b = single("completeUpdates");
  note(qmc_wf_complete_updates(b.h), "qmc_wf_complete_updates");
}

void WaveFunctionComponentGpu::evaluateRatios(VirtualParticleSet& VP, std::vector<ValueType>& ratios)
{
  ensure_device();
  if (!batch_)
    fail("evaluateLog must come first");
  const int n = VP.getTotalNum();
  std::vector<double> pos(3 * (size_t)n), out(n);
  for (int k = 0; k < n; ++k)
    for (int c = 0; c < 3; ++c)
      pos[3 * k + c] = VP.R[k][c];
  note(qmc_wf_evaluate_ratios(batch_->h, slot_, VP.refPtcl, n, pos.data(), out.data()), "qmc_wf_evaluate_ratios");
  for (int k = 0; k < n; ++k)
  {
    ratios[k] = out[k];
    sum_virtual_ += out[k];
  }
  n_virtual_ += n;
}

// ---- batched verbs: one launch per verb for the whole list

void WaveFunctionComponentGpu::multi_evaluateLog(const std::vector<WaveFunctionComponent*>& WFC_list,
                                                 const std::vector<ParticleSet*>& P_list,
                                                 const std::vector<ParticleSet::ParticleGradient_t*>& G_list,
                                                 const std::vector<ParticleSet::ParticleLaplacian_t*>& L_list,
                                                 ParticleSet::ParticleValue_t& values)
{
  make_batch(WFC_list, P_list);
  Batch& b = *batch_;
  note(qmc_wf_evaluate_log(b.h, b.r.data()), "qmc_wf_evaluate_log");
  multi_evaluateGL(WFC_list, P_list, G_list, L_list, false);
  for (int iw = 0; iw < b.W; ++iw)
    values[iw] = cast(WFC_list[iw])->LogValue;
}

void WaveFunctionComponentGpu::multi_evalGrad(const std::vector<WaveFunctionComponent*>& WFC_list,
                                              const std::vector<ParticleSet*>& P_list, int iat,
                                              std::vector<PosType>& grad_now)
{
  Batch& b = batch_of(WFC_list);
  note(qmc_wf_eval_grad(b.h, iat, b.g3.data()), "qmc_wf_eval_grad");
  for (int iw = 0; iw < b.W; ++iw)
    grad_now[iw] = PosType(b.g3[3 * iw], b.g3[3 * iw + 1], b.g3[3 * iw + 2]);
}

void WaveFunctionComponentGpu::multi_ratioGrad(const std::vector<WaveFunctionComponent*>& WFC_list,
                                               const std::vector<ParticleSet*>& P_list, int iat,
                                               std::vector<ValueType>& ratios, std::vector<PosType>& grad_new)
{
  Batch& b = batch_of(WFC_list);
  for (int iw = 0; iw < b.W; ++iw)
    displacements(*P_list[iw], iat, &b.d3[3 * iw]);
  note(qmc_pset_make_move(b.h, iat, b.d3.data()), "qmc_pset_make_move");
  note(qmc_wf_ratio_grad(b.h, iat, b.r.data(), b.g3.data()), "qmc_wf_ratio_grad");
  for (int iw = 0; iw < b.W; ++iw)
  {
    ratios[iw] = b.r[iw];
    for (int c = 0; c < 3; ++c)
      grad_new[iw][c] += b.g3[3 * iw + c];
    auto* m = cast(WFC_list[iw]);
    ++m->n_ratio_grad_;
    m->sum_log_ratio_ += std::log(std::fabs(b.r[iw]));
  }
}

void WaveFunctionComponentGpu::multi_acceptrestoreMove(const std::vector<WaveFunctionComponent*>& WFC_list,
                                                       const std::vector<ParticleSet*>& P_list,
                                                       const std::vector<bool>& isAccepted, int iat)
{
  Batch& b = batch_of(WFC_list);
  for (int iw = 0; iw < b.W; ++iw)
  {
    b.flags[iw] = isAccepted[iw] ? 1 : 0;
    cast(WFC_list[iw])->n_accepted_ += b.flags[iw];
  }
  note(qmc_wf_accept_restore(b.h, iat, b.flags.data()), "qmc_wf_accept_restore");
  note(qmc_pset_accept_reject(b.h, iat, b.flags.data()), "qmc_pset_accept_reject");
}

void WaveFunctionComponentGpu::multi_ratio(const std::vector<WaveFunctionComponent*>& WFC_list,
                                           const std::vector<ParticleSet*>& P_list, int iat,
                                           ParticleSet::ParticleValue_t& ratio_list)
{
  Batch& b = batch_of(WFC_list);
  for (int iw = 0; iw < b.W; ++iw)
    displacements(*P_list[iw], iat, &b.d3[3 * iw]);
  note(qmc_pset_make_move(b.h, iat, b.d3.data()), "qmc_pset_make_move");
  note(qmc_wf_ratio(b.h, iat, b.r.data()), "qmc_wf_ratio");
  for (int iw = 0; iw < b.W; ++iw)
  {
    ratio_list[iw] = b.r[iw];
    auto* m = cast(WFC_list[iw]);
    ++m->n_virtual_;
    m->sum_virtual_ += b.r[iw];
  }
}

void WaveFunctionComponentGpu::multi_evaluateGL(const std::vector<WaveFunctionComponent*>& WFC_list,
                                                const std::vector<ParticleSet*>& P_list,
                                                const std::vector<ParticleSet::ParticleGradient_t*>& G_list,
                                                const std::vector<ParticleSet::ParticleLaplacian_t*>& L_list,
                                                bool fromscratch)
{
  Batch& b    = batch_of(WFC_list);
  const int N = sys_->n_elec;
  b.big.resize((size_t)b.W * N * 4);
  double* G = b.big.data();
  double* L = G + (size_t)b.W * N * 3;
  note(qmc_wf_evaluate_gl(b.h, G, L, b.r.data()), "qmc_wf_evaluate_gl");
  for (int iw = 0; iw < b.W; ++iw)
  {
    auto& Gw = *G_list[iw];
    auto& Lw = *L_list[iw];
    for (int i = 0; i < N; ++i)
    {
      for (int c = 0; c < 3; ++c)
        Gw[i][c] += G[((size_t)iw * N + i) * 3 + c];
      Lw[i] += L[(size_t)iw * N + i];
    }
    cast(WFC_list[iw])->LogValue = b.r[iw];
  }
}

void WaveFunctionComponentGpu::multi_completeUpdates(const std::vector<WaveFunctionComponent*>& WFC_list)
{
  Batch& b = batch_of(WFC_list);
  note(qmc_wf_complete_updates(b.h), "qmc_wf_complete_updates");
}

} // namespace qmcgpu
} // namespace qmcplusplus
