// qmcgpu_wavefunction.cpp -- WaveFunction (the reference's
// QMCWaveFunctions/WaveFunction.h, unchanged) implemented over the device:
// it takes the place of the reference's WaveFunction.cpp at link time.
//
// build_WaveFunction (WaveFunction.cpp:32-140 in the reference) keeps what
// the drivers read from the host ParticleSet -- the electron-electron and
// electron-ion distance tables, whose ID the NLPP loop uses
// (miniqmc.cpp:472-495, NonLocalPP.hpp:115-134) -- and puts the whole
// Slater-Jastrow product (both determinants, J1, J2 and, with -j, J3) into
// one WaveFunctionComponentGpu as Det_up.  Det_dn stays empty and Jastrows
// holds no host component.  Every per-walker verb goes to that component;
// every flex_ verb goes to its multi_ form over the list's device batch.
//
// Contracts kept from the reference: evaluateLog runs only the first time
// (WaveFunction.cpp:178-195); evalGrad returns and ratioGrad assigns the
// whole gradient (ratioGrad zeroes grad, :209-221); restore(iat) drops the
// proposed move; evaluateGL rewrites P.G and P.L and the log value
// (:246-263); flex_evaluateLog also runs only the first time (:300-340).
#include <QMCWaveFunctions/WaveFunction.h>

#include "qmcgpu_adapter.hpp"

namespace qmcplusplus
{
namespace
{
enum AdapterTimers
{
  Timer_GL,
  Timer_CompleteUpdates,
};

TimerNameLevelList_t<AdapterTimers> AdapterTimerNames = {{Timer_GL, "Kinetic Energy", timer_level_coarse},
                                                         {Timer_CompleteUpdates, "Complete Updates",
                                                          timer_level_coarse}};

qmcgpu::WaveFunctionComponentGpu* gpu(WaveFunctionComponent* c)
{
  return static_cast<qmcgpu::WaveFunctionComponentGpu*>(c);
}
} // namespace

void build_WaveFunction(bool useRef, const SPOSet* spo_main, WaveFunction& WF, ParticleSet& ions, ParticleSet& els,
                        const RandomGenerator<QMCTraits::RealType>& RNG, int delay_rank, bool enableJ3)
{
  if (WF.Is_built)
  {
    app_log() << "The wavefunction was built before!" << std::endl;
    return;
  }
  ions.RSoA = ions.R;
  els.RSoA  = els.R;
  // the host distance tables the drivers read (the wavefunction itself
  // evaluates its distances on the device)
  els.addTable(els, DT_SOA);
  WF.ei_TableID = els.addTable(ions, DT_SOA);
  WF.nelup      = els.getTotalNum() / 2;
  auto sys      = qmcgpu::device_system(spo_main, ions, els, enableJ3);
  WF.Det_up     = new qmcgpu::WaveFunctionComponentGpu(sys, delay_rank, els);
  WF.Det_dn     = nullptr;
  WF.setupTimers();
  WF.Is_built = true;
}

WaveFunction::WaveFunction()
    : FirstTime(true), Is_built(false), nelup(0), ei_TableID(1), Det_up(nullptr), Det_dn(nullptr), LogValue(0.0)
{}

WaveFunction::~WaveFunction()
{
  if (Is_built)
  {
    delete Det_up;
    delete Det_dn;
    for (size_t i = 0; i < Jastrows.size(); i++)
      delete Jastrows[i];
  }
}

void WaveFunction::setupTimers() { setup_timers(timers, AdapterTimerNames); }

void WaveFunction::evaluateLog(ParticleSet& P)
{
  if (!FirstTime)
    return;
  P.G      = valT(0);
  P.L      = valT(0);
  LogValue = Det_up->evaluateLog(P, P.G, P.L);
  FirstTime = false;
}

WaveFunction::posT WaveFunction::evalGrad(ParticleSet& P, int iat) { return Det_up->evalGrad(P, iat); }

WaveFunction::valT WaveFunction::ratioGrad(ParticleSet& P, int iat, posT& grad)
{
  grad = valT(0);
  return Det_up->ratioGrad(P, iat, grad);
}

WaveFunction::valT WaveFunction::ratio(ParticleSet& P, int iat) { return Det_up->ratio(P, iat); }

void WaveFunction::acceptMove(ParticleSet& P, int iat) { Det_up->acceptMove(P, iat); }

void WaveFunction::restore(int iat) { gpu(Det_up)->restore(iat); }

void WaveFunction::completeUpdates()
{
  ScopedTimer local_timer(timers[Timer_CompleteUpdates]);
  Det_up->completeUpdates();
}

void WaveFunction::evaluateGL(ParticleSet& P)
{
  ScopedTimer local_timer(timers[Timer_GL]);
  P.G = valT(0);
  P.L = valT(0);
  Det_up->evaluateGL(P, P.G, P.L);
  LogValue = Det_up->LogValue;
}

void WaveFunction::evaluateRatios(VirtualParticleSet& VP, std::vector<valT>& ratios)
{
  Det_up->evaluateRatios(VP, ratios);
}

void WaveFunction::flex_evaluateLog(const std::vector<WaveFunction*>& WF_list,
                                    const std::vector<ParticleSet*>& P_list) const
{
  if (!WF_list[0]->FirstTime)
    return;
  const std::vector<ParticleSet::ParticleGradient_t*> G_list(extract_G_list(P_list));
  const std::vector<ParticleSet::ParticleLaplacian_t*> L_list(extract_L_list(P_list));
  for (size_t iw = 0; iw < P_list.size(); iw++)
  {
    *G_list[iw] = valT(0);
    *L_list[iw] = valT(0);
  }
  ParticleSet::ParticleValue_t values(P_list.size());
  Det_up->multi_evaluateLog(extract_up_list(WF_list), P_list, G_list, L_list, values);
  for (size_t iw = 0; iw < P_list.size(); iw++)
  {
    WF_list[iw]->LogValue  = values[iw];
    WF_list[iw]->FirstTime = false;
  }
}

void WaveFunction::flex_evalGrad(const std::vector<WaveFunction*>& WF_list, const std::vector<ParticleSet*>& P_list,
                                 int iat, std::vector<posT>& grad_now) const
{
  Det_up->multi_evalGrad(extract_up_list(WF_list), P_list, iat, grad_now);
}

void WaveFunction::flex_ratioGrad(const std::vector<WaveFunction*>& WF_list, const std::vector<ParticleSet*>& P_list,
                                  int iat, std::vector<valT>& ratio_list, std::vector<posT>& grad_new) const
{
  for (size_t iw = 0; iw < P_list.size(); iw++)
    grad_new[iw] = valT(0);
  Det_up->multi_ratioGrad(extract_up_list(WF_list), P_list, iat, ratio_list, grad_new);
}

void WaveFunction::flex_acceptrestoreMove(const std::vector<WaveFunction*>& WF_list,
                                          const std::vector<ParticleSet*>& P_list,
                                          const std::vector<bool>& isAccepted, int iat) const
{
  Det_up->multi_acceptrestoreMove(extract_up_list(WF_list), P_list, isAccepted, iat);
}

void WaveFunction::flex_evaluateGL(const std::vector<WaveFunction*>& WF_list,
                                   const std::vector<ParticleSet*>& P_list) const
{
  ScopedTimer local_timer(timers[Timer_GL]);
  const std::vector<ParticleSet::ParticleGradient_t*> G_list(extract_G_list(P_list));
  const std::vector<ParticleSet::ParticleLaplacian_t*> L_list(extract_L_list(P_list));
  for (size_t iw = 0; iw < P_list.size(); iw++)
  {
    *G_list[iw] = valT(0);
    *L_list[iw] = valT(0);
  }
  const std::vector<WaveFunctionComponent*> up_list(extract_up_list(WF_list));
  Det_up->multi_evaluateGL(up_list, P_list, G_list, L_list);
  for (size_t iw = 0; iw < P_list.size(); iw++)
    WF_list[iw]->LogValue = up_list[iw]->LogValue;
}

void WaveFunction::flex_completeUpdates(const std::vector<WaveFunction*>& WF_list) const
{
  ScopedTimer local_timer(timers[Timer_CompleteUpdates]);
  Det_up->multi_completeUpdates(extract_up_list(WF_list));
}

const std::vector<WaveFunctionComponent*> WaveFunction::extract_up_list(const std::vector<WaveFunction*>& WF_list) const
{
  std::vector<WaveFunctionComponent*> up_list;
  for (auto* wf : WF_list)
    up_list.push_back(wf->Det_up);
  return up_list;
}

const std::vector<WaveFunctionComponent*> WaveFunction::extract_dn_list(const std::vector<WaveFunction*>& WF_list) const
{
  std::vector<WaveFunctionComponent*> dn_list;
  for (auto* wf : WF_list)
    dn_list.push_back(wf->Det_dn);
  return dn_list;
}

const std::vector<WaveFunctionComponent*> WaveFunction::extract_jas_list(const std::vector<WaveFunction*>& WF_list,
                                                                         int jas_id) const
{
  std::vector<WaveFunctionComponent*> jas_list;
  for (auto* wf : WF_list)
    jas_list.push_back(wf->Jastrows[jas_id]);
  return jas_list;
}

} // namespace qmcplusplus
