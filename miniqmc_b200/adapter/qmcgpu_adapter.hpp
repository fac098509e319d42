// qmcgpu_adapter.hpp -- the reference's wavefunction interface implemented
// over the C ABI of libqmcgpu (include/qmcgpu.h).
//
// These classes are compiled against the reference's own headers
// (QMCWaveFunctions/SPOSet.h, WaveFunctionComponent.h, WaveFunction.h,
// Particle/ParticleSet.h), so that the reference's drivers
// (Drivers/miniqmc.cpp, Drivers/miniqmc_sync_move.cpp) link against the GPU
// path without a change to their source:
//
//   SPOSetGpu                 SPOSet (SPOSet.h:55-127) evaluated on the
//                             device copy of a spline table
//   WaveFunctionComponentGpu  the whole Slater-Jastrow product of one walker
//                             (WaveFunctionComponent.h:127-252), held as one
//                             slot of a device walker batch; its multi_*
//                             verbs move the whole batch with one launch per
//                             verb, its single-walker verbs act on a batch
//                             of one
//
// qmcgpu_wavefunction.cpp implements WaveFunction (WaveFunction.h) with
// them and takes the place of the reference's WaveFunction.cpp at link time.
//
// Environment:
//   QMCGPU_SPO_FILL=uniform  the table is the library's SplitMix64 fill
//                            (QMC_FILL_UNIFORM, seed QMCGPU_SPO_SEED, 11 by
//                            default) instead of the SPOSet's own table: the
//                            reference's fill makes every orbital of a tile
//                            one field times a scalar (einspline_spo.hpp:
//                            145-156), so its Slater matrices are singular
//   QMCGPU_PRECISION=mixed   FP32 table and walker state (QMC_PREC_MIXED);
//                            FP64 (QMC_PREC_FP64) by default
//   QMCGPU_DEVICE=n          the CUDA device (0 by default)
//   QMCGPU_ADAPTER_REPORT=f  each walker appends one JSON line to f when it
//                            is destroyed (its counters and last log value)
#pragma once

#include <QMCWaveFunctions/SPOSet.h>
#include <QMCWaveFunctions/WaveFunctionComponent.h>
#include <Particle/ParticleSet.h>
#include <Particle/VirtualParticleSet.h>

#include "qmcgpu.h"

#include <memory>
#include <vector>

namespace qmcplusplus
{
namespace qmcgpu
{
/// Checks a C-ABI status.  Numerical failures (QMC_ERR_SINGULAR,
/// QMC_ERR_NONFINITE) are reported once per kind and the run goes on, as the
/// reference's own run goes on with what its LAPACK and arithmetic return;
/// every other failure stops the program with exit code 1, as APP_ABORT does
/// (Configuration.h:35-39).  Returns the status.
int check(int status, const char* what);

/// Stops the program with a message (APP_ABORT).
[[noreturn]] void fail(const char* what);

/// A device system: the spline table, lattice, ions and Jastrow functors
/// that the walkers of one SPO set share.
struct DeviceSystem
{
  qmc_system* sys = nullptr;
  int n_elec = 0, n_orb = 0, components = 0, precision = 0;
  ~DeviceSystem();
};

/// The device system for the reference's SPO set `spo` (an einspline_spo:
/// its table is copied to the device unless QMCGPU_SPO_FILL=uniform), the
/// reference's ions and electrons (lattice, ion positions and species) and
/// the reference's NiO Jastrows (nio.hpp buildJ1 / buildJ2, and buildJeeI
/// when j3).  One per SPO set, made on first use by any thread.
std::shared_ptr<DeviceSystem> device_system(const SPOSet* spo, const ParticleSet& ions, const ParticleSet& els,
                                            bool j3);

/// SPOSet (SPOSet.h) over the device table: values, gradients and the
/// reference's Laplacian (H_xx, einspline_spo.hpp:218) at
/// ParticleSet::activeR(iat).
class SPOSetGpu : public SPOSet
{
public:
  explicit SPOSetGpu(std::shared_ptr<DeviceSystem> sys);
  void evaluate(const ParticleSet& P, int iat, ValueVector_t& psi_v) override;
  void evaluate(const ParticleSet& P, int iat, ValueVector_t& psi_v, GradVector_t& dpsi_v,
                ValueVector_t& d2psi_v) override;

private:
  std::shared_ptr<DeviceSystem> sys_;
  std::vector<double> v_, g_, h_;
};

/// A device walker batch.
struct Batch
{
  qmc_walkers* h = nullptr;
  int W          = 0;
  std::shared_ptr<DeviceSystem> sys;
  std::vector<WaveFunctionComponent*> members;
  Batch(std::shared_ptr<DeviceSystem> s, int n_walkers, int delay);
  ~Batch();
  // scratch, [W] / [W][3] / [W][N][3]
  std::vector<double> d3, r, g3, big;
  std::vector<int> flags;
};

/// The Slater-Jastrow product of one walker on the device.  Its verbs follow
/// the component contract: gradients and Laplacians ADD into the caller's
/// arrays (DiracDeterminant.cpp:121), ratios are returned for the caller to
/// multiply.
class WaveFunctionComponentGpu : public WaveFunctionComponent
{
public:
  WaveFunctionComponentGpu(std::shared_ptr<DeviceSystem> sys, int delay, const ParticleSet& els);
  ~WaveFunctionComponentGpu() override;

  RealType evaluateLog(ParticleSet& P, ParticleSet::ParticleGradient_t& G,
                       ParticleSet::ParticleLaplacian_t& L) override;
  GradType evalGrad(ParticleSet& P, int iat) override;
  ValueType ratioGrad(ParticleSet& P, int iat, GradType& grad_iat) override;
  void acceptMove(ParticleSet& P, int iat) override;
  /// WaveFunction::restore: the proposed move of electron iat is dropped
  void restore(int iat);
  ValueType ratio(ParticleSet& P, int iat) override;
  void evaluateGL(ParticleSet& P, ParticleSet::ParticleGradient_t& G, ParticleSet::ParticleLaplacian_t& L,
                  bool fromscratch = false) override;
  void completeUpdates() override;
  void evaluateRatios(VirtualParticleSet& VP, std::vector<ValueType>& ratios) override;

  void multi_evaluateLog(const std::vector<WaveFunctionComponent*>& WFC_list, const std::vector<ParticleSet*>& P_list,
                         const std::vector<ParticleSet::ParticleGradient_t*>& G_list,
                         const std::vector<ParticleSet::ParticleLaplacian_t*>& L_list,
                         ParticleSet::ParticleValue_t& values) override;
  void multi_evalGrad(const std::vector<WaveFunctionComponent*>& WFC_list, const std::vector<ParticleSet*>& P_list,
                      int iat, std::vector<PosType>& grad_now) override;
  void multi_ratioGrad(const std::vector<WaveFunctionComponent*>& WFC_list, const std::vector<ParticleSet*>& P_list,
                       int iat, std::vector<ValueType>& ratios, std::vector<PosType>& grad_new) override;
  void multi_acceptrestoreMove(const std::vector<WaveFunctionComponent*>& WFC_list,
                               const std::vector<ParticleSet*>& P_list, const std::vector<bool>& isAccepted,
                               int iat) override;
  void multi_ratio(const std::vector<WaveFunctionComponent*>& WFC_list, const std::vector<ParticleSet*>& P_list,
                   int iat, ParticleSet::ParticleValue_t& ratio_list) override;
  void multi_evaluateGL(const std::vector<WaveFunctionComponent*>& WFC_list, const std::vector<ParticleSet*>& P_list,
                        const std::vector<ParticleSet::ParticleGradient_t*>& G_list,
                        const std::vector<ParticleSet::ParticleLaplacian_t*>& L_list,
                        bool fromscratch = false) override;
  void multi_completeUpdates(const std::vector<WaveFunctionComponent*>& WFC_list) override;

private:
  std::shared_ptr<DeviceSystem> sys_;
  int delay_;
  std::shared_ptr<Batch> batch_;
  int slot_ = -1;
  // counters for QMCGPU_ADAPTER_REPORT
  double r0_[3];
  long long n_ratio_grad_ = 0, n_accepted_ = 0, n_virtual_ = 0;
  double sum_log_ratio_ = 0.0, sum_virtual_ = 0.0;
  int first_status_ = 0;

  static WaveFunctionComponentGpu* cast(WaveFunctionComponent* c);
  /// the batch of a multi_* list: the one multi_evaluateLog made for it
  Batch& batch_of(const std::vector<WaveFunctionComponent*>& list) const;
  /// the batch of one walker for a single-walker verb (a batch of one)
  Batch& single(const char* verb);
  void make_batch(const std::vector<WaveFunctionComponent*>& list, const std::vector<ParticleSet*>& P_list);
  int note(int status, const char* what);
};

} // namespace qmcgpu
} // namespace qmcplusplus
