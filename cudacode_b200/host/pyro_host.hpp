// C++ host layer over the C-ABI of include/pyro.h, keeping the names and the
// argument meaning of taillefu/cudacode's host functions for the Monte Carlo
// path (MonteCarlo.cu, Math.cu, Pyrochlore.cu), with RAII and exceptions in
// place of void returns and exit().
#pragma once

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/pyro.h"

namespace pyro_host {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code(code) {}
  int code;
};

// One GPU context holding one lattice and its temperature ladder
// (replaces std::vector<dev> with one entry per GPU).
class Device {
 public:
  Device(int L, const std::vector<double>& temperatures, double J1, double J2, double J3,
         uint64_t seed, int device = 0, int renorm_every = 100)
      : temps_(temperatures) {
    pyro_system_desc s;
    s.L = L;
    s.n_replicas = (int)temps_.size();
    s.replica_offset = 0;
    s.n_temperatures = (int)temps_.size();
    s.temperatures = temps_.data();
    s.J1 = J1;
    s.J2 = J2;
    s.J3 = J3;
    s.J3b = 0.0;
    pyro_config cfg;
    cfg.n_systems = 1;
    cfg.systems = &s;
    cfg.seed = seed;
    cfg.device = device;
    cfg.renorm_every = renorm_every;
    const int rc = pyro_create(&cfg, &ctx_);
    if (rc != PYRO_OK) throw Error(rc, "pyro_create failed");
    L_ = L;
  }
  ~Device() { pyro_destroy(ctx_); }
  Device(const Device&) = delete;
  Device& operator=(const Device&) = delete;

  void check(int rc) const {
    if (rc != PYRO_OK) throw Error(rc, pyro_last_error(ctx_));
  }
  pyro_ctx* ctx() const { return ctx_; }
  int replicas() const { return (int)temps_.size(); }
  int sites() const { return 16 * L_ * L_ * L_; }

 private:
  pyro_ctx* ctx_ = nullptr;
  std::vector<double> temps_;
  int L_ = 0;
};

// GenerateRandomVectorsOnDevice (MonteCarlo.cu:257-293).
inline void GenerateRandomVectorsOnDevice(Device& d) { d.check(pyro_init_random(d.ctx())); }

// MonteCarlo(device, OverRelaxation, ReductionAngle, McSteps, ...)
// (MonteCarlo.cu:176-228): McSteps cycles of one Metropolis sweep and
// OverRelaxation over-relaxation sweeps, no exchange.
inline void MonteCarlo(Device& d, int OverRelaxation, int McSteps) {
  d.check(pyro_cycle(d.ctx(), 1, OverRelaxation, 0, McSteps));
}

// SynchronizeJobs (MonteCarlo.cu:230-245).
inline void SynchronizeJobs(Device& d) { d.check(pyro_synchronize(d.ctx())); }

// TotalEnergyv2(device, Energy) (Math.cu:309-330): FP64 energy of every
// configuration slot.
inline void TotalEnergyv2(Device& d, std::vector<double>& Energy) {
  Energy.resize(d.replicas());
  d.check(pyro_observables(d.ctx(), 0, Energy.data(), nullptr));
}

// Magnetization(NT, device, out) (Pyrochlore.cu:453-466): 3 per replica.
inline void Magnetization(Device& d, std::vector<double>& M) {
  std::vector<double> E(d.replicas());
  M.resize(3 * d.replicas());
  d.check(pyro_observables(d.ctx(), 0, E.data(), M.data()));
}

// TrySwapingTemperatures(CosThetaSolid, Energies, Temperatures, EvenOdd)
// (MonteCarlo.cu:105-172): EvenOdd = 1 pairs (0,1),(2,3)...; returns the
// temperature of each configuration slot.
inline int TrySwapingTemperatures(Device& d, std::vector<double>& Temperatures, int EvenOdd) {
  int accepted = 0;
  d.check(pyro_pt_swap(d.ctx(), EvenOdd ? 0 : 1, &accepted));
  Temperatures.resize(d.replicas());
  d.check(pyro_get_temperatures(d.ctx(), 0, Temperatures.data()));
  return accepted;
}

// ParallelTempering(device, OR, RA, McSteps, EvenOdd, Temperatures, ...,
// Energies) (MonteCarlo.cu:429-470): McSteps sweeps then one exchange of
// alternating parity, energies and temperatures per configuration slot.
inline void ParallelTempering(Device& d, int OverRelaxation, int McSteps,
                              std::vector<double>& Temperatures, std::vector<double>& Energies) {
  d.check(pyro_cycle(d.ctx(), McSteps, McSteps * OverRelaxation, 1, 1));
  TotalEnergyv2(d, Energies);
  Temperatures.resize(d.replicas());
  d.check(pyro_get_temperatures(d.ctx(), 0, Temperatures.data()));
}

// ApplyParallelTemperingDuringMeasure (MonteCarlo.cu:613-657): queues
// McSteps sweeps and one exchange without waiting for them.
inline void ParallelTemperingAsync(Device& d, int OverRelaxation, int McSteps) {
  d.check(pyro_cycle(d.ctx(), McSteps, McSteps * OverRelaxation, 1, 1));
}

// ExtractConfigurationsFromMonteCarlo (Pyrochlore.cu:1608-1617): a
// measurement snapshot of the state the queued Monte Carlo reaches; the
// Monte Carlo queued after it runs while the snapshot is measured.
inline void ExtractConfigurationsFromMonteCarlo(Device& d) { d.check(pyro_snapshot(d.ctx())); }

// Measurement calls read the last snapshot (on) or the live state (off).
inline void MeasureSnapshot(Device& d, bool on) {
  d.check(pyro_set_option(d.ctx(), PYRO_OPT_MEASURE_SNAPSHOT, on ? 1 : 0));
}

// Energies the cycle of the measured state computed, per configuration slot.
inline void CycleEnergies(Device& d, std::vector<double>& Energies) {
  Energies.resize(d.replicas());
  d.check(pyro_last_observables(d.ctx(), 0, Energies.data(), nullptr));
}

// Temperature of each configuration slot in the measured state.
inline void SlotTemperatures(Device& d, std::vector<double>& Temperatures) {
  Temperatures.resize(d.replicas());
  d.check(pyro_get_temperatures(d.ctx(), 0, Temperatures.data()));
}

// CalculateSolidAngle(device, OR, McSteps, ratio, Temperatures, CosThetaSolid)
// (MonteCarlo.cu:371-426): cone width of every temperature for `ratio`
// acceptance.
inline void CalculateSolidAngle(Device& d, int OverRelaxation, double ratio,
                                std::vector<float>& CosThetaSolid) {
  d.check(pyro_tune_cone(d.ctx(), ratio, 50, 10, OverRelaxation));
  CosThetaSolid.resize(d.replicas());
  d.check(pyro_get_cone(d.ctx(), 0, CosThetaSolid.data()));
}

// InitializeCouplings3D(nt, nspc, ..., MagneticField, B, device)
// (Pyrochlore.cu:643-711) for the reference's anisotropic model: the bond
// matrices of J1..J4 (couplings_const, Pyrochlore.cu:169-184) and, with
// MagneticField, the site fields of B (tesla) through the g-tensors of gxy,
// gz (InitializeMagneticField, Pyrochlore.cu:414-450). Energies and
// temperatures are then in the reference's units.
inline void InitializeCouplings3D(Device& d, double J1, double J2, double J3, double J4,
                                  int MagneticField, const double* B, double gxy, double gz) {
  std::vector<double> A(144), f(12, 0.0);
  d.check(pyro_reference_exchange(J1, J2, J3, J4, A.data()));
  if (MagneticField) d.check(pyro_reference_field(gxy, gz, B, f.data()));
  d.check(pyro_set_exchange(d.ctx(), 0, A.data(), MagneticField ? f.data() : nullptr));
}

// Magnetization with the g-tensor (MagnetizationGPU, Pyrochlore.cu:277-342):
// sum_b g_b m_b of every configuration slot, 3 per replica.
inline void MagnetizationG(Device& d, double gxy, double gz, std::vector<double>& M) {
  std::vector<double> g(36), m(12 * d.replicas());
  d.check(pyro_reference_gtensor(gxy, gz, g.data()));
  d.check(pyro_sublattice_magnetisation(d.ctx(), 0, m.data()));
  M.assign(3 * d.replicas(), 0.0);
  for (int r = 0; r < d.replicas(); ++r)
    for (int b = 0; b < 4; ++b)
      for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) M[3 * r + i] += g[9 * b + 3 * i + k] * m[(4 * r + b) * 3 + k];
}

// DoMeasurement / CalculateQuadrupole / CalculateAbsSz / CalculateAbsSumSz
// (Pyrochlore.cu:1047-1100, Math.cu:335-510): the 20 order parameters of
// every configuration slot (pyro_order_parameters layout).
inline void OrderParameters(Device& d, std::vector<double>& out) {
  out.resize(20 * d.replicas());
  d.check(pyro_order_parameters(d.ctx(), 0, out.data()));
}

// Geometric ("log scale") or linear ladder between tmin and tmax
// (the reference's SetupLog/LinearTemperatures, whose source is absent).
inline std::vector<double> Ladder(double tmin, double tmax, int n, bool log_scale) {
  std::vector<double> t(n);
  for (int i = 0; i < n; ++i) {
    const double f = n > 1 ? (double)i / (n - 1) : 0.0;
    t[i] = log_scale ? tmin * std::pow(tmax / tmin, f) : tmin + (tmax - tmin) * f;
  }
  return t;
}

}  // namespace pyro_host
