// pyro_run: command-line driver of the engine, with the option names of the
// reference's main (Pyrochlore.cu:1161-1216) for the Monte Carlo path:
// annealing-free equilibration, cone tuning, parallel tempering, the energy
// per temperature and measure into --Output, and the per-temperature
// statistics files of the reference's measurement loop
// (Pyrochlore.cu:1559-1765): Energies<r>.dat (E, E^2), OrderParameters<r>.dat
// (|m| and m^2 of the A2, E, T, uniform and T' irreps), Quadrupole<r>.dat,
// Sz<r>.dat, SzSum<r>.dat, Magnetization<r>.dat and dchidt<r>.dat, r the
// repetition.
//
//   pyro_run --nx 8 --NumberOfTemperatures 16 --TMin 0.05 --TMax 1 --LogScale
//            --OverRelaxation 4 --McStepsParallelTempering 1
//            --ThermalizationSteps 1000 --NumberOfMeasures 1000 --Rng 56081376
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "measure.hpp"
#include "pyro_host.hpp"

namespace {

struct Options {
  int L = 8;
  int n_temps = 16;
  double tmin = 0.05, tmax = 1.0;
  bool log_scale = false;
  int over_relaxation = 4;
  int mc_steps_pt = 1;
  int thermalization = 1000;
  int n_measures = 1000;
  int pt_every = 1;
  long long seed = 56081376;
  // the reference's anisotropic model (its defaults, Pyrochlore.cu:138-144)
  double J1 = -0.09 / 0.29, J2 = -0.22 / 0.29, J3 = -1.00, J4 = 0.0;
  bool field = false;
  double B[3] = {1.0, 0.0, 0.0};
  double gxy = 1.0, gz = 1.0;
  bool magnetization = false;
  bool order_parameters = false, quadrupole = false, zaxis = false, zaxis_sum = false;
  bool dchidt = false;
  int repetitions = 1;
  // isotropic Heisenberg model in unit-spin convention instead (no reference option)
  bool heisenberg = false;
  double J = 1.0, Jnn2 = 0.0, Jnn3 = 0.0;
  bool reduction_angle = true;
  double ratio = 0.5;
  int device = 0;
  std::string out = "Energies.dat";
};

void usage(const char* prog) {
  std::printf(
      "usage: %s [options]\n"
      "  --nx L                        cubic cells per edge (16 L^3 sites)\n"
      "  --NumberOfTemperatures n      temperature ladder size\n"
      "  --TMin t --TMax t [--LogScale] ladder bounds (geometric with --LogScale)\n"
      "  --OverRelaxation n            over-relaxation sweeps per Metropolis sweep\n"
      "  --McStepsParallelTempering n  Metropolis sweeps between exchanges\n"
      "  --ThermalizationSteps n       exchange cycles before measuring\n"
      "  --NumberOfMeasures n          measured exchange cycles\n"
      "  --Rng seed                    Philox seed\n"
      "  --J1 j --J2 j --J3 j --J4 j   nearest-neighbour couplings of the anisotropic model\n"
      "                                (default YbTiO: -0.09/0.29, -0.22/0.29, -1, 0)\n"
      "  --MagneticField               add the Zeeman field of --Bx --By --Bz (tesla)\n"
      "  --Bx b --By b --Bz b          field (1, 0, 0)\n"
      "  --gxy g --gz g                g-tensor (1, 1)\n"
      "  --Magnetization               also write the g-weighted moment per temperature\n"
      "  --OrderParameters             irrep order parameters (OrderParameters<r>.dat)\n"
      "  --Quadrupole                  quadrupolar order (Quadrupole<r>.dat)\n"
      "  --Zaxis --ZaxisSum            sum |a.S| (Sz<r>.dat), monopole density (SzSum<r>.dat)\n"
      "  --DChiDt                      order parameters times E (dchidt<r>.dat)\n"
      "  --NumberOfRepetitions r       independent runs (seed + r), files suffixed r\n"
      "  --Heisenberg j                isotropic H = j sum S_i.S_j instead (unit spins)\n"
      "  --Jnn2 j --Jnn3 j             isotropic second / third-neighbour couplings\n"
      "  --NoReductionAngle            keep the full-sphere proposal (no cone tuning)\n"
      "  --Ratio r                     target Metropolis acceptance for the cone (0.5)\n"
      "  --Device d                    CUDA device\n"
      "  --Output file                 energy per temperature and measure (Energies.dat)\n",
      prog);
}

bool parse(int argc, char** argv, Options* o) {
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&](const char* name) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "%s: missing value\n", name);
        std::exit(1);
      }
      return argv[++i];
    };
    if (a == "--help" || a == "-h") {
      usage(argv[0]);
      std::exit(0);
    } else if (a == "--nx") o->L = std::atoi(next("--nx"));
    else if (a == "--NumberOfTemperatures") o->n_temps = std::atoi(next(a.c_str()));
    else if (a == "--TMin") o->tmin = std::atof(next(a.c_str()));
    else if (a == "--TMax") o->tmax = std::atof(next(a.c_str()));
    else if (a == "--LogScale") o->log_scale = true;
    else if (a == "--OverRelaxation") o->over_relaxation = std::atoi(next(a.c_str()));
    else if (a == "--McStepsParallelTempering") o->mc_steps_pt = std::atoi(next(a.c_str()));
    else if (a == "--ThermalizationSteps") o->thermalization = std::atoi(next(a.c_str()));
    else if (a == "--NumberOfMeasures") o->n_measures = std::atoi(next(a.c_str()));
    else if (a == "--Rng") o->seed = std::atoll(next(a.c_str()));
    else if (a == "--J1") o->J1 = std::atof(next(a.c_str()));
    else if (a == "--J2") o->J2 = std::atof(next(a.c_str()));
    else if (a == "--J3") o->J3 = std::atof(next(a.c_str()));
    else if (a == "--J4") o->J4 = std::atof(next(a.c_str()));
    else if (a == "--MagneticField") o->field = true;
    else if (a == "--Bx") o->B[0] = std::atof(next(a.c_str()));
    else if (a == "--By") o->B[1] = std::atof(next(a.c_str()));
    else if (a == "--Bz") o->B[2] = std::atof(next(a.c_str()));
    else if (a == "--gxy") o->gxy = std::atof(next(a.c_str()));
    else if (a == "--gz") o->gz = std::atof(next(a.c_str()));
    else if (a == "--Magnetization") o->magnetization = true;
    else if (a == "--OrderParameters") o->order_parameters = true;
    else if (a == "--Quadrupole") o->quadrupole = true;
    else if (a == "--Zaxis") o->zaxis = true;
    else if (a == "--ZaxisSum") o->zaxis_sum = true;
    else if (a == "--DChiDt") o->dchidt = true;
    else if (a == "--NumberOfRepetitions") o->repetitions = std::atoi(next(a.c_str()));
    else if (a == "--Heisenberg") {
      o->heisenberg = true;
      o->J = std::atof(next(a.c_str()));
    } else if (a == "--Jnn2") o->Jnn2 = std::atof(next(a.c_str()));
    else if (a == "--Jnn3") o->Jnn3 = std::atof(next(a.c_str()));
    else if (a == "--NoReductionAngle") o->reduction_angle = false;
    else if (a == "--Ratio") o->ratio = std::atof(next(a.c_str()));
    else if (a == "--Device") o->device = std::atoi(next(a.c_str()));
    else if (a == "--Output") o->out = next(a.c_str());
    else {
      std::fprintf(stderr, "%s: unknown option. See --help for more details.\n", a.c_str());
      return false;
    }
  }
  return true;
}

// One repetition: equilibration, cone tuning, then the measurement loop with
// its statistics files (suffix `rep`); the energy series goes to `series`.
void run(const Options& o, int rep, const std::string& series) {
  const std::vector<double> T = pyro_host::Ladder(o.tmin, o.tmax, o.n_temps, o.log_scale);
  pyro_host::Device dev(o.L, T, o.heisenberg ? o.J : 0.0, o.Jnn2, o.Jnn3,
                        (uint64_t)(o.seed + rep), o.device);
  if (!o.heisenberg)
    pyro_host::InitializeCouplings3D(dev, o.J1, o.J2, o.J3, o.J4, o.field ? 1 : 0, o.B, o.gxy,
                                     o.gz);
  pyro_host::GenerateRandomVectorsOnDevice(dev);
  std::vector<float> cone;
  if (o.reduction_angle) pyro_host::CalculateSolidAngle(dev, o.over_relaxation, o.ratio, cone);
  std::vector<double> temps, energies;
  for (int c = 0; c < o.thermalization; ++c)
    pyro_host::ParallelTempering(dev, o.over_relaxation, o.mc_steps_pt, temps, energies);
  FILE* f = std::fopen(series.c_str(), "w");
  if (!f) throw std::runtime_error("cannot open " + series);
  std::fprintf(f, "# measure, then E/N for T =");
  for (double t : T) std::fprintf(f, " %.6g", t);
  std::fprintf(f, "\n");
  FILE* fm = nullptr;
  if (o.magnetization) {
    const std::string mpath = series + ".magnetization";
    fm = std::fopen(mpath.c_str(), "w");
    if (!fm) {
      std::fclose(f);
      throw std::runtime_error("cannot open " + mpath);
    }
    std::fprintf(fm, "# measure, then (Mx, My, Mz)/N with the g-tensor for each T\n");
  }
  const int nT = (int)T.size();
  const bool need_op = o.order_parameters || o.quadrupole || o.zaxis || o.zaxis_sum || o.dchidt;
  pyro_host::Measure energy_m(nT, 2), op_m(nT, 10), dchi_m(nT, 10), quad_m(nT, 3), sz_m(nT, 1),
      szsum_m(nT, 1), mag_m(nT, 1);
  const std::string sfx = std::to_string(rep) + ".dat";
  auto save = [&]() {
    energy_m.SaveData("Energies" + sfx, T, "E, E^2");
    if (o.order_parameters || o.dchidt)
      op_m.SaveData("OrderParameters" + sfx, T,
                    "|m_A2| |m_E| |m_T| |m_F| |m_T'| then their squares");
    if (o.dchidt) dchi_m.SaveData("dchidt" + sfx, T, "the OrderParameters columns times E");
    if (o.quadrupole)
      quad_m.SaveData("Quadrupole" + sfx, T,
                      "sqrt((2qxx-qyy-qzz)^2 + 3(qzz-qyy)^2), |off-diagonal|, |Q|");
    if (o.zaxis) sz_m.SaveData("Sz" + sfx, T, "sum |a.S| / sqrt 3");
    if (o.zaxis_sum) szsum_m.SaveData("SzSum" + sfx, T, "monopole density");
    if (o.magnetization) mag_m.SaveData("Magnetization" + sfx, T, "|M| with the g-tensor");
  };
  std::vector<double> eT(nT), mT(3 * nT), M, op;
  std::vector<double> e_row(2 * nT), op_row(10 * nT), dchi_row(10 * nT), q_row(3 * nT),
      sz_row(nT), szs_row(nT), mag_row(nT);
  std::vector<int> slot(nT, 0);  // replica holding temperature t
  // Measure cycle m from a snapshot while cycle m + 1 runs on the GPU.
  pyro_host::ParallelTemperingAsync(dev, o.over_relaxation, o.mc_steps_pt);
  pyro_host::ExtractConfigurationsFromMonteCarlo(dev);
  for (int m = 0; m < o.n_measures; ++m) {
    if (m + 1 < o.n_measures)
      pyro_host::ParallelTemperingAsync(dev, o.over_relaxation, o.mc_steps_pt);
    pyro_host::MeasureSnapshot(dev, true);
    pyro_host::CycleEnergies(dev, energies);
    pyro_host::SlotTemperatures(dev, temps);
    if (fm || o.magnetization) pyro_host::MagnetizationG(dev, o.gxy, o.gz, M);
    if (need_op) pyro_host::OrderParameters(dev, op);
    pyro_host::MeasureSnapshot(dev, false);
    if (m + 1 < o.n_measures) pyro_host::ExtractConfigurationsFromMonteCarlo(dev);
    for (size_t r = 0; r < temps.size(); ++r)
      for (int t = 0; t < nT; ++t)
        if (temps[r] == T[t]) slot[t] = (int)r;
    for (int t = 0; t < nT; ++t) {
      const int r = slot[t];
      const double E = energies[r];
      eT[t] = E / dev.sites();
      e_row[2 * t] = E;
      e_row[2 * t + 1] = E * E;
      if (o.magnetization) {
        for (int k = 0; k < 3; ++k) mT[3 * t + k] = M[3 * r + k] / dev.sites();
        mag_row[t] = std::sqrt(M[3 * r] * M[3 * r] + M[3 * r + 1] * M[3 * r + 1] +
                               M[3 * r + 2] * M[3 * r + 2]);
      }
      if (need_op) {
        const double* q = &op[20 * r];
        const double sq[5] = {q[0] * q[0], q[1] * q[1] + q[2] * q[2],
                              q[3] * q[3] + q[4] * q[4] + q[5] * q[5],
                              q[6] * q[6] + q[7] * q[7] + q[8] * q[8],
                              q[9] * q[9] + q[10] * q[10] + q[11] * q[11]};
        for (int k = 0; k < 5; ++k) {
          op_row[10 * t + k] = std::sqrt(sq[k]);
          op_row[10 * t + 5 + k] = sq[k];
        }
        for (int k = 0; k < 10; ++k) dchi_row[10 * t + k] = op_row[10 * t + k] * E;
        const double qxx = q[12], qxy = q[13], qxz = q[14], qyy = q[15], qyz = q[16], qzz = q[17];
        q_row[3 * t] = std::sqrt((2.0 * qxx - qyy - qzz) * (2.0 * qxx - qyy - qzz) +
                                 3.0 * (qzz - qyy) * (qzz - qyy));
        q_row[3 * t + 1] = std::sqrt(qxy * qxy + qxz * qxz + qyz * qyz);
        q_row[3 * t + 2] =
            std::sqrt(qxx * qxx + qyy * qyy + qzz * qzz + qxy * qxy + qxz * qxz + qyz * qyz);
        szs_row[t] = q[18];
        sz_row[t] = q[19];
      }
    }
    energy_m.Accumulate(e_row);
    if (need_op) {
      op_m.Accumulate(op_row);
      dchi_m.Accumulate(dchi_row);
      quad_m.Accumulate(q_row);
      sz_m.Accumulate(sz_row);
      szsum_m.Accumulate(szs_row);
    }
    if (o.magnetization) mag_m.Accumulate(mag_row);
    std::fprintf(f, "%d", m);
    for (double e : eT) std::fprintf(f, " %.12g", e);
    std::fprintf(f, "\n");
    if (fm) {
      std::fprintf(fm, "%d", m);
      for (double v : mT) std::fprintf(fm, " %.12g", v);
      std::fprintf(fm, "\n");
    }
    if (m % 500 == 499) save();
  }
  std::fclose(f);
  if (fm) std::fclose(fm);
  save();
  std::printf("repetition %d: %d measures of %d temperatures (%s, statistics *%s)\n", rep,
              o.n_measures, o.n_temps, series.c_str(), sfx.c_str());
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, &o)) return 1;
  if (o.repetitions < 1) {
    std::fprintf(stderr, "--NumberOfRepetitions must be >= 1\n");
    return 1;
  }
  try {
    for (int rep = 0; rep < o.repetitions; ++rep)
      run(o, rep, rep == 0 ? o.out : o.out + "." + std::to_string(rep));
  } catch (const pyro_host::Error& e) {
    std::fprintf(stderr, "pyro_run: %s (status %d)\n", e.what(), e.code);
    return 2;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "pyro_run: %s\n", e.what());
    return 1;
  }
  return 0;
}
