// pyro_run: command-line driver of the engine, with the option names of the
// reference's main (Pyrochlore.cu:1161-1216) for the Monte Carlo path:
// annealing-free equilibration, cone tuning, parallel tempering, and
// measurement of the energy per temperature into Energies.dat.
//
//   pyro_run --nx 8 --NumberOfTemperatures 16 --TMin 0.05 --TMax 1 --LogScale
//            --OverRelaxation 4 --McStepsParallelTempering 1
//            --ThermalizationSteps 1000 --NumberOfMeasures 1000 --Rng 56081376
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

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

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, &o)) return 1;
  try {
    const std::vector<double> T = pyro_host::Ladder(o.tmin, o.tmax, o.n_temps, o.log_scale);
    pyro_host::Device dev(o.L, T, o.heisenberg ? o.J : 0.0, o.Jnn2, o.Jnn3, (uint64_t)o.seed,
                          o.device);
    if (!o.heisenberg)
      pyro_host::InitializeCouplings3D(dev, o.J1, o.J2, o.J3, o.J4, o.field ? 1 : 0, o.B, o.gxy,
                                       o.gz);
    pyro_host::GenerateRandomVectorsOnDevice(dev);
    std::vector<float> cone;
    if (o.reduction_angle) pyro_host::CalculateSolidAngle(dev, o.over_relaxation, o.ratio, cone);
    std::vector<double> temps, energies;
    for (int c = 0; c < o.thermalization; ++c)
      pyro_host::ParallelTempering(dev, o.over_relaxation, o.mc_steps_pt, temps, energies);
    FILE* f = std::fopen(o.out.c_str(), "w");
    if (!f) {
      std::fprintf(stderr, "cannot open %s\n", o.out.c_str());
      return 1;
    }
    std::fprintf(f, "# measure, then E/N for T =");
    for (double t : T) std::fprintf(f, " %.6g", t);
    std::fprintf(f, "\n");
    FILE* fm = nullptr;
    if (o.magnetization) {
      const std::string mpath = o.out + ".magnetization";
      fm = std::fopen(mpath.c_str(), "w");
      if (!fm) {
        std::fprintf(stderr, "cannot open %s\n", mpath.c_str());
        std::fclose(f);
        return 1;
      }
      std::fprintf(fm, "# measure, then (Mx, My, Mz)/N with the g-tensor for each T\n");
    }
    std::vector<double> eT(T.size()), mT(3 * T.size()), M;
    for (int m = 0; m < o.n_measures; ++m) {
      pyro_host::ParallelTempering(dev, o.over_relaxation, o.mc_steps_pt, temps, energies);
      if (fm) pyro_host::MagnetizationG(dev, o.gxy, o.gz, M);
      for (size_t r = 0; r < temps.size(); ++r)
        for (size_t t = 0; t < T.size(); ++t)
          if (temps[r] == T[t]) {
            eT[t] = energies[r] / dev.sites();
            if (fm)
              for (int k = 0; k < 3; ++k) mT[3 * t + k] = M[3 * r + k] / dev.sites();
          }
      std::fprintf(f, "%d", m);
      for (double e : eT) std::fprintf(f, " %.12g", e);
      std::fprintf(f, "\n");
      if (fm) {
        std::fprintf(fm, "%d", m);
        for (double v : mT) std::fprintf(fm, " %.12g", v);
        std::fprintf(fm, "\n");
      }
    }
    std::fclose(f);
    if (fm) std::fclose(fm);
    std::printf("wrote %d measures of %d temperatures to %s\n", o.n_measures, o.n_temps,
                o.out.c_str());
  } catch (const pyro_host::Error& e) {
    std::fprintf(stderr, "pyro_run: %s (status %d)\n", e.what(), e.code);
    return 2;
  }
  return 0;
}
