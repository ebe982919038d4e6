// Launch interface of the shared-memory-resident small-lattice kernel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lattice.h"

namespace pyro {

constexpr int kSmemThreads = 256;
constexpr int kSmemMaxL = 8;  // 16 L^3 float4 = 128 KiB at L = 8

// n_cycles cycles of (n_metro + n_or sweeps, energy into the history ring)
// of every replica of one system, one CTA per replica.
struct SmemCycleParams {
  SysDev sys;
  float4* spins;  // replica 0 of the system
  const int* temp_of_rep;
  const float* beta;
  const float* cosmax;
  unsigned long long* accepted;
  const unsigned long long* sweep_ctr;
  int n_metro, n_or, n_cycles;
  int renorm_every;
  uint32_t seed_lo, seed_hi;
  double* history;  // may be null
  const unsigned long long* history_count;
  int history_cap, total_temps;
  const ExchangeDev* exch;  // bond matrices (sys.exch >= 0)
  double* energy;           // final-state energy / magnetisation per context replica (or null)
  double* mag;
};

size_t smem_cycle_bytes(int L);
cudaError_t launch_smem_cycles(const SmemCycleParams& p, const NbrTable& tab, cudaStream_t st);

}  // namespace pyro
