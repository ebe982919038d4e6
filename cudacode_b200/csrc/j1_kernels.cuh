// Launch interface of the nearest-neighbour (J1-only) kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lattice.h"

namespace pyro {

constexpr int kJ1Threads = 256;

// One colour pass over all replicas of one J1-only system.
struct J1PassParams {
  float4* spins;  // replica 0 of the system
  int L, L3, n_rep;
  float rcpL;
  int rep_global, rep_key, temp_base;
  float J1;
  const int* temp_of_rep;
  const float* beta;
  const float* cosmax;
  unsigned long long* accepted;
  const unsigned long long* sweep_ctr;
  unsigned long long sweep_off;
  uint32_t seed_lo, seed_hi;
  int renorm_every;
};

// FP64 energy (by tetrahedra) and magnetisation partials of one J1 system;
// partial of (replica r, block b) at partials[partial_begin + r * nblocks + b].
struct J1ObsParams {
  const float4* spins;
  int L, L3, n_rep;
  float rcpL;
  double J1;
  double4* partials;
  int partial_begin;
};

void launch_j1_pass(const J1PassParams& p, int colour, bool metro, cudaStream_t st);
void launch_j1_observables(const J1ObsParams& p, cudaStream_t st);

inline int j1_blocks_per_replica(int L3) { return (L3 + kJ1Threads - 1) / kJ1Threads; }

}  // namespace pyro
