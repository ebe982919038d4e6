// Launch interface of the nearest-neighbour (J1-only) kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lattice.h"

namespace pyro {

constexpr int kJ1Threads = 256;
constexpr int kJ1CycleThreads = 1024;  // CTA size of the cluster-resident cycle kernel

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
  // Bond matrices and Zeeman field of an anisotropic system (exch != 0):
  // xa[b][slot] = A[b][b'] for the three other sublattices b' in increasing
  // order, xf[b] = f[b]. Kernel parameters, so the update's multiply-adds
  // read them from the constant bank.
  int exch;
  float xa[4][3][9];
  float xf[4][3];
  // Programmatic dependent launch: the pass may be launched while the
  // previous kernel of its stream drains; it waits (griddepcontrol.wait)
  // before its first global memory access.
  int pdl;
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
  int pdl;  // programmatic dependent launch (waits for the previous kernel before reading)
};

// A whole cycle (n_metro + n_or sweeps, then observables partials if
// partials != null) of every replica of one J1 system, one thread-block
// cluster of cluster_size CTAs per replica.
struct J1CycleParams {
  J1PassParams pass;  // sweep_off = offset of the first sweep of the cycle
  int n_metro, n_or;
  int cluster_size;
  double J1_64;
  double4* partials;
  int partial_begin;
};

// site_per_thread: one site per thread (more warps in flight) instead of the
// 4 sites of a cell per thread; identical results.
void launch_j1_pass(const J1PassParams& p, int colour, bool metro, bool site_per_thread,
                    cudaStream_t st);
cudaError_t launch_j1_cycle(const J1CycleParams& p, cudaStream_t st);
// Sets the kernel's cluster attributes; reports how many clusters of this
// size can be resident at once (0: size not supported).
cudaError_t j1_cycle_prepare(int cluster_size, int* max_active_clusters);
void launch_j1_observables(const J1ObsParams& p, cudaStream_t st);
// The colour-3 pass (cell form, isotropic J1 only) with the observables
// partials of the resulting state (as launch_j1_observables writes them).
void launch_j1_last_pass(const J1PassParams& p, const J1ObsParams& o, bool metro,
                         cudaStream_t st);

inline int j1_blocks_per_replica(int L3) { return (L3 + kJ1Threads - 1) / kJ1Threads; }

}  // namespace pyro
