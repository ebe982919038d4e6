// Kernel parameter blocks and launchers shared by the C-ABI layer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "lattice.h"

namespace pyro {

constexpr int kPassThreads = 256;
constexpr int kObsThreads = 256;
constexpr int kObsSitesPerThread = 8;

// One colour pass (Metropolis or over-relaxation) over a list of segments.
struct PassParams {
  const PassSeg* segs;
  int nseg;
  const SysDev* sys;
  float4* spins;
  const int* temp_of_rep;       // global replica -> temperature slot (per system)
  const float* beta;            // [temp_base + t]
  const float* cosmax;          // [temp_base + t]
  unsigned long long* accepted; // [temp_base + t]
  const unsigned long long* sweep_ctr;  // device sweep counter (may be null)
  unsigned long long sweep_off; // added to *sweep_ctr (absolute if null)
  uint32_t seed_lo, seed_hi;
  int renorm_every;
  const ExchangeDev* exch;      // bond matrices of anisotropic systems (SysDev::exch >= 0)
  int pdl;                      // programmatic dependent launch (griddepcontrol.wait first)
};

// Energy / magnetisation partial sums, one block per chunk of a replica.
struct ObsSeg {
  int sys;
  int blocks_per_rep;
  int block_begin;    // first CTA of the segment in its launch
  int partial_begin;  // index of the segment's first partial in the shared buffer
};

struct ObsParams {
  const ObsSeg* segs;
  int nseg;
  const SysDev* sys;
  const float4* spins;
  double4* partials;  // one per block: (E, Mx, My, Mz)
  const ExchangeDev* exch;
};

struct ExchangeParams {
  const SysDev* sys;
  int n_sys;
  int sys_first;               // first system handled (blockIdx.x offset)
  const double* energy;        // by global replica of the system (+ e_base)
  int energy_is_global;        // 1: energy indexed from 0 by global replica id of the system
  const double* beta64;        // [temp_base + t]
  int* temp_of_rep;            // [temp_base + global replica]
  int* rep_of_temp;            // [temp_base + t]
  unsigned long long* swap_count;  // per system
  unsigned long long* swap_acc;    // [temp_base + t], accepted swaps of pair (t, t+1)
  unsigned long long* swap_try;    // [temp_base + t]
  int* last_accepted;              // per system, accepted pairs of this call
  int parity;                      // 0/1, or -1: (swap_count % 2)
  uint32_t seed_lo, seed_hi;
  double* history;                 // [slot * total_temps + temp_base + t] or null
  unsigned long long* history_count;  // cycles recorded (single counter)
  int history_cap;
  int total_temps;
  unsigned long long* sweep_ctr;   // advanced by sweep_advance (block 0) if non-null
  unsigned long long sweep_advance;
  int do_swap;
  // Non-null: the block first sums its system's observables partials into
  // energy and mag (as obs_finalise_kernel does, same order), so a cycle
  // needs no separate finalise launch.
  const double4* partials;
  const ObsSeg* obs_segs;
  double* energy_out;  // [rep_ctx_base + r]
  double* mag_out;     // [3 (rep_ctx_base + r) + k]
};

void launch_colour_pass(const PassParams& p, const NbrTable& tab, int n_blocks, bool metro,
                        bool j1_only, cudaStream_t st);
void launch_init_random(float4* spins, const SysDev* sys_host, const SysDev* sys_dev, int n_sys,
                        uint32_t seed_lo, uint32_t seed_hi, cudaStream_t st);
void launch_observables(const ObsParams& p, const NbrTable& tab, int n_blocks, cudaStream_t st);
// Sums partials of every replica of every system in fixed order.
void launch_obs_finalise(const double4* partials, const ObsSeg* segs, int nseg, const SysDev* sys,
                         int total_reps, const int* rep_sys, const int* rep_local,
                         double* energy_rep, double* mag_rep, cudaStream_t st);
void launch_exchange(const ExchangeParams& p, int n_sys, int max_pairs, cudaStream_t st);
void launch_advance(unsigned long long* ctr, unsigned long long by, cudaStream_t st);
void launch_check_spins(const float4* spins, long long n, float tol, unsigned long long* first_bad,
                        cudaStream_t st);

}  // namespace pyro
