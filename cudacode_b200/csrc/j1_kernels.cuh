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
  // Per-pass launches of isotropic systems with L = 16 or 32 use kernels
  // compiled for that L (shift decode, compile-time plane offsets) when set.
  int fixed_l;
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

// A whole cycle of one J1 system as one launch over a work queue (the
// work-queue cycle kernel). A work item is one colour pass of one
// kJ1Threads-cell chunk of one replica: one CTA of the per-pass kernel
// (cell form), or a quarter of it (site form, one FCC corner). Items are
// numbered replica group by replica group, pass by pass, the chunks of pass
// k starting at chunk dep * k so that an item's inputs were issued a whole
// pass earlier. The grid has one CTA per item; each CTA takes the next
// ticket of an atomic counter as its item. Before it starts, the item of
// pass k on chunk q waits until pass k - 1 is complete on chunks
// q - dep .. q + dep (every chunk holding a neighbour of its cells):
// progress[rep][chunk] counts the items completed on that chunk, released
// after the item's stores and acquired before the dependants' loads. An item
// only waits on items with smaller tickets, all of them taken by CTAs that
// are running, so the launch always makes progress; every wait is bounded
// all the same (spin_limit polls), after which the kernel sets *status = 1
// and the waiting CTAs return.
struct J1WaveParams {
  J1PassParams pass;  // whole system; sweep_off = offset of the cycle's first sweep
  J1ObsParams obs;    // observables partials (with_obs), as launch_j1_observables writes them
  int n_metro, n_or;
  int group;       // replicas per group
  int n_chunks;    // chunks of kJ1Threads cells per replica
  int dep;         // dependency half-width, in chunks
  // After the 4 (n_metro + n_or) colour passes, an observables pass (one
  // cell-form item per chunk) writes the FP64 energy and magnetisation
  // partials of the state the last pass left.
  int with_obs;
  // Items per chunk of a Metropolis / over-relaxation pass: 1 (cell form)
  // or 4 (site form, one per FCC corner), as the kernel variant's forms.
  int sub_metro, sub_or;
  unsigned int* progress;  // [n_rep][n_chunks], zero at launch
  unsigned int* queue;     // next ticket, zero at launch
  int* status;             // set to 1 when a wait gave up
  int n_items;             // = grid size
  unsigned int spin_limit;
  int stall_item;          // diagnostics: this item never reports completion (-1: none)
};

// forms: bit 0 Metropolis passes in the site form, bit 1 over-relaxation
// passes in the site form.
cudaError_t launch_j1_wave(const J1WaveParams& p, int forms, cudaStream_t st);

// A cycle of one J1 system as skewed launches: replica group g (of w.group
// replicas) runs its pass k (k < 4 (n_metro + n_or): colour passes; k ==
// 4 (n_metro + n_or), with w.with_obs: its energy partials) in launch
// t = stagger g + k, so every launch holds the passes of about
// passes / stagger groups at once (one launch fills the GPU; their spins
// stay in L2) and needs no synchronisation inside: its items belong to
// different replicas, and consecutive passes of a group are in consecutive
// launches of one stream. Items and their code are the work-queue kernel's
// (w.queue, w.progress and w.status are unused).
struct J1SkewParams {
  J1WaveParams w;
  int t;         // launch index, 0 .. stagger (n_groups - 1) + passes - 1
  int stagger;   // launches between the starts of consecutive groups
  int n_groups;  // ceil(n_rep / group)
};
__host__ __device__ inline int skew_passes(const J1WaveParams& w) {
  return 4 * (w.n_metro + w.n_or) + (w.with_obs ? 1 : 0);
}
__host__ __device__ inline int skew_sub(const J1WaveParams& w, int k) {
  return k < 4 * w.n_metro ? w.sub_metro : (k < 4 * (w.n_metro + w.n_or) ? w.sub_or : 1);
}
__host__ __device__ inline int skew_first_group(const J1SkewParams& sp) {
  const int lag = sp.t - (skew_passes(sp.w) - 1);
  const int g = lag <= 0 ? 0 : (lag + sp.stagger - 1) / sp.stagger;
  return g;
}
__host__ __device__ inline int skew_last_group(const J1SkewParams& sp) {
  const int g = sp.t / sp.stagger;
  return g < sp.n_groups - 1 ? g : sp.n_groups - 1;
}
// Items (CTAs) of launch sp.t.
int j1_skew_items(const J1SkewParams& sp);
cudaError_t launch_j1_skew(const J1SkewParams& sp, int forms, cudaStream_t st);
// Dependency half-width in chunks for lattice size L.
int j1_wave_dep(int L);

// log2 L of the fixed-L per-pass kernels that launch_j1_pass and
// launch_j1_last_pass use for `p` (0: the run-time-L kernels).
int j1_fixed_log2(const J1PassParams& p);

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
