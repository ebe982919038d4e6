// The engine context (one per GPU) shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/pyro.h"
#include "gen_wave.cuh"
#include "kernels.cuh"
#include "lattice.h"

namespace pyro {
struct TetState;  // learned tetrahedron move (tet_capi.cu)
constexpr int kMaxChains = 8;
}

struct pyro_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string err;
  uint64_t seed = 0;
  int renorm_every = 0;
  pyro::NbrTable tab;

  std::vector<pyro::SysDev> sys;
  std::vector<pyro::ExchangeDev> exch;  // bond matrices of the anisotropic systems (SysDev::exch)
  pyro::ExchangeDev* d_exch = nullptr;
  std::vector<std::vector<double>> ladders;
  pyro::SysDev* d_sys = nullptr;
  int total_temps = 0;
  int total_reps = 0;  // replicas held

  float4* d_spins = nullptr;
  long long n_spins = 0;

  int* d_temp_of_rep = nullptr;
  int* d_rep_of_temp = nullptr;
  float* d_beta = nullptr;
  double* d_beta64 = nullptr;
  float* d_cosmax = nullptr;
  unsigned long long* d_accepted = nullptr;
  unsigned long long* d_swap_acc = nullptr;
  unsigned long long* d_swap_try = nullptr;
  unsigned long long* d_swap_count = nullptr;
  int* d_last_accepted = nullptr;

  double* d_energy = nullptr;
  double* d_mag = nullptr;
  int* d_rep_sys = nullptr;
  int* d_rep_local = nullptr;

  // Observables: obs_segs covers every system in the global partial
  // numbering (read by the finalise kernel); obs_generic is the subset run by
  // the generic kernel (launch-local block_begin, global partial_begin);
  // J1-only systems on the specialised path are listed in obs_j1.
  std::vector<pyro::ObsSeg> obs_segs, obs_generic;
  std::vector<int> obs_j1;
  // Systems swept by the specialised J1 kernels: obs_j1 (isotropic) plus the
  // 4-colour systems with bond matrices (their observables run generic).
  std::vector<int> j1_sys;
  pyro::ObsSeg* d_obs_segs = nullptr;
  pyro::ObsSeg* d_obs_generic = nullptr;
  int obs_generic_blocks = 0;
  int partials_cap = 0;
  double4* d_partials = nullptr;

  // Colour passes: generic segments, plus (system, colour) launches of the
  // specialised J1 kernel.
  int n_passes = 4;
  bool use_j1_kernel = true;
  // Per-pass J1 kernel form for Metropolis / over-relaxation passes:
  // one site per thread (true) or the 4 sites of a cell per thread.
  bool j1_metro_site_mode = true;
  bool j1_or_site_mode = false;
  int j1_fixed_l = 1;  // fixed-L per-pass kernels for L = 16, 32 (PYRO_OPT_J1_FIXED_L)
  // Cycle kernel for J1 systems: 0 per-pass launches, 1 cluster-resident,
  // 2 the work-queue kernel (one launch per system per cycle).
  int cycle_kernel = 0;
  // Work-queue kernel: per J1 system, a queue ticket (padded to 128 bytes)
  // and the per-(replica, chunk) progress counters; zeroed before each
  // launch. wave_status is set by a dependency wait that gave up.
  unsigned int* d_wave = nullptr;
  size_t wave_words = 0;
  int* d_wave_status = nullptr;
  int* h_wave_status = nullptr;  // pinned copy, read after a synchronising call
  int wave_stall_item = -1;
  // Work-queue kernel of the 16-colour systems (same option): its units and
  // groups, and a queue ticket (padded) plus one progress counter per (unit,
  // chunk), zeroed before each launch.
  pyro::GenWaveUnit* d_gwave_units = nullptr;
  pyro::GenWaveGroup* d_gwave_groups = nullptr;
  int* d_gwave_chunk_unit = nullptr;
  size_t gwave_chunk_cap = 0;
  unsigned int* d_gwave = nullptr;
  size_t gwave_units_cap = 0, gwave_groups_cap = 0, gwave_words = 0;
  int gwave_n_groups = 0;
  long long gwave_chunks = 0;  // chunks of one pass over every unit
  int smem_kernel = 1;
  int rep_group = 0;    // per-pass J1 kernels over groups of this many replicas (0: all)
  int gen_group_mb = 0; // generic kernels over groups of replicas of about this many MB (0: off)
  struct GenGroup {
    std::vector<std::vector<pyro::PassSeg>> pass_segs;  // per pass
    std::vector<int> pass_blocks;
    std::vector<pyro::PassSeg*> d_pass_segs;
    std::vector<char> all16;  // every segment of the pass is a 16-colour system
  };
  std::vector<char> pass_all16;  // same, for the ungrouped generic lists
  int far_kernel = 1;  // compile-time-offset kernel for 16-colour passes
  int pdl = 1;         // programmatic dependent launch of the per-pass J1 kernels
  int tet_grouped = 1;  // learned sweeps inside the replica groups
  int fused_obs = 1;    // energy partials from a group's last pass (grouped J1 path)
  bool defer_finalise = false;  // while a cycle is captured: its exchange kernel finalises
  std::vector<GenGroup> gen_groups;
  int n_chains = 1;     // concurrent streams the replica groups are dealt to
  cudaStream_t chain_stream[pyro::kMaxChains] = {};
  cudaEvent_t chain_event[pyro::kMaxChains] = {};
  // PYRO_OPT_CHAIN_STAGGER: each odd chain starts after the preceding
  // chain's first chain_stagger passes (0: all chains start together)
  int chain_stagger = 0;
  cudaEvent_t stagger_event[pyro::kMaxChains] = {};
  cudaEvent_t fork_event = nullptr;  // cycles without exchange of L <= 8 systems in shared memory
  int cluster_size = 16;
  bool cluster_checked = false;
  std::vector<std::vector<pyro::PassSeg>> pass_segs;
  std::vector<std::vector<std::pair<int, int>>> pass_j1;
  std::vector<pyro::PassSeg*> d_pass_segs;
  std::vector<int> pass_blocks;

  unsigned long long* d_sweep = nullptr;
  unsigned long long h_sweep = 0;
  unsigned long long metro_sweeps_since_reset = 0;
  unsigned long long* d_scratch_u64 = nullptr;

  double* d_history = nullptr;
  int history_cap = 0;
  unsigned long long* d_history_count = nullptr;

  std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> graphs;
  std::map<std::tuple<int, int, int, int>, unsigned long long> graph_kernels;
  unsigned long long launches = 0;  // kernels run by graph replays and direct calls

  // Structure-factor scratch, grown on demand.
  double2* d_sq_s1 = nullptr;
  double2* d_sq_s2 = nullptr;
  double2* d_sq_tw = nullptr;
  double* d_sq_out = nullptr;
  size_t sq_s1 = 0, sq_s2 = 0, sq_tw = 0, sq_out = 0;
  bool sq_ready = false;  // DFT kernels' shared-memory limit raised

  pyro::TetState* tet = nullptr;

  // Measurement snapshot (pyro_snapshot): copies of every system's spins, of
  // the replica <-> temperature maps and of the last cycle's FP64 energies
  // and magnetisations, taken on snap_stream; with measure_snapshot set the
  // measurement calls read them there while later cycles run.
  float4* d_snap = nullptr;
  int* d_snap_temp_of_rep = nullptr;
  int* d_snap_rep_of_temp = nullptr;
  double* d_snap_energy = nullptr;
  double* d_snap_mag = nullptr;
  cudaStream_t snap_stream = nullptr;
  cudaEvent_t snap_start = nullptr, snap_done = nullptr;
  bool snap_taken = false;
  int measure_snapshot = 0;

  // Per-sublattice magnetisation partials, grown on demand (exchange.cu).
  double* d_submag = nullptr;
  size_t submag_cap = 0;
  // Order-parameter scratch, grown on demand (order.cu), bytes.
  void* d_order = nullptr;
  size_t order_cap = 0;
};

namespace pyro {

// Systems on the isotropic nearest-neighbour-only paths (specialised J1
// kernels, learned tetrahedron move).
inline bool j1_only(const SysDev& s) { return s.n_colours == 4 && s.shells == 1 && s.exch < 0; }
// Systems the specialised nearest-neighbour sweep kernels can run: J1-only,
// or bond matrices with no further shells.
inline bool j1_sweepable(const SysDev& s) {
  return s.n_colours == 4 && (j1_only(s) || (s.exch >= 0 && (s.shells & ~1) == 0));
}

// NVTX range around a C-ABI call (header-only NVTX 3: inert unless a
// profiler attaches), so timelines show cycles, measurements and training.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

inline int fail(pyro_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

// What the measurement calls read: the live state on the context stream,
// or (measure_snapshot) the last pyro_snapshot on the measurement stream.
inline const float4* measure_spins(const pyro_ctx* c) {
  return c->measure_snapshot ? c->d_snap : c->d_spins;
}
inline cudaStream_t measure_stream(const pyro_ctx* c) {
  return c->measure_snapshot ? c->snap_stream : c->stream;
}
inline const int* measure_temp_of_rep(const pyro_ctx* c) {
  return c->measure_snapshot ? c->d_snap_temp_of_rep : c->d_temp_of_rep;
}
inline const int* measure_rep_of_temp(const pyro_ctx* c) {
  return c->measure_snapshot ? c->d_snap_rep_of_temp : c->d_rep_of_temp;
}

// Drops the captured cycle graphs and rebuilds the pass schedules (after a
// change of kernel options or of a system's Hamiltonian).
int rebuild_schedule(pyro_ctx* ctx);

// Frees the learned-move state (tet_capi.cu).
void tet_free(pyro_ctx* ctx);
// Queues n learned tetrahedron sweeps of every J1-only system (tet_capi.cu).
int queue_tet_sweeps(pyro_ctx* ctx, int n);
// Queues n learned sweeps of replicas [r0, r0 + cnt) of system si on stream
// st (a replica group of the grouped cycle; a no-op for other systems), and
// advances the learned-move sweep counter by n on the context stream.
int queue_tet_group(pyro_ctx* ctx, int si, int r0, int cnt, int n, cudaStream_t st);
void tet_advance(pyro_ctx* ctx, int n);
// Adds n to the learned-move proposal count (acceptance statistics).
void tet_count_sweeps(pyro_ctx* ctx, unsigned long long n);
// Learned-move sweep counter (device), read / set synchronously.
unsigned long long tet_counter(pyro_ctx* ctx);
void tet_set_counter(pyro_ctx* ctx, unsigned long long v);

}  // namespace pyro

#define PYRO_CK(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return ::pyro::fail(ctx, PYRO_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define PYRO_CK_LAUNCH()                                                                \
  do {                                                                                  \
    cudaError_t e_ = cudaGetLastError();                                                \
    if (e_ != cudaSuccess)                                                              \
      return ::pyro::fail(ctx, PYRO_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)
