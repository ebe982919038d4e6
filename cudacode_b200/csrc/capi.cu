// C-ABI implementation: context, memory layout, pass schedules, CUDA graph of
// the sweep + exchange cycle, and the host-side wrappers of include/pyro.h.
//
// The reference keeps this state in `struct dev` (fields used at
// MonteCarlo.cu:15-245, Pyrochlore.cu:74-133) and drives it from one pthread
// per GPU; here one context owns one GPU's memory and all calls are
// stream-ordered on the context's stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/pyro.h"
#include "ctx.h"
#include "j1_kernels.cuh"
#include "kernels.cuh"
#include "lattice.h"
#include "far_kernels.cuh"
#include "smem_kernels.cuh"
#include "sq_kernels.cuh"

using namespace pyro;

namespace {

template <typename T>
cudaError_t alloc(T** p, size_t n) {
  return cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(n, 1));
}

PassParams pass_params(pyro_ctx* ctx, int pass) {
  PassParams p;
  p.segs = ctx->d_pass_segs[pass];
  p.nseg = (int)ctx->pass_segs[pass].size();
  p.sys = ctx->d_sys;
  p.spins = ctx->d_spins;
  p.temp_of_rep = ctx->d_temp_of_rep;
  p.beta = ctx->d_beta;
  p.cosmax = ctx->d_cosmax;
  p.accepted = ctx->d_accepted;
  p.sweep_ctr = ctx->d_sweep;
  p.sweep_off = 0;
  p.seed_lo = (uint32_t)(ctx->seed & 0xffffffffu);
  p.seed_hi = (uint32_t)(ctx->seed >> 32);
  p.renorm_every = ctx->renorm_every;
  p.exch = ctx->d_exch;
  p.pdl = ctx->pdl;
  return p;
}

// Queues one sweep (all colour passes) with the given offset from *d_sweep.
J1PassParams j1_params(pyro_ctx* ctx, int si, unsigned long long off) {
  const SysDev& s = ctx->sys[si];
  J1PassParams p;
  p.spins = ctx->d_spins + s.spin_off;
  p.L = s.L;
  p.L3 = s.L3;
  p.n_rep = s.n_rep;
  p.rcpL = 1.0f / (float)s.L;
  p.rep_global = s.rep_global;
  p.rep_key = s.rep_key;
  p.temp_base = s.temp_base;
  p.J1 = s.J1;
  p.temp_of_rep = ctx->d_temp_of_rep;
  p.beta = ctx->d_beta;
  p.cosmax = ctx->d_cosmax;
  p.accepted = ctx->d_accepted;
  p.sweep_ctr = ctx->d_sweep;
  p.sweep_off = off;
  p.seed_lo = (uint32_t)(ctx->seed & 0xffffffffu);
  p.seed_hi = (uint32_t)(ctx->seed >> 32);
  p.renorm_every = ctx->renorm_every;
  p.exch = s.exch >= 0 ? 1 : 0;
  p.pdl = ctx->pdl;
  p.fixed_l = ctx->j1_fixed_l;
  std::memset(p.xa, 0, sizeof p.xa);
  std::memset(p.xf, 0, sizeof p.xf);
  if (s.exch >= 0) {
    const ExchangeDev& X = ctx->exch[s.exch];
    for (int b = 0; b < 4; ++b) {
      for (int t = 0, slot = 0; t < 4; ++t) {
        if (t == b) continue;
        for (int q = 0; q < 9; ++q) p.xa[b][slot][q] = X.A[4 * b + t][q];
        ++slot;
      }
      for (int q = 0; q < 3; ++q) p.xf[b][q] = X.f[b][q];
    }
  }
  return p;
}

int queue_sweep(pyro_ctx* ctx, bool metro, unsigned long long off, bool skip_j1 = false) {
  for (int pass = 0; pass < ctx->n_passes; ++pass) {
    for (const auto& sc : ctx->pass_j1[pass]) {
      if (skip_j1) break;
      const bool site_mode = metro ? ctx->j1_metro_site_mode : ctx->j1_or_site_mode;
      launch_j1_pass(j1_params(ctx, sc.first, off), sc.second, metro, site_mode, ctx->stream);
      PYRO_CK_LAUNCH();
    }
    if (ctx->pass_blocks[pass] == 0) continue;
    PassParams p = pass_params(ctx, pass);
    p.sweep_off = off;
    if (ctx->far_kernel && ctx->pass_all16[pass])
      launch_far_pass(p, pass, ctx->pass_blocks[pass], metro, ctx->stream);
    else
      launch_colour_pass(p, ctx->tab, ctx->pass_blocks[pass], metro, /*j1_only=*/false,
                         ctx->stream);
    PYRO_CK_LAUNCH();
  }
  return PYRO_OK;
}

int queue_observables(pyro_ctx* ctx, bool skip_j1 = false) {
  for (int si : ctx->obs_j1) {
    if (skip_j1) break;
    const SysDev& s = ctx->sys[si];
    J1ObsParams jp;
    jp.spins = ctx->d_spins + s.spin_off;
    jp.L = s.L;
    jp.L3 = s.L3;
    jp.n_rep = s.n_rep;
    jp.rcpL = 1.0f / (float)s.L;
    jp.J1 = s.J64[0];
    jp.partials = ctx->d_partials;
    jp.partial_begin = ctx->obs_segs[si].partial_begin;
    jp.pdl = ctx->pdl;
    launch_j1_observables(jp, ctx->stream);
    PYRO_CK_LAUNCH();
  }
  if (ctx->obs_generic_blocks > 0) {
    ObsParams op;
    op.segs = ctx->d_obs_generic;
    op.nseg = (int)ctx->obs_generic.size();
    op.sys = ctx->d_sys;
    op.spins = ctx->d_spins;
    op.partials = ctx->d_partials;
    op.exch = ctx->d_exch;
    launch_observables(op, ctx->tab, ctx->obs_generic_blocks, ctx->stream);
    PYRO_CK_LAUNCH();
  }
  if (ctx->defer_finalise) return PYRO_OK;  // the cycle's exchange kernel sums the partials
  launch_obs_finalise(ctx->d_partials, ctx->d_obs_segs, (int)ctx->obs_segs.size(), ctx->d_sys,
                      ctx->total_reps, ctx->d_rep_sys, ctx->d_rep_local, ctx->d_energy, ctx->d_mag,
                      ctx->stream);
  PYRO_CK_LAUNCH();
  return PYRO_OK;
}

// Checks once that the cluster size can be resident; falls back to smaller
// clusters, then to per-pass launches.
int check_cluster(pyro_ctx* ctx) {
  if (ctx->cluster_checked) return PYRO_OK;
  ctx->cluster_checked = true;
  if (ctx->cycle_kernel != 1) return PYRO_OK;
  for (int cs = ctx->cluster_size; cs >= 1; cs = cs > 8 ? 8 : cs / 2) {
    int n = 0;
    cudaError_t e = j1_cycle_prepare(cs, &n);
    if (e == cudaSuccess && n > 0) {
      ctx->cluster_size = cs;
      return PYRO_OK;
    }
    cudaGetLastError();
  }
  ctx->cycle_kernel = 0;
  return PYRO_OK;
}

// The cluster-resident cycle kernel runs isotropic J1 systems only; with a
// bond-matrix system on the J1 path every J1 system takes per-pass kernels.
bool use_cycle_kernel(const pyro_ctx* ctx) {
  return ctx->cycle_kernel == 1 && ctx->use_j1_kernel && !ctx->obs_j1.empty() &&
         ctx->j1_sys.size() == ctx->obs_j1.size();
}

// The work-queue cycle kernel runs the J1 systems of a cycle without
// learned sweeps.
bool use_wave_kernel(const pyro_ctx* ctx, int n_metro, int n_or, int n_tet) {
  return ctx->cycle_kernel == 2 && ctx->use_j1_kernel && !ctx->j1_sys.empty() && n_tet == 0 &&
         n_metro + n_or > 0;
}

constexpr size_t kWaveTicketWords = 32;  // a system's queue ticket, padded to 128 bytes

// Work-queue buffers for the current systems (allocated outside any capture).
int prepare_wave(pyro_ctx* ctx) {
  size_t words = 0;
  for (int si : ctx->j1_sys) {
    const SysDev& s = ctx->sys[si];
    words += kWaveTicketWords + (size_t)s.n_rep * j1_blocks_per_replica(s.L3);
  }
  if (words > ctx->wave_words) {
    if (ctx->d_wave) cudaFree(ctx->d_wave);
    ctx->d_wave = nullptr;
    ctx->wave_words = 0;
    PYRO_CK(alloc(&ctx->d_wave, words));
    ctx->wave_words = words;
  }
  if (!ctx->d_wave_status) {
    PYRO_CK(cudaHostAlloc((void**)&ctx->h_wave_status, sizeof(int), cudaHostAllocDefault));
    *ctx->h_wave_status = 0;
    PYRO_CK(alloc(&ctx->d_wave_status, 1));
    PYRO_CK(cudaMemset(ctx->d_wave_status, 0, sizeof(int)));
  }
  return PYRO_OK;
}

// One work-queue launch per J1 system: n_metro + n_or sweeps and, with
// with_obs, the energy partials of isotropic systems (the others' come from
// the generic observables kernel).
int queue_wave(pyro_ctx* ctx, int n_metro, int n_or, bool with_obs) {
  if (!ctx->d_wave || !ctx->d_wave_status) return fail(ctx, PYRO_ERR_STATE, "work queue not prepared");
  PYRO_CK(cudaMemsetAsync(ctx->d_wave, 0, ctx->wave_words * sizeof(unsigned int), ctx->stream));
  const int forms = (ctx->j1_metro_site_mode ? 1 : 0) | (ctx->j1_or_site_mode ? 2 : 0);
  size_t off = 0;
  for (int si : ctx->j1_sys) {
    const SysDev& s = ctx->sys[si];
    J1WaveParams w;
    std::memset(&w, 0, sizeof w);
    w.pass = j1_params(ctx, si, 0);
    w.pass.pdl = 0;
    w.n_metro = n_metro;
    w.n_or = n_or;
    w.group = ctx->rep_group > 0 ? std::min(ctx->rep_group, s.n_rep) : s.n_rep;
    w.n_chunks = j1_blocks_per_replica(s.L3);
    w.dep = j1_wave_dep(s.L);
    w.with_obs = with_obs && s.exch < 0 ? 1 : 0;
    w.obs.spins = ctx->d_spins + s.spin_off;
    w.obs.L = s.L;
    w.obs.L3 = s.L3;
    w.obs.n_rep = s.n_rep;
    w.obs.rcpL = 1.0f / (float)s.L;
    w.obs.J1 = s.J64[0];
    w.obs.partials = ctx->d_partials;
    w.obs.partial_begin = ctx->obs_segs[si].partial_begin;
    w.sub_metro = (forms & 1) ? 4 : 1;
    w.sub_or = (forms & 2) ? 4 : 1;
    w.queue = ctx->d_wave + off;
    w.progress = ctx->d_wave + off + kWaveTicketWords;
    w.status = ctx->d_wave_status;
    const long long items = (long long)s.n_rep * w.n_chunks *
                            (4ll * n_metro * w.sub_metro + 4ll * n_or * w.sub_or + w.with_obs);
    if (items > 0x7fffffffll) return fail(ctx, PYRO_ERR_ARG, "work-queue kernel: too many items");
    w.n_items = (int)items;
    w.spin_limit = ctx->wave_stall_item >= 0 ? 4096u : (1u << 20);
    w.stall_item = ctx->wave_stall_item;
    PYRO_CK(launch_j1_wave(w, forms, ctx->stream));
    off += kWaveTicketWords + (size_t)s.n_rep * w.n_chunks;
  }
  return PYRO_OK;
}

// The work-queue kernel of 16-colour systems runs, with PYRO_OPT_CYCLE_KERNEL
// 2, the systems off the nearest-neighbour path when every one of them is an
// isotropic 16-colour system (J2 or J3 set, no bond matrices).
bool use_gen_wave(const pyro_ctx* ctx, int n_metro, int n_or, int n_tet) {
  if (ctx->cycle_kernel != 2 || n_tet != 0 || n_metro + n_or <= 0) return false;
  bool any = false;
  for (int i = 0; i < (int)ctx->sys.size(); ++i) {
    if (std::find(ctx->j1_sys.begin(), ctx->j1_sys.end(), i) != ctx->j1_sys.end()) continue;
    const SysDev& s = ctx->sys[i];
    if (s.n_colours != 16 || s.exch >= 0) return false;
    any = true;
  }
  return any;
}

// Units (system, replica) of the 16-colour systems in groups of about
// PYRO_OPT_GROUP_MB MB of spins (one group when 0), their progress counters
// and the queue (allocated outside any capture).
int prepare_gen_wave(pyro_ctx* ctx) {
  std::vector<GenWaveUnit> units;
  std::vector<GenWaveGroup> groups;
  const double budget = ctx->gen_group_mb > 0 ? (double)ctx->gen_group_mb * 1048576.0 : 1e300;
  double bytes = 0.0;
  int prog = 0;
  for (int i = 0; i < (int)ctx->sys.size(); ++i) {
    if (std::find(ctx->j1_sys.begin(), ctx->j1_sys.end(), i) != ctx->j1_sys.end()) continue;
    const SysDev& s = ctx->sys[i];
    const double per_rep = 16.0 * 16.0 * s.L3;
    const int nq = (s.L3 + kPassThreads - 1) / kPassThreads;
    for (int r = 0; r < s.n_rep; ++r) {
      if (groups.empty() || (bytes > 0.0 && bytes + per_rep > budget)) {
        GenWaveGroup g;
        g.unit_begin = (int)units.size();
        g.n_units = 0;
        g.chunks = 0;
        g.chunk_prefix = 0;
        groups.push_back(g);
        bytes = 0.0;
      }
      GenWaveGroup& g = groups.back();
      GenWaveUnit u;
      u.sys = i;
      u.rep = r;
      u.n_chunks = nq;
      u.dep = (2 * s.L * s.L + kPassThreads - 1) / kPassThreads + 1;
      u.prog_off = prog;
      u.chunk_begin = g.chunks;
      units.push_back(u);
      g.n_units += 1;
      g.chunks += nq;
      prog += nq;
      bytes += per_rep;
    }
  }
  if (units.empty()) return fail(ctx, PYRO_ERR_STATE, "work queue: no 16-colour systems");
  if (units.size() > ctx->gwave_units_cap) {
    if (ctx->d_gwave_units) cudaFree(ctx->d_gwave_units);
    ctx->d_gwave_units = nullptr;
    ctx->gwave_units_cap = 0;
    PYRO_CK(alloc(&ctx->d_gwave_units, units.size()));
    ctx->gwave_units_cap = units.size();
  }
  if (groups.size() > ctx->gwave_groups_cap) {
    if (ctx->d_gwave_groups) cudaFree(ctx->d_gwave_groups);
    ctx->d_gwave_groups = nullptr;
    ctx->gwave_groups_cap = 0;
    PYRO_CK(alloc(&ctx->d_gwave_groups, groups.size()));
    ctx->gwave_groups_cap = groups.size();
  }
  const size_t words = kWaveTicketWords + (size_t)prog;
  if (words > ctx->gwave_words) {
    if (ctx->d_gwave) cudaFree(ctx->d_gwave);
    ctx->d_gwave = nullptr;
    ctx->gwave_words = 0;
    PYRO_CK(alloc(&ctx->d_gwave, words));
    ctx->gwave_words = words;
  }
  long long chunks = 0;
  for (auto& g : groups) {
    g.chunk_prefix = (int)chunks;
    chunks += g.chunks;
  }
  std::vector<int> chunk_unit;
  chunk_unit.reserve((size_t)chunks);
  for (int ui = 0; ui < (int)units.size(); ++ui)
    for (int q = 0; q < units[ui].n_chunks; ++q) chunk_unit.push_back(ui);
  if (chunk_unit.size() > ctx->gwave_chunk_cap) {
    if (ctx->d_gwave_chunk_unit) cudaFree(ctx->d_gwave_chunk_unit);
    ctx->d_gwave_chunk_unit = nullptr;
    ctx->gwave_chunk_cap = 0;
    PYRO_CK(alloc(&ctx->d_gwave_chunk_unit, chunk_unit.size()));
    ctx->gwave_chunk_cap = chunk_unit.size();
  }
  PYRO_CK(cudaMemcpy(ctx->d_gwave_chunk_unit, chunk_unit.data(), sizeof(int) * chunk_unit.size(),
                     cudaMemcpyHostToDevice));
  ctx->gwave_n_groups = (int)groups.size();
  ctx->gwave_chunks = chunks;
  PYRO_CK(cudaMemcpy(ctx->d_gwave_units, units.data(), sizeof(GenWaveUnit) * units.size(),
                     cudaMemcpyHostToDevice));
  PYRO_CK(cudaMemcpy(ctx->d_gwave_groups, groups.data(), sizeof(GenWaveGroup) * groups.size(),
                     cudaMemcpyHostToDevice));
  if (!ctx->d_wave_status) {
    PYRO_CK(cudaHostAlloc((void**)&ctx->h_wave_status, sizeof(int), cudaHostAllocDefault));
    *ctx->h_wave_status = 0;
    PYRO_CK(alloc(&ctx->d_wave_status, 1));
    PYRO_CK(cudaMemset(ctx->d_wave_status, 0, sizeof(int)));
  }
  return PYRO_OK;
}

// One work-queue launch for the 16-colour systems: n_metro + n_or sweeps
// (their energies come from the observables kernel after it).
int queue_gen_wave(pyro_ctx* ctx, int n_metro, int n_or) {
  if (!ctx->d_gwave || !ctx->d_wave_status) return fail(ctx, PYRO_ERR_STATE, "work queue not prepared");
  const long long item = 16ll * (n_metro + n_or) * ctx->gwave_chunks;
  if (item > 0x7fffffffll) return fail(ctx, PYRO_ERR_ARG, "work-queue kernel: too many items");
  PYRO_CK(cudaMemsetAsync(ctx->d_gwave, 0, ctx->gwave_words * sizeof(unsigned int), ctx->stream));
  GenWaveParams w;
  std::memset(&w, 0, sizeof w);
  w.pass = pass_params(ctx, 0);
  w.pass.segs = nullptr;
  w.pass.nseg = 0;
  w.pass.sweep_off = 0;
  w.pass.pdl = 0;
  w.units = ctx->d_gwave_units;
  w.groups = ctx->d_gwave_groups;
  w.chunk_unit = ctx->d_gwave_chunk_unit;
  w.n_groups = ctx->gwave_n_groups;
  w.n_metro = n_metro;
  w.n_or = n_or;
  w.queue = ctx->d_gwave;
  w.progress = ctx->d_gwave + kWaveTicketWords;
  w.status = ctx->d_wave_status;
  w.n_items = (int)item;
  w.spin_limit = ctx->wave_stall_item >= 0 ? 4096u : (1u << 20);
  w.stall_item = ctx->wave_stall_item;
  PYRO_CK(launch_gen_wave(w, ctx->stream));
  return PYRO_OK;
}

// The skewed multi-group launches run the J1 systems of a cycle without
// learned sweeps.
bool use_skew_kernel(const pyro_ctx* ctx, int n_metro, int n_or, int n_tet) {
  return ctx->cycle_kernel == 3 && ctx->use_j1_kernel && !ctx->j1_sys.empty() && n_tet == 0 &&
         n_metro + n_or > 0;
}

// Skewed launches per J1 system: replica groups of PYRO_OPT_REPLICA_GROUP
// (0: 2), about PYRO_OPT_CHAINS groups in flight per launch.
int queue_skew(pyro_ctx* ctx, int n_metro, int n_or, bool with_obs) {
  const int forms = (ctx->j1_metro_site_mode ? 1 : 0) | (ctx->j1_or_site_mode ? 2 : 0);
  for (int si : ctx->j1_sys) {
    const SysDev& s = ctx->sys[si];
    J1SkewParams sp;
    std::memset(&sp, 0, sizeof sp);
    J1WaveParams& w = sp.w;
    w.pass = j1_params(ctx, si, 0);
    w.n_metro = n_metro;
    w.n_or = n_or;
    w.group = std::min(ctx->rep_group > 0 ? ctx->rep_group : 2, s.n_rep);
    w.n_chunks = j1_blocks_per_replica(s.L3);
    w.with_obs = with_obs && s.exch < 0 ? 1 : 0;
    w.obs.spins = ctx->d_spins + s.spin_off;
    w.obs.L = s.L;
    w.obs.L3 = s.L3;
    w.obs.n_rep = s.n_rep;
    w.obs.rcpL = 1.0f / (float)s.L;
    w.obs.J1 = s.J64[0];
    w.obs.partials = ctx->d_partials;
    w.obs.partial_begin = ctx->obs_segs[si].partial_begin;
    w.sub_metro = (forms & 1) ? 4 : 1;
    w.sub_or = (forms & 2) ? 4 : 1;
    w.stall_item = -1;
    sp.n_groups = (s.n_rep + w.group - 1) / w.group;
    const int passes = skew_passes(w);
    const int in_flight = std::max(1, ctx->n_chains);
    sp.stagger = std::max(1, (passes + in_flight - 1) / in_flight);
    const int launches = sp.stagger * (sp.n_groups - 1) + passes;
    for (int t = 0; t < launches; ++t) {
      sp.t = t;
      PYRO_CK(launch_j1_skew(sp, forms, ctx->stream));
    }
  }
  return PYRO_OK;
}

// Queues the copy of the work-queue kernel's status word to pinned host
// memory (read by wave_status_result after the stream synchronised).
int queue_wave_status(pyro_ctx* ctx) {
  if (!ctx->d_wave_status) return PYRO_OK;
  PYRO_CK(cudaMemcpyAsync(ctx->h_wave_status, ctx->d_wave_status, sizeof(int),
                          cudaMemcpyDeviceToHost, ctx->stream));
  return PYRO_OK;
}

// After the stream synchronised: a dependency wait that gave up turns into
// PYRO_ERR_TIMEOUT, and the status word is cleared.
int wave_status_result(pyro_ctx* ctx) {
  if (!ctx->d_wave_status || *ctx->h_wave_status == 0) return PYRO_OK;
  *ctx->h_wave_status = 0;
  PYRO_CK(cudaMemset(ctx->d_wave_status, 0, sizeof(int)));
  return fail(ctx, PYRO_ERR_TIMEOUT,
              "work-queue cycle kernel: a dependency wait ran out; the spins are partly updated");
}

// Synchronous check of the status word (for calls that synchronise anyway).
int check_wave_status(pyro_ctx* ctx) {
  if (!ctx->d_wave_status) return PYRO_OK;
  int rc = queue_wave_status(ctx);
  if (rc) return rc;
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return wave_status_result(ctx);
}

// n_metro Metropolis + n_or over-relaxation sweeps of every system, and (if
// with_obs) the observables partials and their per-replica sums.
// Per-pass J1 kernels in replica groups: every sweep of one group of
// rep_group replicas before the next group, so that a group's spins stay in
// L2 across its passes. Same updates, same order within each replica.
// Grouped schedule: J1 systems in groups of rep_group replicas (per-pass J1
// kernels) and the other systems in groups of about gen_group_mb MB (generic
// kernel), each group running all its sweeps before the next group, the
// groups dealt round-robin to `chains` streams that fork from and join back
// into the context stream (parallel branches of a captured graph), so a
// group's spins stay in L2 across its passes and one chain's launch gaps are
// filled by another's kernels. Same updates, same order within each replica.
// With with_obs, the FP64 energy partials of an isotropic J1 group are
// computed on its chain right after its last pass, while its spins are still
// in L2 (instead of one lattice-wide read from HBM after all groups).
// n_tet learned tetrahedron sweeps of a J1-only group follow its plain
// sweeps on the same chain (before its energy partials).
int queue_grouped(pyro_ctx* ctx, int n_metro, int n_or, bool j1_grouped, bool gen_grouped,
                  bool with_obs, int n_tet) {
  const int chains = std::max(1, std::min(ctx->n_chains, kMaxChains));
  if (chains > 1) {
    for (int c = 0; c < chains; ++c) {
      if (!ctx->chain_stream[c])
        PYRO_CK(cudaStreamCreateWithFlags(&ctx->chain_stream[c], cudaStreamNonBlocking));
      if (!ctx->chain_event[c])
        PYRO_CK(cudaEventCreateWithFlags(&ctx->chain_event[c], cudaEventDisableTiming));
    }
    if (!ctx->fork_event) PYRO_CK(cudaEventCreateWithFlags(&ctx->fork_event, cudaEventDisableTiming));
    PYRO_CK(cudaEventRecord(ctx->fork_event, ctx->stream));
    for (int c = 0; c < chains; ++c) PYRO_CK(cudaStreamWaitEvent(ctx->chain_stream[c], ctx->fork_event, 0));
  }
  // staggered start: each odd chain c waits for chain c - 1's first
  // `stagger` passes (recorded when chain c - 1 has queued them)
  // (at most one group's passes: chain c - 1's first group is queued before
  // chain c's, so the event is recorded before it is waited on)
  const int stagger = chains > 1 ? std::min(ctx->chain_stagger, 4 * (n_metro + n_or)) : 0;
  int chain_passes[kMaxChains] = {};
  bool chain_started[kMaxChains] = {};
  auto before_pass = [&](int c) -> int {
    if (stagger > 0 && (c & 1) && !chain_started[c])
      PYRO_CK(cudaStreamWaitEvent(ctx->chain_stream[c], ctx->stagger_event[c - 1], 0));
    chain_started[c] = true;
    return PYRO_OK;
  };
  auto after_pass = [&](int c) -> int {
    if (stagger > 0 && !(c & 1) && c + 1 < chains && ++chain_passes[c] == stagger)
      PYRO_CK(cudaEventRecord(ctx->stagger_event[c], ctx->chain_stream[c]));
    return PYRO_OK;
  };
  if (stagger > 0)
    for (int c = 0; c + 1 < chains; c += 2)
      if (!ctx->stagger_event[c])
        PYRO_CK(cudaEventCreateWithFlags(&ctx->stagger_event[c], cudaEventDisableTiming));
  int gi = 0;
  if (j1_grouped) {
    for (int si : ctx->j1_sys) {
      const SysDev& s = ctx->sys[si];
      for (int r0 = 0; r0 < s.n_rep; r0 += ctx->rep_group, ++gi) {
        cudaStream_t st = chains > 1 ? ctx->chain_stream[gi % chains] : ctx->stream;
        const int cnt = std::min(ctx->rep_group, s.n_rep - r0);
        J1ObsParams jp;
        jp.spins = ctx->d_spins + s.spin_off + (long long)r0 * 16 * s.L3;
        jp.L = s.L;
        jp.L3 = s.L3;
        jp.n_rep = cnt;
        jp.rcpL = 1.0f / (float)s.L;
        jp.J1 = s.J64[0];
        jp.partials = ctx->d_partials;
        jp.partial_begin = ctx->obs_segs[si].partial_begin + r0 * j1_blocks_per_replica(s.L3);
        jp.pdl = ctx->pdl;
        // the group's energy partials from its last pass when that pass runs
        // in the cell form (isotropic J1, no learned sweeps after it)
        const int n_sw = n_metro + n_or;
        const bool last_metro = n_or == 0;
        const bool fuse = ctx->fused_obs && with_obs && s.exch < 0 && n_tet == 0 && n_sw > 0 &&
                          !(last_metro ? ctx->j1_metro_site_mode : ctx->j1_or_site_mode);
        const int ch = chains > 1 ? (gi % chains) : 0;
        for (int k = 0; k < n_sw; ++k) {
          const bool metro = k < n_metro;
          for (int colour = 0; colour < 4; ++colour) {
            J1PassParams p = j1_params(ctx, si, (unsigned long long)k);
            p.spins += (long long)r0 * 16 * s.L3;
            p.n_rep = cnt;
            p.rep_global += r0;
            p.rep_key += r0;
            if (int rc = before_pass(ch)) return rc;
            if (fuse && k == n_sw - 1 && colour == 3)
              launch_j1_last_pass(p, jp, metro, st);
            else
              launch_j1_pass(p, colour, metro,
                             metro ? ctx->j1_metro_site_mode : ctx->j1_or_site_mode, st);
            PYRO_CK_LAUNCH();
            if (int rc = after_pass(ch)) return rc;
          }
        }
        if (n_tet > 0) {
          const int rc = queue_tet_group(ctx, si, r0, cnt, n_tet, st);
          if (rc) return rc;
        }
        if (with_obs && s.exch < 0 && !fuse) {
          launch_j1_observables(jp, st);
          PYRO_CK_LAUNCH();
        }
      }
    }
  }
  if (gen_grouped) {
    for (const auto& G : ctx->gen_groups) {
      cudaStream_t st = chains > 1 ? ctx->chain_stream[gi % chains] : ctx->stream;
      ++gi;
      for (int k = 0; k < n_metro + n_or; ++k) {
        const bool metro = k < n_metro;
        for (int pass = 0; pass < ctx->n_passes; ++pass) {
          if (G.pass_blocks[pass] == 0) continue;
          PassParams p = pass_params(ctx, pass);
          p.segs = G.d_pass_segs[pass];
          p.nseg = (int)G.pass_segs[pass].size();
          p.sweep_off = (unsigned long long)k;
          if (ctx->far_kernel && G.all16[pass])
            launch_far_pass(p, pass, G.pass_blocks[pass], metro, st);
          else
            launch_colour_pass(p, ctx->tab, G.pass_blocks[pass], metro, false, st);
          PYRO_CK_LAUNCH();
        }
      }
    }
  }
  if (chains > 1) {
    for (int c = 0; c < chains; ++c) {
      PYRO_CK(cudaEventRecord(ctx->chain_event[c], ctx->chain_stream[c]));
      PYRO_CK(cudaStreamWaitEvent(ctx->stream, ctx->chain_event[c], 0));
    }
  }
  return PYRO_OK;
}

// Generic (non-J1-path) sweeps of every system, ungrouped.
int queue_generic_sweeps(pyro_ctx* ctx, int n_metro, int n_or) {
  int rc = PYRO_OK;
  for (int i = 0; i < n_metro && rc == PYRO_OK; ++i) rc = queue_sweep(ctx, true, i, true);
  for (int i = 0; i < n_or && rc == PYRO_OK; ++i) rc = queue_sweep(ctx, false, n_metro + i, true);
  return rc;
}

// The J1 systems run per-pass kernels in replica groups.
bool j1_grouped_path(const pyro_ctx* ctx) {
  return !use_cycle_kernel(ctx) && ctx->rep_group > 0 && ctx->use_j1_kernel &&
         !ctx->j1_sys.empty();
}

// n_tet > 0 only on the J1 grouped path with every J1-only system on it
// (tet_in_groups): each group's learned sweeps follow its plain sweeps.
int queue_cycle_body(pyro_ctx* ctx, int n_metro, int n_or, bool with_obs, int n_tet = 0) {
  int rc = check_cluster(ctx);
  if (rc) return rc;
  const bool skew = use_skew_kernel(ctx, n_metro, n_or, n_tet);
  const bool j1_wave = use_wave_kernel(ctx, n_metro, n_or, n_tet);
  const bool gen_wave = use_gen_wave(ctx, n_metro, n_or, n_tet);
  if (skew || j1_wave || gen_wave) {
    // the 16-colour systems in their work-queue launch, or the other systems
    // on their usual kernels; then the J1 systems' launches
    if (gen_wave)
      rc = queue_gen_wave(ctx, n_metro, n_or);
    else if (!ctx->gen_groups.empty())
      rc = queue_grouped(ctx, n_metro, n_or, false, true, with_obs, 0);
    else
      rc = queue_generic_sweeps(ctx, n_metro, n_or);
    if (rc == PYRO_OK && (skew || j1_wave))
      rc = skew ? queue_skew(ctx, n_metro, n_or, with_obs) : queue_wave(ctx, n_metro, n_or, with_obs);
    else if (rc == PYRO_OK && !ctx->j1_sys.empty())
      rc = PYRO_ERR_STATE;  // J1 systems take the J1 work queue whenever the 16-colour ones do
    if (rc == PYRO_OK && with_obs) rc = queue_observables(ctx, /*skip_j1=*/skew || j1_wave);
    return rc;
  }
  const bool cyc = use_cycle_kernel(ctx);
  const bool j1_grouped = j1_grouped_path(ctx);
  const bool gen_grouped = !ctx->gen_groups.empty();
  if (n_tet > 0 && !j1_grouped) return fail(ctx, PYRO_ERR_STATE, "learned sweeps need replica groups");
  if (j1_grouped || gen_grouped) {
    rc = queue_grouped(ctx, n_metro, n_or, j1_grouped, gen_grouped, with_obs, n_tet);
    if (rc) return rc;
    if (n_tet > 0) {
      tet_advance(ctx, n_tet);
      PYRO_CK_LAUNCH();
    }
    if (!gen_grouped) rc = queue_generic_sweeps(ctx, n_metro, n_or);
    if (rc) return rc;
    if (!j1_grouped) {  // J1 systems ungrouped: their per-pass kernels or the cluster kernel
      if (cyc) {
        for (int si : ctx->obs_j1) {
          J1CycleParams cp;
          cp.pass = j1_params(ctx, si, 0);
          cp.n_metro = n_metro;
          cp.n_or = n_or;
          cp.cluster_size = ctx->cluster_size;
          cp.J1_64 = ctx->sys[si].J64[0];
          cp.partials = with_obs ? ctx->d_partials : nullptr;
          cp.partial_begin = ctx->obs_segs[si].partial_begin;
          PYRO_CK(launch_j1_cycle(cp, ctx->stream));
        }
      } else {
        for (int k = 0; k < n_metro + n_or; ++k)
          for (int pass = 0; pass < ctx->n_passes; ++pass)
            for (const auto& sc : ctx->pass_j1[pass]) {
              const bool metro = k < n_metro;
              launch_j1_pass(j1_params(ctx, sc.first, (unsigned long long)k), sc.second, metro,
                             metro ? ctx->j1_metro_site_mode : ctx->j1_or_site_mode, ctx->stream);
              PYRO_CK_LAUNCH();
            }
      }
    }
    // J1 observables were queued per group when grouped
    if (with_obs) rc = queue_observables(ctx, (cyc && !j1_grouped) || j1_grouped);
    return rc;
  }
  if (cyc) {
    for (int si : ctx->obs_j1) {
      J1CycleParams cp;
      cp.pass = j1_params(ctx, si, 0);
      cp.n_metro = n_metro;
      cp.n_or = n_or;
      cp.cluster_size = ctx->cluster_size;
      cp.J1_64 = ctx->sys[si].J64[0];
      cp.partials = with_obs ? ctx->d_partials : nullptr;
      cp.partial_begin = ctx->obs_segs[si].partial_begin;
      PYRO_CK(launch_j1_cycle(cp, ctx->stream));
    }
  }
  for (int i = 0; i < n_metro && rc == PYRO_OK; ++i) rc = queue_sweep(ctx, true, i, cyc);
  for (int i = 0; i < n_or && rc == PYRO_OK; ++i) rc = queue_sweep(ctx, false, n_metro + i, cyc);
  if (rc) return rc;
  if (with_obs) rc = queue_observables(ctx, cyc);
  return rc;
}

ExchangeParams exchange_params(pyro_ctx* ctx) {
  ExchangeParams x;
  std::memset(&x, 0, sizeof(x));
  x.sys = ctx->d_sys;
  x.n_sys = (int)ctx->sys.size();
  x.sys_first = 0;
  x.energy = ctx->d_energy;
  x.energy_is_global = 0;
  x.beta64 = ctx->d_beta64;
  x.temp_of_rep = ctx->d_temp_of_rep;
  x.rep_of_temp = ctx->d_rep_of_temp;
  x.swap_count = ctx->d_swap_count;
  x.swap_acc = ctx->d_swap_acc;
  x.swap_try = ctx->d_swap_try;
  x.last_accepted = ctx->d_last_accepted;
  x.parity = -1;
  x.seed_lo = (uint32_t)(ctx->seed & 0xffffffffu);
  x.seed_hi = (uint32_t)(ctx->seed >> 32);
  x.history = nullptr;
  x.history_count = ctx->d_history_count;
  x.history_cap = ctx->history_cap;
  x.total_temps = ctx->total_temps;
  x.sweep_ctr = nullptr;
  x.sweep_advance = 0;
  x.do_swap = 1;
  return x;
}

int max_pairs(const pyro_ctx* ctx) {
  int m = 1;
  for (const auto& s : ctx->sys) m = std::max(m, (s.n_temp + 1) / 2);
  return m;
}

bool sharded(const pyro_ctx* ctx) {
  for (const auto& s : ctx->sys)
    if (s.n_rep != s.n_temp) return true;
  return false;
}

void free_all(pyro_ctx* c) {
  tet_free(c);
  for (auto& g : c->gen_groups)
    for (auto* p : g.d_pass_segs)
      if (p) cudaFree(p);
  c->gen_groups.clear();
  for (int i = 0; i < kMaxChains; ++i) {
    if (c->chain_stream[i]) cudaStreamDestroy(c->chain_stream[i]);
    if (c->chain_event[i]) cudaEventDestroy(c->chain_event[i]);
    if (c->stagger_event[i]) cudaEventDestroy(c->stagger_event[i]);
    c->chain_stream[i] = nullptr;
    c->chain_event[i] = nullptr;
    c->stagger_event[i] = nullptr;
  }
  if (c->fork_event) cudaEventDestroy(c->fork_event);
  c->fork_event = nullptr;
  for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
  c->graphs.clear();
  c->graph_kernels.clear();
  void* ptrs[] = {c->d_sys,         c->d_spins,        c->d_temp_of_rep, c->d_rep_of_temp,
                  c->d_beta,        c->d_beta64,       c->d_cosmax,      c->d_accepted,
                  c->d_swap_acc,    c->d_swap_try,     c->d_swap_count,  c->d_last_accepted,
                  c->d_energy,      c->d_mag,          c->d_rep_sys,     c->d_rep_local,
                  c->d_obs_segs,    c->d_partials,     c->d_sweep,       c->d_scratch_u64,
                  c->d_history,     c->d_history_count, c->d_obs_generic,
                  c->d_sq_s1,       c->d_sq_s2,        c->d_sq_tw,
                  c->d_sq_out,      c->d_exch,         c->d_submag,      c->d_order,
                  c->d_wave,        c->d_wave_status,  c->d_snap,        c->d_snap_temp_of_rep,
                  c->d_snap_rep_of_temp, c->d_snap_energy, c->d_snap_mag,
                  c->d_gwave_units, c->d_gwave_groups, c->d_gwave, c->d_gwave_chunk_unit};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (c->snap_stream) cudaStreamDestroy(c->snap_stream);
  if (c->snap_start) cudaEventDestroy(c->snap_start);
  if (c->snap_done) cudaEventDestroy(c->snap_done);
  c->snap_stream = nullptr;
  c->snap_start = c->snap_done = nullptr;
  c->d_snap = nullptr;
  c->snap_taken = false;
  c->measure_snapshot = 0;
  if (c->h_wave_status) cudaFreeHost(c->h_wave_status);
  c->h_wave_status = nullptr;
  c->d_wave = nullptr;
  c->d_wave_status = nullptr;
  c->wave_words = 0;
  c->d_gwave_units = nullptr;
  c->d_gwave_groups = nullptr;
  c->d_gwave = nullptr;
  c->d_gwave_chunk_unit = nullptr;
  c->gwave_units_cap = c->gwave_groups_cap = c->gwave_words = c->gwave_chunk_cap = 0;
  for (auto* p : c->d_pass_segs)
    if (p) cudaFree(p);
  c->d_pass_segs.clear();
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  c->stream = nullptr;
}

// Pass p runs colour p of 16-colour systems, and colour p/4 of 4-colour
// systems when p % 4 == 0 (every pass if all systems use 4 colours).
// J1-only systems go to the specialised kernel unless use_j1_kernel is off.
int build_schedule(pyro_ctx* ctx) {
  for (auto* p : ctx->d_pass_segs)
    if (p) cudaFree(p);
  ctx->d_pass_segs.clear();
  if (ctx->d_obs_segs) cudaFree(ctx->d_obs_segs);
  if (ctx->d_obs_generic) cudaFree(ctx->d_obs_generic);
  ctx->d_obs_segs = ctx->d_obs_generic = nullptr;
  ctx->n_passes = 4;
  for (const auto& s : ctx->sys) ctx->n_passes = std::max(ctx->n_passes, s.n_colours);
  ctx->pass_segs.assign(ctx->n_passes, {});
  ctx->pass_j1.assign(ctx->n_passes, {});
  ctx->pass_blocks.assign(ctx->n_passes, 0);
  auto j1_path = [&](const SysDev& s) { return ctx->use_j1_kernel && j1_sweepable(s); };
  for (int pass = 0; pass < ctx->n_passes; ++pass) {
    int blocks = 0;
    for (int i = 0; i < (int)ctx->sys.size(); ++i) {
      const SysDev& s = ctx->sys[i];
      int colour = -1;
      if (s.n_colours == ctx->n_passes) colour = pass;
      else if (pass % 4 == 0) colour = pass / 4;
      if (colour < 0) continue;
      if (j1_path(s)) {
        ctx->pass_j1[pass].push_back({i, colour});
        continue;
      }
      PassSeg g;
      g.sys = i;
      g.colour = colour;
      g.blocks_per_rep = (s.units_per_colour + kPassThreads - 1) / kPassThreads;
      g.block_begin = blocks;
      g.rep_begin = 0;
      blocks += g.blocks_per_rep * s.n_rep;
      ctx->pass_segs[pass].push_back(g);
    }
    ctx->pass_blocks[pass] = blocks;
  }
  ctx->pass_all16.assign(ctx->n_passes, 1);
  for (int pass = 0; pass < ctx->n_passes; ++pass)
    for (const PassSeg& g : ctx->pass_segs[pass])
      if (ctx->sys[g.sys].n_colours != 16 || ctx->sys[g.sys].exch >= 0) ctx->pass_all16[pass] = 0;
  ctx->obs_segs.clear();
  ctx->obs_generic.clear();
  ctx->obs_j1.clear();
  ctx->j1_sys.clear();
  int partial = 0, gblocks = 0;
  for (int i = 0; i < (int)ctx->sys.size(); ++i) {
    const SysDev& s = ctx->sys[i];
    ObsSeg g;
    g.sys = i;
    g.partial_begin = partial;
    g.block_begin = partial;
    if (j1_path(s)) ctx->j1_sys.push_back(i);
    if (j1_path(s) && s.exch < 0) {
      g.blocks_per_rep = j1_blocks_per_replica(s.L3);
      ctx->obs_j1.push_back(i);
    } else {
      g.blocks_per_rep = (16 * s.L3 + kObsThreads * kObsSitesPerThread - 1) /
                         (kObsThreads * kObsSitesPerThread);
      ObsSeg gg = g;
      gg.block_begin = gblocks;
      gblocks += g.blocks_per_rep * s.n_rep;
      ctx->obs_generic.push_back(gg);
    }
    partial += g.blocks_per_rep * s.n_rep;
    ctx->obs_segs.push_back(g);
  }
  ctx->obs_generic_blocks = gblocks;
  if (partial > ctx->partials_cap) return fail(ctx, PYRO_ERR_STATE, "partials buffer too small");
  ctx->d_pass_segs.assign(ctx->n_passes, nullptr);
  PYRO_CK(alloc(&ctx->d_obs_segs, ctx->obs_segs.size()));
  PYRO_CK(cudaMemcpy(ctx->d_obs_segs, ctx->obs_segs.data(), sizeof(ObsSeg) * ctx->obs_segs.size(),
                     cudaMemcpyHostToDevice));
  PYRO_CK(alloc(&ctx->d_obs_generic, ctx->obs_generic.size()));
  if (!ctx->obs_generic.empty())
    PYRO_CK(cudaMemcpy(ctx->d_obs_generic, ctx->obs_generic.data(),
                       sizeof(ObsSeg) * ctx->obs_generic.size(), cudaMemcpyHostToDevice));
  for (int pass = 0; pass < ctx->n_passes; ++pass) {
    PYRO_CK(alloc(&ctx->d_pass_segs[pass], ctx->pass_segs[pass].size()));
    if (!ctx->pass_segs[pass].empty())
      PYRO_CK(cudaMemcpy(ctx->d_pass_segs[pass], ctx->pass_segs[pass].data(),
                         sizeof(PassSeg) * ctx->pass_segs[pass].size(), cudaMemcpyHostToDevice));
  }
  // Replica groups of the generic path: consecutive (system, replica) ranges
  // of about gen_group_mb MB each; every group gets its own segment list per
  // pass, so all its sweeps can run while its spins stay in L2.
  for (auto& g : ctx->gen_groups)
    for (auto* p : g.d_pass_segs)
      if (p) cudaFree(p);
  ctx->gen_groups.clear();
  if (ctx->gen_group_mb > 0) {
    const double budget = (double)ctx->gen_group_mb * 1048576.0;
    struct Range { int sys, r0, n; };
    std::vector<std::vector<Range>> groups(1);
    double bytes = 0.0;
    for (int i = 0; i < (int)ctx->sys.size(); ++i) {
      const SysDev& s = ctx->sys[i];
      if (j1_path(s)) continue;
      const double per_rep = 16.0 * 16.0 * s.L3;
      for (int r = 0; r < s.n_rep; ++r) {
        if (bytes > 0.0 && bytes + per_rep > budget) {
          groups.emplace_back();
          bytes = 0.0;
        }
        auto& cur = groups.back();
        if (!cur.empty() && cur.back().sys == i && cur.back().r0 + cur.back().n == r) ++cur.back().n;
        else cur.push_back({i, r, 1});
        bytes += per_rep;
      }
    }
    if (groups.back().empty()) groups.pop_back();
    for (const auto& gr : groups) {
      pyro_ctx::GenGroup G;
      G.pass_segs.assign(ctx->n_passes, {});
      G.pass_blocks.assign(ctx->n_passes, 0);
      G.d_pass_segs.assign(ctx->n_passes, nullptr);
      G.all16.assign(ctx->n_passes, 1);
      for (int pass = 0; pass < ctx->n_passes; ++pass) {
        int blocks = 0;
        for (const Range& rg : gr) {
          const SysDev& s = ctx->sys[rg.sys];
          int colour = -1;
          if (s.n_colours == ctx->n_passes) colour = pass;
          else if (pass % 4 == 0) colour = pass / 4;
          if (colour < 0) continue;
          PassSeg g;
          g.sys = rg.sys;
          g.colour = colour;
          g.blocks_per_rep = (s.units_per_colour + kPassThreads - 1) / kPassThreads;
          g.block_begin = blocks;
          g.rep_begin = rg.r0;
          blocks += g.blocks_per_rep * rg.n;
          G.pass_segs[pass].push_back(g);
          if (s.n_colours != 16 || s.exch >= 0) G.all16[pass] = 0;
        }
        G.pass_blocks[pass] = blocks;
        PYRO_CK(alloc(&G.d_pass_segs[pass], G.pass_segs[pass].size()));
        if (!G.pass_segs[pass].empty())
          PYRO_CK(cudaMemcpy(G.d_pass_segs[pass], G.pass_segs[pass].data(),
                             sizeof(PassSeg) * G.pass_segs[pass].size(), cudaMemcpyHostToDevice));
      }
      ctx->gen_groups.push_back(std::move(G));
    }
  }
  return PYRO_OK;
}

int validate(const pyro_config* cfg, std::string* why) {
  if (!cfg || cfg->n_systems <= 0 || !cfg->systems) {
    *why = "config: need n_systems >= 1 and a systems array";
    return PYRO_ERR_ARG;
  }
  for (int i = 0; i < cfg->n_systems; ++i) {
    const pyro_system_desc& d = cfg->systems[i];
    char buf[160];
    if (d.L < 2 || d.L > 256) {
      snprintf(buf, sizeof buf, "system %d: L=%d out of range [2, 256]", i, d.L);
      *why = buf;
      return PYRO_ERR_ARG;
    }
    if (d.n_temperatures < 1 || d.n_replicas < 1 || d.replica_offset < 0 ||
        d.replica_offset + d.n_replicas > d.n_temperatures) {
      snprintf(buf, sizeof buf, "system %d: replicas [%d, %d) not inside the ladder of %d", i,
               d.replica_offset, d.replica_offset + d.n_replicas, d.n_temperatures);
      *why = buf;
      return PYRO_ERR_ARG;
    }
    if (!d.temperatures) {
      snprintf(buf, sizeof buf, "system %d: temperatures is NULL", i);
      *why = buf;
      return PYRO_ERR_ARG;
    }
    for (int t = 0; t < d.n_temperatures; ++t) {
      const double T = d.temperatures[t];
      if (!(T > 0.0) || !std::isfinite(T) || (t > 0 && !(T > d.temperatures[t - 1]))) {
        snprintf(buf, sizeof buf, "system %d: temperatures must be finite, > 0, increasing", i);
        *why = buf;
        return PYRO_ERR_ARG;
      }
    }
    const double J[4] = {d.J1, d.J2, d.J3, d.J3b};
    for (double j : J)
      if (!std::isfinite(j)) {
        snprintf(buf, sizeof buf, "system %d: couplings must be finite", i);
        *why = buf;
        return PYRO_ERR_ARG;
      }
    // A 16-colour class holds sites that are a lattice vector apart; with
    // L = 2 the J2/J3 shells would reach a periodic image of the same site.
    if ((d.J2 != 0.0 || d.J3 != 0.0 || d.J3b != 0.0) && d.L < 3) {
      snprintf(buf, sizeof buf, "system %d: J2/J3 need L >= 3", i);
      *why = buf;
      return PYRO_ERR_ARG;
    }
  }
  if (cfg->renorm_every < 0) {
    *why = "renorm_every must be >= 0";
    return PYRO_ERR_ARG;
  }
  return PYRO_OK;
}

}  // namespace

namespace pyro {
int rebuild_schedule(pyro_ctx* ctx) {
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_kernels.clear();
  return build_schedule(ctx);
}
}  // namespace pyro

extern "C" {

int pyro_version(void) { return 1; }

int pyro_neighbour_table(int site, int* out120) {
  if (site < 0 || site >= kSitesPerCell || !out120) return PYRO_ERR_ARG;
  NbrTable tab;
  if (!build_neighbour_table(&tab)) return PYRO_ERR_STATE;
  for (int k = 0; k < kMaxNbr; ++k) {
    const NbrEntry e = tab.e[site][k];
    out120[4 * k] = e.dx;
    out120[4 * k + 1] = e.dy;
    out120[4 * k + 2] = e.dz;
    out120[4 * k + 3] = e.t;
  }
  return PYRO_OK;
}

const char* pyro_last_error(const pyro_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int pyro_create(const pyro_config* cfg, pyro_ctx** out) {
  if (!out) return PYRO_ERR_ARG;
  *out = nullptr;
  std::string why;
  int rc = validate(cfg, &why);
  if (rc != PYRO_OK) {
    fprintf(stderr, "pyro_create: %s\n", why.c_str());
    return rc;
  }
  pyro_ctx* ctx = new pyro_ctx();
  ctx->device = cfg->device;
  ctx->seed = cfg->seed;
  ctx->renorm_every = cfg->renorm_every;
  if (!build_neighbour_table(&ctx->tab)) {
    delete ctx;
    return PYRO_ERR_STATE;
  }
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) {
    fprintf(stderr, "pyro_create: cudaSetDevice(%d): %s\n", cfg->device, cudaGetErrorString(e));
    delete ctx;
    return PYRO_ERR_CUDA;
  }
  auto bail = [&](int code) {
    fprintf(stderr, "pyro_create: %s\n", ctx->err.c_str());
    free_all(ctx);
    delete ctx;
    return code;
  };
#define CREATE_CK(call)                                                              \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
      return bail(e_ == cudaErrorMemoryAllocation ? PYRO_ERR_NOMEM : PYRO_ERR_CUDA); \
    }                                                                                \
  } while (0)
  CREATE_CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  ctx->own_stream = true;

  // Systems, temperature slots and replica maps.
  long long spin_off = 0;
  int temp_base = 0, rep_ctx = 0;
  int max_colours = 4;
  std::vector<int> h_temp_of_rep, h_rep_of_temp;
  std::vector<float> h_beta, h_cos;
  std::vector<double> h_beta64;
  std::vector<int> h_rep_sys, h_rep_local;
  for (int i = 0; i < cfg->n_systems; ++i) {
    const pyro_system_desc& d = cfg->systems[i];
    SysDev s;
    std::memset(&s, 0, sizeof s);
    s.L = d.L;
    s.L3 = d.L * d.L * d.L;
    const bool far = d.J2 != 0.0 || d.J3 != 0.0 || d.J3b != 0.0;
    s.n_colours = far ? 16 : 4;
    max_colours = std::max(max_colours, s.n_colours);
    s.units_per_colour = 16 * s.L3 / s.n_colours;
    s.n_rep = d.n_replicas;
    s.rep_global = d.replica_offset;
    s.rep_key = temp_base + d.replica_offset;
    s.swap_key = i;
    s.rep_ctx_base = rep_ctx;
    s.temp_base = temp_base;
    s.n_temp = d.n_temperatures;
    s.spin_off = spin_off;
    s.rcpL = 1.0f / (float)d.L;
    s.J1 = (float)d.J1;
    s.J2 = (float)d.J2;
    s.J3a = (float)d.J3;
    s.J3b = (float)d.J3b;
    s.J64[0] = d.J1;
    s.J64[1] = d.J2;
    s.J64[2] = d.J3;
    s.J64[3] = d.J3b;
    s.shells = (d.J1 != 0.0 ? 1 : 0) | (d.J2 != 0.0 ? 2 : 0) | (d.J3 != 0.0 ? 4 : 0) |
               (d.J3b != 0.0 ? 8 : 0);
    s.exch = -1;
    ctx->sys.push_back(s);
    ctx->ladders.emplace_back(d.temperatures, d.temperatures + d.n_temperatures);
    for (int t = 0; t < d.n_temperatures; ++t) {
      h_temp_of_rep.push_back(t);
      h_rep_of_temp.push_back(t);
      h_beta.push_back((float)(1.0 / d.temperatures[t]));
      h_beta64.push_back(1.0 / d.temperatures[t]);
      h_cos.push_back(-1.0f);
    }
    for (int r = 0; r < d.n_replicas; ++r) {
      h_rep_sys.push_back(i);
      h_rep_local.push_back(r);
    }
    spin_off += (long long)d.n_replicas * 16 * s.L3;
    temp_base += d.n_temperatures;
    rep_ctx += d.n_replicas;
  }
  ctx->total_temps = temp_base;
  ctx->total_reps = rep_ctx;
  ctx->n_spins = spin_off;
  ctx->n_passes = max_colours;

  ctx->partials_cap = 0;
  for (const auto& sd : ctx->sys)
    ctx->partials_cap += sd.n_rep * ((16 * sd.L3 + kObsThreads * kObsSitesPerThread - 1) /
                                     (kObsThreads * kObsSitesPerThread));
  const int nS = (int)ctx->sys.size(), nT = ctx->total_temps, nR = ctx->total_reps;
  CREATE_CK(alloc(&ctx->d_sys, nS));
  CREATE_CK(alloc(&ctx->d_spins, ctx->n_spins));
  CREATE_CK(alloc(&ctx->d_temp_of_rep, nT));
  CREATE_CK(alloc(&ctx->d_rep_of_temp, nT));
  CREATE_CK(alloc(&ctx->d_beta, nT));
  CREATE_CK(alloc(&ctx->d_beta64, nT));
  CREATE_CK(alloc(&ctx->d_cosmax, nT));
  CREATE_CK(alloc(&ctx->d_accepted, nT));
  CREATE_CK(alloc(&ctx->d_swap_acc, nT));
  CREATE_CK(alloc(&ctx->d_swap_try, nT));
  CREATE_CK(alloc(&ctx->d_swap_count, nS));
  CREATE_CK(alloc(&ctx->d_last_accepted, nS));
  CREATE_CK(alloc(&ctx->d_energy, nR));
  CREATE_CK(alloc(&ctx->d_mag, 3 * nR));
  CREATE_CK(alloc(&ctx->d_rep_sys, nR));
  CREATE_CK(alloc(&ctx->d_rep_local, nR));
  CREATE_CK(alloc(&ctx->d_partials, ctx->partials_cap));
  CREATE_CK(alloc(&ctx->d_sweep, 1));
  CREATE_CK(alloc(&ctx->d_scratch_u64, 4));
  CREATE_CK(alloc(&ctx->d_history_count, 1));
  CREATE_CK(cudaMemcpy(ctx->d_sys, ctx->sys.data(), sizeof(SysDev) * nS, cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemcpy(ctx->d_temp_of_rep, h_temp_of_rep.data(), sizeof(int) * nT,
                       cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemcpy(ctx->d_rep_of_temp, h_rep_of_temp.data(), sizeof(int) * nT,
                       cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemcpy(ctx->d_beta, h_beta.data(), sizeof(float) * nT, cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemcpy(ctx->d_beta64, h_beta64.data(), sizeof(double) * nT, cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemcpy(ctx->d_cosmax, h_cos.data(), sizeof(float) * nT, cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemcpy(ctx->d_rep_sys, h_rep_sys.data(), sizeof(int) * nR, cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemcpy(ctx->d_rep_local, h_rep_local.data(), sizeof(int) * nR,
                       cudaMemcpyHostToDevice));
  CREATE_CK(cudaMemset(ctx->d_accepted, 0, sizeof(unsigned long long) * nT));
  CREATE_CK(cudaMemset(ctx->d_swap_acc, 0, sizeof(unsigned long long) * nT));
  CREATE_CK(cudaMemset(ctx->d_swap_try, 0, sizeof(unsigned long long) * nT));
  CREATE_CK(cudaMemset(ctx->d_swap_count, 0, sizeof(unsigned long long) * nS));
  CREATE_CK(cudaMemset(ctx->d_last_accepted, 0, sizeof(int) * nS));
  CREATE_CK(cudaMemset(ctx->d_sweep, 0, sizeof(unsigned long long)));
  CREATE_CK(cudaMemset(ctx->d_history_count, 0, sizeof(unsigned long long)));
  CREATE_CK(cudaMemset(ctx->d_spins, 0, sizeof(float4) * ctx->n_spins));
#undef CREATE_CK
  rc = build_schedule(ctx);
  if (rc != PYRO_OK) return bail(rc);
  *out = ctx;
  return PYRO_OK;
}

int pyro_destroy(pyro_ctx* ctx) {
  if (!ctx) return PYRO_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
  return PYRO_OK;
}

int pyro_set_stream(pyro_ctx* ctx, void* cuda_stream) {
  if (!ctx) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_kernels.clear();
  if (ctx->own_stream && ctx->stream) {
    PYRO_CK(cudaStreamSynchronize(ctx->stream));
    cudaStreamDestroy(ctx->stream);
  }
  ctx->stream = (cudaStream_t)cuda_stream;
  ctx->own_stream = false;
  return PYRO_OK;
}

int pyro_set_option(pyro_ctx* ctx, int option, int value) {
  if (!ctx) return PYRO_ERR_ARG;
  if (option == PYRO_OPT_MEASURE_SNAPSHOT) {  // no kernel schedule depends on it
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "measure snapshot option is 0 or 1");
    if (value && !ctx->snap_taken) return fail(ctx, PYRO_ERR_STATE, "no snapshot taken yet");
    ctx->measure_snapshot = value;
    return PYRO_OK;
  }
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  if (option == PYRO_OPT_J1_KERNEL) {
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "J1 kernel option is 0 or 1");
    ctx->use_j1_kernel = value == 1;
  } else if (option == PYRO_OPT_FAR_KERNEL) {
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "far kernel option is 0 or 1");
    ctx->far_kernel = value;
  } else if (option == PYRO_OPT_PDL) {
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "PDL option is 0 or 1");
    ctx->pdl = value;
  } else if (option == PYRO_OPT_FUSED_OBS) {
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "fused observables option is 0 or 1");
    ctx->fused_obs = value;
  } else if (option == PYRO_OPT_TET_GROUPED) {
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "tet grouped option is 0 or 1");
    ctx->tet_grouped = value;
  } else if (option == PYRO_OPT_GROUP_MB) {
    if (value < 0) return fail(ctx, PYRO_ERR_ARG, "group size in MB must be >= 0");
    ctx->gen_group_mb = value;
  } else if (option == PYRO_OPT_CHAINS) {
    if (value < 1 || value > kMaxChains) return fail(ctx, PYRO_ERR_ARG, "chains is 1..8");
    ctx->n_chains = value;
  } else if (option == PYRO_OPT_REPLICA_GROUP) {
    if (value < 0) return fail(ctx, PYRO_ERR_ARG, "replica group must be >= 0");
    ctx->rep_group = value;
  } else if (option == PYRO_OPT_SMEM_KERNEL) {
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "smem kernel option is 0 or 1");
    ctx->smem_kernel = value;
  } else if (option == PYRO_OPT_J1_SITE_MODE) {
    if (value < 0 || value > 3) return fail(ctx, PYRO_ERR_ARG, "J1 site mode is 0..3");
    ctx->j1_metro_site_mode = (value & 1) != 0;
    ctx->j1_or_site_mode = (value & 2) != 0;
  } else if (option == PYRO_OPT_CYCLE_KERNEL) {
    if (value < 0 || value > 3) return fail(ctx, PYRO_ERR_ARG, "cycle kernel option is 0..3");
    ctx->cycle_kernel = value;
    ctx->cluster_checked = false;
  } else if (option == PYRO_OPT_WAVE_STALL) {
    if (value < -1) return fail(ctx, PYRO_ERR_ARG, "stall item is -1 (off) or an item index");
    ctx->wave_stall_item = value;
  } else if (option == PYRO_OPT_CHAIN_STAGGER) {
    if (value < 0) return fail(ctx, PYRO_ERR_ARG, "chain stagger must be >= 0");
    ctx->chain_stagger = value;
  } else if (option == PYRO_OPT_J1_FIXED_L) {
    if (value != 0 && value != 1) return fail(ctx, PYRO_ERR_ARG, "fixed-L option is 0 or 1");
    ctx->j1_fixed_l = value;
  } else if (option == PYRO_OPT_CLUSTER_SIZE) {
    if (value < 1 || value > 16) return fail(ctx, PYRO_ERR_ARG, "cluster size is 1..16");
    ctx->cluster_size = value;
    ctx->cluster_checked = false;
  } else {
    return fail(ctx, PYRO_ERR_ARG, "unknown option");
  }
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_kernels.clear();
  return build_schedule(ctx);
}

int pyro_get_option(pyro_ctx* ctx, int option, int* value) {
  if (!ctx || !value) return PYRO_ERR_ARG;
  int rc = check_cluster(ctx);
  if (rc) return rc;
  switch (option) {
    case PYRO_OPT_J1_KERNEL: *value = ctx->use_j1_kernel ? 1 : 0; break;
    case PYRO_OPT_CYCLE_KERNEL: *value = ctx->cycle_kernel; break;
    case PYRO_OPT_CLUSTER_SIZE: *value = ctx->cluster_size; break;
    case PYRO_OPT_SMEM_KERNEL: *value = ctx->smem_kernel; break;
    case PYRO_OPT_REPLICA_GROUP: *value = ctx->rep_group; break;
    case PYRO_OPT_CHAINS: *value = ctx->n_chains; break;
    case PYRO_OPT_GROUP_MB: *value = ctx->gen_group_mb; break;
    case PYRO_OPT_FAR_KERNEL: *value = ctx->far_kernel; break;
    case PYRO_OPT_PDL: *value = ctx->pdl; break;
    case PYRO_OPT_TET_GROUPED: *value = ctx->tet_grouped; break;
    case PYRO_OPT_FUSED_OBS: *value = ctx->fused_obs; break;
    case PYRO_OPT_WAVE_STALL: *value = ctx->wave_stall_item; break;
    case PYRO_OPT_MEASURE_SNAPSHOT: *value = ctx->measure_snapshot; break;
    case PYRO_OPT_J1_FIXED_L: *value = ctx->j1_fixed_l; break;
    case PYRO_OPT_CHAIN_STAGGER: *value = ctx->chain_stagger; break;
    case PYRO_OPT_J1_SITE_MODE:
      *value = (ctx->j1_metro_site_mode ? 1 : 0) | (ctx->j1_or_site_mode ? 2 : 0);
      break;
    default: return fail(ctx, PYRO_ERR_ARG, "unknown option");
  }
  return PYRO_OK;
}

// Times each kernel variant on `cycles` real cycles (they advance the chain:
// every variant computes the same updates) and keeps the fastest.
int pyro_autotune(pyro_ctx* ctx, int n_metro, int n_or, int cycles, int* chosen) {
  NvtxRange nvtx_range("pyro_autotune");
  if (!ctx) return PYRO_ERR_ARG;
  if (cycles < 1 || n_metro < 0 || n_or < 0 || n_metro + n_or < 1)
    return fail(ctx, PYRO_ERR_ARG, "autotune: need cycles >= 1 and at least one sweep");
  struct Variant { int j1, cyc, cs, site, group, chains, gen_mb, stagger; };
  bool any_j1 = false, any_gen = false;
  for (const auto& s : ctx->sys) {
    if (j1_sweepable(s)) any_j1 = true;
    else any_gen = true;
  }
  std::vector<Variant> vs;
  int n_j1 = 0;  // stage 1: the J1 variants, first in vs
  if (any_j1) {
    const Variant j1v[] = {{0, 0, 16, 1, 0, 1, 0}, {1, 0, 16, 1, 0, 1, 0}, {1, 0, 16, 3, 0, 1, 0},
                           {1, 0, 16, 1, 8, 1, 0}, {1, 0, 16, 1, 4, 2, 0}, {1, 0, 16, 3, 4, 2, 0},
                           {1, 0, 16, 1, 3, 2, 0}, {1, 0, 16, 1, 2, 2, 0}, {1, 0, 16, 1, 2, 3, 0},
                           {1, 0, 16, 1, 3, 3, 0}, {1, 0, 16, 1, 2, 4, 0}, {1, 0, 16, 1, 1, 4, 0},
                           {1, 1, 16, 1, 0, 1, 0}, {1, 1, 10, 1, 0, 1, 0}, {1, 0, 16, 1, 6, 2, 0},
                           {1, 0, 16, 1, 4, 3, 0}, {1, 0, 16, 1, 5, 2, 0}, {1, 0, 16, 3, 2, 4, 0},
                           {1, 0, 16, 3, 2, 2, 0}, {1, 0, 16, 3, 1, 4, 0}, {1, 0, 16, 1, 2, 6, 0},
                           {1, 0, 16, 1, 1, 8, 0}, {1, 0, 16, 1, 1, 6, 0},
                           // the work-queue cycle kernel: forms, replica groups
                           {1, 2, 16, 3, 2, 1, 0}, {1, 2, 16, 3, 4, 1, 0}, {1, 2, 16, 3, 8, 1, 0},
                           {1, 2, 16, 3, 16, 1, 0}, {1, 2, 16, 3, 0, 1, 0}, {1, 2, 16, 1, 4, 1, 0},
                           {1, 2, 16, 1, 8, 1, 0}, {1, 2, 16, 2, 8, 1, 0},
                           // skewed multi-group launches: forms, group size, groups in flight
                           {1, 3, 16, 3, 2, 4, 0}, {1, 3, 16, 3, 2, 8, 0}, {1, 3, 16, 3, 1, 8, 0},
                           {1, 3, 16, 3, 4, 4, 0}, {1, 3, 16, 1, 2, 4, 0}, {1, 3, 16, 1, 2, 8, 0},
                           {1, 3, 16, 1, 4, 4, 0}, {1, 3, 16, 3, 4, 2, 0},
                           // Metropolis passes in the cell form too (fixed-L kernels)
                           {1, 0, 16, 0, 2, 4, 0}, {1, 0, 16, 0, 4, 2, 0}, {1, 0, 16, 0, 3, 3, 0},
                           {1, 0, 16, 0, 1, 8, 0},
                           // odd chains started one Metropolis sweep after their partner
                           {1, 0, 16, 1, 2, 4, 0, 4}, {1, 0, 16, 1, 2, 4, 0, 8}, {1, 0, 16, 1, 3, 3, 0, 4},
                           {1, 0, 16, 1, 1, 8, 0, 4}, {1, 0, 16, 0, 2, 4, 0, 4}};
    vs.insert(vs.end(), std::begin(j1v), std::end(j1v));
    n_j1 = (int)vs.size();
  }
  if (any_gen) {
    const int base = vs.size();  // filled with the best J1 knobs after stage 1
    const Variant gv[] = {{1, 0, 16, 1, 0, 1, 0},  {1, 0, 16, 1, 0, 1, 24}, {1, 0, 16, 1, 0, 1, 40},
                          {1, 0, 16, 1, 0, 1, 64}, {1, 0, 16, 1, 0, 2, 24}, {1, 0, 16, 1, 0, 2, 40},
                          {1, 0, 16, 1, 0, 3, 24},
                          // the work queue over every 16-colour system (contexts without J1
                          // systems: with them, stage 2 keeps the J1 winner's cycle kernel)
                          {1, 2, 16, 1, 0, 1, 0},  {1, 2, 16, 1, 0, 1, 24}, {1, 2, 16, 1, 0, 1, 64}};
    vs.insert(vs.end(), std::begin(gv), std::end(gv));
    (void)base;
  }
  const bool swap = !sharded(ctx);
  cudaEvent_t a, b;
  PYRO_CK(cudaEventCreate(&a));
  PYRO_CK(cudaEventCreate(&b));
  auto apply = [&](const Variant& v) {
    int rc = pyro_set_option(ctx, PYRO_OPT_J1_KERNEL, v.j1);
    if (!rc) rc = pyro_set_option(ctx, PYRO_OPT_CYCLE_KERNEL, v.cyc);
    if (!rc) rc = pyro_set_option(ctx, PYRO_OPT_CLUSTER_SIZE, v.cs);
    if (!rc) rc = pyro_set_option(ctx, PYRO_OPT_J1_SITE_MODE, v.site);
    if (!rc) rc = pyro_set_option(ctx, PYRO_OPT_REPLICA_GROUP, v.group);
    if (!rc) rc = pyro_set_option(ctx, PYRO_OPT_CHAINS, v.chains);
    if (!rc) rc = pyro_set_option(ctx, PYRO_OPT_GROUP_MB, v.gen_mb);
    if (!rc) rc = pyro_set_option(ctx, PYRO_OPT_CHAIN_STAGGER, v.stagger);
    if (!rc) rc = check_cluster(ctx);
    return rc;
  };
  float best = 1e30f;
  int best_i = -1;
  for (int i = 0; i < (int)vs.size(); ++i) {
    Variant v = vs[i];
    if (i >= n_j1 && best_i >= 0 && best_i < n_j1) {
      // stage 2 (generic groups) keeps the J1 knobs of stage 1's winner
      const Variant& w = vs[best_i];
      v.j1 = w.j1;
      v.cyc = w.cyc;
      v.cs = w.cs;
      v.site = w.site;
      v.group = w.group;
      if (v.chains == 1) v.chains = w.chains;
      vs[i] = v;
    }
    int rc = apply(v);
    if (rc) continue;
    if (v.cyc == 1 && (ctx->cycle_kernel != 1 || ctx->cluster_size != v.cs)) continue;
    if (v.cyc >= 2 && ctx->cycle_kernel != v.cyc) continue;
    if ((rc = pyro_cycle(ctx, n_metro, n_or, swap, 1))) return rc;  // build the graph
    float ms = 1e30f;
    for (int rep = 0; rep < 2; ++rep) {  // best of two timings
      PYRO_CK(cudaEventRecord(a, ctx->stream));
      if ((rc = pyro_cycle(ctx, n_metro, n_or, swap, cycles))) return rc;
      PYRO_CK(cudaEventRecord(b, ctx->stream));
      PYRO_CK(cudaEventSynchronize(b));
      float t = 0.f;
      PYRO_CK(cudaEventElapsedTime(&t, a, b));
      ms = std::min(ms, t);
    }
    if (ms < best) {
      best = ms;
      best_i = i;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (best_i < 0) return fail(ctx, PYRO_ERR_STATE, "autotune: no variant ran");
  int rc = apply(vs[best_i]);
  if (chosen) *chosen = best_i;
  return rc;
}

void* pyro_get_stream(const pyro_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int pyro_synchronize(pyro_ctx* ctx) {
  if (!ctx) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return check_wave_status(ctx);
}

int pyro_set_system_keys(pyro_ctx* ctx, int system, int key_base, int swap_key) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || key_base < 0 || swap_key < 0)
    return fail(ctx, PYRO_ERR_ARG, "set_system_keys: bad system or negative key");
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  SysDev& s = ctx->sys[system];
  s.rep_key = key_base + s.rep_global;
  s.swap_key = swap_key;
  PYRO_CK(cudaMemcpy(ctx->d_sys, ctx->sys.data(), sizeof(SysDev) * ctx->sys.size(),
                     cudaMemcpyHostToDevice));
  return rebuild_schedule(ctx);  // the captured cycles hold the old keys
}

int pyro_snapshot(pyro_ctx* ctx) {
  NvtxRange nvtx_range("pyro_snapshot");
  if (!ctx) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  if (!ctx->snap_stream) {
    PYRO_CK(cudaStreamCreateWithFlags(&ctx->snap_stream, cudaStreamNonBlocking));
    PYRO_CK(cudaEventCreateWithFlags(&ctx->snap_start, cudaEventDisableTiming));
    PYRO_CK(cudaEventCreateWithFlags(&ctx->snap_done, cudaEventDisableTiming));
    PYRO_CK(alloc(&ctx->d_snap, (size_t)ctx->n_spins));
    PYRO_CK(alloc(&ctx->d_snap_temp_of_rep, (size_t)ctx->total_temps));
    PYRO_CK(alloc(&ctx->d_snap_rep_of_temp, (size_t)ctx->total_temps));
    PYRO_CK(alloc(&ctx->d_snap_energy, (size_t)ctx->total_reps));
    PYRO_CK(alloc(&ctx->d_snap_mag, (size_t)3 * ctx->total_reps));
  }
  // The copy starts when the context stream reaches this point, after any
  // measurement of the previous snapshot (same measurement stream); the
  // context stream's next update waits until the copy has read the spins.
  cudaStream_t ms = ctx->snap_stream;
  PYRO_CK(cudaEventRecord(ctx->snap_start, ctx->stream));
  PYRO_CK(cudaStreamWaitEvent(ms, ctx->snap_start, 0));
  PYRO_CK(cudaMemcpyAsync(ctx->d_snap, ctx->d_spins, sizeof(float4) * (size_t)ctx->n_spins,
                          cudaMemcpyDeviceToDevice, ms));
  PYRO_CK(cudaMemcpyAsync(ctx->d_snap_temp_of_rep, ctx->d_temp_of_rep,
                          sizeof(int) * ctx->total_temps, cudaMemcpyDeviceToDevice, ms));
  PYRO_CK(cudaMemcpyAsync(ctx->d_snap_rep_of_temp, ctx->d_rep_of_temp,
                          sizeof(int) * ctx->total_temps, cudaMemcpyDeviceToDevice, ms));
  PYRO_CK(cudaMemcpyAsync(ctx->d_snap_energy, ctx->d_energy, sizeof(double) * ctx->total_reps,
                          cudaMemcpyDeviceToDevice, ms));
  PYRO_CK(cudaMemcpyAsync(ctx->d_snap_mag, ctx->d_mag, sizeof(double) * 3 * ctx->total_reps,
                          cudaMemcpyDeviceToDevice, ms));
  PYRO_CK(cudaEventRecord(ctx->snap_done, ms));
  PYRO_CK(cudaStreamWaitEvent(ctx->stream, ctx->snap_done, 0));
  ctx->snap_taken = true;
  return PYRO_OK;
}

int pyro_system_info(const pyro_ctx* ctx, int system, int* L, int* n_sites, int* n_replicas,
                     int* n_colours) {
  if (!ctx || system < 0 || system >= (int)ctx->sys.size()) return PYRO_ERR_ARG;
  const SysDev& s = ctx->sys[system];
  if (L) *L = s.L;
  if (n_sites) *n_sites = 16 * s.L3;
  if (n_replicas) *n_replicas = s.n_rep;
  if (n_colours) *n_colours = s.n_colours;
  return PYRO_OK;
}

int pyro_init_random(pyro_ctx* ctx) {
  if (!ctx) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  launch_init_random(ctx->d_spins, ctx->sys.data(), ctx->d_sys, (int)ctx->sys.size(),
                     (uint32_t)(ctx->seed & 0xffffffffu), (uint32_t)(ctx->seed >> 32), ctx->stream);
  PYRO_CK_LAUNCH();
  return PYRO_OK;
}

static int spin_copy(pyro_ctx* ctx, int system, void* dst, const void* src, cudaMemcpyKind kind,
                     bool to_device, bool sync) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || (!dst && !src))
    return fail(ctx, PYRO_ERR_ARG, "spin copy: bad system or null pointer");
  PYRO_CK(cudaSetDevice(ctx->device));
  const SysDev& s = ctx->sys[system];
  const size_t bytes = sizeof(float4) * (size_t)s.n_rep * 16 * s.L3;
  float4* dev = ctx->d_spins + s.spin_off;
  if (to_device) PYRO_CK(cudaMemcpyAsync(dev, src, bytes, kind, ctx->stream));
  else PYRO_CK(cudaMemcpyAsync(dst, dev, bytes, kind, ctx->stream));
  if (!sync) return PYRO_OK;
  if (!to_device) {
    const int rc = queue_wave_status(ctx);
    if (rc) return rc;
  }
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return to_device ? PYRO_OK : wave_status_result(ctx);
}

int pyro_set_spins(pyro_ctx* ctx, int system, const float* host_xyzw) {
  if (!host_xyzw) return fail(ctx, PYRO_ERR_ARG, "set_spins: null pointer");
  return spin_copy(ctx, system, nullptr, host_xyzw, cudaMemcpyHostToDevice, true, true);
}
int pyro_get_spins(pyro_ctx* ctx, int system, float* host_xyzw) {
  if (!host_xyzw) return fail(ctx, PYRO_ERR_ARG, "get_spins: null pointer");
  return spin_copy(ctx, system, host_xyzw, nullptr, cudaMemcpyDeviceToHost, false, true);
}
// The reference's host layout: per replica three planes x, y, z of 16 L^3
// values each (site index s L^3 + cell, as here), replicas one after another.
int pyro_set_spins_planar(pyro_ctx* ctx, int system, const double* host_planes) {
  if (!ctx) return PYRO_ERR_ARG;
  if (!host_planes) return fail(ctx, PYRO_ERR_ARG, "set_spins_planar: null pointer");
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "set_spins_planar: bad system");
  const SysDev& s = ctx->sys[system];
  const size_t n = (size_t)16 * s.L3;
  std::vector<float> buf(4 * n * (size_t)s.n_rep);
  for (size_t r = 0; r < (size_t)s.n_rep; ++r) {
    const double* x = host_planes + 3 * n * r;
    for (size_t i = 0; i < n; ++i) {
      float* o = buf.data() + 4 * (n * r + i);
      o[0] = (float)x[i];
      o[1] = (float)x[n + i];
      o[2] = (float)x[2 * n + i];
      o[3] = 0.0f;
    }
  }
  return spin_copy(ctx, system, nullptr, buf.data(), cudaMemcpyHostToDevice, true, true);
}

int pyro_get_spins_planar(pyro_ctx* ctx, int system, double* host_planes) {
  if (!ctx) return PYRO_ERR_ARG;
  if (!host_planes) return fail(ctx, PYRO_ERR_ARG, "get_spins_planar: null pointer");
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "get_spins_planar: bad system");
  const SysDev& s = ctx->sys[system];
  const size_t n = (size_t)16 * s.L3;
  std::vector<float> buf(4 * n * (size_t)s.n_rep);
  const int rc = spin_copy(ctx, system, buf.data(), nullptr, cudaMemcpyDeviceToHost, false, true);
  if (rc) return rc;
  for (size_t r = 0; r < (size_t)s.n_rep; ++r) {
    double* x = host_planes + 3 * n * r;
    for (size_t i = 0; i < n; ++i) {
      const float* v = buf.data() + 4 * (n * r + i);
      x[i] = v[0];
      x[n + i] = v[1];
      x[2 * n + i] = v[2];
    }
  }
  return PYRO_OK;
}

int pyro_set_spins_device(pyro_ctx* ctx, int system, const float* dev_xyzw) {
  if (!dev_xyzw) return fail(ctx, PYRO_ERR_ARG, "set_spins_device: null pointer");
  return spin_copy(ctx, system, nullptr, dev_xyzw, cudaMemcpyDeviceToDevice, true, false);
}
int pyro_get_spins_device(pyro_ctx* ctx, int system, float* dev_xyzw) {
  if (!dev_xyzw) return fail(ctx, PYRO_ERR_ARG, "get_spins_device: null pointer");
  return spin_copy(ctx, system, dev_xyzw, nullptr, cudaMemcpyDeviceToDevice, false, false);
}

static int run_sweeps(pyro_ctx* ctx, int n, bool metro) {
  NvtxRange nvtx_range("pyro_sweeps");
  if (!ctx) return PYRO_ERR_ARG;
  if (n < 0) return fail(ctx, PYRO_ERR_ARG, "n_sweeps must be >= 0");
  if (n == 0) return PYRO_OK;
  PYRO_CK(cudaSetDevice(ctx->device));
  int rc = queue_cycle_body(ctx, metro ? n : 0, metro ? 0 : n, false);
  if (rc != PYRO_OK) return rc;
  launch_advance(ctx->d_sweep, (unsigned long long)n, ctx->stream);
  PYRO_CK_LAUNCH();
  ctx->h_sweep += (unsigned long long)n;
  if (metro) ctx->metro_sweeps_since_reset += (unsigned long long)n;
  return PYRO_OK;
}

int pyro_metropolis_sweep(pyro_ctx* ctx, int n_sweeps) { return run_sweeps(ctx, n_sweeps, true); }
int pyro_overrelax_sweep(pyro_ctx* ctx, int n_sweeps) { return run_sweeps(ctx, n_sweeps, false); }

int pyro_set_cone(pyro_ctx* ctx, int system, const float* cosmax) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !cosmax)
    return fail(ctx, PYRO_ERR_ARG, "set_cone: bad system or null pointer");
  const SysDev& s = ctx->sys[system];
  for (int t = 0; t < s.n_temp; ++t)
    if (!(cosmax[t] >= -1.0f && cosmax[t] < 1.0f))
      return fail(ctx, PYRO_ERR_ARG, "set_cone: cos(theta_max) must lie in [-1, 1)");
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemcpyAsync(ctx->d_cosmax + s.temp_base, cosmax, sizeof(float) * s.n_temp,
                          cudaMemcpyHostToDevice, ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return PYRO_OK;
}

int pyro_get_cone(pyro_ctx* ctx, int system, float* cosmax) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !cosmax)
    return fail(ctx, PYRO_ERR_ARG, "get_cone: bad system or null pointer");
  const SysDev& s = ctx->sys[system];
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemcpyAsync(cosmax, ctx->d_cosmax + s.temp_base, sizeof(float) * s.n_temp,
                          cudaMemcpyDeviceToHost, ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return PYRO_OK;
}

int pyro_get_acceptance(pyro_ctx* ctx, int system, uint64_t* accepted, uint64_t* proposed) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !accepted)
    return fail(ctx, PYRO_ERR_ARG, "get_acceptance: bad system or null pointer");
  const SysDev& s = ctx->sys[system];
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemcpyAsync(accepted, ctx->d_accepted + s.temp_base,
                          sizeof(unsigned long long) * s.n_temp, cudaMemcpyDeviceToHost,
                          ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  if (proposed) {
    // Each temperature slot holds exactly one replica during every sweep;
    // in a sharded context only the slots of held replicas are counted here.
    const uint64_t per = (uint64_t)16 * s.L3 * ctx->metro_sweeps_since_reset;
    for (int t = 0; t < s.n_temp; ++t) proposed[t] = s.n_rep == s.n_temp ? per : 0;
  }
  return PYRO_OK;
}

int pyro_reset_acceptance(pyro_ctx* ctx) {
  if (!ctx) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemsetAsync(ctx->d_accepted, 0, sizeof(unsigned long long) * ctx->total_temps,
                          ctx->stream));
  ctx->metro_sweeps_since_reset = 0;
  return PYRO_OK;
}

int pyro_tune_cone(pyro_ctx* ctx, double target, int iterations, int sweeps_per_iteration,
                   int n_or) {
  if (!ctx) return PYRO_ERR_ARG;
  if (!(target > 0.0 && target < 1.0) || iterations < 0 || sweeps_per_iteration < 1 || n_or < 0)
    return fail(ctx, PYRO_ERR_ARG, "tune_cone: need 0 < target < 1, iterations >= 0, sweeps >= 1");
  if (sharded(ctx))
    return fail(ctx, PYRO_ERR_STATE, "tune_cone: needs every replica of the ladder in one context");
  std::vector<float> cosv;
  std::vector<uint64_t> acc, prop;
  for (int it = 0; it < iterations; ++it) {
    int rc = pyro_reset_acceptance(ctx);
    if (rc) return rc;
    for (int k = 0; k < sweeps_per_iteration; ++k) {
      if ((rc = pyro_metropolis_sweep(ctx, 1))) return rc;
      if (n_or > 0 && (rc = pyro_overrelax_sweep(ctx, n_or))) return rc;
    }
    bool done = true;
    for (int si = 0; si < (int)ctx->sys.size(); ++si) {
      const SysDev& s = ctx->sys[si];
      cosv.resize(s.n_temp);
      acc.resize(s.n_temp);
      prop.resize(s.n_temp);
      if ((rc = pyro_get_acceptance(ctx, si, acc.data(), prop.data()))) return rc;
      if ((rc = pyro_get_cone(ctx, si, cosv.data()))) return rc;
      for (int t = 0; t < s.n_temp; ++t) {
        const double ratio = prop[t] ? (double)acc[t] / (double)prop[t] : target;
        if (std::fabs(ratio - target) > 0.02) done = false;
        double theta = std::acos(std::max(-1.0, std::min(1.0, (double)cosv[t])));
        const double f = std::max(0.5, std::min(2.0, ratio / target));
        theta = std::max(1e-4, std::min(M_PI, theta * f));
        float c = (float)std::cos(theta);
        if (c >= 1.0f) c = std::nextafter(1.0f, 0.0f);
        if (c < -1.0f) c = -1.0f;
        cosv[t] = c;
      }
      if ((rc = pyro_set_cone(ctx, si, cosv.data()))) return rc;
    }
    if (done) break;
  }
  return pyro_reset_acceptance(ctx);
}

int pyro_observables_device(pyro_ctx* ctx, int system, double* dev_energy,
                            double* dev_magnetisation3) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "observables: bad system");
  PYRO_CK(cudaSetDevice(ctx->device));
  int rc = queue_observables(ctx);
  if (rc) return rc;
  ctx->launches += ctx->obs_j1.size() + (ctx->obs_generic_blocks > 0 ? 1 : 0) + 1;
  const SysDev& s = ctx->sys[system];
  if (dev_energy)
    PYRO_CK(cudaMemcpyAsync(dev_energy, ctx->d_energy + s.rep_ctx_base, sizeof(double) * s.n_rep,
                            cudaMemcpyDeviceToDevice, ctx->stream));
  if (dev_magnetisation3)
    PYRO_CK(cudaMemcpyAsync(dev_magnetisation3, ctx->d_mag + 3 * s.rep_ctx_base,
                            sizeof(double) * 3 * s.n_rep, cudaMemcpyDeviceToDevice, ctx->stream));
  return PYRO_OK;
}

int pyro_last_observables_device(pyro_ctx* ctx, int system, double* dev_energy,
                                 double* dev_magnetisation3) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "last_observables: bad system");
  PYRO_CK(cudaSetDevice(ctx->device));
  const SysDev& s = ctx->sys[system];
  if (dev_energy)
    PYRO_CK(cudaMemcpyAsync(dev_energy, ctx->d_energy + s.rep_ctx_base, sizeof(double) * s.n_rep,
                            cudaMemcpyDeviceToDevice, ctx->stream));
  if (dev_magnetisation3)
    PYRO_CK(cudaMemcpyAsync(dev_magnetisation3, ctx->d_mag + 3 * s.rep_ctx_base,
                            sizeof(double) * 3 * s.n_rep, cudaMemcpyDeviceToDevice, ctx->stream));
  return PYRO_OK;
}

int pyro_last_observables(pyro_ctx* ctx, int system, double* energy, double* magnetisation3) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "last_observables: bad system");
  PYRO_CK(cudaSetDevice(ctx->device));
  const SysDev& s = ctx->sys[system];
  if (ctx->measure_snapshot) {  // the energies the snapshot's cycle computed
    const cudaStream_t st = ctx->snap_stream;
    if (energy)
      PYRO_CK(cudaMemcpyAsync(energy, ctx->d_snap_energy + s.rep_ctx_base,
                              sizeof(double) * s.n_rep, cudaMemcpyDeviceToHost, st));
    if (magnetisation3)
      PYRO_CK(cudaMemcpyAsync(magnetisation3, ctx->d_snap_mag + 3 * s.rep_ctx_base,
                              sizeof(double) * 3 * s.n_rep, cudaMemcpyDeviceToHost, st));
    PYRO_CK(cudaStreamSynchronize(st));
    return PYRO_OK;
  }
  if (energy)
    PYRO_CK(cudaMemcpyAsync(energy, ctx->d_energy + s.rep_ctx_base, sizeof(double) * s.n_rep,
                            cudaMemcpyDeviceToHost, ctx->stream));
  if (magnetisation3)
    PYRO_CK(cudaMemcpyAsync(magnetisation3, ctx->d_mag + 3 * s.rep_ctx_base,
                            sizeof(double) * 3 * s.n_rep, cudaMemcpyDeviceToHost, ctx->stream));
  const int rc = queue_wave_status(ctx);
  if (rc) return rc;
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return wave_status_result(ctx);
}

namespace {
// True for page-locked host memory that the device can copy from or to
// asynchronously.
bool pinned_host(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}
}  // namespace

int pyro_set_cone_async(pyro_ctx* ctx, int system, const float* pinned_cosmax) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !pinned_cosmax)
    return fail(ctx, PYRO_ERR_ARG, "set_cone_async: bad system or null pointer");
  PYRO_CK(cudaSetDevice(ctx->device));
  if (!pinned_host(pinned_cosmax))
    return fail(ctx, PYRO_ERR_ARG, "set_cone_async: the buffer is not pinned host memory");
  const SysDev& s = ctx->sys[system];
  for (int t = 0; t < s.n_temp; ++t)
    if (!(pinned_cosmax[t] >= -1.0f && pinned_cosmax[t] < 1.0f))
      return fail(ctx, PYRO_ERR_ARG, "set_cone_async: cos(theta_max) must lie in [-1, 1)");
  PYRO_CK(cudaMemcpyAsync(ctx->d_cosmax + s.temp_base, pinned_cosmax, sizeof(float) * s.n_temp,
                          cudaMemcpyHostToDevice, ctx->stream));
  return PYRO_OK;
}

int pyro_last_observables_async(pyro_ctx* ctx, int system, double* pinned_energy,
                                double* pinned_magnetisation3) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "last_observables_async: bad system");
  if (ctx->measure_snapshot)
    return fail(ctx, PYRO_ERR_STATE, "last_observables_async: not in the snapshot mode");
  PYRO_CK(cudaSetDevice(ctx->device));
  if ((pinned_energy && !pinned_host(pinned_energy)) ||
      (pinned_magnetisation3 && !pinned_host(pinned_magnetisation3)))
    return fail(ctx, PYRO_ERR_ARG, "last_observables_async: a buffer is not pinned host memory");
  const SysDev& s = ctx->sys[system];
  if (pinned_energy)
    PYRO_CK(cudaMemcpyAsync(pinned_energy, ctx->d_energy + s.rep_ctx_base,
                            sizeof(double) * s.n_rep, cudaMemcpyDeviceToHost, ctx->stream));
  if (pinned_magnetisation3)
    PYRO_CK(cudaMemcpyAsync(pinned_magnetisation3, ctx->d_mag + 3 * s.rep_ctx_base,
                            sizeof(double) * 3 * s.n_rep, cudaMemcpyDeviceToHost, ctx->stream));
  return PYRO_OK;
}

int pyro_observables(pyro_ctx* ctx, int system, double* energy, double* magnetisation3) {
  NvtxRange nvtx_range("pyro_observables");
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "observables: bad system");
  PYRO_CK(cudaSetDevice(ctx->device));
  int rc = queue_observables(ctx);
  if (rc) return rc;
  const SysDev& s = ctx->sys[system];
  if (energy)
    PYRO_CK(cudaMemcpyAsync(energy, ctx->d_energy + s.rep_ctx_base, sizeof(double) * s.n_rep,
                            cudaMemcpyDeviceToHost, ctx->stream));
  if (magnetisation3)
    PYRO_CK(cudaMemcpyAsync(magnetisation3, ctx->d_mag + 3 * s.rep_ctx_base,
                            sizeof(double) * 3 * s.n_rep, cudaMemcpyDeviceToHost, ctx->stream));
  rc = queue_wave_status(ctx);
  if (rc) return rc;
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return wave_status_result(ctx);
}

int pyro_get_temperatures(pyro_ctx* ctx, int system, double* temperature_of_replica) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !temperature_of_replica)
    return fail(ctx, PYRO_ERR_ARG, "get_temperatures: bad system or null pointer");
  const SysDev& s = ctx->sys[system];
  std::vector<int> t(s.n_temp);
  PYRO_CK(cudaSetDevice(ctx->device));
  const cudaStream_t st = measure_stream(ctx);
  PYRO_CK(cudaMemcpyAsync(t.data(), measure_temp_of_rep(ctx) + s.temp_base,
                          sizeof(int) * s.n_temp, cudaMemcpyDeviceToHost, st));
  PYRO_CK(cudaStreamSynchronize(st));
  for (int g = 0; g < s.n_temp; ++g) temperature_of_replica[g] = ctx->ladders[system][t[g]];
  return PYRO_OK;
}

int pyro_get_permutation(pyro_ctx* ctx, int system, int* replica_of_temperature) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !replica_of_temperature)
    return fail(ctx, PYRO_ERR_ARG, "get_permutation: bad system or null pointer");
  const SysDev& s = ctx->sys[system];
  PYRO_CK(cudaSetDevice(ctx->device));
  const cudaStream_t st = measure_stream(ctx);
  PYRO_CK(cudaMemcpyAsync(replica_of_temperature, measure_rep_of_temp(ctx) + s.temp_base,
                          sizeof(int) * s.n_temp, cudaMemcpyDeviceToHost, st));
  PYRO_CK(cudaStreamSynchronize(st));
  return PYRO_OK;
}

int pyro_pt_swap(pyro_ctx* ctx, int parity, int* n_accepted) {
  if (!ctx) return PYRO_ERR_ARG;
  if (parity > 1) return fail(ctx, PYRO_ERR_ARG, "pt_swap: parity must be 0, 1 or < 0 (auto)");
  if (sharded(ctx))
    return fail(ctx, PYRO_ERR_STATE,
                "pt_swap: context holds part of the ladder; use pyro_pt_swap_global");
  PYRO_CK(cudaSetDevice(ctx->device));
  int rc = queue_observables(ctx);
  if (rc) return rc;
  ExchangeParams x = exchange_params(ctx);
  x.parity = parity < 0 ? -1 : parity;
  launch_exchange(x, (int)ctx->sys.size(), max_pairs(ctx), ctx->stream);
  PYRO_CK_LAUNCH();
  if (n_accepted) {
    std::vector<int> a(ctx->sys.size());
    PYRO_CK(cudaMemcpyAsync(a.data(), ctx->d_last_accepted, sizeof(int) * a.size(),
                            cudaMemcpyDeviceToHost, ctx->stream));
    PYRO_CK(cudaStreamSynchronize(ctx->stream));
    int sum = 0;
    for (int v : a) sum += v;
    *n_accepted = sum;
  }
  return PYRO_OK;
}

int pyro_pt_swap_global(pyro_ctx* ctx, int system, const double* dev_energy_all, int parity) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !dev_energy_all)
    return fail(ctx, PYRO_ERR_ARG, "pt_swap_global: bad system or null pointer");
  if (parity > 1) return fail(ctx, PYRO_ERR_ARG, "pt_swap_global: parity must be 0, 1 or < 0");
  PYRO_CK(cudaSetDevice(ctx->device));
  ExchangeParams x = exchange_params(ctx);
  x.sys_first = system;
  x.energy = dev_energy_all;
  x.energy_is_global = 1;
  x.parity = parity < 0 ? -1 : parity;
  x.history_count = nullptr;
  launch_exchange(x, 1, (ctx->sys[system].n_temp + 1) / 2, ctx->stream);
  PYRO_CK_LAUNCH();
  ctx->launches += 1;
  return PYRO_OK;
}

int pyro_get_swap_stats(pyro_ctx* ctx, int system, uint64_t* accepted, uint64_t* attempted) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "get_swap_stats: bad system");
  const SysDev& s = ctx->sys[system];
  PYRO_CK(cudaSetDevice(ctx->device));
  if (accepted)
    PYRO_CK(cudaMemcpyAsync(accepted, ctx->d_swap_acc + s.temp_base, 8 * s.n_temp,
                            cudaMemcpyDeviceToHost, ctx->stream));
  if (attempted)
    PYRO_CK(cudaMemcpyAsync(attempted, ctx->d_swap_try + s.temp_base, 8 * s.n_temp,
                            cudaMemcpyDeviceToHost, ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return PYRO_OK;
}

int pyro_enable_history(pyro_ctx* ctx, int capacity_cycles) {
  if (!ctx) return PYRO_ERR_ARG;
  if (capacity_cycles < 0) return fail(ctx, PYRO_ERR_ARG, "history capacity must be >= 0");
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_kernels.clear();
  if (ctx->d_history) cudaFree(ctx->d_history);
  ctx->d_history = nullptr;
  ctx->history_cap = capacity_cycles;
  if (capacity_cycles > 0)
    PYRO_CK(alloc(&ctx->d_history, (size_t)capacity_cycles * ctx->total_temps));
  PYRO_CK(cudaMemset(ctx->d_history_count, 0, sizeof(unsigned long long)));
  return PYRO_OK;
}

int pyro_get_history(pyro_ctx* ctx, int system, double* out, int* n_cycles) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !out || !n_cycles)
    return fail(ctx, PYRO_ERR_ARG, "get_history: bad system or null pointer");
  if (!ctx->d_history) return fail(ctx, PYRO_ERR_STATE, "get_history: history not enabled");
  PYRO_CK(cudaSetDevice(ctx->device));
  unsigned long long count = 0;
  PYRO_CK(cudaMemcpyAsync(&count, ctx->d_history_count, 8, cudaMemcpyDeviceToHost, ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  const int n = (int)std::min<unsigned long long>(count, (unsigned long long)ctx->history_cap);
  std::vector<double> all((size_t)ctx->history_cap * ctx->total_temps);
  PYRO_CK(cudaMemcpy(all.data(), ctx->d_history, sizeof(double) * all.size(),
                     cudaMemcpyDeviceToHost));
  const SysDev& s = ctx->sys[system];
  // Oldest first: when the ring wrapped, start at the oldest slot.
  const unsigned long long first = count > (unsigned long long)ctx->history_cap
                                       ? count % (unsigned long long)ctx->history_cap
                                       : 0ull;
  for (int c = 0; c < n; ++c) {
    const size_t slot = (size_t)((first + c) % ctx->history_cap);
    for (int t = 0; t < s.n_temp; ++t)
      out[(size_t)c * s.n_temp + t] = all[slot * ctx->total_temps + s.temp_base + t];
  }
  *n_cycles = n;
  return PYRO_OK;
}

// Small lattices: every system fits one CTA's shared memory.
static bool use_smem_path(const pyro_ctx* ctx) {
  if (!ctx->smem_kernel) return false;
  for (const auto& s : ctx->sys)
    if (s.L > kSmemMaxL) return false;
  return true;
}

// Cycles without exchange on the shared-memory kernel: one launch per system
// for all cycles; the energy of every cycle goes to the history ring.
static int run_smem_cycles(pyro_ctx* ctx, int n_metro, int n_or, int n_cycles) {
  for (int si = 0; si < (int)ctx->sys.size(); ++si) {
    const SysDev& s = ctx->sys[si];
    SmemCycleParams p;
    p.sys = s;
    p.spins = ctx->d_spins + s.spin_off;
    p.temp_of_rep = ctx->d_temp_of_rep;
    p.beta = ctx->d_beta;
    p.cosmax = ctx->d_cosmax;
    p.accepted = ctx->d_accepted;
    p.sweep_ctr = ctx->d_sweep;
    p.n_metro = n_metro;
    p.n_or = n_or;
    p.n_cycles = n_cycles;
    p.renorm_every = ctx->renorm_every;
    p.seed_lo = (uint32_t)(ctx->seed & 0xffffffffu);
    p.seed_hi = (uint32_t)(ctx->seed >> 32);
    p.history = ctx->d_history;
    p.history_count = ctx->d_history_count;
    p.history_cap = ctx->history_cap;
    p.total_temps = ctx->total_temps;
    p.exch = ctx->d_exch;
    p.energy = ctx->d_energy;
    p.mag = ctx->d_mag;
    PYRO_CK(launch_smem_cycles(p, ctx->tab, ctx->stream));
    ctx->launches += 1;
  }
  launch_advance(ctx->d_sweep, (unsigned long long)(n_metro + n_or) * n_cycles, ctx->stream);
  PYRO_CK_LAUNCH();
  if (ctx->d_history) {
    launch_advance(ctx->d_history_count, (unsigned long long)n_cycles, ctx->stream);
    PYRO_CK_LAUNCH();
  }
  ctx->h_sweep += (unsigned long long)(n_metro + n_or) * n_cycles;
  ctx->metro_sweeps_since_reset += (unsigned long long)n_metro * n_cycles;
  return PYRO_OK;
}

// Learned sweeps can run inside the replica groups: the J1 grouped path
// covers every J1-only system.
static bool tet_in_groups(const pyro_ctx* ctx) {
  if (!ctx->tet_grouped || !j1_grouped_path(ctx)) return false;
  for (int i = 0; i < (int)ctx->sys.size(); ++i)
    if (j1_only(ctx->sys[i]) &&
        std::find(ctx->j1_sys.begin(), ctx->j1_sys.end(), i) == ctx->j1_sys.end())
      return false;
  return true;
}

static int run_cycles(pyro_ctx* ctx, int n_metro, int n_or, int n_tet, int do_swap, int n_cycles) {
  NvtxRange nvtx_range("pyro_cycle");
  if (!ctx) return PYRO_ERR_ARG;
  if (n_metro < 0 || n_or < 0 || n_tet < 0 || n_cycles < 0)
    return fail(ctx, PYRO_ERR_ARG, "cycle: counts must be >= 0");
  if (do_swap && sharded(ctx))
    return fail(ctx, PYRO_ERR_STATE,
                "cycle: a sharded context exchanges through pyro_pt_swap_global");
  if (n_tet > 0 && !ctx->tet)
    return fail(ctx, PYRO_ERR_STATE, "cycle: learned moves need pyro_tet_init first");
  if (n_cycles == 0) return PYRO_OK;
  PYRO_CK(cudaSetDevice(ctx->device));
  if (!do_swap && n_tet == 0 && use_smem_path(ctx)) return run_smem_cycles(ctx, n_metro, n_or, n_cycles);
  const auto key = std::make_tuple(n_metro, n_or, n_tet, do_swap ? 1 : 0);
  auto it = ctx->graphs.find(key);
  if (it == ctx->graphs.end()) {
    cudaGraph_t g;
    int rc = check_cluster(ctx);  // sets kernel attributes: not inside a capture
    if (rc) return rc;
    if (use_wave_kernel(ctx, n_metro, n_or, n_tet) && (rc = prepare_wave(ctx))) return rc;
    if (use_gen_wave(ctx, n_metro, n_or, n_tet) && (rc = prepare_gen_wave(ctx))) return rc;
    PYRO_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
    ctx->defer_finalise = true;  // the exchange kernel below finalises the observables
    if (n_tet == 0) {
      rc = queue_cycle_body(ctx, n_metro, n_or, true);
    } else if (tet_in_groups(ctx)) {
      // each replica group's learned sweeps on its own chain
      rc = queue_cycle_body(ctx, n_metro, n_or, true, n_tet);
    } else {
      rc = queue_cycle_body(ctx, n_metro, n_or, false);
      if (rc == PYRO_OK) rc = queue_tet_sweeps(ctx, n_tet);
      if (rc == PYRO_OK) rc = queue_observables(ctx);
    }
    ctx->defer_finalise = false;
    if (rc == PYRO_OK) {
      ExchangeParams x = exchange_params(ctx);
      x.partials = ctx->d_partials;
      x.obs_segs = ctx->d_obs_segs;
      x.energy_out = ctx->d_energy;
      x.mag_out = ctx->d_mag;
      x.do_swap = do_swap ? 1 : 0;
      x.parity = -1;
      x.history = ctx->d_history;
      x.sweep_ctr = ctx->d_sweep;
      x.sweep_advance = (unsigned long long)(n_metro + n_or);
      launch_exchange(x, (int)ctx->sys.size(), max_pairs(ctx), ctx->stream);
      if (cudaGetLastError() != cudaSuccess) rc = PYRO_ERR_CUDA;
    }
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (rc != PYRO_OK) return fail(ctx, rc, "cycle: capture failed: " + ctx->err);
    if (e != cudaSuccess)
      return fail(ctx, PYRO_ERR_CUDA, std::string("cycle: end capture: ") + cudaGetErrorString(e));
    // kernels in the graph (for the launch count)
    size_t n_nodes = 0;
    unsigned long long n_kernels = 0;
    if (cudaGraphGetNodes(g, nullptr, &n_nodes) == cudaSuccess && n_nodes > 0) {
      std::vector<cudaGraphNode_t> nodes(n_nodes);
      if (cudaGraphGetNodes(g, nodes.data(), &n_nodes) == cudaSuccess)
        for (auto nd : nodes) {
          cudaGraphNodeType ty;
          if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel)
            ++n_kernels;
        }
    }
    cudaGraphExec_t ge;
    e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess)
      return fail(ctx, PYRO_ERR_CUDA, std::string("cycle: instantiate: ") + cudaGetErrorString(e));
    it = ctx->graphs.emplace(key, ge).first;
    ctx->graph_kernels[key] = n_kernels;
  }
  for (int c = 0; c < n_cycles; ++c) PYRO_CK(cudaGraphLaunch(it->second, ctx->stream));
  ctx->launches += ctx->graph_kernels[key] * (unsigned long long)n_cycles;
  ctx->h_sweep += (unsigned long long)(n_metro + n_or) * n_cycles;
  ctx->metro_sweeps_since_reset += (unsigned long long)n_metro * n_cycles;
  if (n_tet > 0) tet_count_sweeps(ctx, (unsigned long long)n_tet * n_cycles);
  return PYRO_OK;
}

int pyro_cycle(pyro_ctx* ctx, int n_metro, int n_or, int do_swap, int n_cycles) {
  return run_cycles(ctx, n_metro, n_or, 0, do_swap, n_cycles);
}

int pyro_cycle_tet(pyro_ctx* ctx, int n_metro, int n_or, int n_tet, int do_swap, int n_cycles) {
  return run_cycles(ctx, n_metro, n_or, n_tet, do_swap, n_cycles);
}

int pyro_get_launch_count(pyro_ctx* ctx, uint64_t* launches) {
  if (!ctx || !launches) return PYRO_ERR_ARG;
  *launches = ctx->launches;
  return PYRO_OK;
}

int pyro_get_sweep_count(pyro_ctx* ctx, uint64_t* sweeps) {
  if (!ctx || !sweeps) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  unsigned long long v = 0;
  PYRO_CK(cudaMemcpyAsync(&v, ctx->d_sweep, 8, cudaMemcpyDeviceToHost, ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  *sweeps = v;
  return PYRO_OK;
}

int pyro_check_spins(pyro_ctx* ctx, float tol, long long* first_bad) {
  if (!ctx) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  const unsigned long long none = ~0ull;
  PYRO_CK(cudaMemcpyAsync(ctx->d_scratch_u64, &none, 8, cudaMemcpyHostToDevice, ctx->stream));
  launch_check_spins(ctx->d_spins, ctx->n_spins, tol, ctx->d_scratch_u64, ctx->stream);
  PYRO_CK_LAUNCH();
  unsigned long long v = none;
  PYRO_CK(cudaMemcpyAsync(&v, ctx->d_scratch_u64, 8, cudaMemcpyDeviceToHost, ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  if (first_bad) *first_bad = v == none ? -1 : (long long)v;
  if (v != none) return fail(ctx, PYRO_ERR_NAN, "check_spins: non-finite or non-unit spin");
  return PYRO_OK;
}

static int grow(pyro_ctx* ctx, double2** p, size_t* cap, size_t n) {
  if (n <= *cap && *p) return PYRO_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  cudaError_t e = cudaMalloc((void**)p, sizeof(double2) * n);
  if (e != cudaSuccess)
    return fail(ctx, e == cudaErrorMemoryAllocation ? PYRO_ERR_NOMEM : PYRO_ERR_CUDA,
                std::string("structure factor scratch: ") + cudaGetErrorString(e));
  *cap = n;
  return PYRO_OK;
}

int pyro_structure_factor(pyro_ctx* ctx, int system, int replica, int G, int stride, double* out) {
  NvtxRange nvtx_range("pyro_structure_factor");
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size() || !out)
    return fail(ctx, PYRO_ERR_ARG, "structure_factor: bad system or null pointer");
  const SysDev& sd = ctx->sys[system];
  if (G < 2 || G > 256 || (G & 1) || stride < 1 || stride > 4 * sd.L)
    return fail(ctx, PYRO_ERR_ARG, "structure_factor: need even 2 <= G <= 256, 1 <= stride <= 4L");
  if (replica < -1 || replica >= sd.n_rep)
    return fail(ctx, PYRO_ERR_ARG, "structure_factor: replica out of range");
  PYRO_CK(cudaSetDevice(ctx->device));
  const cudaStream_t st = measure_stream(ctx);
  if (!ctx->sq_ready) {
    PYRO_CK(sq_prepare());
    ctx->sq_ready = true;
  }
  const int L = sd.L;
  int g = L, b = stride;  // gcd(L, stride)
  while (b) {
    const int t = g % b;
    g = b;
    b = t;
  }
  SqParams p;
  p.L = L;
  p.G = G;
  p.stride = stride;
  p.Lf = L / g;
  p.R = std::min(G, p.Lf);
  p.residues = G > p.Lf ? 1 : 0;
  for (int s = 0; s < 16; ++s) site_pos4(s, &p.pos4[3 * s]);
  const int r0 = replica < 0 ? 0 : replica, r1 = replica < 0 ? sd.n_rep : replica + 1;
  p.inv_n_norm = 1.0 / ((double)16 * sd.L3 * (double)(r1 - r0));
  // replicas per launch sequence: at most 1 GiB of scratch (at least one replica)
  const size_t per_rep = sq_scratch_per_replica(p);
  const int batch = (int)std::max<size_t>(1, std::min<size_t>(r1 - r0, (1ull << 30) / per_rep));
  const size_t G3 = (size_t)G * G * G;
  // d_sq_s1: scratch; d_sq_tw: 4L basis-phase roots, then the Lf DFT roots;
  // d_sq_s2: the R steps (ints)
  int rc = grow(ctx, &ctx->d_sq_s1, &ctx->sq_s1, (per_rep * batch + 15) / 16);
  if (!rc) rc = grow(ctx, &ctx->d_sq_tw, &ctx->sq_tw, (size_t)4 * L + p.Lf);
  if (!rc) rc = grow(ctx, &ctx->d_sq_s2, &ctx->sq_s2, (size_t)(p.R + 3) / 4);
  if (!rc) rc = grow(ctx, (double2**)&ctx->d_sq_out, &ctx->sq_out, (G3 + 1) / 2);
  if (rc) return rc;
  std::vector<double2> tw(4 * L + p.Lf);
  for (int j = 0; j < 4 * L; ++j) {
    const double ang = -2.0 * M_PI * (double)j / (4.0 * L);
    tw[j] = make_double2(std::cos(ang), std::sin(ang));
  }
  for (int j = 0; j < p.Lf; ++j) {
    const double ang = -2.0 * M_PI * (double)j / (double)p.Lf;
    tw[4 * L + j] = make_double2(std::cos(ang), std::sin(ang));
  }
  std::vector<int> steps(p.R);
  const long long sred = stride / g;
  for (int k = 0; k < p.R; ++k) {
    const long long w = p.residues ? k : k - G / 2;
    const long long v = (sred * w) % p.Lf;
    steps[k] = (int)(v < 0 ? v + p.Lf : v);
  }
  PYRO_CK(cudaMemcpyAsync(ctx->d_sq_tw, tw.data(), sizeof(double2) * tw.size(),
                          cudaMemcpyHostToDevice, st));
  PYRO_CK(cudaMemcpyAsync(ctx->d_sq_s2, steps.data(), sizeof(int) * steps.size(),
                          cudaMemcpyHostToDevice, st));
  PYRO_CK(cudaMemsetAsync(ctx->d_sq_out, 0, sizeof(double) * G3, st));
  p.tw4 = ctx->d_sq_tw;
  for (int r = r0; r < r1; r += batch) {
    const int n = std::min(batch, r1 - r);
    launch_structure_factor(measure_spins(ctx) + sd.spin_off + (long long)r * 16 * sd.L3, n, p,
                            ctx->d_sq_tw + 4 * L, (const int*)ctx->d_sq_s2, ctx->d_sq_s1,
                            ctx->d_sq_out, st);
    PYRO_CK_LAUNCH();
  }
  PYRO_CK(cudaMemcpyAsync(out, ctx->d_sq_out, sizeof(double) * G3, cudaMemcpyDeviceToHost, st));
  PYRO_CK(cudaStreamSynchronize(st));
  return PYRO_OK;
}

}  // extern "C"
