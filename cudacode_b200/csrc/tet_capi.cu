// C-ABI of the learned tetrahedron proposal: network weights, the MH-corrected
// tetrahedron sweep, sample collection from the plain chains, and maximum-
// likelihood training with the tensor-core forward/backward kernels and Adam.
// This path has no counterpart in taillefu/cudacode.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pyro.h"
#include "../../include/pyro_math.h"
#include "ctx.h"
#include "tet_mlp.cuh"

namespace pyro {

struct TetState {
  float* d_master = nullptr;  // kMlpParams FP32 weights
  float* d_m = nullptr;       // Adam moments
  float* d_v = nullptr;
  float* d_grad = nullptr;
  unsigned char* d_image = nullptr;  // kImgBytes weight image
  unsigned long long* d_ctr = nullptr;       // tetrahedron sweeps done
  unsigned long long* d_accepted = nullptr;  // per temperature slot
  unsigned long long proposed_sweeps = 0;    // since the last reset
  double* d_loss = nullptr;
  int* d_idx = nullptr;
  int idx_cap = 0;
  float* d_feat = nullptr;  // sample ring [cap][16]
  float* d_targ = nullptr;  // [cap][12]
  long long cap = 0;
  long long written = 0;  // samples ever written
  int adam_step = 0;
  uint64_t seed = 0;
  int sweep_kernel = 2;   // 0 per pass, 1 cluster (one launch per call), 2 per pass, lane pairs
  int closure = 1;        // site 3 from its exact conditional (1) or the network's vMF (0)
  int forward_umma = 1;   // batched forward on tcgen05 (1) or mma.sync (0)
  int* d_err = nullptr;   // set by the tcgen05 forward if a wait ran out
  int cluster_max = 8;    // largest cluster size tried
  int cluster_ok = -1;    // -1 unknown, else the usable size (0: none)
};

void tet_free(pyro_ctx* ctx) {
  if (!ctx || !ctx->tet) return;
  TetState* t = ctx->tet;
  void* ptrs[] = {t->d_err,    t->d_master, t->d_m,     t->d_v,    t->d_grad, t->d_image, t->d_ctr,
                  t->d_accepted, t->d_loss, t->d_idx, t->d_feat, t->d_targ};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete t;
  ctx->tet = nullptr;
}

}  // namespace pyro

using namespace pyro;

namespace {

int need_tet(pyro_ctx* ctx) {
  if (!ctx) return PYRO_ERR_ARG;
  if (!ctx->tet) return fail(ctx, PYRO_ERR_STATE, "learned move: call pyro_tet_init first");
  return PYRO_OK;
}

bool j1_only_system(const SysDev& s) { return j1_only(s); }

// He-style initial weights from Philox (host), zero biases; the direction
// outputs start as a random linear map, log kappa near 0.
void init_weights(uint64_t seed, std::vector<float>& w) {
  w.assign(kMlpParams, 0.0f);
  auto fill = [&](int off, int fan_in, int n, uint32_t tag) {
    const float sc = std::sqrt(2.0f / (float)fan_in);
    for (int i = 0; i < n; i += 2) {
      uint32_t r[4];
      pyro_philox((uint32_t)i, tag, 0u, PYRO_PURPOSE_TET + 9, (uint32_t)(seed & 0xffffffffu),
                  (uint32_t)(seed >> 32), r);
      // Box-Muller from two uniforms in (0, 1]
      const double u1 = ((r[0] >> 8) + 1.0) / 16777216.0, u2 = (r[1] >> 8) / 16777216.0;
      const double rad = std::sqrt(-2.0 * std::log(u1));
      w[off + i] = (float)(sc * rad * std::cos(2.0 * M_PI * u2));
      if (i + 1 < n) w[off + i + 1] = (float)(sc * rad * std::sin(2.0 * M_PI * u2));
    }
  };
  fill(kOffW1, 13, kMlpIn * kMlpHidden, 1);
  fill(kOffW2, kMlpHidden, kMlpHidden * kMlpHidden, 2);
  fill(kOffW3, kMlpHidden, kMlpHidden * kMlpOut, 3);
  for (int i = kOffW3; i < kOffW3 + kMlpHidden * kMlpOut; ++i) w[i] *= 0.25f;
  for (int r = 13; r < 16; ++r)  // padded inputs are always zero
    for (int o = 0; o < kMlpHidden; ++o) w[kOffW1 + r * kMlpHidden + o] = 0.0f;
}

TetMoveParams move_params(pyro_ctx* ctx, int si, unsigned long long off) {
  const SysDev& s = ctx->sys[si];
  TetMoveParams p;
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
  p.accepted = ctx->tet->d_accepted;
  p.tet_ctr = ctx->tet->d_ctr;
  p.tet_off = off;
  p.seed_lo = (uint32_t)(ctx->seed & 0xffffffffu);
  p.seed_hi = (uint32_t)(ctx->seed >> 32);
  p.image = ctx->tet->d_image;
  p.closure = ctx->tet->closure;
  p.pdl = ctx->pdl;
  p.err = ctx->tet->d_err;
  p.trace = nullptr;
  return p;
}

}  // namespace

namespace pyro {

unsigned long long tet_counter(pyro_ctx* ctx) {
  unsigned long long v = 0;
  if (ctx->tet) cudaMemcpy(&v, ctx->tet->d_ctr, 8, cudaMemcpyDeviceToHost);
  return v;
}

void tet_set_counter(pyro_ctx* ctx, unsigned long long v) {
  if (ctx->tet) cudaMemcpy(ctx->tet->d_ctr, &v, 8, cudaMemcpyHostToDevice);
}

void tet_count_sweeps(pyro_ctx* ctx, unsigned long long n) {
  if (ctx->tet) ctx->tet->proposed_sweeps += n;
}

// Cluster size of the one-launch sweep kernel (form 1), 0 if no cluster
// can be resident (the per-pass kernels run instead); checked once.
static int tet_cluster_size(TetState* t) {
  if (t->sweep_kernel != 1) return 0;
  if (t->cluster_ok < 0) {
    t->cluster_ok = 0;
    for (int cs = t->cluster_max; cs >= 1; --cs) {
      int n_active = 0;
      if (tet_cluster_prepare(cs, &n_active) == cudaSuccess && n_active > 0) {
        t->cluster_ok = cs;
        break;
      }
      cudaGetLastError();
    }
  }
  return t->cluster_ok;
}

// Queues n tetrahedron sweeps (4 passes each) over every J1-only system;
// offsets from the device counter, which this call advances.
int queue_tet_sweeps(pyro_ctx* ctx, int n) {
  TetState* t = ctx->tet;  // sweep_kernel: 0 per pass, 1 cluster, 2 per pass with lane pairs
  const int cluster = tet_cluster_size(t);
  if (cluster > 0) {
    for (int si = 0; si < (int)ctx->sys.size(); ++si) {
      if (!j1_only_system(ctx->sys[si])) continue;
      const int cs = std::min(cluster, tet_chunks(ctx->sys[si].L3));
      PYRO_CK(launch_tet_sweep_cluster(move_params(ctx, si, 0), n, cs, ctx->stream));
    }
  } else {
    for (int k = 0; k < n; ++k)
      for (int f = 0; f < 4; ++f)
        for (int si = 0; si < (int)ctx->sys.size(); ++si) {
          if (!j1_only_system(ctx->sys[si])) continue;
          launch_tet_move(move_params(ctx, si, (unsigned long long)k), f, t->sweep_kernel,
                          ctx->stream);
          PYRO_CK_LAUNCH();
        }
  }
  tet_advance(ctx, n);
  PYRO_CK_LAUNCH();
  return PYRO_OK;
}

// n sweeps of replicas [r0, r0 + cnt) of system si on stream st (one replica
// group of the grouped cycle; the sweeps of a replica are the same updates
// in the same order as in queue_tet_sweeps). The caller advances the
// counter once for all groups (tet_advance).
int queue_tet_group(pyro_ctx* ctx, int si, int r0, int cnt, int n, cudaStream_t st) {
  const SysDev& s = ctx->sys[si];
  if (!j1_only_system(s) || n <= 0) return PYRO_OK;
  TetState* t = ctx->tet;
  auto group = [&](unsigned long long k) {
    TetMoveParams p = move_params(ctx, si, k);
    p.spins += (long long)r0 * 16 * s.L3;
    p.n_rep = cnt;
    p.rep_global += r0;
    p.rep_key += r0;
    return p;
  };
  const int cluster = tet_cluster_size(t);
  if (cluster > 0) {
    PYRO_CK(launch_tet_sweep_cluster(group(0), n, std::min(cluster, tet_chunks(s.L3)), st));
    return PYRO_OK;
  }
  for (int k = 0; k < n; ++k)
    for (int f = 0; f < 4; ++f) {
      launch_tet_move(group((unsigned long long)k), f, t->sweep_kernel, st);
      PYRO_CK_LAUNCH();
    }
  return PYRO_OK;
}

void tet_advance(pyro_ctx* ctx, int n) {
  launch_advance(ctx->tet->d_ctr, (unsigned long long)n, ctx->stream);
}

}  // namespace pyro

extern "C" {

int pyro_tet_init(pyro_ctx* ctx, uint64_t seed, long long sample_capacity) {
  if (!ctx) return PYRO_ERR_ARG;
  if (sample_capacity < 0) return fail(ctx, PYRO_ERR_ARG, "tet_init: capacity must be >= 0");
  bool any = false;
  for (const auto& s : ctx->sys) any = any || j1_only_system(s);
  if (!any) return fail(ctx, PYRO_ERR_STATE, "tet_init: the learned move needs a J1-only system");
  PYRO_CK(cudaSetDevice(ctx->device));
  tet_free(ctx);
  TetState* t = new TetState();
  ctx->tet = t;
  t->seed = seed;
  t->cap = sample_capacity;
  PYRO_CK(cudaMalloc((void**)&t->d_master, sizeof(float) * kMlpParams));
  PYRO_CK(cudaMalloc((void**)&t->d_m, sizeof(float) * kMlpParams));
  PYRO_CK(cudaMalloc((void**)&t->d_v, sizeof(float) * kMlpParams));
  PYRO_CK(cudaMalloc((void**)&t->d_grad, sizeof(float) * kMlpParams));
  PYRO_CK(cudaMalloc((void**)&t->d_image, kImgTotal));
  PYRO_CK(cudaMalloc((void**)&t->d_err, sizeof(int)));
  PYRO_CK(cudaMemset(t->d_err, 0, sizeof(int)));
  PYRO_CK(cudaMalloc((void**)&t->d_ctr, sizeof(unsigned long long)));
  PYRO_CK(cudaMalloc((void**)&t->d_accepted, sizeof(unsigned long long) * ctx->total_temps));
  PYRO_CK(cudaMalloc((void**)&t->d_loss, sizeof(double)));
  if (t->cap > 0) {
    PYRO_CK(cudaMalloc((void**)&t->d_feat, sizeof(float) * 16 * t->cap));
    PYRO_CK(cudaMalloc((void**)&t->d_targ, sizeof(float) * 12 * t->cap));
  }
  std::vector<float> w;
  init_weights(seed, w);
  PYRO_CK(cudaMemcpy(t->d_master, w.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
  PYRO_CK(cudaMemset(t->d_m, 0, sizeof(float) * kMlpParams));
  PYRO_CK(cudaMemset(t->d_v, 0, sizeof(float) * kMlpParams));
  PYRO_CK(cudaMemset(t->d_ctr, 0, sizeof(unsigned long long)));
  PYRO_CK(cudaMemset(t->d_accepted, 0, sizeof(unsigned long long) * ctx->total_temps));
  launch_mlp_pack(t->d_master, t->d_image, ctx->stream);
  PYRO_CK_LAUNCH();
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_kernels.clear();
  return PYRO_OK;
}

int pyro_tet_set_weights(pyro_ctx* ctx, const float* w, int n) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (!w || n != kMlpParams) return fail(ctx, PYRO_ERR_ARG, "tet_set_weights: need 6288 floats");
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemcpyAsync(ctx->tet->d_master, w, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice,
                          ctx->stream));
  launch_mlp_pack(ctx->tet->d_master, ctx->tet->d_image, ctx->stream);
  PYRO_CK_LAUNCH();
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return PYRO_OK;
}

int pyro_tet_get_weights(pyro_ctx* ctx, float* w, int n) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (!w || n != kMlpParams) return fail(ctx, PYRO_ERR_ARG, "tet_get_weights: need 6288 floats");
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemcpyAsync(w, ctx->tet->d_master, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost,
                          ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  return PYRO_OK;
}

int pyro_tet_set_kernel(pyro_ctx* ctx, int cluster) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (cluster < 0 || cluster > 3) return fail(ctx, PYRO_ERR_ARG, "tet kernel option is 0..3");
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  ctx->tet->sweep_kernel = cluster;
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_kernels.clear();
  return PYRO_OK;
}

int pyro_tet_set_proposal(pyro_ctx* ctx, int kind) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (kind != 0 && kind != 1) return fail(ctx, PYRO_ERR_ARG, "tet proposal kind is 0 or 1");
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  ctx->tet->closure = kind;
  for (auto& kv : ctx->graphs) cudaGraphExecDestroy(kv.second);
  ctx->graphs.clear();
  ctx->graph_kernels.clear();
  return PYRO_OK;
}

int pyro_tet_trace_pass(pyro_ctx* ctx, int system, int corner, int form, float* records) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (system < 0 || system >= (int)ctx->sys.size() || !j1_only_system(ctx->sys[system]))
    return fail(ctx, PYRO_ERR_ARG, "tet_trace_pass: not a J1-only system");
  if (corner < 0 || corner > 3 || (form != 0 && form != 3) || !records)
    return fail(ctx, PYRO_ERR_ARG, "tet_trace_pass: corner 0..3, form 0 or 3, records");
  PYRO_CK(cudaSetDevice(ctx->device));
  const SysDev& s = ctx->sys[system];
  const size_t n = (size_t)s.n_rep * s.L3 * kTetTraceFloats;
  float* d = nullptr;
  PYRO_CK(cudaMalloc((void**)&d, sizeof(float) * n));
  TetMoveParams p = move_params(ctx, system, 0);
  p.trace = d;
  p.pdl = 0;
  launch_tet_move(p, corner, form, ctx->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(records, d, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d);
  if (e != cudaSuccess)
    return fail(ctx, PYRO_ERR_CUDA, std::string("tet_trace_pass: ") + cudaGetErrorString(e));
  int err = 0;
  PYRO_CK(cudaMemcpy(&err, ctx->tet->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(ctx->tet->d_err, 0, sizeof(int));
    return fail(ctx, PYRO_ERR_TIMEOUT,
                "tet: a tensor-core MMA of the learned move did not complete in time");
  }
  return PYRO_OK;
}

int pyro_tet_sweep(pyro_ctx* ctx, int n_sweeps) {
  NvtxRange nvtx_range("pyro_tet_sweep");
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (n_sweeps < 0) return fail(ctx, PYRO_ERR_ARG, "tet_sweep: n_sweeps must be >= 0");
  PYRO_CK(cudaSetDevice(ctx->device));
  rc = queue_tet_sweeps(ctx, n_sweeps);
  if (rc) return rc;
  ctx->tet->proposed_sweeps += (unsigned long long)n_sweeps;
  return PYRO_OK;
}

int pyro_tet_acceptance(pyro_ctx* ctx, int system, uint64_t* accepted, uint64_t* proposed) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (system < 0 || system >= (int)ctx->sys.size() || !accepted)
    return fail(ctx, PYRO_ERR_ARG, "tet_acceptance: bad system or null pointer");
  const SysDev& s = ctx->sys[system];
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemcpyAsync(accepted, ctx->tet->d_accepted + s.temp_base, 8 * s.n_temp,
                          cudaMemcpyDeviceToHost, ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  if (proposed)
    for (int t = 0; t < s.n_temp; ++t)
      proposed[t] = s.n_rep == s.n_temp ? (uint64_t)4 * s.L3 * ctx->tet->proposed_sweeps : 0;
  int err = 0;
  PYRO_CK(cudaMemcpy(&err, ctx->tet->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(ctx->tet->d_err, 0, sizeof(int));
    return fail(ctx, PYRO_ERR_TIMEOUT,
                "tet: a tensor-core MMA of the learned move did not complete in time");
  }
  return PYRO_OK;
}

int pyro_tet_reset_acceptance(pyro_ctx* ctx) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaMemsetAsync(ctx->tet->d_accepted, 0, 8 * ctx->total_temps, ctx->stream));
  ctx->tet->proposed_sweeps = 0;
  return PYRO_OK;
}

int pyro_tet_collect(pyro_ctx* ctx, int system, int stride, long long* n_written) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (system < 0 || system >= (int)ctx->sys.size() || stride < 1)
    return fail(ctx, PYRO_ERR_ARG, "tet_collect: bad system or stride");
  const SysDev& s = ctx->sys[system];
  if (!j1_only_system(s)) return fail(ctx, PYRO_ERR_STATE, "tet_collect: system is not J1-only");
  TetState* t = ctx->tet;
  if (t->cap == 0) return fail(ctx, PYRO_ERR_STATE, "tet_collect: no sample buffer (capacity 0)");
  PYRO_CK(cudaSetDevice(ctx->device));
  TetCollectParams p;
  p.spins = ctx->d_spins + s.spin_off;
  p.L = s.L;
  p.L3 = s.L3;
  p.n_rep = s.n_rep;
  p.rcpL = 1.0f / (float)s.L;
  p.rep_global = s.rep_global;
  p.temp_base = s.temp_base;
  p.J1 = s.J1;
  p.temp_of_rep = ctx->d_temp_of_rep;
  p.beta = ctx->d_beta;
  p.stride = stride;
  p.features = t->d_feat;
  p.targets = t->d_targ;
  p.cap = (int)t->cap;
  p.head = t->written % t->cap;
  launch_tet_collect(p, ctx->stream);
  PYRO_CK_LAUNCH();
  const long long n = tet_collect_count(s.L3, s.n_rep, stride);
  t->written += n;
  if (n_written) *n_written = n;
  return PYRO_OK;
}

int pyro_tet_samples(pyro_ctx* ctx, float* features, float* targets, long long max_n,
                     long long* n_out) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  TetState* t = ctx->tet;
  const long long avail = t->written < t->cap ? t->written : t->cap;
  const long long n = avail < max_n ? avail : max_n;
  PYRO_CK(cudaSetDevice(ctx->device));
  if (n > 0 && features)
    PYRO_CK(cudaMemcpyAsync(features, t->d_feat, sizeof(float) * 16 * n, cudaMemcpyDeviceToHost,
                            ctx->stream));
  if (n > 0 && targets)
    PYRO_CK(cudaMemcpyAsync(targets, t->d_targ, sizeof(float) * 12 * n, cudaMemcpyDeviceToHost,
                            ctx->stream));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  if (n_out) *n_out = n;
  return PYRO_OK;
}

int pyro_tet_train(pyro_ctx* ctx, int steps, int batch, float lr, double* mean_loss) {
  NvtxRange nvtx_range("pyro_tet_train");
  int rc = need_tet(ctx);
  if (rc) return rc;
  TetState* t = ctx->tet;
  const long long avail = t->written < t->cap ? t->written : t->cap;
  if (steps < 0 || batch < 1 || !(lr > 0.0f)) return fail(ctx, PYRO_ERR_ARG, "tet_train: bad args");
  if (avail < 1) return fail(ctx, PYRO_ERR_STATE, "tet_train: no samples collected");
  PYRO_CK(cudaSetDevice(ctx->device));
  if (t->idx_cap < batch) {
    if (t->d_idx) cudaFree(t->d_idx);
    t->d_idx = nullptr;
    PYRO_CK(cudaMalloc((void**)&t->d_idx, sizeof(int) * batch));
    t->idx_cap = batch;
  }
  double last = 0.0;
  for (int k = 0; k < steps; ++k) {
    ++t->adam_step;
    launch_draw_batch(t->d_idx, batch, avail, (uint32_t)(t->seed & 0xffffffffu),
                      (uint32_t)(t->seed >> 32), (uint32_t)t->adam_step, ctx->stream);
    PYRO_CK(cudaMemsetAsync(t->d_grad, 0, sizeof(float) * kMlpParams, ctx->stream));
    PYRO_CK(cudaMemsetAsync(t->d_loss, 0, sizeof(double), ctx->stream));
    launch_mlp_gradient(t->d_feat, t->d_targ, t->d_idx, batch, t->d_image, t->d_grad, t->d_loss,
                        ctx->stream);
    PYRO_CK_LAUNCH();
    launch_adam(t->d_master, t->d_m, t->d_v, t->d_grad, kMlpParams, lr, 0.9f, 0.999f, 1e-8f,
                1.0f / (float)batch, t->adam_step, ctx->stream);
    PYRO_CK_LAUNCH();
    launch_mlp_pack(t->d_master, t->d_image, ctx->stream);
    PYRO_CK_LAUNCH();
  }
  if (mean_loss)
    PYRO_CK(cudaMemcpyAsync(&last, t->d_loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  // the move kernels start copying the weight image before their dependency
  // wait: no move may be queued behind the pack kernel
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  if (mean_loss) *mean_loss = last / (double)batch;
  return PYRO_OK;
}

int pyro_tet_set_forward(pyro_ctx* ctx, int tensor_memory) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (tensor_memory != 0 && tensor_memory != 1)
    return fail(ctx, PYRO_ERR_ARG, "tet_set_forward: 0 (mma.sync) or 1 (tcgen05)");
  ctx->tet->forward_umma = tensor_memory;
  return PYRO_OK;
}

// Network outputs of n device-resident feature rows on the chosen kernel.
static int tet_forward_queue(pyro_ctx* ctx, const float* d_in, int n, float* d_out) {
  TetState* t = ctx->tet;
  if (t->forward_umma) {
    PYRO_CK(launch_umma_forward(d_in, n, t->d_image, d_out, t->d_err, ctx->stream));
  } else {
    launch_mlp_forward(d_in, n, t->d_image, d_out, ctx->stream);
    PYRO_CK_LAUNCH();
  }
  ctx->launches += 1;
  return PYRO_OK;
}

static int tet_forward_check(pyro_ctx* ctx) {
  TetState* t = ctx->tet;
  if (!t->forward_umma || !t->d_err) return PYRO_OK;
  int err = 0;
  PYRO_CK(cudaMemcpy(&err, t->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    cudaMemset(t->d_err, 0, sizeof(int));
    return fail(ctx, PYRO_ERR_TIMEOUT, "tet_forward: a tensor-core MMA did not complete in time");
  }
  return PYRO_OK;
}

int pyro_tet_forward_device(pyro_ctx* ctx, const float* dev_features, int n, float* dev_out16) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (!dev_features || !dev_out16 || n < 1) return fail(ctx, PYRO_ERR_ARG, "tet_forward: bad args");
  PYRO_CK(cudaSetDevice(ctx->device));
  return tet_forward_queue(ctx, dev_features, n, dev_out16);
}

// Test paths: host features in, host outputs / gradients out.
int pyro_tet_forward(pyro_ctx* ctx, const float* features, int n, float* out) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (!features || !out || n < 1) return fail(ctx, PYRO_ERR_ARG, "tet_forward: bad args");
  PYRO_CK(cudaSetDevice(ctx->device));
  float *d_in = nullptr, *d_out = nullptr;
  PYRO_CK(cudaMalloc((void**)&d_in, sizeof(float) * 16 * n));
  cudaError_t e = cudaMalloc((void**)&d_out, sizeof(float) * 16 * n);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_in, features, sizeof(float) * 16 * n, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) {
    rc = tet_forward_queue(ctx, d_in, n, d_out);
    if (rc) {
      cudaFree(d_in);
      cudaFree(d_out);
      return rc;
    }
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, d_out, sizeof(float) * 16 * n, cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_in);
  if (d_out) cudaFree(d_out);
  if (e != cudaSuccess) return fail(ctx, PYRO_ERR_CUDA, std::string("tet_forward: ") + cudaGetErrorString(e));
  return tet_forward_check(ctx);
}

int pyro_tet_gradient(pyro_ctx* ctx, const float* features, const float* targets, int n,
                      float* grad, double* loss_sum) {
  int rc = need_tet(ctx);
  if (rc) return rc;
  if (!features || !targets || !grad || n < 1) return fail(ctx, PYRO_ERR_ARG, "tet_gradient: bad args");
  PYRO_CK(cudaSetDevice(ctx->device));
  float *d_f = nullptr, *d_t = nullptr;
  PYRO_CK(cudaMalloc((void**)&d_f, sizeof(float) * 16 * n));
  cudaError_t e = cudaMalloc((void**)&d_t, sizeof(float) * 12 * n);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_f, features, sizeof(float) * 16 * n, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_t, targets, sizeof(float) * 12 * n, cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->tet->d_grad, 0, sizeof(float) * kMlpParams, ctx->stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(ctx->tet->d_loss, 0, sizeof(double), ctx->stream);
  if (e == cudaSuccess) {
    launch_mlp_gradient(d_f, d_t, nullptr, n, ctx->tet->d_image, ctx->tet->d_grad,
                        ctx->tet->d_loss, ctx->stream);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(grad, ctx->tet->d_grad, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost,
                        ctx->stream);
  double l = 0.0;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&l, ctx->tet->d_loss, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(d_f);
  if (d_t) cudaFree(d_t);
  if (e != cudaSuccess) return fail(ctx, PYRO_ERR_CUDA, std::string("tet_gradient: ") + cudaGetErrorString(e));
  if (loss_sum) *loss_sum = l;
  return PYRO_OK;
}

}  // extern "C"
