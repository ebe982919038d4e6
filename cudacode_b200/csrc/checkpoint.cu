// Checkpoint / resume and the reference's configuration files.
//
// Checkpoint: one file with the full chain state. Philox is counter-based,
// so no generator state is stored: the seed, the sweep and exchange counters
// and (if present) the learned-move counter and weights determine every
// future random number. Layout (little endian):
//   "PYROCKP1", u32 version, u32 n_systems, u64 seed, i32 renorm_every,
//   u32 has_tet, u64 sweeps, u64 tet_sweeps,
//   per system: i32 L, n_replicas, replica_offset, n_temperatures,
//               f64 J1, J2, J3, J3b,
//               u32 has_exchange, [f64 A[144], f64 f[12] if has_exchange],
//               f64 T[n_temperatures],
//               i32 temperature_of_replica[n_temperatures],
//               i32 replica_of_temperature[n_temperatures],
//               f32 cosmax[n_temperatures], u64 swap_count,
//   [f32 weights[6288] if has_tet], float4 spins of every system,
//   u64 FNV-1a checksum of all preceding bytes.
// A missing, short or corrupt file gives PYRO_ERR_IO; a file written for
// another configuration gives PYRO_ERR_ARG. The reference stores only spins
// (SaveConfigurations, Math.cu:618-658) and temperatures (SaveTemperatures,
// source absent).
//
// Configuration files: SaveConfigurations / ReadConfigurations
// (Math.cu:618-701) write, per temperature, "<prefix><k>.dat" with k = 0 for
// the highest temperature, each holding repetitions of the spins as
// consecutive (x, y, z) doubles in the reference's site order (site plane,
// then cell), appended when `append` is set.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pyro.h"
#include "ctx.h"
#include "tet_mlp.cuh"

using namespace pyro;

namespace {

const char kMagic[8] = {'P', 'Y', 'R', 'O', 'C', 'K', 'P', '1'};
const uint32_t kVersion = 2;  // 1: no exchange block (isotropic systems only)

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) {
      h ^= c[i];
      h *= 1099511628211ull;
    }
  }
};

struct Writer {
  std::vector<unsigned char> buf;
  template <typename T>
  void put(const T& v) {
    const unsigned char* c = (const unsigned char*)&v;
    buf.insert(buf.end(), c, c + sizeof(T));
  }
  void put_bytes(const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    buf.insert(buf.end(), c, c + n);
  }
};

struct Reader {
  const unsigned char* p;
  size_t n, off = 0;
  bool ok = true;
  template <typename T>
  T get() {
    T v{};
    if (off + sizeof(T) > n) {
      ok = false;
      return v;
    }
    std::memcpy(&v, p + off, sizeof(T));
    off += sizeof(T);
    return v;
  }
  bool get_bytes(void* dst, size_t k) {
    if (off + k > n) return ok = false;
    std::memcpy(dst, p + off, k);
    off += k;
    return true;
  }
};

}  // namespace

extern "C" {

int pyro_save_checkpoint(pyro_ctx* ctx, const char* path) {
  if (!ctx || !path) return PYRO_ERR_ARG;
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  Writer w;
  w.put_bytes(kMagic, 8);
  w.put(kVersion);
  w.put((uint32_t)ctx->sys.size());
  w.put((uint64_t)ctx->seed);
  w.put((int32_t)ctx->renorm_every);
  const uint32_t has_tet = ctx->tet ? 1u : 0u;
  w.put(has_tet);
  uint64_t sweeps = 0, tet_sweeps = 0;
  PYRO_CK(cudaMemcpy(&sweeps, ctx->d_sweep, 8, cudaMemcpyDeviceToHost));
  if (has_tet) tet_sweeps = tet_counter(ctx);
  w.put(sweeps);
  w.put(tet_sweeps);
  for (size_t si = 0; si < ctx->sys.size(); ++si) {
    const SysDev& s = ctx->sys[si];
    w.put((int32_t)s.L);
    w.put((int32_t)s.n_rep);
    w.put((int32_t)s.rep_global);
    w.put((int32_t)s.n_temp);
    for (int k = 0; k < 4; ++k) w.put(s.J64[k]);
    w.put((uint32_t)(s.exch >= 0 ? 1 : 0));
    if (s.exch >= 0) {
      const ExchangeDev& X = ctx->exch[s.exch];
      for (int p = 0; p < 16; ++p)
        for (int q = 0; q < 9; ++q) w.put(X.A64[p][q]);
      for (int b = 0; b < 4; ++b)
        for (int q = 0; q < 3; ++q) w.put(X.f64[b][q]);
    }
    for (double T : ctx->ladders[si]) w.put(T);
    std::vector<int> tor(s.n_temp), rot(s.n_temp);
    std::vector<float> cone(s.n_temp);
    uint64_t swaps = 0;
    PYRO_CK(cudaMemcpy(tor.data(), ctx->d_temp_of_rep + s.temp_base, 4 * s.n_temp,
                       cudaMemcpyDeviceToHost));
    PYRO_CK(cudaMemcpy(rot.data(), ctx->d_rep_of_temp + s.temp_base, 4 * s.n_temp,
                       cudaMemcpyDeviceToHost));
    PYRO_CK(cudaMemcpy(cone.data(), ctx->d_cosmax + s.temp_base, 4 * s.n_temp,
                       cudaMemcpyDeviceToHost));
    PYRO_CK(cudaMemcpy(&swaps, ctx->d_swap_count + si, 8, cudaMemcpyDeviceToHost));
    w.put_bytes(tor.data(), 4 * tor.size());
    w.put_bytes(rot.data(), 4 * rot.size());
    w.put_bytes(cone.data(), 4 * cone.size());
    w.put(swaps);
  }
  if (has_tet) {
    std::vector<float> wts(kMlpParams);
    int rc = pyro_tet_get_weights(ctx, wts.data(), kMlpParams);
    if (rc) return rc;
    w.put_bytes(wts.data(), 4 * wts.size());
  }
  const size_t spin_bytes = sizeof(float4) * (size_t)ctx->n_spins;
  const size_t head = w.buf.size();
  w.buf.resize(head + spin_bytes);
  PYRO_CK(cudaMemcpy(w.buf.data() + head, ctx->d_spins, spin_bytes, cudaMemcpyDeviceToHost));
  Fnv f;
  f.add(w.buf.data(), w.buf.size());
  w.put(f.h);
  const std::string tmp = std::string(path) + ".tmp";
  FILE* fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) return fail(ctx, PYRO_ERR_IO, std::string("save_checkpoint: cannot open ") + tmp);
  const size_t wrote = std::fwrite(w.buf.data(), 1, w.buf.size(), fp);
  const int closed = std::fclose(fp);
  if (wrote != w.buf.size() || closed != 0 || std::rename(tmp.c_str(), path) != 0)
    return fail(ctx, PYRO_ERR_IO, std::string("save_checkpoint: write failed: ") + path);
  return PYRO_OK;
}

int pyro_load_checkpoint(pyro_ctx* ctx, const char* path) {
  if (!ctx || !path) return PYRO_ERR_ARG;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) return fail(ctx, PYRO_ERR_IO, std::string("load_checkpoint: cannot open ") + path);
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof chunk, fp)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  std::fclose(fp);
  if (buf.size() < 8 + 8 || std::memcmp(buf.data(), kMagic, 8) != 0)
    return fail(ctx, PYRO_ERR_IO, "load_checkpoint: not a checkpoint file");
  Fnv f;
  f.add(buf.data(), buf.size() - 8);
  uint64_t stored;
  std::memcpy(&stored, buf.data() + buf.size() - 8, 8);
  if (stored != f.h) return fail(ctx, PYRO_ERR_IO, "load_checkpoint: checksum mismatch (corrupt)");
  Reader r{buf.data(), buf.size() - 8};
  r.off = 8;
  const uint32_t version = r.get<uint32_t>();
  const uint32_t n_sys = r.get<uint32_t>();
  const uint64_t seed = r.get<uint64_t>();
  const int32_t renorm = r.get<int32_t>();
  const uint32_t has_tet = r.get<uint32_t>();
  const uint64_t sweeps = r.get<uint64_t>();
  const uint64_t tet_sweeps = r.get<uint64_t>();
  if (!r.ok || (version != kVersion && version != 1))
    return fail(ctx, PYRO_ERR_IO, "load_checkpoint: bad header");
  if (n_sys != ctx->sys.size() || seed != ctx->seed || renorm != ctx->renorm_every)
    return fail(ctx, PYRO_ERR_ARG, "load_checkpoint: written for another configuration");
  struct SysState {
    std::vector<int> tor, rot;
    std::vector<float> cone;
    uint64_t swaps;
  };
  std::vector<SysState> st(n_sys);
  for (uint32_t si = 0; si < n_sys; ++si) {
    const SysDev& s = ctx->sys[si];
    const int L = r.get<int32_t>(), R = r.get<int32_t>(), off = r.get<int32_t>(),
              nT = r.get<int32_t>();
    double J[4];
    for (double& j : J) j = r.get<double>();
    if (!r.ok) return fail(ctx, PYRO_ERR_IO, "load_checkpoint: truncated");
    if (L != s.L || R != s.n_rep || off != s.rep_global || nT != s.n_temp)
      return fail(ctx, PYRO_ERR_ARG, "load_checkpoint: lattice or replicas differ");
    for (int k = 0; k < 4; ++k)
      if (J[k] != s.J64[k]) return fail(ctx, PYRO_ERR_ARG, "load_checkpoint: couplings differ");
    const uint32_t has_x = version >= 2 ? r.get<uint32_t>() : 0u;
    if (!r.ok) return fail(ctx, PYRO_ERR_IO, "load_checkpoint: truncated");
    if ((has_x != 0) != (s.exch >= 0))
      return fail(ctx, PYRO_ERR_ARG, "load_checkpoint: exchange matrices differ");
    if (has_x) {
      const ExchangeDev& X = ctx->exch[s.exch];
      bool same = true;
      for (int p = 0; p < 16; ++p)
        for (int q = 0; q < 9; ++q) same = (r.get<double>() == X.A64[p][q]) && same;
      for (int b = 0; b < 4; ++b)
        for (int q = 0; q < 3; ++q) same = (r.get<double>() == X.f64[b][q]) && same;
      if (!r.ok) return fail(ctx, PYRO_ERR_IO, "load_checkpoint: truncated");
      if (!same) return fail(ctx, PYRO_ERR_ARG, "load_checkpoint: exchange matrices differ");
    }
    for (int t = 0; t < nT; ++t)
      if (r.get<double>() != ctx->ladders[si][t])
        return fail(ctx, PYRO_ERR_ARG, "load_checkpoint: temperature ladder differs");
    st[si].tor.resize(nT);
    st[si].rot.resize(nT);
    st[si].cone.resize(nT);
    r.get_bytes(st[si].tor.data(), 4 * nT);
    r.get_bytes(st[si].rot.data(), 4 * nT);
    r.get_bytes(st[si].cone.data(), 4 * nT);
    st[si].swaps = r.get<uint64_t>();
    if (!r.ok) return fail(ctx, PYRO_ERR_IO, "load_checkpoint: truncated");
  }
  std::vector<float> wts;
  if (has_tet) {
    wts.resize(kMlpParams);
    if (!r.get_bytes(wts.data(), 4 * wts.size()))
      return fail(ctx, PYRO_ERR_IO, "load_checkpoint: truncated");
  }
  const size_t spin_bytes = sizeof(float4) * (size_t)ctx->n_spins;
  if (r.n - r.off != spin_bytes)
    return fail(ctx, PYRO_ERR_IO, "load_checkpoint: spin payload has the wrong size");
  // All checks passed: install the state.
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  PYRO_CK(cudaMemcpy(ctx->d_spins, buf.data() + r.off, spin_bytes, cudaMemcpyHostToDevice));
  PYRO_CK(cudaMemcpy(ctx->d_sweep, &sweeps, 8, cudaMemcpyHostToDevice));
  ctx->h_sweep = sweeps;
  for (uint32_t si = 0; si < n_sys; ++si) {
    const SysDev& s = ctx->sys[si];
    PYRO_CK(cudaMemcpy(ctx->d_temp_of_rep + s.temp_base, st[si].tor.data(), 4 * s.n_temp,
                       cudaMemcpyHostToDevice));
    PYRO_CK(cudaMemcpy(ctx->d_rep_of_temp + s.temp_base, st[si].rot.data(), 4 * s.n_temp,
                       cudaMemcpyHostToDevice));
    PYRO_CK(cudaMemcpy(ctx->d_cosmax + s.temp_base, st[si].cone.data(), 4 * s.n_temp,
                       cudaMemcpyHostToDevice));
    PYRO_CK(cudaMemcpy(ctx->d_swap_count + si, &st[si].swaps, 8, cudaMemcpyHostToDevice));
  }
  if (has_tet) {
    if (!ctx->tet) {
      int rc = pyro_tet_init(ctx, 0, 0);
      if (rc) return rc;
    }
    int rc = pyro_tet_set_weights(ctx, wts.data(), kMlpParams);
    if (rc) return rc;
    tet_set_counter(ctx, tet_sweeps);
  }
  return PYRO_OK;
}

int pyro_save_configurations(pyro_ctx* ctx, int system, const char* prefix, int append) {
  if (!ctx || !prefix) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "save_configurations: bad system");
  const SysDev& s = ctx->sys[system];
  if (s.n_rep != s.n_temp)
    return fail(ctx, PYRO_ERR_STATE, "save_configurations: context holds part of the ladder");
  const size_t n = (size_t)16 * s.L3;
  std::vector<float4> spins((size_t)s.n_rep * n);
  std::vector<int> rot(s.n_temp);
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  PYRO_CK(cudaMemcpy(spins.data(), ctx->d_spins + s.spin_off, sizeof(float4) * spins.size(),
                     cudaMemcpyDeviceToHost));
  PYRO_CK(cudaMemcpy(rot.data(), ctx->d_rep_of_temp + s.temp_base, 4 * s.n_temp,
                     cudaMemcpyDeviceToHost));
  std::vector<double> aos(3 * n);
  for (int k = 0; k < s.n_temp; ++k) {
    const int t = s.n_temp - 1 - k;  // k = 0: highest temperature
    const int rep = rot[t];
    for (size_t i = 0; i < n; ++i) {
      const float4 v = spins[(size_t)rep * n + i];
      aos[3 * i] = v.x;
      aos[3 * i + 1] = v.y;
      aos[3 * i + 2] = v.z;
    }
    const std::string name = std::string(prefix) + std::to_string(k) + ".dat";
    FILE* fp = std::fopen(name.c_str(), append ? "ab" : "wb");
    if (!fp) return fail(ctx, PYRO_ERR_IO, "save_configurations: cannot open " + name);
    const size_t wrote = std::fwrite(aos.data(), sizeof(double), aos.size(), fp);
    if (std::fclose(fp) != 0 || wrote != aos.size())
      return fail(ctx, PYRO_ERR_IO, "save_configurations: write failed: " + name);
  }
  return PYRO_OK;
}

int pyro_read_configurations(pyro_ctx* ctx, int system, const char* prefix, int repetition) {
  if (!ctx || !prefix || repetition < 0) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "read_configurations: bad system");
  const SysDev& s = ctx->sys[system];
  if (s.n_rep != s.n_temp)
    return fail(ctx, PYRO_ERR_STATE, "read_configurations: context holds part of the ladder");
  const size_t n = (size_t)16 * s.L3;
  std::vector<float4> spins((size_t)s.n_rep * n);
  std::vector<int> rot(s.n_temp);
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  PYRO_CK(cudaMemcpy(rot.data(), ctx->d_rep_of_temp + s.temp_base, 4 * s.n_temp,
                     cudaMemcpyDeviceToHost));
  std::vector<double> aos(3 * n);
  for (int k = 0; k < s.n_temp; ++k) {
    const std::string name = std::string(prefix) + std::to_string(k) + ".dat";
    FILE* fp = std::fopen(name.c_str(), "rb");
    if (!fp) return fail(ctx, PYRO_ERR_IO, "read_configurations: cannot open " + name);
    const bool seek_ok =
        std::fseek(fp, (long)(sizeof(double) * aos.size() * (size_t)repetition), SEEK_SET) == 0;
    const size_t got = seek_ok ? std::fread(aos.data(), sizeof(double), aos.size(), fp) : 0;
    std::fclose(fp);
    if (got != aos.size())
      return fail(ctx, PYRO_ERR_IO, "read_configurations: " + name + " is too short");
    const int rep = rot[s.n_temp - 1 - k];
    for (size_t i = 0; i < n; ++i)
      spins[(size_t)rep * n + i] =
          make_float4((float)aos[3 * i], (float)aos[3 * i + 1], (float)aos[3 * i + 2], 0.0f);
  }
  PYRO_CK(cudaMemcpy(ctx->d_spins + s.spin_off, spins.data(), sizeof(float4) * spins.size(),
                     cudaMemcpyHostToDevice));
  return PYRO_OK;
}

}  // extern "C"
