// Bond-dependent nearest-neighbour exchange and Zeeman field: the
// reference's anisotropic pyrochlore model in this engine's convention.
//
// The reference's Hamiltonian (TotalEnergy, Pyrochlore.cu:468-523, with the
// spin-1/2 factor S^2 = 1/4 and unit vectors n) is
//   E = -(1/4) sum_<ij> n_i^T C[b_i][b_j] n_j - (1/2) sum_i F[b_i] . n_i,
// C the 3x3 bond matrices of couplings_const (Pyrochlore.cu:169-184) and F
// the site fields of InitializeMagneticField (Pyrochlore.cu:414-450). Here
//   E = sum_<ij> n_i^T A[b_i][b_j] n_j - sum_i f[b_i] . n_i,
// so A = -C / 4 and f = F / 2 reproduce the reference's energies (and
// temperatures) exactly.
//
// The bond matrices are generated from the lattice symmetry rather than
// copied: for sublattices a != b with basis vectors B_a, B_b (units a/4,
// tetrahedron centre c = (1/2, 1/2, 1/2)), d = B_b - B_a has two components
// +-1 (axes i, j) and a zero one (axis k); m = the unit vector along axis k
// pointing from c to the bond midpoint. Then
//   C = -J1 (e_i e_i^T + e_j e_j^T) - J2 e_k e_k^T
//       - J3 d_i d_j (e_i e_j^T + e_j e_i^T) + [D]_x,   D = J4 (m x d),
// [D]_x the antisymmetric matrix with entries eps_abg D_g (a
// Dzyaloshinskii-Moriya term). The g-tensor of sublattice b is
// g_b = gxy I + (gz - gxy) z_b z_b^T, z_b = (B_b - c) / |B_b - c| its local
// <111> axis, and F_b = mu_B g_b B (B in tesla, mu_B = 0.0578838261305
// meV/T). Tests compare both against the reference's literal tables.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/pyro.h"
#include "ctx.h"

using namespace pyro;

namespace {

const int kBasis[4][3] = {{0, 0, 0}, {1, 1, 0}, {0, 1, 1}, {1, 0, 1}};  // units a/4

void bond_matrix(int a, int b, double J1, double J2, double J3, double J4, double C[3][3]) {
  int d[3], k = -1;
  for (int q = 0; q < 3; ++q) {
    d[q] = kBasis[b][q] - kBasis[a][q];
    if (d[q] == 0) k = q;
  }
  const int i = (k + 1) % 3, j = (k + 2) % 3;
  // m: +-e_k, the side of the bond midpoint relative to the centre
  double m[3] = {0.0, 0.0, 0.0};
  m[k] = kBasis[a][k] == 1 ? 1.0 : -1.0;
  const double D[3] = {J4 * (m[1] * d[2] - m[2] * d[1]), J4 * (m[2] * d[0] - m[0] * d[2]),
                       J4 * (m[0] * d[1] - m[1] * d[0])};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) C[r][c] = 0.0;
  C[i][i] = -J1;
  C[j][j] = -J1;
  C[k][k] = -J2;
  C[i][j] = C[j][i] = -J3 * d[i] * d[j];
  // [D]_x: entry (r, c) = eps_{r c g} D_g
  C[0][1] += D[2];
  C[1][0] -= D[2];
  C[1][2] += D[0];
  C[2][1] -= D[0];
  C[2][0] += D[1];
  C[0][2] -= D[1];
}

constexpr int kMagThreads = 256;
constexpr int kMagSitesPerThread = 8;

// FP64 sum of the spins of one site plane (one cubic-cell site s, so one
// sublattice s & 3) of one replica over a chunk of cells: block (chunk, s,
// replica) -> partials[((rep * 16 + s) * chunks + chunk) * 3 + k].
__global__ void __launch_bounds__(kMagThreads) plane_sum_kernel(const float4* __restrict__ spins,
                                                                int L3, int chunks,
                                                                double* partials) {
  const int chunk = blockIdx.x, s = blockIdx.y, rep = blockIdx.z;
  const float4* plane = spins + ((long long)rep * 16 + s) * L3;
  double x = 0.0, y = 0.0, z = 0.0;
  for (int k = 0; k < kMagSitesPerThread; ++k) {
    const int c = (chunk * kMagSitesPerThread + k) * kMagThreads + threadIdx.x;
    if (c < L3) {
      const float4 v = __ldg(plane + c);
      x += v.x;
      y += v.y;
      z += v.z;
    }
  }
  __shared__ double red[3][kMagThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_down_sync(0xffffffffu, x, o);
    y += __shfl_down_sync(0xffffffffu, y, o);
    z += __shfl_down_sync(0xffffffffu, z, o);
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = x;
    red[1][w] = y;
    red[2][w] = z;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int q = 0; q < kMagThreads / 32; ++q) {
      sx += red[0][q];
      sy += red[1][q];
      sz += red[2][q];
    }
    double* o = partials + (((long long)rep * 16 + s) * chunks + chunk) * 3;
    o[0] = sx;
    o[1] = sy;
    o[2] = sz;
  }
}

// out[(rep * 4 + b) * 3 + k]: planes b, 4 + b, 8 + b, 12 + b and their chunks
// in a fixed order (deterministic).
__global__ void sublattice_finalise_kernel(const double* __restrict__ partials, int n_rep,
                                           int chunks, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // (rep, b, k)
  if (i >= n_rep * 12) return;
  const int rep = i / 12, b = (i / 3) % 4, k = i % 3;
  double v = 0.0;
  for (int f = 0; f < 4; ++f)
    for (int c = 0; c < chunks; ++c)
      v += partials[(((long long)rep * 16 + 4 * f + b) * chunks + c) * 3 + k];
  out[i] = v;
}

bool finite_all(const double* v, int n) {
  for (int q = 0; q < n; ++q)
    if (!std::isfinite(v[q])) return false;
  return true;
}

}  // namespace

extern "C" {

int pyro_reference_exchange(double J1, double J2, double J3, double J4, double* exchange144) {
  if (!exchange144) return PYRO_ERR_ARG;
  std::memset(exchange144, 0, sizeof(double) * 144);
  for (int a = 0; a < 4; ++a)
    for (int b = 0; b < 4; ++b) {
      if (a == b) continue;
      double C[3][3];
      bond_matrix(a, b, J1, J2, J3, J4, C);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) exchange144[(4 * a + b) * 9 + 3 * r + c] = -0.25 * C[r][c];
    }
  return PYRO_OK;
}

int pyro_reference_field(double gxy, double gz, const double* B3, double* field12) {
  if (!B3 || !field12) return PYRO_ERR_ARG;
  const double mu_b = 0.0578838261305;  // meV / T
  for (int b = 0; b < 4; ++b) {
    double z[3];
    for (int q = 0; q < 3; ++q) z[q] = (kBasis[b][q] - 0.5) / std::sqrt(0.75);
    for (int r = 0; r < 3; ++r) {
      double v = 0.0;
      for (int c = 0; c < 3; ++c) v += ((r == c ? gxy : 0.0) + (gz - gxy) * z[r] * z[c]) * B3[c];
      field12[3 * b + r] = 0.5 * mu_b * v;
    }
  }
  return PYRO_OK;
}

int pyro_set_exchange(pyro_ctx* ctx, int system, const double* exchange144,
                      const double* field12) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "set_exchange: no such system");
  if (!exchange144 && field12)
    return fail(ctx, PYRO_ERR_ARG, "set_exchange: a field needs bond matrices");
  if (exchange144) {
    if (!finite_all(exchange144, 144) || (field12 && !finite_all(field12, 12)))
      return fail(ctx, PYRO_ERR_ARG, "set_exchange: non-finite value");
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        if (a == b) continue;
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) {
            const double x = exchange144[(4 * a + b) * 9 + 3 * r + c];
            const double y = exchange144[(4 * b + a) * 9 + 3 * c + r];
            if (std::fabs(x - y) > 1e-12 * (1.0 + std::fabs(x)))
              return fail(ctx, PYRO_ERR_ARG,
                          "set_exchange: A[b][a] must be the transpose of A[a][b]");
          }
      }
  }
  PYRO_CK(cudaSetDevice(ctx->device));
  PYRO_CK(cudaStreamSynchronize(ctx->stream));
  SysDev& s = ctx->sys[system];
  if (exchange144) {
    ExchangeDev X;
    std::memset(&X, 0, sizeof X);
    for (int a = 0; a < 4; ++a)
      for (int b = 0; b < 4; ++b) {
        if (a == b) continue;  // same-sublattice pairs are never nearest neighbours
        for (int q = 0; q < 9; ++q) {
          X.A64[4 * a + b][q] = exchange144[(4 * a + b) * 9 + q];
          X.A[4 * a + b][q] = (float)X.A64[4 * a + b][q];
        }
      }
    if (field12)
      for (int b = 0; b < 4; ++b)
        for (int q = 0; q < 3; ++q) {
          X.f64[b][q] = field12[3 * b + q];
          X.f[b][q] = (float)X.f64[b][q];
        }
    if (s.exch < 0) {
      s.exch = (int)ctx->exch.size();
      ctx->exch.push_back(X);
    } else {
      ctx->exch[s.exch] = X;
    }
  } else {
    s.exch = -1;  // its entry of ctx->exch stays, unused
  }
  if (ctx->d_exch) PYRO_CK(cudaFree(ctx->d_exch));
  ctx->d_exch = nullptr;
  if (!ctx->exch.empty()) {
    PYRO_CK(cudaMalloc((void**)&ctx->d_exch, sizeof(ExchangeDev) * ctx->exch.size()));
    PYRO_CK(cudaMemcpy(ctx->d_exch, ctx->exch.data(), sizeof(ExchangeDev) * ctx->exch.size(),
                       cudaMemcpyHostToDevice));
  }
  PYRO_CK(cudaMemcpy(ctx->d_sys, ctx->sys.data(), sizeof(SysDev) * ctx->sys.size(),
                     cudaMemcpyHostToDevice));
  return rebuild_schedule(ctx);
}

int pyro_reference_gtensor(double gxy, double gz, double* g36) {
  if (!g36) return PYRO_ERR_ARG;
  for (int b = 0; b < 4; ++b) {
    double z[3];
    for (int q = 0; q < 3; ++q) z[q] = (kBasis[b][q] - 0.5) / std::sqrt(0.75);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        g36[9 * b + 3 * r + c] = (r == c ? gxy : 0.0) + (gz - gxy) * z[r] * z[c];
  }
  return PYRO_OK;
}

int pyro_sublattice_magnetisation(pyro_ctx* ctx, int system, double* out) {
  NvtxRange nvtx_range("pyro_sublattice_magnetisation");
  if (!ctx || !out) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "sublattice_magnetisation: no such system");
  const SysDev& s = ctx->sys[system];
  const int chunks = (s.L3 + kMagThreads * kMagSitesPerThread - 1) / (kMagThreads * kMagSitesPerThread);
  const size_t need = (size_t)s.n_rep * 16 * chunks * 3 + (size_t)s.n_rep * 12;
  PYRO_CK(cudaSetDevice(ctx->device));
  if (need > ctx->submag_cap || !ctx->d_submag) {
    if (ctx->d_submag) PYRO_CK(cudaFree(ctx->d_submag));
    ctx->d_submag = nullptr;
    ctx->submag_cap = 0;
    const cudaError_t e = cudaMalloc((void**)&ctx->d_submag, sizeof(double) * need);
    if (e != cudaSuccess)
      return fail(ctx, e == cudaErrorMemoryAllocation ? PYRO_ERR_NOMEM : PYRO_ERR_CUDA,
                  std::string("sublattice_magnetisation scratch: ") + cudaGetErrorString(e));
    ctx->submag_cap = need;
  }
  double* partials = ctx->d_submag;
  double* d_out = ctx->d_submag + (size_t)s.n_rep * 16 * chunks * 3;
  const cudaStream_t st = measure_stream(ctx);
  plane_sum_kernel<<<dim3(chunks, 16, s.n_rep), kMagThreads, 0, st>>>(
      measure_spins(ctx) + s.spin_off, s.L3, chunks, partials);
  PYRO_CK_LAUNCH();
  sublattice_finalise_kernel<<<(s.n_rep * 12 + 127) / 128, 128, 0, st>>>(partials, s.n_rep,
                                                                       chunks, d_out);
  PYRO_CK_LAUNCH();
  ctx->launches += 2;
  PYRO_CK(cudaMemcpyAsync(out, d_out, sizeof(double) * 12 * s.n_rep, cudaMemcpyDeviceToHost, st));
  PYRO_CK(cudaStreamSynchronize(st));
  return PYRO_OK;
}

int pyro_get_exchange(pyro_ctx* ctx, int system, double* exchange144, double* field12,
                      int* is_set) {
  if (!ctx) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "get_exchange: no such system");
  const SysDev& s = ctx->sys[system];
  if (is_set) *is_set = s.exch >= 0 ? 1 : 0;
  if (s.exch < 0) return PYRO_OK;
  const ExchangeDev& X = ctx->exch[s.exch];
  if (exchange144)
    for (int p = 0; p < 16; ++p)
      for (int q = 0; q < 9; ++q) exchange144[9 * p + q] = X.A64[p][q];
  if (field12)
    for (int b = 0; b < 4; ++b)
      for (int q = 0; q < 3; ++q) field12[3 * b + q] = X.f64[b][q];
  return PYRO_OK;
}

}  // extern "C"
