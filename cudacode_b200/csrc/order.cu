// Order parameters of the pyrochlore spin configurations, FP64, one pass
// over the lattice per call.
//
// Per replica (sums over the whole lattice; the reference computes the same
// quantities per cubic cell and reduces them over cells):
//   [0..11]  irreducible-representation components (Measurement,
//            Pyrochlore.cu:526-641): linear combinations of the four
//            sublattice magnetisations M_b = sum of S over sublattice b,
//            m_r = sum_b c_rb . M_b with the table kIrrep below;
//   [12..17] quadrupole sum_i (S_i^a S_i^b - delta_ab / 3), ab = xx, xy, xz,
//            yy, yz, zz (_CudaQuadrupolarOrder, Math.cu:335-372);
//   [18]     monopole density sum_cells (1/4) sum_{up-tetrahedra t of the
//            cell} |sum_b a_b . S_{4t+b}| (CudaCalculateMonopoleSquare,
//            Math.cu:386-476);
//   [19]     sum_i |a_b . S_i| / sqrt 3 (CudaCalculateAbsSz, Math.cu:478-510);
// with a_b the sublattice axes (1,1,1), (-1,-1,1), (1,-1,-1), (-1,1,-1)
// (unnormalised, the reference's orientation of the local <111> axes).
// The Ising map (CudaCalculateIsingConf, Math.cu:513-541) gives per cell a
// 16-bit mask, bit 4t + b set where a_b . S < 0.
//
// The irrep table has to equal the reference's definition of its order
// parameters, so it is restated here in terms of the local frames: row 0
// (A2) a_b / sqrt 3; rows 1, 2 (E) the local x and y axes
// (-2,1,1), (2,-1,1), (-2,-1,-1), (2,1,-1) / sqrt 6 and (0,-1,1), (0,1,1),
// (0,1,-1), (0,-1,-1) / sqrt 2; rows 6..8 the uniform magnetisation; rows
// 3..5 and 9..11 the two remaining three-component irreps, each component
// a pattern of +-1/sqrt 2 on two axes.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/pyro.h"
#include "ctx.h"

using namespace pyro;

namespace {

constexpr int kOrdThreads = 256;
constexpr int kOrdCellsPerThread = 2;
constexpr int kOrdQ = 20;      // per-replica outputs
constexpr int kOrdPart = 20;   // per-block partials: 12 sublattice sums, 6 quadrupole, 2

__device__ __forceinline__ double warp_sum_o(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block (chunk, replica): cells [chunk * per_block, ...). Partials layout
// [rep][chunk][kOrdPart]: M_b (12), Q (6), monopole, |Sz|.
__global__ void __launch_bounds__(kOrdThreads) order_partials_kernel(const float4* __restrict__ spins,
                                                                     int L3, int chunks,
                                                                     double* partials) {
  const int chunk = blockIdx.x, rep = blockIdx.y;
  const float4* rb = spins + (long long)rep * 16 * L3;
  const double ax[4][3] = {{1, 1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, 1, -1}};
  double acc[kOrdPart];
#pragma unroll
  for (int q = 0; q < kOrdPart; ++q) acc[q] = 0.0;
  for (int k = 0; k < kOrdCellsPerThread; ++k) {
    const int cell = (chunk * kOrdCellsPerThread + k) * kOrdThreads + threadIdx.x;
    if (cell >= L3) break;
    double mono = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      double charge = 0.0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const float4 v = __ldg(rb + (4 * t + b) * L3 + cell);
        const double x = v.x, y = v.y, z = v.z;
        acc[3 * b] += x;
        acc[3 * b + 1] += y;
        acc[3 * b + 2] += z;
        acc[12] += x * x - 1.0 / 3.0;
        acc[13] += x * y;
        acc[14] += x * z;
        acc[15] += y * y - 1.0 / 3.0;
        acc[16] += y * z;
        acc[17] += z * z - 1.0 / 3.0;
        const double p = x * ax[b][0] + y * ax[b][1] + z * ax[b][2];
        charge += p;
        acc[19] += fabs(p);
      }
      mono += fabs(charge);
    }
    acc[18] += 0.25 * mono;
  }
  __shared__ double red[kOrdPart][kOrdThreads / 32];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < kOrdPart; ++q) {
    const double v = warp_sum_o(acc[q]);
    if (lane == 0) red[q][w] = v;
  }
  __syncthreads();
  if (threadIdx.x < kOrdPart) {
    double s = 0.0;
    for (int i = 0; i < kOrdThreads / 32; ++i) s += red[threadIdx.x][i];
    partials[((long long)rep * chunks + chunk) * kOrdPart + threadIdx.x] = s;
  }
}

// Fixed-order sum of the partials of each replica.
__global__ void order_finalise_kernel(const double* __restrict__ partials, int n_rep, int chunks,
                                      double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_rep * kOrdPart) return;
  const int rep = i / kOrdPart, q = i % kOrdPart;
  double v = 0.0;
  for (int c = 0; c < chunks; ++c) v += partials[((long long)rep * chunks + c) * kOrdPart + q];
  out[i] = v;
}

__global__ void ising_kernel(const float4* __restrict__ spins, int L3, int* out) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= L3) return;
  const float ax[4][3] = {{1, 1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, 1, -1}};
  int mask = 0;
  for (int s = 0; s < 16; ++s) {
    const float4 v = __ldg(spins + s * L3 + cell);
    const double p = (double)v.x * ax[s & 3][0] + (double)v.y * ax[s & 3][1] +
                     (double)v.z * ax[s & 3][2];
    mask |= (p < 0.0 ? 1 : 0) << s;
  }
  out[cell] = mask;
}

// Irrep table: kIrrep[r][b] = coefficient vector of M_b in component r, in
// units of the row's normalisation kNorm[r].
const int kIrrep[12][4][3] = {
    {{1, 1, 1}, {-1, -1, 1}, {1, -1, -1}, {-1, 1, -1}},        // A2
    {{-2, 1, 1}, {2, -1, 1}, {-2, -1, -1}, {2, 1, -1}},        // E, local x
    {{0, -1, 1}, {0, 1, 1}, {0, 1, -1}, {0, -1, -1}},          // E, local y
    {{0, -1, 1}, {0, -1, -1}, {0, 1, -1}, {0, 1, 1}},          // T (first), x
    {{1, 0, -1}, {1, 0, 1}, {-1, 0, -1}, {-1, 0, 1}},          //            y
    {{-1, 1, 0}, {1, -1, 0}, {1, 1, 0}, {-1, -1, 0}},          //            z
    {{1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}},              // uniform, x
    {{0, 1, 0}, {0, 1, 0}, {0, 1, 0}, {0, 1, 0}},              //          y
    {{0, 0, 1}, {0, 0, 1}, {0, 0, 1}, {0, 0, 1}},              //          z
    {{0, -1, -1}, {0, -1, 1}, {0, 1, 1}, {0, 1, -1}},          // T (second), x
    {{-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {1, 0, 1}},          //             y
    {{-1, -1, 0}, {1, 1, 0}, {1, -1, 0}, {-1, 1, 0}},          //             z
};

double irrep_norm(int r) {
  if (r == 0) return 1.0 / std::sqrt(3.0);
  if (r == 1) return 1.0 / std::sqrt(6.0);
  if (r >= 6 && r <= 8) return 1.0;
  return 1.0 / std::sqrt(2.0);
}

int grow_scratch(pyro_ctx* ctx, size_t need) {
  if (need <= ctx->order_cap && ctx->d_order) return PYRO_OK;
  if (ctx->d_order) PYRO_CK(cudaFree(ctx->d_order));
  ctx->d_order = nullptr;
  ctx->order_cap = 0;
  const cudaError_t e = cudaMalloc((void**)&ctx->d_order, need);
  if (e != cudaSuccess)
    return fail(ctx, e == cudaErrorMemoryAllocation ? PYRO_ERR_NOMEM : PYRO_ERR_CUDA,
                std::string("order parameter scratch: ") + cudaGetErrorString(e));
  ctx->order_cap = need;
  return PYRO_OK;
}

}  // namespace

extern "C" {

int pyro_order_parameters(pyro_ctx* ctx, int system, double* out) {
  NvtxRange nvtx_range("pyro_order_parameters");
  if (!ctx || !out) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "order_parameters: no such system");
  const SysDev& s = ctx->sys[system];
  PYRO_CK(cudaSetDevice(ctx->device));
  const int chunks = (s.L3 + kOrdThreads * kOrdCellsPerThread - 1) / (kOrdThreads * kOrdCellsPerThread);
  const size_t n_part = (size_t)s.n_rep * chunks * kOrdPart;
  const size_t n_out = (size_t)s.n_rep * kOrdPart;
  int rc = grow_scratch(ctx, sizeof(double) * (n_part + n_out));
  if (rc) return rc;
  double* part = reinterpret_cast<double*>(ctx->d_order);
  double* d_out = part + n_part;
  const cudaStream_t st = measure_stream(ctx);
  order_partials_kernel<<<dim3(chunks, s.n_rep), kOrdThreads, 0, st>>>(
      measure_spins(ctx) + s.spin_off, s.L3, chunks, part);
  PYRO_CK_LAUNCH();
  order_finalise_kernel<<<(int)((n_out + 127) / 128), 128, 0, st>>>(part, s.n_rep, chunks, d_out);
  PYRO_CK_LAUNCH();
  ctx->launches += 2;
  std::string buf;
  buf.resize(sizeof(double) * n_out);
  double* h = reinterpret_cast<double*>(&buf[0]);
  PYRO_CK(cudaMemcpyAsync(h, d_out, sizeof(double) * n_out, cudaMemcpyDeviceToHost, st));
  PYRO_CK(cudaStreamSynchronize(st));
  for (int r = 0; r < s.n_rep; ++r) {
    const double* p = h + (size_t)r * kOrdPart;
    double* o = out + (size_t)r * kOrdQ;
    for (int q = 0; q < 12; ++q) {
      double v = 0.0;
      for (int b = 0; b < 4; ++b)
        for (int k = 0; k < 3; ++k) v += kIrrep[q][b][k] * p[3 * b + k];
      o[q] = irrep_norm(q) * v;
    }
    for (int q = 12; q < 18; ++q) o[q] = p[q];
    o[18] = p[18];
    o[19] = p[19] / std::sqrt(3.0);
  }
  return PYRO_OK;
}

int pyro_ising_configuration(pyro_ctx* ctx, int system, int replica, int* out) {
  if (!ctx || !out) return PYRO_ERR_ARG;
  if (system < 0 || system >= (int)ctx->sys.size())
    return fail(ctx, PYRO_ERR_ARG, "ising_configuration: no such system");
  const SysDev& s = ctx->sys[system];
  if (replica < 0 || replica >= s.n_rep)
    return fail(ctx, PYRO_ERR_ARG, "ising_configuration: no such replica");
  PYRO_CK(cudaSetDevice(ctx->device));
  int rc = grow_scratch(ctx, sizeof(int) * (size_t)s.L3);
  if (rc) return rc;
  int* d = reinterpret_cast<int*>(ctx->d_order);
  const cudaStream_t st = measure_stream(ctx);
  ising_kernel<<<(s.L3 + 255) / 256, 256, 0, st>>>(
      measure_spins(ctx) + s.spin_off + (long long)replica * 16 * s.L3, s.L3, d);
  PYRO_CK_LAUNCH();
  ctx->launches += 1;
  PYRO_CK(cudaMemcpyAsync(out, d, sizeof(int) * s.L3, cudaMemcpyDeviceToHost, st));
  PYRO_CK(cudaStreamSynchronize(st));
  return PYRO_OK;
}

}  // extern "C"
