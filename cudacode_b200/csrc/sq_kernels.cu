// Static spin structure factor S(q), FP64, for sm_100a.
//
//   S(q) = (1/N) sum_a | sum_i S_i^a exp(-i q . r_i) |^2,
//   q = (2 pi / L) stride (h, k, l),  h, k, l in [-G/2, G/2),
//   r_i = cell (x, y, z) + basis position p_s of site s (units of a).
//
// The phase of a cell coordinate, exp(-2 pi i stride h x / L), depends on x
// only modulo L' = L / gcd(L, stride), and on h only modulo L'. So:
//   1. fold: each site plane s of each replica is summed over the cells
//      that agree modulo L' in all three coordinates (an L'^3 array of the
//      three spin components, FP64), one read of the spins;
//   2. three one-dimensional DFT passes over the folded cube (z, then y,
//      then x), each a batched complex matrix product of the L'-point axis
//      with the twiddles of R wave numbers (the L' roots of unity and each
//      wave number's step in shared memory), R = the number of distinct
//      wave numbers needed (G when G <= L', else the L' residues);
//   3. combine: for every q of the G^3 grid, the basis phases
//      exp(-i q . p_s) (which are not periodic in L') applied to the 16 site
//      planes' transforms, |.|^2 summed over the components and over the
//      replicas.
// Every pass runs over all replicas of a batch in one launch.
//
// Replaces the cuFFT-backed StructFactor path of the reference (_vzabsmtgpu,
// Math.cu:721-741; lattice and Fourier set-up Pyrochlore.cu:1303-1419), whose
// classes are not part of the published code.
#include <cuda_runtime.h>

#include "sq_kernels.cuh"

namespace pyro {
namespace {

constexpr int kSqThreads = 256;
constexpr int kTileM = 32;  // inner indices per CTA of a DFT pass

// fold[r][s][a][z'][y'][x'] = sum over cells (x, y, z) = (x', y', z') mod L'.
__global__ void __launch_bounds__(kSqThreads)
    sq_fold_kernel(const float4* __restrict__ spins, SqParams p, int n_rep, double* fold) {
  const int Lf = p.Lf, L = p.L, g = L / Lf;
  const long long L3f = (long long)Lf * Lf * Lf;
  const long long total = (long long)n_rep * 16 * L3f;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int xf = (int)(idx % Lf);
    const int yf = (int)((idx / Lf) % Lf);
    const int zf = (int)((idx / ((long long)Lf * Lf)) % Lf);
    const long long rs = idx / L3f;  // r * 16 + s
    const float4* plane = spins + rs * L * L * L;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int mz = 0; mz < g; ++mz)
      for (int my = 0; my < g; ++my) {
        const float4* row = plane + ((long long)(zf + mz * Lf) * L + (yf + my * Lf)) * L + xf;
        for (int mx = 0; mx < g; ++mx) {
          const float4 v = __ldg(row + mx * Lf);
          sx += v.x;
          sy += v.y;
          sz += v.z;
        }
      }
    double* out = fold + rs * 3 * L3f + ((long long)zf * Lf + yf) * Lf + xf;
    out[0] = sx;
    out[L3f] = sy;
    out[2 * L3f] = sz;
  }
}

// One DFT pass: for every batch b and inner index i,
//   out[b][k][i] = sum_j in[b][j][i] exp(-2 pi i step[k] j / n),  k < R,  j < n (= L'),
// step[k] = stride' w(k) mod L' for the k-th wave number w(k). The input is
// real (kReal, the folded spins) or complex. When I == 1 the axis is the
// innermost dimension: a tile then takes kTileM consecutive batches as its
// inner index (in[b][j] at b n + j, out at b R + k). Shared memory: the n
// roots of unity, the [n][kTileM] input slab and the R steps; the twiddle
// index of each output advances by its step per j (no division in the loop).
template <bool kReal>
__global__ void __launch_bounds__(kSqThreads)
    sq_dft_kernel(const void* __restrict__ in_v, long long n_batch, int n, long long I, int R,
                  const double2* __restrict__ roots, const int* __restrict__ steps,
                  double2* out) {
  extern __shared__ double2 sh[];
  double2* rt = sh;                     // [n]
  double2* tile = sh + n;               // [n][kTileM]
  int* st = (int*)(tile + n * kTileM);  // [R]
  for (int e = threadIdx.x; e < n; e += blockDim.x) rt[e] = roots[e];
  for (int e = threadIdx.x; e < R; e += blockDim.x) st[e] = steps[e];
  const bool axis_inner = I == 1;
  const long long tiles_per_batch = axis_inner ? 1 : (I + kTileM - 1) / kTileM;
  long long b0 = (long long)blockIdx.x / tiles_per_batch;
  const long long i0 = ((long long)blockIdx.x - b0 * tiles_per_batch) * kTileM;
  if (axis_inner) b0 *= kTileM;
  const long long m_count =
      axis_inner ? min((long long)kTileM, n_batch - b0) : min((long long)kTileM, I - i0);
  // stage the [n][m] slab (coalesced along the contiguous dimension)
  for (int e = threadIdx.x; e < n * kTileM; e += blockDim.x) {
    int j, m;
    if (axis_inner) {
      j = e % n;
      m = e / n;
    } else {
      m = e % kTileM;
      j = e / kTileM;
    }
    double2 v = make_double2(0.0, 0.0);
    if (m < m_count) {
      const long long addr = axis_inner ? (b0 + m) * n + j : (b0 * n + j) * I + i0 + m;
      if (kReal) v.x = ((const double*)in_v)[addr];
      else v = ((const double2*)in_v)[addr];
    }
    tile[j * kTileM + m] = v;
  }
  __syncthreads();
  // outputs: kTileM x R per tile, four wave numbers per thread
  constexpr int kKq = 4;
  const int k_groups = (R + kKq - 1) / kKq;
  for (int w = threadIdx.x; w < kTileM * k_groups; w += blockDim.x) {
    int m, kg;
    if (axis_inner) {  // consecutive threads: consecutive k groups of one batch
      kg = w % k_groups;
      m = w / k_groups;
    } else {  // consecutive threads: consecutive inner indices
      m = w % kTileM;
      kg = w / kTileM;
    }
    if (m >= m_count) continue;
    const int k0 = kg * kKq;
    double re[kKq], im[kKq];
    int ix[kKq], sp[kKq];
#pragma unroll
    for (int q = 0; q < kKq; ++q) {
      re[q] = im[q] = 0.0;
      ix[q] = 0;
      sp[q] = k0 + q < R ? st[k0 + q] : 0;
    }
    for (int j = 0; j < n; ++j) {
      const double2 v = tile[j * kTileM + m];
#pragma unroll
      for (int q = 0; q < kKq; ++q) {
        const double2 t = rt[ix[q]];
        if (kReal) {
          re[q] = fma(v.x, t.x, re[q]);
          im[q] = fma(v.x, t.y, im[q]);
        } else {
          re[q] = fma(v.x, t.x, fma(-v.y, t.y, re[q]));
          im[q] = fma(v.x, t.y, fma(v.y, t.x, im[q]));
        }
        ix[q] += sp[q];
        if (ix[q] >= n) ix[q] -= n;
      }
    }
#pragma unroll
    for (int q = 0; q < kKq; ++q) {
      const int k = k0 + q;
      if (k >= R) continue;
      const long long addr = axis_inner ? (b0 + m) * R + k : (b0 * R + k) * I + i0 + m;
      out[addr] = make_double2(re[q], im[q]);
    }
  }
}

// sq[(h' G + k') G + l'] += (1/(N nrep)) sum_r sum_a |sum_s ph_s(q) A[r][s][a][l][k][h]|^2,
// (l, k, h) the transform indices of the wave numbers of q.
__global__ void __launch_bounds__(kSqThreads)
    sq_combine_kernel(const double2* __restrict__ A, SqParams p, int n_rep, double* sq) {
  const int G = p.G, R = p.R;
  const long long G3 = (long long)G * G * G;
  const long long R3 = (long long)R * R * R;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < G3;
       idx += (long long)gridDim.x * blockDim.x) {
    const int hi = (int)(idx / ((long long)G * G));
    const int ki = (int)((idx / G) % G);
    const int li = (int)(idx % G);
    const int h = hi - G / 2, k = ki - G / 2, l = li - G / 2;
    auto tindex = [&](int wv) {  // transform index of wave number wv
      if (p.residues) {
        const int r = wv % p.Lf;
        return r < 0 ? r + p.Lf : r;
      }
      return wv + G / 2;
    };
    const long long t = ((long long)tindex(l) * R + tindex(k)) * R + tindex(h);
    double2 ph[16];
    const int L4 = 4 * p.L;
#pragma unroll
    for (int s = 0; s < 16; ++s) {
      long long e = (long long)p.stride * ((long long)h * p.pos4[3 * s] +
                                           (long long)k * p.pos4[3 * s + 1] +
                                           (long long)l * p.pos4[3 * s + 2]);
      e %= L4;
      if (e < 0) e += L4;
      ph[s] = p.tw4[e];
    }
    double total = 0.0;
    for (int r = 0; r < n_rep; ++r)
      for (int a = 0; a < 3; ++a) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int s = 0; s < 16; ++s) {
          const double2 v = A[((long long)(r * 16 + s) * 3 + a) * R3 + t];
          re += v.x * ph[s].x - v.y * ph[s].y;
          im += v.x * ph[s].y + v.y * ph[s].x;
        }
        total += re * re + im * im;
      }
    sq[idx] += total * p.inv_n_norm;
  }
}

int grid_for(long long n) {
  const long long b = (n + kSqThreads - 1) / kSqThreads;
  return (int)(b > 148 * 16 ? 148 * 16 : (b < 1 ? 1 : b));
}

size_t dft_smem(int n, int R) {
  return sizeof(double2) * ((size_t)n + (size_t)n * kTileM) + sizeof(int) * (size_t)R;
}

template <bool kReal>
void launch_dft(const void* in, long long n_batch, int n, long long I, int R,
                const double2* roots, const int* steps, double2* out, cudaStream_t st) {
  const long long tiles = I == 1 ? (n_batch + kTileM - 1) / kTileM
                                 : n_batch * ((I + kTileM - 1) / kTileM);
  sq_dft_kernel<kReal><<<(unsigned)tiles, kSqThreads, dft_smem(n, R), st>>>(in, n_batch, n, I, R,
                                                                           roots, steps, out);
}

}  // namespace

size_t sq_scratch_per_replica(const SqParams& p) {
  const size_t L3f = (size_t)p.Lf * p.Lf * p.Lf;
  const size_t fold = 48 * L3f * sizeof(double);
  const size_t a1 = 48 * (size_t)p.R * p.Lf * p.Lf * sizeof(double2);
  const size_t a2 = 48 * (size_t)p.R * p.R * p.Lf * sizeof(double2);
  const size_t a3 = 48 * (size_t)p.R * p.R * p.R * sizeof(double2);
  return fold + a1 + a2 + a3;
}

cudaError_t sq_prepare() {
  const int smem = (int)dft_smem(256, 256);  // L' <= L <= 256, R <= 256
  cudaError_t e = cudaFuncSetAttribute(sq_dft_kernel<true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(sq_dft_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
  return e;
}

void launch_structure_factor(const float4* spins, int n_rep, const SqParams& p,
                             const double2* roots, const int* steps, void* scratch, double* sq,
                             cudaStream_t st) {
  const int Lf = p.Lf, R = p.R;
  const long long L3f = (long long)Lf * Lf * Lf;
  char* base = (char*)scratch;
  double* fold = (double*)base;
  base += (size_t)n_rep * 48 * L3f * sizeof(double);
  double2* a1 = (double2*)base;
  base += (size_t)n_rep * 48 * R * (size_t)Lf * Lf * sizeof(double2);
  double2* a2 = (double2*)base;
  base += (size_t)n_rep * 48 * (size_t)R * R * Lf * sizeof(double2);
  double2* a3 = (double2*)base;
  const long long planes = (long long)n_rep * 48;  // (r, s, a)
  sq_fold_kernel<<<grid_for((long long)n_rep * 16 * L3f), kSqThreads, 0, st>>>(spins, p, n_rep,
                                                                              fold);
  // z: [(r,s,a)][z'][(y',x')] -> [(r,s,a)][l][(y',x')]
  launch_dft<true>(fold, planes, Lf, (long long)Lf * Lf, R, roots, steps, a1, st);
  // y: [(r,s,a,l)][y'][x'] -> [(r,s,a,l)][k][x']
  launch_dft<false>(a1, planes * R, Lf, Lf, R, roots, steps, a2, st);
  // x: [(r,s,a,l,k)][x'] -> [(r,s,a,l,k)][h]
  launch_dft<false>(a2, planes * R * R, Lf, 1, R, roots, steps, a3, st);
  sq_combine_kernel<<<grid_for((long long)p.G * p.G * p.G), kSqThreads, 0, st>>>(a3, p, n_rep,
                                                                                 sq);
}

}  // namespace pyro
