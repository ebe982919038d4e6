// Static spin structure factor S(q), FP64, for sm_100a.
//
//   S(q) = (1/N) sum_a | sum_i S_i^a exp(-i q . r_i) |^2,
//   q = (2 pi / L) stride (h, k, l),  h, k, l in [-G/2, G/2),
//   r_i = cell (x, y, z) + basis position p_s of site s (units of a).
//
// The sum over sites factorises: for each of the 16 site planes s and each
// spin component a, a three-dimensional discrete Fourier transform over the
// L^3 cells (done as three one-dimensional passes, x then y then z, each
// producing only the G wave numbers asked for), then a sum over s with the
// basis phase exp(-i q . p_s). Twiddles come from one table
// w[j] = exp(-2 pi i j / (4 L)) (basis positions are multiples of a/4).
//
// Replaces the cuFFT-backed StructFactor path of the reference (_vzabsmtgpu,
// Math.cu:721-741; lattice and Fourier set-up Pyrochlore.cu:1303-1419), whose
// classes are not part of the published code.
#include <cuda_runtime.h>

#include "sq_kernels.cuh"

namespace pyro {
namespace {

__device__ __forceinline__ int wrap_mod(long long v, int m) {
  long long r = v % m;
  return (int)(r < 0 ? r + m : r);
}

// Pass x: lines (rep, s, a, z, y) of L real inputs -> G complex outputs.
__global__ void sq_x_kernel(const float4* __restrict__ spins, SqParams p, double2* out) {
  const int line = blockIdx.x;  // ((s * 3 + a) * L + z) * L + y
  const int L = p.L;
  const int y = line % L;
  const int z = (line / L) % L;
  const int a = (line / (L * L)) % 3;
  const int s = line / (3 * L * L);
  const float4* row = spins + (long long)s * L * L * L + ((long long)z * L + y) * L;
  for (int hi = threadIdx.x; hi < p.G; hi += blockDim.x) {
    const int h = hi - p.G / 2;
    double re = 0.0, im = 0.0;
    for (int x = 0; x < L; ++x) {
      const float4 v = row[x];
      const double sa = a == 0 ? v.x : (a == 1 ? v.y : v.z);
      const double2 w = p.tw[4 * wrap_mod((long long)p.stride * h * x, L)];
      re += sa * w.x;
      im += sa * w.y;
    }
    out[(long long)line * p.G + hi] = make_double2(re, im);
  }
}

// Pass y: in [(s,a,z)][y][h] -> out [(s,a,z)][k][h].
__global__ void sq_y_kernel(const double2* __restrict__ in, SqParams p, double2* out) {
  const int L = p.L, G = p.G;
  const long long plane = blockIdx.x;  // (s*3 + a) * L + z
  const double2* src = in + plane * L * G;
  double2* dst = out + plane * G * G;
  for (int idx = threadIdx.x; idx < G * G; idx += blockDim.x) {
    const int ki = idx / G, hi = idx - ki * G;
    const int k = ki - G / 2;
    double re = 0.0, im = 0.0;
    for (int y = 0; y < L; ++y) {
      const double2 v = src[(long long)y * G + hi];
      const double2 w = p.tw[4 * wrap_mod((long long)p.stride * k * y, L)];
      re += v.x * w.x - v.y * w.y;
      im += v.x * w.y + v.y * w.x;
    }
    dst[idx] = make_double2(re, im);
  }
}

// Pass z: in [(s,a)][z][k][h] -> out [(s,a)][l][k][h].
__global__ void sq_z_kernel(const double2* __restrict__ in, SqParams p, double2* out) {
  const int L = p.L, G = p.G;
  const long long sa = blockIdx.y;  // s * 3 + a
  const double2* src = in + sa * L * G * G;
  double2* dst = out + sa * G * G * G;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < (long long)G * G * G;
       idx += (long long)gridDim.x * blockDim.x) {
    const int li = (int)(idx / (G * G));
    const int kh = (int)(idx - (long long)li * G * G);
    const int l = li - G / 2;
    double re = 0.0, im = 0.0;
    for (int z = 0; z < L; ++z) {
      const double2 v = src[(long long)z * G * G + kh];
      const double2 w = p.tw[4 * wrap_mod((long long)p.stride * l * z, L)];
      re += v.x * w.x - v.y * w.y;
      im += v.x * w.y + v.y * w.x;
    }
    dst[idx] = make_double2(re, im);
  }
}

// S(q) += (1/N) sum_a |sum_s exp(-i q.p_s) A_s^a(q)|^2 for one replica.
__global__ void sq_combine_kernel(const double2* __restrict__ A, SqParams p, double* sq) {
  const int G = p.G, L = p.L;
  const long long G3 = (long long)G * G * G;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < G3;
       idx += (long long)gridDim.x * blockDim.x) {
    const int li = (int)(idx / (G * G));
    const int ki = (int)((idx / G) % G);
    const int hi = (int)(idx % G);
    const int h = hi - G / 2, k = ki - G / 2, l = li - G / 2;
    double total = 0.0;
    for (int a = 0; a < 3; ++a) {
      double re = 0.0, im = 0.0;
      for (int s = 0; s < 16; ++s) {
        const long long ph =
            (long long)p.stride * ((long long)h * p.pos4[3 * s] + (long long)k * p.pos4[3 * s + 1] +
                                   (long long)l * p.pos4[3 * s + 2]);
        const double2 w = p.tw[wrap_mod(ph, 4 * L)];
        const double2 v = A[(long long)(s * 3 + a) * G3 + idx];
        re += v.x * w.x - v.y * w.y;
        im += v.x * w.y + v.y * w.x;
      }
      total += re * re + im * im;
    }
    // out index (h', k', l') with h' = h + G/2: [(h' G + k') G + l']
    const long long o = ((long long)hi * G + ki) * G + li;
    sq[o] += total * p.inv_n_norm;
  }
}

}  // namespace

void launch_structure_factor_replica(const float4* rep_spins, const SqParams& p, double2* s1,
                                     double2* s2, double2* s3, double* sq, cudaStream_t st) {
  const int L = p.L, G = p.G;
  sq_x_kernel<<<48 * L * L, 64, 0, st>>>(rep_spins, p, s1);
  sq_y_kernel<<<48 * L, 256, 0, st>>>(s1, p, s2);
  long long n = (long long)G * G * G;
  int bx = (int)((n + 255) / 256);
  if (bx > 1024) bx = 1024;
  sq_z_kernel<<<dim3(bx, 48), 256, 0, st>>>(s2, p, s3);
  int bc = (int)((n + 255) / 256);
  if (bc > 4096) bc = 4096;
  sq_combine_kernel<<<bc, 256, 0, st>>>(s3, p, sq);
}

}  // namespace pyro
