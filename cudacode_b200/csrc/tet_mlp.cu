// Learned tetrahedron proposal for the J1 pyrochlore antiferromagnet, sm_100a.
//
// The up-tetrahedron at FCC corner f of a cubic cell holds the sites
// 4f..4f+3 of that cell; every other bond of those sites goes to a
// down-tetrahedron, i.e. to up-tetrahedra of the other three corners. So the
// tetrahedra of one corner share no bond and are moved together in one pass
// (4 passes = one sweep over all up-tetrahedra).
//
// For each tetrahedron the external field of site k is h_k = J1 * (sum of its
// three down-tetrahedron neighbours). A 16 -> 64 -> 64 -> 16 MLP (hard-swish, BF16
// weights and activations, FP32 accumulation with mma.sync m16n8k16 on the
// tensor cores) maps (h_0..h_3 / 3, log(beta) / 3) to a von Mises-Fisher
// distribution vMF(mu_k, kappa_k) per site. The joint proposal of the four
// spins is independent of their current values, so the Metropolis-Hastings
// ratio is
//   exp(-beta (E(S') - E(S))) * q(S) / q(S'),
//   log q(S) - log q(S') = sum_k kappa_k mu_k . (S_k - S'_k),
// with E the exact FP32 energy of the tetrahedron (its 6 internal bonds and
// the external fields). Detailed balance holds whatever the network outputs.
// vMF sampling on the sphere follows Wood (1994): w = 1 + log(u + (1 - u)
// e^{-2 kappa}) / kappa, azimuth uniform, frame of Duff et al. (2017).
//
// The network is trained by maximum likelihood on tetrahedron configurations
// collected from the plain chains; the gradient kernel runs the same forward
// pass and its backward pass on the tensor cores, one warp per 32 samples.
// This move has no counterpart in taillefu/cudacode.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "../../include/pyro_math.h"
#include "lattice.h"
#include "tet_mlp.cuh"
#include "tet_umma.cuh"

namespace pyro {
namespace {

constexpr int kTetThreads = 128;      // training / test kernels: 4 warps x 32 rows
constexpr int kTetMoveThreads = 256;  // move kernel: 8 warps x 32 tetrahedra
constexpr int kLdB = 40;          // padded row of 32 batch entries (bf16)
constexpr int kLdOut = 17;        // padded row of 16 floats

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) {
  return *reinterpret_cast<const uint32_t*>(p);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

// Four 8x8 BF16 matrices from shared memory (ldmatrix .x4): lane l gives the
// 16-byte row address of matrix l / 8, row l % 8; register q receives this
// lane's pair of matrix q (row lane / 4, columns 2 (lane % 4) and + 1), which
// is the B fragment layout of mma m16n8k16 for a [n][k] (k-contiguous) matrix.
__device__ __forceinline__ void ldsm_x4(const __nv_bfloat16* p, uint32_t (&r)[4]) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a)
               : "memory");
}

// D = A * B + D, m16n8k16, BF16 inputs, FP32 accumulators.
__device__ __forceinline__ void mma_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2,
                                         uint32_t a3, uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Hard-swish, x * clamp(x + 3, 0, 6) / 6 (Howard et al. 2019): smooth
// enough for a proposal network, and plain FMA-pipe arithmetic. With SiLU the
// special-function unit (two operations per activation) bounded the move's
// per-pass latency.
__device__ __forceinline__ float hswish(float x) {
  return x * fminf(fmaxf(x + 3.0f, 0.0f), 6.0f) * (1.0f / 6.0f);
}
__device__ __forceinline__ float hswish_grad(float x) {
  return x <= -3.0f ? 0.0f : (x >= 3.0f ? 1.0f : x * (1.0f / 3.0f) + 0.5f);
}

// Weights staged in shared memory: the weight image, copied verbatim.
struct MlpSmem {
  const __nv_bfloat16* w1t;  // [64][kLdIn]
  const __nv_bfloat16* w2t;  // [64][kLdH]
  const __nv_bfloat16* w3t;  // [16][kLdH]
  const __nv_bfloat16* w2;   // [64][kLdH]  (backward)
  const __nv_bfloat16* w3;   // [64][kLdIn] (backward)
  const float* b1;           // [64]
  const float* b2;           // [64]
  const float* b3;           // [16]
};

constexpr int kSmemWeightsFwd = kImgFwdBytes;
constexpr int kSmemWeightsAll = kImgBytes;

__device__ MlpSmem carve_weights(const unsigned char* base) {
  MlpSmem w;
  w.w1t = reinterpret_cast<const __nv_bfloat16*>(base + kImgW1t);
  w.w2t = reinterpret_cast<const __nv_bfloat16*>(base + kImgW2t);
  w.w3t = reinterpret_cast<const __nv_bfloat16*>(base + kImgW3t);
  w.w2 = reinterpret_cast<const __nv_bfloat16*>(base + kImgW2);
  w.w3 = reinterpret_cast<const __nv_bfloat16*>(base + kImgW3);
  w.b1 = reinterpret_cast<const float*>(base + kImgB1);
  w.b2 = reinterpret_cast<const float*>(base + kImgB2);
  w.b3 = reinterpret_cast<const float*>(base + kImgB3);
  return w;
}

// Starts the copy of the first `bytes` of the weight image into shared
// memory (16-byte cp.async granules, L2 only); stage_wait() completes it for
// the whole CTA. Between the two a kernel issues its spin loads, so the two
// memory latencies overlap.
__device__ __forceinline__ void stage_weights(unsigned char* smem, const unsigned char* image,
                                              int bytes) {
  for (int i = threadIdx.x * 16; i < bytes; i += blockDim.x * 16) {
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem + i);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(image + i)
                 : "memory");
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__device__ __forceinline__ void stage_wait() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
}

// Forward pass of one 16-row m-tile of a warp. feat: [rows][kLdIn] bf16 row
// major (the tile starts at row r_base). Returns outputs in C-fragment
// layout; optionally keeps pre-activations and writes activations
// feature-major (bf16, [feature][kLdB]) for the weight-gradient GEMMs.
struct TileFwd {
  float o[2][4];
  float pre1[8][4];
  float pre2[8][4];
};

template <bool kKeep>
__device__ __forceinline__ void tile_forward(const __nv_bfloat16* feat, int r_base, const MlpSmem& w,
                                             TileFwd& f, __nv_bfloat16* h1t,
                                             __nv_bfloat16* h2t) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = r_base + g, r1 = r0 + 8;
  // layer 1: [16 x 16] x [16 x 64]
  const uint32_t a0 = ld32(feat + r0 * kLdIn + 2 * t), a1 = ld32(feat + r1 * kLdIn + 2 * t);
  const uint32_t a2 = ld32(feat + r0 * kLdIn + 8 + 2 * t), a3 = ld32(feat + r1 * kLdIn + 8 + 2 * t);
  float h1[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    h1[j][0] = h1[j][2] = w.b1[8 * j + 2 * t];
    h1[j][1] = h1[j][3] = w.b1[8 * j + 2 * t + 1];
    const __nv_bfloat16* bw = w.w1t + (8 * j + g) * kLdIn + 2 * t;
    mma_bf16(h1[j], a0, a1, a2, a3, ld32(bw), ld32(bw + 8));
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (kKeep) f.pre1[j][e] = h1[j][e];
      h1[j][e] = hswish(h1[j][e]);
    }
  if (kKeep) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      h1t[c * kLdB + r0] = __float2bfloat16_rn(h1[j][0]);
      h1t[(c + 1) * kLdB + r0] = __float2bfloat16_rn(h1[j][1]);
      h1t[c * kLdB + r1] = __float2bfloat16_rn(h1[j][2]);
      h1t[(c + 1) * kLdB + r1] = __float2bfloat16_rn(h1[j][3]);
    }
  }
  // layer 2: [16 x 64] x [64 x 64]
  float h2[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    h2[j][0] = h2[j][2] = w.b2[8 * j + 2 * t];
    h2[j][1] = h2[j][3] = w.b2[8 * j + 2 * t + 1];
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const uint32_t x0 = pack_bf16(h1[2 * kk][0], h1[2 * kk][1]);
    const uint32_t x1 = pack_bf16(h1[2 * kk][2], h1[2 * kk][3]);
    const uint32_t x2 = pack_bf16(h1[2 * kk + 1][0], h1[2 * kk + 1][1]);
    const uint32_t x3 = pack_bf16(h1[2 * kk + 1][2], h1[2 * kk + 1][3]);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const __nv_bfloat16* bw = w.w2t + (8 * j + g) * kLdH + 16 * kk + 2 * t;
      mma_bf16(h2[j], x0, x1, x2, x3, ld32(bw), ld32(bw + 8));
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (kKeep) f.pre2[j][e] = h2[j][e];
      h2[j][e] = hswish(h2[j][e]);
    }
  if (kKeep) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      h2t[c * kLdB + r0] = __float2bfloat16_rn(h2[j][0]);
      h2t[(c + 1) * kLdB + r0] = __float2bfloat16_rn(h2[j][1]);
      h2t[c * kLdB + r1] = __float2bfloat16_rn(h2[j][2]);
      h2t[(c + 1) * kLdB + r1] = __float2bfloat16_rn(h2[j][3]);
    }
  }
  // layer 3: [16 x 64] x [64 x 16]
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    f.o[j][0] = f.o[j][2] = w.b3[8 * j + 2 * t];
    f.o[j][1] = f.o[j][3] = w.b3[8 * j + 2 * t + 1];
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const uint32_t x0 = pack_bf16(h2[2 * kk][0], h2[2 * kk][1]);
    const uint32_t x1 = pack_bf16(h2[2 * kk][2], h2[2 * kk][3]);
    const uint32_t x2 = pack_bf16(h2[2 * kk + 1][0], h2[2 * kk + 1][1]);
    const uint32_t x3 = pack_bf16(h2[2 * kk + 1][2], h2[2 * kk + 1][3]);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const __nv_bfloat16* bw = w.w3t + (8 * j + g) * kLdH + 16 * kk + 2 * t;
      mma_bf16(f.o[j], x0, x1, x2, x3, ld32(bw), ld32(bw + 8));
    }
  }
}

// The network of the learned move for one 16-row m-tile: tile_forward's
// operands and accumulations, with the hidden activations rounded to BF16
// first and evaluated by hswish_bf16x2 (tile_forward rounds after an FP32
// activation), and the weight fragments fetched by ldmatrix (one
// instruction per two n-tiles instead of four 32-bit loads). Used by every
// mma.sync form of the move, so they agree bit for bit; the batched forward
// and the training keep tile_forward.
__device__ __forceinline__ void tile_forward_move(const __nv_bfloat16* feat, int r_base,
                                                  const MlpSmem& w, TileFwd& f) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = r_base + g, r1 = r0 + 8;
  // ldmatrix row of this lane: matrix lane / 8 of an x4 load covers n-tile
  // j + (lane / 16) and k half (lane / 8) % 2 of a 16-wide k step
  const int bn = 8 * (lane >> 4) + (lane & 7), bk = 8 * ((lane >> 3) & 1);
  const uint32_t a0 = ld32(feat + r0 * kLdIn + 2 * t), a1 = ld32(feat + r1 * kLdIn + 2 * t);
  const uint32_t a2 = ld32(feat + r0 * kLdIn + 8 + 2 * t), a3 = ld32(feat + r1 * kLdIn + 8 + 2 * t);
  float h1[8][4];
#pragma unroll
  for (int j = 0; j < 8; j += 2) {
    uint32_t b[4];
    ldsm_x4(w.w1t + (8 * j + bn) * kLdIn + bk, b);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      h1[j + q][0] = h1[j + q][2] = w.b1[8 * (j + q) + 2 * t];
      h1[j + q][1] = h1[j + q][3] = w.b1[8 * (j + q) + 2 * t + 1];
      mma_bf16(h1[j + q], a0, a1, a2, a3, b[2 * q], b[2 * q + 1]);
    }
  }
  float h2[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    h2[j][0] = h2[j][2] = w.b2[8 * j + 2 * t];
    h2[j][1] = h2[j][3] = w.b2[8 * j + 2 * t + 1];
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const uint32_t x0 = hswish_bf16x2(pack_bf16(h1[2 * kk][0], h1[2 * kk][1]));
    const uint32_t x1 = hswish_bf16x2(pack_bf16(h1[2 * kk][2], h1[2 * kk][3]));
    const uint32_t x2 = hswish_bf16x2(pack_bf16(h1[2 * kk + 1][0], h1[2 * kk + 1][1]));
    const uint32_t x3 = hswish_bf16x2(pack_bf16(h1[2 * kk + 1][2], h1[2 * kk + 1][3]));
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      uint32_t b[4];
      ldsm_x4(w.w2t + (8 * j + bn) * kLdH + 16 * kk + bk, b);
      mma_bf16(h2[j], x0, x1, x2, x3, b[0], b[1]);
      mma_bf16(h2[j + 1], x0, x1, x2, x3, b[2], b[3]);
    }
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    f.o[j][0] = f.o[j][2] = w.b3[8 * j + 2 * t];
    f.o[j][1] = f.o[j][3] = w.b3[8 * j + 2 * t + 1];
  }
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const uint32_t x0 = hswish_bf16x2(pack_bf16(h2[2 * kk][0], h2[2 * kk][1]));
    const uint32_t x1 = hswish_bf16x2(pack_bf16(h2[2 * kk][2], h2[2 * kk][3]));
    const uint32_t x2 = hswish_bf16x2(pack_bf16(h2[2 * kk + 1][0], h2[2 * kk + 1][1]));
    const uint32_t x3 = hswish_bf16x2(pack_bf16(h2[2 * kk + 1][2], h2[2 * kk + 1][3]));
    uint32_t b[4];
    ldsm_x4(w.w3t + bn * kLdH + 16 * kk + bk, b);
    mma_bf16(f.o[0], x0, x1, x2, x3, b[0], b[1]);
    mma_bf16(f.o[1], x0, x1, x2, x3, b[2], b[3]);
  }
}

__device__ __forceinline__ void store_out(const TileFwd& f, int r_base, float* out) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = r_base + g, r1 = r0 + 8;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    out[r0 * kLdOut + 8 * j + 2 * t] = f.o[j][0];
    out[r0 * kLdOut + 8 * j + 2 * t + 1] = f.o[j][1];
    out[r1 * kLdOut + 8 * j + 2 * t] = f.o[j][2];
    out[r1 * kLdOut + 8 * j + 2 * t + 1] = f.o[j][3];
  }
}

// Network outputs -> (mu_k, kappa_k) for the four sites.
struct VmfParams {
  pyro_vec3 mu[4];
  float kappa[4];
  float z[4];      // clamped log kappa
  bool z_in[4];    // log kappa strictly inside the clamp range
  float onorm[4];  // |o_k| before normalisation
};

__device__ __forceinline__ VmfParams vmf_params(const float* o) {
  VmfParams v;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float x = o[4 * k], y = o[4 * k + 1], z = o[4 * k + 2];
    float n = sqrtf(x * x + y * y + z * z);
    pyro_vec3 m;
    if (n > 1e-20f) {
      m.x = x / n;
      m.y = y / n;
      m.z = z / n;
    } else {
      m.x = 0.0f;
      m.y = 0.0f;
      m.z = 1.0f;
      n = 1e-20f;
    }
    v.mu[k] = m;
    v.onorm[k] = n;
    const float lz = o[4 * k + 3];
    v.z[k] = fminf(fmaxf(lz, kLogKappaMin), kLogKappaMax);
    v.z_in[k] = lz > kLogKappaMin && lz < kLogKappaMax;
    v.kappa[k] = expf(v.z[k]);
  }
  return v;
}

// Cell frame (periodic neighbour rows), as in the J1 kernels.
struct Frame {
  int zo[3], yo[3], xo[3];
};

__device__ __forceinline__ Frame cell_frame(int cell, int L, float rcpL) {
  int q = (int)((float)cell * rcpL);
  int r = cell - q * L;
  if (r < 0) { --q; r += L; } else if (r >= L) { ++q; r -= L; }
  int q2 = (int)((float)q * rcpL);
  int r2 = q - q2 * L;
  if (r2 < 0) { --q2; r2 += L; } else if (r2 >= L) { ++q2; r2 -= L; }
  const int x = r, y = r2, z = q2, L2 = L * L;
  Frame f;
  f.xo[0] = x == 0 ? L - 1 : x - 1;
  f.xo[1] = x;
  f.xo[2] = x == L - 1 ? 0 : x + 1;
  f.yo[0] = (y == 0 ? L - 1 : y - 1) * L;
  f.yo[1] = y * L;
  f.yo[2] = (y == L - 1 ? 0 : y + 1) * L;
  f.zo[0] = (z == 0 ? L - 1 : z - 1) * L2;
  f.zo[1] = z * L2;
  f.zo[2] = (z == L - 1 ? 0 : z + 1) * L2;
  return f;
}

// kL2: read through L2 only (the cluster kernel rewrites the lattice between
// passes of one launch, so an SM's L1 may hold stale lines).
template <bool kL2>
__device__ __forceinline__ float4 ld_spin(const float4* p) {
  if (kL2) return __ldcg(p);
  return __ldg(p);
}

template <int S, int K, bool kL2 = false>
__device__ __forceinline__ float4 nbr(const float4* __restrict__ rep, const Frame& f, int L3) {
  constexpr NbrEntry e = j1_neighbour(S, K);
  return ld_spin<kL2>(rep + f.zo[e.dz + 1] + f.yo[e.dy + 1] + f.xo[e.dx + 1] + e.t * L3);
}

// External field of site S (sum of its three down-tetrahedron neighbours).
template <int S, bool kL2 = false>
__device__ __forceinline__ pyro_vec3 ext_field(const float4* __restrict__ rep, const Frame& f,
                                               int L3, float J1) {
  constexpr int k0 = j1_down_index(S, 0), k1 = j1_down_index(S, 1), k2 = j1_down_index(S, 2);
  const float4 a = nbr<S, k0, kL2>(rep, f, L3), b = nbr<S, k1, kL2>(rep, f, L3),
               c = nbr<S, k2, kL2>(rep, f, L3);
  pyro_vec3 h;
  h.x = J1 * ((a.x + b.x) + c.x);
  h.y = J1 * ((a.y + b.y) + c.y);
  h.z = J1 * ((a.z + b.z) + c.z);
  return h;
}

template <int F, bool kL2 = false>
__device__ __forceinline__ void tet_fields(const float4* __restrict__ rep, const Frame& fr, int L3,
                                           float J1, pyro_vec3 h[4]) {
  h[0] = ext_field<4 * F + 0, kL2>(rep, fr, L3, J1);
  h[1] = ext_field<4 * F + 1, kL2>(rep, fr, L3, J1);
  h[2] = ext_field<4 * F + 2, kL2>(rep, fr, L3, J1);
  h[3] = ext_field<4 * F + 3, kL2>(rep, fr, L3, J1);
}

__device__ __forceinline__ float dot3(pyro_vec3 a, pyro_vec3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}

__device__ __forceinline__ float tet_energy(const pyro_vec3 s[4], const pyro_vec3 h[4], float J1) {
  const float bonds = dot3(s[0], s[1]) + dot3(s[0], s[2]) + dot3(s[0], s[3]) + dot3(s[1], s[2]) +
                      dot3(s[1], s[3]) + dot3(s[2], s[3]);
  return J1 * bonds + dot3(s[0], h[0]) + dot3(s[1], h[1]) + dot3(s[2], h[2]) + dot3(s[3], h[3]);
}

__device__ __forceinline__ void write_features(__nv_bfloat16* row, const pyro_vec3 h[4], float beta) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    row[3 * k] = __float2bfloat16_rn(h[k].x * (1.0f / 3.0f));
    row[3 * k + 1] = __float2bfloat16_rn(h[k].y * (1.0f / 3.0f));
    row[3 * k + 2] = __float2bfloat16_rn(h[k].z * (1.0f / 3.0f));
  }
  row[12] = __float2bfloat16_rn(logf(beta) * (1.0f / 3.0f));
  row[13] = row[14] = row[15] = __float2bfloat16_rn(0.0f);
}

// Uniform in (0, 1] from the top 23 bits of a Philox word (mantissa fill,
// integer pipe only).
__device__ __forceinline__ float tet_uniform(uint32_t r) {
  return 2.0f - __uint_as_float(0x3f800000u | (r >> 9));
}

// Uniform in (0, 1] for the MH test from the low bits of the words whose top
// 23 bits feed the proposals of sites 0 and 1 (9 + 9 + 5 bits of r[0..2]),
// bits that no other draw of the move uses.
__device__ __forceinline__ float tet_test_uniform(const uint32_t r[4]) {
  const uint32_t m = ((r[0] & 0x1ffu) << 14) | ((r[1] & 0x1ffu) << 5) | (r[2] & 0x1fu);
  return 2.0f - __uint_as_float(0x3f800000u | m);
}

// Rotation of (sin t cos p, sin t sin p, cos t) onto the axis n, in the
// frame of Duff et al. (2017), with the approximate reciprocal (|sgn + n.z|
// >= 1).
__device__ __forceinline__ pyro_vec3 about_axis_fast(pyro_vec3 n, float ct, float st, float cp,
                                                     float sp) {
  const float sgn = copysignf(1.0f, n.z);
  const float a = __fdividef(-1.0f, sgn + n.z);
  const float b = n.x * n.y * a;
  const float c1 = st * cp, c2 = st * sp;
  pyro_vec3 o;
  o.x = ct * n.x + c2 * b + c1 * (sgn * n.x * n.x * a + 1.0f);
  o.y = ct * n.y + c2 * (n.y * n.y * a + sgn) + c1 * (sgn * b);
  o.z = ct * n.z - c2 * n.y - c1 * (sgn * n.x);
  return o;
}

// vMF(mu, kappa) sample on the sphere (Wood 1994): w = 1 + log(u + (1 - u)
// e^{-2 kappa}) / kappa, azimuth 2 pi v. The sampler runs on the hardware
// approximations; the MH ratio is evaluated with the vMF density at the
// value drawn.
__device__ __forceinline__ pyro_vec3 vmf_sample(pyro_vec3 mu, float kappa, float u, float v) {
  float w = 1.0f + __fdividef(__logf(u + (1.0f - u) * __expf(-2.0f * kappa)), kappa);
  w = fminf(1.0f, fmaxf(-1.0f, w));
  const float q = 1.0f - w * w;
  const float st = q > 0.0f ? q * rsqrtf(q) : 0.0f;
  float sp, cp;
  pyro_sincospif(2.0f * v, &sp, &cp);
  return about_axis_fast(mu, w, st, cp, sp);
}

// Proposal for one site from its four network outputs o[0..3]: mu = o_xyz /
// |o_xyz|, kappa = exp(clamp(o_w)); returns the sample and the site's term
// kappa mu . (s - s') of log q(S) - log q(S').
struct SiteMove {
  pyro_vec3 sn;
  float lq;
};

__device__ __forceinline__ SiteMove site_move(const float* o, pyro_vec3 s, uint32_t ru,
                                              uint32_t rv) {
  const float x = o[0], y = o[1], z = o[2];
  const float n2 = x * x + y * y + z * z;
  pyro_vec3 mu;
  if (n2 > 1e-30f) {
    const float inv = rsqrtf(n2);
    mu.x = x * inv;
    mu.y = y * inv;
    mu.z = z * inv;
  } else {
    mu.x = 0.0f;
    mu.y = 0.0f;
    mu.z = 1.0f;
  }
  const float kappa = __expf(fminf(fmaxf(o[3], kLogKappaMin), kLogKappaMax));
  SiteMove m;
  m.sn = vmf_sample(mu, kappa, tet_uniform(ru), tet_uniform(rv));
  m.lq = kappa * (dot3(mu, s) - dot3(mu, m.sn));
  return m;
}

// log(sinh k / k) up to a constant, k - log k + log(1 - e^{-2k}): the
// normalisation of a vMF density of concentration k > 0.
__device__ __forceinline__ float vmf_log_norm(float k) {
  return (k - __logf(k)) + __logf(1.0f - __expf(-2.0f * k));
}

// Natural parameter f = -beta (J1 (s0 + s1 + s2) + h3) of site 3's exact
// conditional distribution p(s3 | s0, s1, s2) ~ exp(f . s3), as an axis and a
// concentration (at least exp(kLogKappaMin), the network's smallest).
__device__ __forceinline__ pyro_vec3 closure_axis(pyro_vec3 s0, pyro_vec3 s1, pyro_vec3 s2,
                                                  pyro_vec3 h3, float beta, float J1,
                                                  float* kappa) {
  pyro_vec3 f;
  f.x = -beta * (J1 * ((s0.x + s1.x) + s2.x) + h3.x);
  f.y = -beta * (J1 * ((s0.y + s1.y) + s2.y) + h3.y);
  f.z = -beta * (J1 * ((s0.z + s1.z) + s2.z) + h3.z);
  const float n2 = f.x * f.x + f.y * f.y + f.z * f.z;
  pyro_vec3 mu;
  float k = 0.0f;
  if (n2 > 1e-30f) {
    const float inv = rsqrtf(n2);
    mu.x = f.x * inv;
    mu.y = f.y * inv;
    mu.z = f.z * inv;
    k = n2 * inv;
  } else {
    mu.x = 0.0f;
    mu.y = 0.0f;
    mu.z = 1.0f;
  }
  *kappa = fmaxf(k, kKappaFloor);
  return mu;
}

// Site 3 drawn from its exact conditional distribution given the proposed
// sites 0-2 (a0..a2) and its external field: a vMF whose natural parameter
// is closure_axis. Returns the sample and the site's term of log q(S) -
// log q(S'): `rev` (closure_reverse: the density of the current s3 under the
// conditional of the current sites 0-2) minus the density of the sample. The
// joint proposal q = (network vMFs of sites 0-2) x (this conditional) is
// exactly computable in both directions, so the MH test stays exact; site 3
// is integrated out of the mismatch between q and the Boltzmann weight,
// which raises the acceptance of the joint move.
__device__ __forceinline__ float closure_reverse(pyro_vec3 b0, pyro_vec3 b1, pyro_vec3 b2,
                                                 pyro_vec3 s3, pyro_vec3 h3, float beta,
                                                 float J1) {
  float ko;
  const pyro_vec3 mo = closure_axis(b0, b1, b2, h3, beta, J1, &ko);
  return ko * dot3(mo, s3) - vmf_log_norm(ko);
}

__device__ __forceinline__ SiteMove closure_move(pyro_vec3 a0, pyro_vec3 a1, pyro_vec3 a2,
                                                 float rev, pyro_vec3 h3, float beta, float J1,
                                                 uint32_t ru, uint32_t rv) {
  float kn;
  const pyro_vec3 mn = closure_axis(a0, a1, a2, h3, beta, J1, &kn);
  SiteMove m;
  m.sn = vmf_sample(mn, kn, tet_uniform(ru), tet_uniform(rv));
  m.lq = rev - (kn * dot3(mn, m.sn) - vmf_log_norm(kn));
  return m;
}

// Proposal, MH test and write-back of one tetrahedron of corner F from its
// network outputs o[16], its fields h and spins s. Returns 1 if accepted.
// p.closure: site 3 from its exact conditional (closure_move) instead of the
// network's fourth vMF.
template <int F>
__device__ __forceinline__ int tet_finish(const TetMoveParams& p, int rep, int cell, float beta,
                                          unsigned long long sweep, const pyro_vec3 h[4],
                                          const pyro_vec3 s[4], const float* o) {
  const uint32_t key_tet = (uint32_t)(F * p.L3 + cell);
  uint32_t r0[4], r1[4];
  pyro_philox(key_tet, (uint32_t)(p.rep_key + rep), (uint32_t)sweep, PYRO_PURPOSE_TET + 0,
              p.seed_lo, p.seed_hi, r0);
  pyro_philox(key_tet, (uint32_t)(p.rep_key + rep), (uint32_t)sweep, PYRO_PURPOSE_TET + 1,
              p.seed_lo, p.seed_hi, r1);
  const SiteMove m0 = site_move(o + 0, s[0], r0[0], r0[1]);
  const SiteMove m1 = site_move(o + 4, s[1], r0[2], r0[3]);
  const SiteMove m2 = site_move(o + 8, s[2], r1[0], r1[1]);
  const SiteMove m3 =
      p.closure ? closure_move(m0.sn, m1.sn, m2.sn,
                               closure_reverse(s[0], s[1], s[2], s[3], h[3], beta, p.J1), h[3],
                               beta, p.J1, r1[2], r1[3])
                : site_move(o + 12, s[3], r1[2], r1[3]);
  const pyro_vec3 sn[4] = {m0.sn, m1.sn, m2.sn, m3.sn};
  const float dE = tet_energy(sn, h, p.J1) - tet_energy(s, h, p.J1);
  const float log_q = (m0.lq + m1.lq) + (m2.lq + m3.lq);
  const float log_r = -beta * dE + log_q;
  const int accepted = log_r >= 0.0f || tet_test_uniform(r0) < __expf(log_r);
  if (p.trace) {
    float* t = p.trace + ((long long)rep * p.L3 + cell) * kTetTraceFloats;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      t[3 * k] = s[k].x;
      t[3 * k + 1] = s[k].y;
      t[3 * k + 2] = s[k].z;
      t[12 + 3 * k] = h[k].x;
      t[12 + 3 * k + 1] = h[k].y;
      t[12 + 3 * k + 2] = h[k].z;
      t[40 + 3 * k] = sn[k].x;
      t[40 + 3 * k + 1] = sn[k].y;
      t[40 + 3 * k + 2] = sn[k].z;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) t[24 + i] = o[i];
    t[52] = log_r;
    t[53] = (float)accepted;
    t[54] = tet_test_uniform(r0);
    t[55] = beta;
  }
  if (accepted) {
    float4* wb = p.spins + (long long)rep * 16 * p.L3;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      wb[(4 * F + k) * p.L3 + cell] = make_float4(sn[k].x, sn[k].y, sn[k].z, 0.0f);
  }
  return accepted;
}

// One warp's 32 tetrahedra of corner F (one per lane; lanes with
// active == false only feed the warp-wide MMAs): features, network, vMF
// proposals, MH test, write-back. Returns 1 if this lane's move was accepted.
// kWait: the weight copy of this CTA is still in flight (stage_weights) and
// is completed after the spin loads, a CTA-wide barrier.
template <int F, bool kL2, bool kWait>
__device__ __forceinline__ int tet_warp_step(const TetMoveParams& p, const MlpSmem& w, bool active,
                                             int rep, int cell, float beta,
                                             unsigned long long sweep, __nv_bfloat16* feat,
                                             float* out) {
  const int lane = threadIdx.x & 31;
  const float4* rb = p.spins + (long long)rep * 16 * p.L3;
  pyro_vec3 h[4], s[4];
  if (active) {
    const Frame fr = cell_frame(cell, p.L, p.rcpL);
    tet_fields<F, kL2>(rb, fr, p.L3, p.J1, h);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 v = ld_spin<kL2>(rb + (4 * F + k) * p.L3 + cell);
      s[k].x = v.x;
      s[k].y = v.y;
      s[k].z = v.z;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      h[k].x = h[k].y = h[k].z = 0.0f;
      s[k].x = s[k].y = 0.0f;
      s[k].z = 1.0f;
    }
  }
  write_features(feat + lane * kLdIn, h, active ? beta : 1.0f);
  if (kWait) stage_wait();
  else __syncwarp();
  TileFwd fw;
  tile_forward_move(feat, 0, w, fw);
  store_out(fw, 0, out);
  tile_forward_move(feat, 16, w, fw);
  store_out(fw, 16, out);
  __syncwarp();
  int accepted = 0;
  if (active) {
    float o[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) o[i] = out[lane * kLdOut + i];
    accepted = tet_finish<F>(p, rep, cell, beta, sweep, h, s, o);
  }
  return accepted;
}

// Offset of down-tetrahedron neighbour M of site S from replica start.
template <int S, int M>
__device__ __forceinline__ int down_off(const Frame& f, int L3) {
  constexpr NbrEntry e = j1_neighbour(S, j1_down_index(S, M));
  return f.zo[e.dz + 1] + f.yo[e.dy + 1] + f.xo[e.dx + 1] + e.t * L3;
}

// Down neighbour M of site 4F + 2 half + K, the site chosen per lane by a
// select instead of a branch, so that all loads of a lane issue together.
template <int F, int K, int M>
__device__ __forceinline__ int pair_down_off(const Frame& f, int L3, int half) {
  const int lo = down_off<4 * F + K, M>(f, L3), hi = down_off<4 * F + 2 + K, M>(f, L3);
  return half ? hi : lo;
}

// Same move with two lanes per tetrahedron (16 per warp, one MMA m-tile):
// lane l < 16 handles sites 0 and 1 of tetrahedron l, lane l + 16 sites 2
// and 3 (their fields, proposals and stores), which halves the serial work
// of a warp. Lane l then gathers the partner's values and evaluates the
// energy change and the proposal ratio with exactly the single-lane
// expressions, so the decisions are identical. Returns 1 on the lower lane
// of an accepted move. kWait as in tet_warp_step.
template <int F, bool kL2, bool kWait>
__device__ __forceinline__ int tet_pair_step(const TetMoveParams& p, const MlpSmem& w, bool active,
                                             int rep, int cell, float beta,
                                             unsigned long long sweep, __nv_bfloat16* feat,
                                             float* out) {
  const int lane = threadIdx.x & 31;
  const int half = lane >> 4;  // 0: sites 0, 1; 1: sites 2, 3
  const int row = lane & 15;
  // rep and cell are valid on inactive lanes too (their loads are in bounds;
  // they write nothing)
  const float4* rb = p.spins + (long long)rep * 16 * p.L3;
  const Frame fr = cell_frame(cell, p.L, p.rcpL);
  float4 nb[2][3], own[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) own[k] = ld_spin<kL2>(rb + (4 * F + 2 * half + k) * p.L3 + cell);
  nb[0][0] = ld_spin<kL2>(rb + pair_down_off<F, 0, 0>(fr, p.L3, half));
  nb[0][1] = ld_spin<kL2>(rb + pair_down_off<F, 0, 1>(fr, p.L3, half));
  nb[0][2] = ld_spin<kL2>(rb + pair_down_off<F, 0, 2>(fr, p.L3, half));
  nb[1][0] = ld_spin<kL2>(rb + pair_down_off<F, 1, 0>(fr, p.L3, half));
  nb[1][1] = ld_spin<kL2>(rb + pair_down_off<F, 1, 1>(fr, p.L3, half));
  nb[1][2] = ld_spin<kL2>(rb + pair_down_off<F, 1, 2>(fr, p.L3, half));
  // random words (no dependence on the spins) while the loads are in flight:
  // this lane's two proposals (and, on the lower lane, the acceptance test)
  const uint32_t key_tet = (uint32_t)(F * p.L3 + cell);
  uint32_t r[4];
  pyro_philox(key_tet, (uint32_t)(p.rep_key + rep), (uint32_t)sweep, PYRO_PURPOSE_TET + half,
              p.seed_lo, p.seed_hi, r);
  // external fields in ext_field's order
  pyro_vec3 h[2], s[2];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    h[k].x = p.J1 * ((nb[k][0].x + nb[k][1].x) + nb[k][2].x);
    h[k].y = p.J1 * ((nb[k][0].y + nb[k][1].y) + nb[k][2].y);
    h[k].z = p.J1 * ((nb[k][0].z + nb[k][1].z) + nb[k][2].z);
    s[k].x = own[k].x;
    s[k].y = own[k].y;
    s[k].z = own[k].z;
  }
  // the reverse term of site 3's conditional (upper lane) needs only the
  // current spins: evaluated before the network
  float rev3 = 0.0f;
  if (p.closure) {
    pyro_vec3 b0, b1;
    b0.x = __shfl_up_sync(0xffffffffu, s[0].x, 16);
    b0.y = __shfl_up_sync(0xffffffffu, s[0].y, 16);
    b0.z = __shfl_up_sync(0xffffffffu, s[0].z, 16);
    b1.x = __shfl_up_sync(0xffffffffu, s[1].x, 16);
    b1.y = __shfl_up_sync(0xffffffffu, s[1].y, 16);
    b1.z = __shfl_up_sync(0xffffffffu, s[1].z, 16);
    rev3 = closure_reverse(b0, b1, s[0], s[1], h[1], beta, p.J1);
  }
  __nv_bfloat16* frow = feat + row * kLdIn;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int c = 3 * (2 * half + k);
    frow[c] = __float2bfloat16_rn(h[k].x * (1.0f / 3.0f));
    frow[c + 1] = __float2bfloat16_rn(h[k].y * (1.0f / 3.0f));
    frow[c + 2] = __float2bfloat16_rn(h[k].z * (1.0f / 3.0f));
  }
  if (half == 0) {
    frow[12] = __float2bfloat16_rn(logf(active ? beta : 1.0f) * (1.0f / 3.0f));
    frow[13] = frow[14] = frow[15] = __float2bfloat16_rn(0.0f);
  }
  if (kWait) stage_wait();
  else __syncwarp();
  TileFwd fw;
  tile_forward_move(feat, 0, w, fw);
  store_out(fw, 0, out);
  __syncwarp();
  // this lane's two sites: network outputs 8 * half .. 8 * half + 7
  float o[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) o[i] = out[row * kLdOut + 8 * half + i];
  const SiteMove ma = site_move(o + 0, s[0], r[0], r[1]);
  // every lane draws its second network site (on the upper lane the draw for
  // site 3 is discarded when site 3 comes from its conditional): no branch,
  // so the two draws of a lane overlap
  SiteMove mb = site_move(o + 4, s[1], r[2], r[3]);
  if (p.closure) {
    // site 3 (upper lane) is conditional on the lower lane's proposed sites 0, 1
    pyro_vec3 a0, a1;
    a0.x = __shfl_up_sync(0xffffffffu, ma.sn.x, 16);
    a0.y = __shfl_up_sync(0xffffffffu, ma.sn.y, 16);
    a0.z = __shfl_up_sync(0xffffffffu, ma.sn.z, 16);
    a1.x = __shfl_up_sync(0xffffffffu, mb.sn.x, 16);
    a1.y = __shfl_up_sync(0xffffffffu, mb.sn.y, 16);
    a1.z = __shfl_up_sync(0xffffffffu, mb.sn.z, 16);
    if (half == 1) mb = closure_move(a0, a1, ma.sn, rev3, h[1], beta, p.J1, r[2], r[3]);
  }
  const pyro_vec3 sn[2] = {ma.sn, mb.sn};
  const float lq_half = ma.lq + mb.lq;
  // gather sites 2, 3 on the lower lane
  pyro_vec3 S[4], SN[4], H[4];
  S[0] = s[0];
  S[1] = s[1];
  SN[0] = sn[0];
  SN[1] = sn[1];
  H[0] = h[0];
  H[1] = h[1];
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    S[2 + k].x = __shfl_down_sync(0xffffffffu, s[k].x, 16);
    S[2 + k].y = __shfl_down_sync(0xffffffffu, s[k].y, 16);
    S[2 + k].z = __shfl_down_sync(0xffffffffu, s[k].z, 16);
    SN[2 + k].x = __shfl_down_sync(0xffffffffu, sn[k].x, 16);
    SN[2 + k].y = __shfl_down_sync(0xffffffffu, sn[k].y, 16);
    SN[2 + k].z = __shfl_down_sync(0xffffffffu, sn[k].z, 16);
    H[2 + k].x = __shfl_down_sync(0xffffffffu, h[k].x, 16);
    H[2 + k].y = __shfl_down_sync(0xffffffffu, h[k].y, 16);
    H[2 + k].z = __shfl_down_sync(0xffffffffu, h[k].z, 16);
  }
  const float lq_hi = __shfl_down_sync(0xffffffffu, lq_half, 16);
  uint32_t acc_word = 0;
  if (half == 0 && active) {
    const float dE = tet_energy(SN, H, p.J1) - tet_energy(S, H, p.J1);
    const float log_q = lq_half + lq_hi;
    const float log_r = -beta * dE + log_q;
    acc_word = (log_r >= 0.0f || tet_test_uniform(r) < __expf(log_r)) ? 1u : 0u;
  }
  const uint32_t accepted = __shfl_sync(0xffffffffu, acc_word, row);
  if (accepted && active) {
    float4* wb = p.spins + (long long)rep * 16 * p.L3;
#pragma unroll
    for (int k = 0; k < 2; ++k)
      wb[(4 * F + 2 * half + k) * p.L3 + cell] = make_float4(sn[k].x, sn[k].y, sn[k].z, 0.0f);
  }
  return half == 0 ? (int)accepted : 0;
}

// Acceptance per temperature slot: lanes of a warp that share a slot add
// once (a warp may straddle two replicas).
__device__ __forceinline__ void count_accepted(const TetMoveParams& p, int tslot, int accepted) {
  const int lane = threadIdx.x & 31;
  const unsigned peers = __match_any_sync(0xffffffffu, tslot);
  const unsigned acc_mask = __ballot_sync(0xffffffffu, accepted) & peers;
  if (lane == __ffs(peers) - 1 && acc_mask)
    atomicAdd(p.accepted + p.temp_base + tslot, (unsigned long long)__popc(acc_mask));
}

// Start of a per-pass kernel that may overlap the drain of the previous
// kernel of its stream (programmatic dependent launch): that kernel must be
// complete, its writes visible, before the first global access.
__device__ __forceinline__ void pass_prologue() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <int F>
__global__ void __launch_bounds__(kTetMoveThreads) tet_move_kernel(const TetMoveParams p) {
  pass_prologue();
  extern __shared__ __align__(16) unsigned char smem[];
  const MlpSmem w = carve_weights(smem);
  __nv_bfloat16* feat_all = reinterpret_cast<__nv_bfloat16*>(smem + kSmemWeightsFwd);
  float* out_all = reinterpret_cast<float*>(smem + kSmemWeightsFwd + kTetMoveThreads * kLdIn * 2);
  stage_weights(smem, p.image, kImgFwdBytes);
  const int warp = threadIdx.x >> 5;
  const long long tet = (long long)blockIdx.x * kTetMoveThreads + threadIdx.x;  // rep * L3 + cell
  const bool active = tet < (long long)p.n_rep * p.L3;
  const int rep = active ? (int)(tet / p.L3) : 0;
  const int cell = active ? (int)(tet - (long long)rep * p.L3) : 0;
  const int tslot = p.temp_of_rep[p.temp_base + p.rep_global + rep];
  const float beta = p.beta[p.temp_base + tslot];
  const unsigned long long sweep = (p.tet_ctr ? *p.tet_ctr : 0ull) + p.tet_off;
  const int acc = tet_warp_step<F, false, true>(p, w, active, rep, cell, beta, sweep,
                                          feat_all + warp * 32 * kLdIn,
                                          out_all + warp * 32 * kLdOut);
  count_accepted(p, tslot, acc);
}

// Per-pass kernel, two lanes per tetrahedron (256 threads = 128 tetrahedra).
template <int F>
__global__ void __launch_bounds__(kTetMoveThreads) tet_move_pair_kernel(const TetMoveParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  // The weight image is written only by the pack kernel, and every call that
  // packs synchronises its stream before returning, so no kernel that this
  // one may overlap writes it: its copy starts before the dependency wait.
  stage_weights(smem, p.image, kImgFwdBytes);
  pass_prologue();
  const MlpSmem w = carve_weights(smem);
  __nv_bfloat16* feat_all = reinterpret_cast<__nv_bfloat16*>(smem + kSmemWeightsFwd);
  float* out_all = reinterpret_cast<float*>(smem + kSmemWeightsFwd + kTetMoveThreads * kLdIn * 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long tet = (long long)blockIdx.x * (kTetMoveThreads / 2) + warp * 16 + (lane & 15);
  const bool active = tet < (long long)p.n_rep * p.L3;
  const int rep = active ? (int)(tet / p.L3) : 0;
  const int cell = active ? (int)(tet - (long long)rep * p.L3) : 0;
  const int tslot = p.temp_of_rep[p.temp_base + p.rep_global + rep];
  const float beta = p.beta[p.temp_base + tslot];
  const unsigned long long sweep = (p.tet_ctr ? *p.tet_ctr : 0ull) + p.tet_off;
  const int acc = tet_pair_step<F, false, true>(p, w, active, rep, cell, beta, sweep,
                                          feat_all + warp * 32 * kLdIn,
                                          out_all + warp * 32 * kLdOut);
  count_accepted(p, tslot, acc);
}

// The move with the network on the 5th-generation tensor cores: one thread
// per tetrahedron, 128 per CTA (tensor-memory lane = thread = row); fields
// and spins as tet_warp_step, the network of tet_umma.cuh, then the same
// proposal and MH test. A wait that runs out sets *p.err and skips the moves
// of the CTA.
template <int F>
__global__ void __launch_bounds__(umma::kURows) tet_move_umma_kernel(const TetMoveParams p) {
  pass_prologue();
  extern __shared__ __align__(16) unsigned char smem[];
  umma::stage_network(smem, p.image);
  umma::setup(smem);
  const long long tet = (long long)blockIdx.x * umma::kURows + threadIdx.x;  // rep * L3 + cell
  const bool active = tet < (long long)p.n_rep * p.L3;
  const int rep = active ? (int)(tet / p.L3) : 0;
  const int cell = active ? (int)(tet - (long long)rep * p.L3) : 0;
  const int tslot = p.temp_of_rep[p.temp_base + p.rep_global + rep];
  const float beta = p.beta[p.temp_base + tslot];
  const unsigned long long sweep = (p.tet_ctr ? *p.tet_ctr : 0ull) + p.tet_off;
  const float4* rb = p.spins + (long long)rep * 16 * p.L3;
  pyro_vec3 h[4], s[4];
  if (active) {
    const Frame fr = cell_frame(cell, p.L, p.rcpL);
    tet_fields<F, false>(rb, fr, p.L3, p.J1, h);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 v = __ldg(rb + (4 * F + k) * p.L3 + cell);
      s[k].x = v.x;
      s[k].y = v.y;
      s[k].z = v.z;
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      h[k].x = h[k].y = h[k].z = 0.0f;
      s[k].x = s[k].y = 0.0f;
      s[k].z = 1.0f;
    }
  }
  // features, rounded to BF16 as write_features does
  float x[kMlpIn];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    x[3 * k] = h[k].x * (1.0f / 3.0f);
    x[3 * k + 1] = h[k].y * (1.0f / 3.0f);
    x[3 * k + 2] = h[k].z * (1.0f / 3.0f);
  }
  x[12] = logf(active ? beta : 1.0f) * (1.0f / 3.0f);
  x[13] = x[14] = x[15] = 0.0f;
  umma::store_row(smem + umma::kUA0, threadIdx.x, kMlpIn, x);
  const uint32_t tmem = umma::ready(smem);
  uint32_t parity = 0;
  float o[kMlpOut];
  const bool ok = umma::network<true>(smem, tmem, o, &parity);
  int acc = 0;
  if (ok && active) acc = tet_finish<F>(p, rep, cell, beta, sweep, h, s, o);
  if (!ok && threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
  count_accepted(p, tslot, acc);
  umma::teardown(smem, tmem, ok, parity);
}

__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// n_sweeps tetrahedron sweeps of one replica per thread-block cluster: the
// four corner passes of a sweep are separated by cluster barriers, the
// weights are staged once, and the CTAs of the cluster split the replica's
// L^3 tetrahedra of a corner in chunks of kTetMoveThreads. Same proposals and
// decisions as the per-pass kernel.
__global__ void __launch_bounds__(kTetMoveThreads) tet_sweep_cluster_kernel(const TetMoveParams p,
                                                                            int n_sweeps,
                                                                            int csize) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MlpSmem w = carve_weights(smem);
  __nv_bfloat16* feat_all = reinterpret_cast<__nv_bfloat16*>(smem + kSmemWeightsFwd);
  float* out_all = reinterpret_cast<float*>(smem + kSmemWeightsFwd + kTetMoveThreads * kLdIn * 2);
  stage_weights(smem, p.image, kImgFwdBytes);
  stage_wait();
  const int warp = threadIdx.x >> 5;
  __nv_bfloat16* feat = feat_all + warp * 32 * kLdIn;
  float* out = out_all + warp * 32 * kLdOut;
  const int rep = blockIdx.x / csize, rank = blockIdx.x - rep * csize;
  const int tslot = p.temp_of_rep[p.temp_base + p.rep_global + rep];
  const float beta = p.beta[p.temp_base + tslot];
  const unsigned long long base = (p.tet_ctr ? *p.tet_ctr : 0ull) + p.tet_off;
  const int n_chunks = (p.L3 + kTetMoveThreads - 1) / kTetMoveThreads;
  int acc = 0;
  for (int k = 0; k < n_sweeps; ++k) {
    const unsigned long long sweep = base + (unsigned long long)k;
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
      for (int c = rank; c < n_chunks; c += csize) {
        const int cell = c * kTetMoveThreads + threadIdx.x;
        const bool active = cell < p.L3;
        const int cl = active ? cell : 0;
        switch (f) {
          case 0: acc += tet_warp_step<0, true, false>(p, w, active, rep, cl, beta, sweep, feat, out); break;
          case 1: acc += tet_warp_step<1, true, false>(p, w, active, rep, cl, beta, sweep, feat, out); break;
          case 2: acc += tet_warp_step<2, true, false>(p, w, active, rep, cl, beta, sweep, feat, out); break;
          default: acc += tet_warp_step<3, true, false>(p, w, active, rep, cl, beta, sweep, feat, out); break;
        }
      }
      cluster_sync_all();
    }
  }
  // every lane of this CTA belongs to one replica: plain warp sum
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0 && acc > 0)
    atomicAdd(p.accepted + p.temp_base + tslot, (unsigned long long)acc);
}

template <int F>
__device__ __forceinline__ void collect_one(const TetCollectParams& p, int rep, int cell, float* feat,
                                            float* targ) {
  const float4* rb = p.spins + (long long)rep * 16 * p.L3;
  const Frame fr = cell_frame(cell, p.L, p.rcpL);
  pyro_vec3 h[4];
  tet_fields<F>(rb, fr, p.L3, p.J1, h);
  const int g = p.rep_global + rep;
  const float beta = p.beta[p.temp_base + p.temp_of_rep[p.temp_base + g]];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    feat[3 * k] = h[k].x * (1.0f / 3.0f);
    feat[3 * k + 1] = h[k].y * (1.0f / 3.0f);
    feat[3 * k + 2] = h[k].z * (1.0f / 3.0f);
    const float4 v = __ldg(rb + (4 * F + k) * p.L3 + cell);
    targ[3 * k] = v.x;
    targ[3 * k + 1] = v.y;
    targ[3 * k + 2] = v.z;
  }
  feat[12] = logf(beta) * (1.0f / 3.0f);
  feat[13] = feat[14] = feat[15] = 0.0f;
}

__global__ void tet_collect_kernel(const TetCollectParams p) {
  const long long per_class_rep = (p.L3 + p.stride - 1) / p.stride;
  const long long total = 4ll * p.n_rep * per_class_rep;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(i / ((long long)p.n_rep * per_class_rep));
    const long long rest = i - (long long)f * p.n_rep * per_class_rep;
    const int rep = (int)(rest / per_class_rep);
    const int cell = (int)(rest - (long long)rep * per_class_rep) * p.stride;
    const long long slot = (p.head + i) % p.cap;
    float* feat = p.features + slot * 16;
    float* targ = p.targets + slot * 12;
    switch (f) {
      case 0: collect_one<0>(p, rep, cell, feat, targ); break;
      case 1: collect_one<1>(p, rep, cell, feat, targ); break;
      case 2: collect_one<2>(p, rep, cell, feat, targ); break;
      default: collect_one<3>(p, rep, cell, feat, targ); break;
    }
  }
}

// One BF16 matrix region of the weight image: rows x ld entries, the first
// `cols` of a row taken from the master array (element (r, c) at
// m[off + r * rs + c * cs]), the padding zero.
__device__ __forceinline__ void pack_region(const float* __restrict__ m, unsigned char* image,
                                            int region, int rows, int ld, int cols, int off,
                                            int rs, int cs, int tid, int nthreads) {
  __nv_bfloat16* dst = reinterpret_cast<__nv_bfloat16*>(image + region);
  for (int i = tid; i < rows * ld; i += nthreads) {
    const int r = i / ld, c = i - r * ld;
    dst[i] = __float2bfloat16_rn(c < cols ? m[off + r * rs + c * cs] : 0.0f);
  }
}

// An N x K operand W^T (element (n, k) = m[off + k * N + n]) in the
// canonical K-major core-matrix layout of the tensor-memory MMA.
__device__ __forceinline__ void pack_core(const float* __restrict__ m, unsigned char* image,
                                          int region, int N, int K, int off, int tid, int nthreads) {
  __nv_bfloat16* dst = reinterpret_cast<__nv_bfloat16*>(image + region);
  for (int i = tid; i < N * K; i += nthreads) {
    const int n = i / K, k = i - n * K;
    const int byte = (n / 8) * (K / 8) * 128 + (k / 8) * 128 + (n % 8) * 16 + (k % 8) * 2;
    dst[byte / 2] = __float2bfloat16_rn(m[off + k * N + n]);
  }
}

__global__ void mlp_pack_kernel(const float* __restrict__ m, unsigned char* image) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  // forward operands, [out][in]: element (o, i) = W[i][o]
  pack_region(m, image, kImgW1t, kMlpHidden, kLdIn, kMlpIn, kOffW1, 1, kMlpHidden, tid, nt);
  pack_region(m, image, kImgW2t, kMlpHidden, kLdH, kMlpHidden, kOffW2, 1, kMlpHidden, tid, nt);
  pack_region(m, image, kImgW3t, kMlpOut, kLdH, kMlpHidden, kOffW3, 1, kMlpOut, tid, nt);
  // backward operands, [in][out]
  pack_region(m, image, kImgW2, kMlpHidden, kLdH, kMlpHidden, kOffW2, kMlpHidden, 1, tid, nt);
  pack_region(m, image, kImgW3, kMlpHidden, kLdIn, kMlpOut, kOffW3, kMlpOut, 1, tid, nt);
  // forward operands in the tcgen05 core-matrix layout, element (n, k) = W[k][n]
  pack_core(m, image, kImgU1, kMlpHidden, kMlpIn, kOffW1, tid, nt);
  pack_core(m, image, kImgU2, kMlpHidden, kMlpHidden, kOffW2, tid, nt);
  pack_core(m, image, kImgU3, kMlpOut, kMlpHidden, kOffW3, tid, nt);
  float* b = reinterpret_cast<float*>(image + kImgB1);  // b1, b2, b3 contiguous
  for (int i = tid; i < 2 * kMlpHidden + kMlpOut; i += nt)
    b[i] = i < kMlpHidden ? m[kOffB1 + i]
                          : (i < 2 * kMlpHidden ? m[kOffB2 + i - kMlpHidden]
                                                : m[kOffB3 + i - 2 * kMlpHidden]);
}

__global__ void __launch_bounds__(kTetThreads) mlp_forward_kernel(const float* __restrict__ features,
                                                                  int n,
                                                                  const unsigned char* image,
                                                                  float* out) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MlpSmem w = carve_weights(smem);
  __nv_bfloat16* feat_all = reinterpret_cast<__nv_bfloat16*>(smem + kSmemWeightsFwd);
  float* out_all = reinterpret_cast<float*>(smem + kSmemWeightsFwd + kTetThreads * kLdIn * 2);
  stage_weights(smem, image, kImgFwdBytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __nv_bfloat16* feat = feat_all + warp * 32 * kLdIn;
  float* o = out_all + warp * 32 * kLdOut;
  const long long row = (long long)blockIdx.x * kTetThreads + threadIdx.x;
  for (int i = 0; i < 16; ++i)
    feat[lane * kLdIn + i] = __float2bfloat16_rn(row < n ? features[row * 16 + i] : 0.0f);
  stage_wait();
  TileFwd fw;
  tile_forward<false>(feat, 0, w, fw, nullptr, nullptr);
  store_out(fw, 0, o);
  tile_forward<false>(feat, 16, w, fw, nullptr, nullptr);
  store_out(fw, 16, o);
  __syncwarp();
  if (row < n)
    for (int i = 0; i < 16; ++i) out[row * 16 + i] = o[lane * kLdOut + i];
}

// Per-warp shared buffers of the gradient kernel.
struct GradWarpSmem {
  __nv_bfloat16* feat;  // [32][kLdIn] row major
  __nv_bfloat16* xt;    // [16][kLdB]  feature major
  __nv_bfloat16* h1t;   // [64][kLdB]
  __nv_bfloat16* h2t;   // [64][kLdB]
  __nv_bfloat16* dorow;  // [32][kLdIn] dL/do row major
  __nv_bfloat16* dot;   // [16][kLdB]
  __nv_bfloat16* da2t;  // [64][kLdB]
  __nv_bfloat16* da1t;  // [64][kLdB]
  float* out;           // [32][kLdOut]
};
constexpr int kGradWarpBytes =
    (32 * kLdIn + 16 * kLdB + 64 * kLdB * 2 + 32 * kLdIn + 16 * kLdB + 64 * kLdB * 2) * 2 +
    32 * kLdOut * 4;
constexpr int kGradSmem = kSmemWeightsAll + 4 * kGradWarpBytes + kMlpParams * 4;

__device__ GradWarpSmem carve_warp(unsigned char* base) {
  GradWarpSmem s;
  __nv_bfloat16* b = reinterpret_cast<__nv_bfloat16*>(base);
  s.feat = b;
  s.xt = s.feat + 32 * kLdIn;
  s.h1t = s.xt + 16 * kLdB;
  s.h2t = s.h1t + 64 * kLdB;
  s.dorow = s.h2t + 64 * kLdB;
  s.dot = s.dorow + 32 * kLdIn;
  s.da2t = s.dot + 16 * kLdB;
  s.da1t = s.da2t + 64 * kLdB;
  s.out = reinterpret_cast<float*>(s.da1t + 64 * kLdB);
  return s;
}

// sum over the 8 row groups (lanes with equal lane % 4)
__device__ __forceinline__ float group_sum(float v) {
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 16);
  return v;
}

// Weight-gradient GEMM of one warp: G[m][n] += sum_b AT[m][b] * BT[n][b],
// AT: [M][kLdB], BT: [N][kLdB] (feature major, 32 batch entries), added to
// the shared FP32 gradient block at `grad` with row stride n_total.
template <int M, int N>
__device__ __forceinline__ void weight_grad(const __nv_bfloat16* at, const __nv_bfloat16* bt,
                                            float* grad, int n_total) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mt = 0; mt < M / 16; ++mt) {
    float c[N / 8][4];
#pragma unroll
    for (int j = 0; j < N / 8; ++j) c[j][0] = c[j][1] = c[j][2] = c[j][3] = 0.0f;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      const __nv_bfloat16* ar = at + (16 * mt + g) * kLdB + 16 * ks + 2 * t;
      const uint32_t a0 = ld32(ar), a1 = ld32(ar + 8 * kLdB), a2 = ld32(ar + 8),
                     a3 = ld32(ar + 8 * kLdB + 8);
#pragma unroll
      for (int j = 0; j < N / 8; ++j) {
        const __nv_bfloat16* br = bt + (8 * j + g) * kLdB + 16 * ks + 2 * t;
        mma_bf16(c[j], a0, a1, a2, a3, ld32(br), ld32(br + 8));
      }
    }
#pragma unroll
    for (int j = 0; j < N / 8; ++j) {
      const int r0 = 16 * mt + g, col = 8 * j + 2 * t;
      atomicAdd(grad + r0 * n_total + col, c[j][0]);
      atomicAdd(grad + r0 * n_total + col + 1, c[j][1]);
      atomicAdd(grad + (r0 + 8) * n_total + col, c[j][2]);
      atomicAdd(grad + (r0 + 8) * n_total + col + 1, c[j][3]);
    }
  }
}

// Negative log-likelihood of the targets under the vMF mixture of one sample
// and its gradient with respect to the 16 network outputs.
__device__ __forceinline__ float nll_and_grad(const float* o, const float* s, float* d) {
  const VmfParams v = vmf_params(o);
  float loss = 0.0f;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float kap = v.kappa[k];
    pyro_vec3 sk;
    sk.x = s[3 * k];
    sk.y = s[3 * k + 1];
    sk.z = s[3 * k + 2];
    const float m = dot3(v.mu[k], sk);
    const float em = -expm1f(-2.0f * kap);  // 1 - e^{-2 kappa}
    // log f = z - log(2 pi) - log(1 - e^{-2 kappa}) + kappa (m - 1)
    loss -= v.z[k] - 1.8378770664093453f - logf(em) + kap * (m - 1.0f);
    const float r = 2.0f * kap / expm1f(2.0f * kap);
    d[4 * k + 3] = v.z_in[k] ? -(1.0f - r + kap * (m - 1.0f)) : 0.0f;
    // d/d mu = -kappa s; through mu = o / |o|
    const float inv = 1.0f / v.onorm[k];
    d[4 * k + 0] = -kap * (sk.x - m * v.mu[k].x) * inv;
    d[4 * k + 1] = -kap * (sk.y - m * v.mu[k].y) * inv;
    d[4 * k + 2] = -kap * (sk.z - m * v.mu[k].z) * inv;
  }
  return loss;
}

__global__ void __launch_bounds__(kTetThreads) mlp_gradient_kernel(
    const float* __restrict__ features, const float* __restrict__ targets, const int* idx, int n,
    const unsigned char* image, float* grad, double* loss_sum) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MlpSmem w = carve_weights(smem);
  unsigned char* wbase = smem + kSmemWeightsAll;
  float* g_acc = reinterpret_cast<float*>(wbase + 4 * kGradWarpBytes);
  stage_weights(smem, image, kImgBytes);
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) g_acc[i] = 0.0f;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  GradWarpSmem ws = carve_warp(wbase + warp * kGradWarpBytes);
  stage_wait();
  float loss_local = 0.0f;
  for (long long base = (long long)blockIdx.x * kTetThreads; base < n;
       base += (long long)gridDim.x * kTetThreads) {
    const long long row = base + threadIdx.x;
    const bool valid = row < n;
    const long long src = valid ? (idx ? (long long)idx[row] : row) : 0;
    float tg[12];
    for (int i = 0; i < 16; ++i) {
      const float x = valid ? features[src * 16 + i] : 0.0f;
      const __nv_bfloat16 xb = __float2bfloat16_rn(x);
      ws.feat[lane * kLdIn + i] = xb;
      ws.xt[i * kLdB + lane] = xb;
    }
    for (int i = 0; i < 12; ++i) tg[i] = valid ? targets[src * 12 + i] : 0.0f;
    __syncwarp();
    // forward + output gradient, tile by tile
    TileFwd fw[2];
    tile_forward<true>(ws.feat, 0, w, fw[0], ws.h1t, ws.h2t);
    store_out(fw[0], 0, ws.out);
    tile_forward<true>(ws.feat, 16, w, fw[1], ws.h1t, ws.h2t);
    store_out(fw[1], 16, ws.out);
    __syncwarp();
    {
      float o[16], d[16];
      for (int i = 0; i < 16; ++i) o[i] = ws.out[lane * kLdOut + i];
      const float l = nll_and_grad(o, tg, d);
      if (valid) loss_local += l;
      for (int i = 0; i < 16; ++i) {
        const __nv_bfloat16 db = __float2bfloat16_rn(valid ? d[i] : 0.0f);
        ws.dorow[lane * kLdIn + i] = db;
        ws.dot[i * kLdB + lane] = db;
        if (valid) atomicAdd(&g_acc[kOffB3 + i], d[i]);  // bias b3, FP32
      }
    }
    __syncwarp();
    // backward through layers 3 and 2, tile by tile
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
      const int r0 = 16 * mt + g, r1 = r0 + 8;
      const uint32_t a0 = ld32(ws.dorow + r0 * kLdIn + 2 * t), a1 = ld32(ws.dorow + r1 * kLdIn + 2 * t);
      const uint32_t a2 = ld32(ws.dorow + r0 * kLdIn + 8 + 2 * t),
                     a3 = ld32(ws.dorow + r1 * kLdIn + 8 + 2 * t);
      float da2[8][4];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        da2[j][0] = da2[j][1] = da2[j][2] = da2[j][3] = 0.0f;
        const __nv_bfloat16* bw = w.w3 + (8 * j + g) * kLdIn + 2 * t;
        mma_bf16(da2[j], a0, a1, a2, a3, ld32(bw), ld32(bw + 8));
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
#pragma unroll
        for (int e = 0; e < 4; ++e) da2[j][e] *= hswish_grad(fw[mt].pre2[j][e]);
        const int c = 8 * j + 2 * t;
        ws.da2t[c * kLdB + r0] = __float2bfloat16_rn(da2[j][0]);
        ws.da2t[(c + 1) * kLdB + r0] = __float2bfloat16_rn(da2[j][1]);
        ws.da2t[c * kLdB + r1] = __float2bfloat16_rn(da2[j][2]);
        ws.da2t[(c + 1) * kLdB + r1] = __float2bfloat16_rn(da2[j][3]);
        const float s0 = group_sum(da2[j][0] + da2[j][2]), s1 = group_sum(da2[j][1] + da2[j][3]);
        if (g == 0) {
          atomicAdd(&g_acc[kOffB2 + c], s0);
          atomicAdd(&g_acc[kOffB2 + c + 1], s1);
        }
      }
      float da1[8][4];
#pragma unroll
      for (int j = 0; j < 8; ++j) da1[j][0] = da1[j][1] = da1[j][2] = da1[j][3] = 0.0f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint32_t x0 = pack_bf16(da2[2 * kk][0], da2[2 * kk][1]);
        const uint32_t x1 = pack_bf16(da2[2 * kk][2], da2[2 * kk][3]);
        const uint32_t x2 = pack_bf16(da2[2 * kk + 1][0], da2[2 * kk + 1][1]);
        const uint32_t x3 = pack_bf16(da2[2 * kk + 1][2], da2[2 * kk + 1][3]);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const __nv_bfloat16* bw = w.w2 + (8 * j + g) * kLdH + 16 * kk + 2 * t;
          mma_bf16(da1[j], x0, x1, x2, x3, ld32(bw), ld32(bw + 8));
        }
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
#pragma unroll
        for (int e = 0; e < 4; ++e) da1[j][e] *= hswish_grad(fw[mt].pre1[j][e]);
        const int c = 8 * j + 2 * t;
        ws.da1t[c * kLdB + r0] = __float2bfloat16_rn(da1[j][0]);
        ws.da1t[(c + 1) * kLdB + r0] = __float2bfloat16_rn(da1[j][1]);
        ws.da1t[c * kLdB + r1] = __float2bfloat16_rn(da1[j][2]);
        ws.da1t[(c + 1) * kLdB + r1] = __float2bfloat16_rn(da1[j][3]);
        const float s0 = group_sum(da1[j][0] + da1[j][2]), s1 = group_sum(da1[j][1] + da1[j][3]);
        if (g == 0) {
          atomicAdd(&g_acc[kOffB1 + c], s0);
          atomicAdd(&g_acc[kOffB1 + c + 1], s1);
        }
      }
    }
    __syncwarp();
    // weight gradients: dW1 = X^T dA1, dW2 = H1^T dA2, dW3 = H2^T dO
    weight_grad<16, 64>(ws.xt, ws.da1t, g_acc + kOffW1, 64);
    weight_grad<64, 64>(ws.h1t, ws.da2t, g_acc + kOffW2, 64);
    weight_grad<64, 16>(ws.h2t, ws.dot, g_acc + kOffW3, 16);
    __syncwarp();
  }
  // loss: warp sum, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) loss_local += __shfl_down_sync(0xffffffffu, loss_local, o);
  if (lane == 0) atomicAdd(loss_sum, (double)loss_local);
  __syncthreads();
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x)
    if (g_acc[i] != 0.0f) atomicAdd(grad + i, g_acc[i]);
}

__global__ void adam_kernel(float* w, float* m, float* v, const float* g, int n, float lr,
                            float b1, float b2, float eps, float scale, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float gi = g[i] * scale;
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void draw_batch_kernel(int* idx, int n, long long n_avail, uint32_t seed_lo,
                                  uint32_t seed_hi, uint32_t step) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t r[4];
    pyro_philox((uint32_t)i, step, 0u, PYRO_PURPOSE_TET + 8, seed_lo, seed_hi, r);
    const unsigned long long x = ((unsigned long long)r[0] << 32) | r[1];
    idx[i] = (int)(x % (unsigned long long)n_avail);
  }
}

constexpr int kTetSmem = kSmemWeightsFwd + kTetThreads * kLdIn * 2 + kTetThreads * kLdOut * 4;
constexpr int kTetMoveSmem =
    kSmemWeightsFwd + kTetMoveThreads * kLdIn * 2 + kTetMoveThreads * kLdOut * 4;

}  // namespace

void launch_mlp_pack(const float* master, unsigned char* image, cudaStream_t st) {
  mlp_pack_kernel<<<(kImgBytes / 2 + 255) / 256, 256, 0, st>>>(master, image);
}

namespace {
template <typename Kernel>
void launch_move(Kernel k, int blocks, const TetMoveParams& p, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks, 1, 1);
  cfg.blockDim = dim3(kTetMoveThreads, 1, 1);
  cfg.dynamicSmemBytes = kTetMoveSmem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = p.pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, k, p);  // errors are read back with cudaGetLastError
}
}  // namespace

void launch_tet_move(const TetMoveParams& p, int f, int form, cudaStream_t st) {
  const long long n = (long long)p.n_rep * p.L3;
  if (form == 3) {
    const int blocks = (int)((n + umma::kURows - 1) / umma::kURows);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks, 1, 1);
    cfg.blockDim = dim3(umma::kURows, 1, 1);
    cfg.dynamicSmemBytes = umma::kUSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = p.pdl ? 1 : 0;
    switch (f) {
      case 0: cudaLaunchKernelEx(&cfg, tet_move_umma_kernel<0>, p); break;
      case 1: cudaLaunchKernelEx(&cfg, tet_move_umma_kernel<1>, p); break;
      case 2: cudaLaunchKernelEx(&cfg, tet_move_umma_kernel<2>, p); break;
      default: cudaLaunchKernelEx(&cfg, tet_move_umma_kernel<3>, p); break;
    }
    return;  // errors are read back with cudaGetLastError
  }
  if (form == 2) {
    const int half = kTetMoveThreads / 2;
    const int blocks = (int)((n + half - 1) / half);
    switch (f) {
      case 0: launch_move(tet_move_pair_kernel<0>, blocks, p, st); break;
      case 1: launch_move(tet_move_pair_kernel<1>, blocks, p, st); break;
      case 2: launch_move(tet_move_pair_kernel<2>, blocks, p, st); break;
      default: launch_move(tet_move_pair_kernel<3>, blocks, p, st); break;
    }
    return;
  }
  const int blocks = (int)((n + kTetMoveThreads - 1) / kTetMoveThreads);
  switch (f) {
    case 0: launch_move(tet_move_kernel<0>, blocks, p, st); break;
    case 1: launch_move(tet_move_kernel<1>, blocks, p, st); break;
    case 2: launch_move(tet_move_kernel<2>, blocks, p, st); break;
    default: launch_move(tet_move_kernel<3>, blocks, p, st); break;
  }
}

cudaError_t tet_cluster_prepare(int csize, int* max_active) {
  *max_active = 0;
  cudaError_t e = cudaFuncSetAttribute(tet_sweep_cluster_kernel,
                                       cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(csize * 8, 1, 1);
  cfg.blockDim = dim3(kTetMoveThreads, 1, 1);
  cfg.dynamicSmemBytes = kTetMoveSmem;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaOccupancyMaxActiveClusters(max_active, tet_sweep_cluster_kernel, &cfg);
}

cudaError_t launch_tet_sweep_cluster(const TetMoveParams& p, int n_sweeps, int csize,
                                     cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(csize * p.n_rep, 1, 1);
  cfg.blockDim = dim3(kTetMoveThreads, 1, 1);
  cfg.dynamicSmemBytes = kTetMoveSmem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, tet_sweep_cluster_kernel, p, n_sweeps, csize);
}

int tet_chunks(int L3) { return (L3 + kTetMoveThreads - 1) / kTetMoveThreads; }

long long tet_collect_count(int L3, int n_rep, int stride) {
  return 4ll * n_rep * ((L3 + stride - 1) / stride);
}

void launch_tet_collect(const TetCollectParams& p, cudaStream_t st) {
  const long long n = tet_collect_count(p.L3, p.n_rep, p.stride);
  long long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  tet_collect_kernel<<<(int)blocks, 256, 0, st>>>(p);
}

void launch_mlp_forward(const float* features, int n, const unsigned char* image, float* out,
                        cudaStream_t st) {
  const int blocks = (n + kTetThreads - 1) / kTetThreads;
  mlp_forward_kernel<<<blocks, kTetThreads, kTetSmem, st>>>(features, n, image, out);
}

void launch_mlp_gradient(const float* features, const float* targets, const int* idx, int n,
                         const unsigned char* image, float* grad, double* loss,
                         cudaStream_t st) {
  static bool attr_set = false;
  if (!attr_set) {
    cudaFuncSetAttribute(mlp_gradient_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kGradSmem);
    attr_set = true;
  }
  int blocks = (n + kTetThreads - 1) / kTetThreads;
  if (blocks > 148 * 2) blocks = 148 * 2;
  if (blocks < 1) blocks = 1;
  mlp_gradient_kernel<<<blocks, kTetThreads, kGradSmem, st>>>(features, targets, idx, n, image,
                                                               grad, loss);
}

void launch_adam(float* master, float* m, float* v, const float* grad, int n, float lr,
                 float beta1, float beta2, float eps, float scale, int step, cudaStream_t st) {
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  adam_kernel<<<(n + 255) / 256, 256, 0, st>>>(master, m, v, grad, n, lr, beta1, beta2, eps, scale,
                                               c1, c2);
}

void launch_draw_batch(int* idx, int n, long long n_avail, uint32_t seed_lo, uint32_t seed_hi,
                       uint32_t step, cudaStream_t st) {
  draw_batch_kernel<<<(n + 255) / 256, 256, 0, st>>>(idx, n, n_avail, seed_lo, seed_hi, step);
}

}  // namespace pyro
