// Learned tetrahedron proposal: a 16 -> 64 -> 64 -> 16 MLP (BF16 weights,
// FP32 accumulation on the tensor cores) that maps the external fields of the
// four spins of an up-tetrahedron (and beta) to a von Mises-Fisher
// distribution for each of them. The joint move draws sites 0-2 from the
// network's vMFs and site 3 either from the network's fourth vMF or from its
// exact conditional distribution given the three new spins and its external
// field (a vMF too); it is accepted with the exact Metropolis-Hastings ratio.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyro {

constexpr int kMlpIn = 16;   // 12 field components / 3, log(beta) / 3, 3 zeros
constexpr int kMlpHidden = 64;
constexpr int kMlpOut = 16;  // per site k: mu direction (3, unnormalised), log kappa
// FP32 master layout (row = input feature, contiguous = output feature):
constexpr int kOffW1 = 0;                                  // [16][64]
constexpr int kOffB1 = kOffW1 + kMlpIn * kMlpHidden;       // [64]
constexpr int kOffW2 = kOffB1 + kMlpHidden;                // [64][64]
constexpr int kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;   // [64]
constexpr int kOffW3 = kOffB2 + kMlpHidden;                // [64][16]
constexpr int kOffB3 = kOffW3 + kMlpHidden * kMlpOut;      // [16]
constexpr int kMlpParams = kOffB3 + kMlpOut;               // 6288
constexpr float kLogKappaMin = -4.0f, kLogKappaMax = 6.0f;
constexpr float kKappaFloor = 0.018315639f;  // exp(kLogKappaMin)

// The weights as the byte image of the kernels' shared-memory copy: BF16
// operand matrices in padded rows (conflict-free fragment loads), FP32
// biases. Forward operands are the transposed matrices ([out][in], input
// contiguous), backward operands the master orientation ([in][out]). The
// forward part comes first, so forward-only kernels copy a prefix; every
// offset is a multiple of 16 bytes, so a CTA stages the image with 16-byte
// asynchronous copies.
constexpr int kLdIn = 24;  // padded row of 16 bf16 (48 B)
constexpr int kLdH = 72;   // padded row of 64 bf16 (144 B)
constexpr int kImgW1t = 0;                                   // bf16 [64][kLdIn]
constexpr int kImgW2t = kImgW1t + kMlpHidden * kLdIn * 2;    // bf16 [64][kLdH]
constexpr int kImgW3t = kImgW2t + kMlpHidden * kLdH * 2;     // bf16 [16][kLdH]
constexpr int kImgB1 = kImgW3t + kMlpOut * kLdH * 2;         // f32 [64]
constexpr int kImgB2 = kImgB1 + kMlpHidden * 4;              // f32 [64]
constexpr int kImgB3 = kImgB2 + kMlpHidden * 4;              // f32 [16]
constexpr int kImgFwdBytes = kImgB3 + kMlpOut * 4;
constexpr int kImgW2 = kImgFwdBytes;                         // bf16 [64][kLdH]
constexpr int kImgW3 = kImgW2 + kMlpHidden * kLdH * 2;       // bf16 [64][kLdIn]
constexpr int kImgBytes = kImgW3 + kMlpHidden * kLdIn * 2;
// The forward operands again in the tensor-memory MMA's canonical K-major
// layout (8-row x 16-byte core matrices, no swizzle): element (n, k) of an
// N x K operand at (n / 8) * (K / 8) * 128 + (k / 8) * 128 + (n % 8) * 16 +
// (k % 8) * 2 bytes.
constexpr int kImgU1 = kImgBytes;                            // W1^T, N=64, K=16
constexpr int kImgU2 = kImgU1 + kMlpHidden * kMlpIn * 2;     // W2^T, N=64, K=64
constexpr int kImgU3 = kImgU2 + kMlpHidden * kMlpHidden * 2; // W3^T, N=16, K=64
constexpr int kImgTotal = kImgU3 + kMlpOut * kMlpHidden * 2;
static_assert(kImgW2t % 16 == 0 && kImgW3t % 16 == 0 && kImgB1 % 16 == 0 &&
                  kImgFwdBytes % 16 == 0 && kImgW3 % 16 == 0 && kImgBytes % 16 == 0,
              "16-byte staging granules");
static_assert(kImgU2 % 16 == 0 && kImgU3 % 16 == 0 && kImgTotal % 16 == 0, "core matrices");

struct TetMoveParams {
  float4* spins;  // replica 0 of the system
  int L, L3, n_rep;
  float rcpL;
  int rep_global, rep_key, temp_base;
  float J1;
  const int* temp_of_rep;
  const float* beta;
  unsigned long long* accepted;  // [temp_base + t]
  const unsigned long long* tet_ctr;
  unsigned long long tet_off;
  uint32_t seed_lo, seed_hi;
  const unsigned char* image;  // kImgBytes weight image
  int closure;                 // 1: site 3 from its exact conditional, 0: the network's vMF
  int pdl;                     // programmatic dependent launch of the per-pass kernels
  int* err;                    // set to 1 if a tensor-core wait of the tcgen05 form ran out
  // Diagnostics (null in the Monte Carlo): one record of kTetTraceFloats per
  // tetrahedron at trace[(rep * L3 + cell) * kTetTraceFloats] (forms 0 and 3).
  float* trace;
};

// Trace record of one learned move: spins before (12), external fields (12),
// network outputs (16), proposal (12), log of the MH ratio as evaluated,
// decision (0 / 1), the test uniform, beta.
constexpr int kTetTraceFloats = 56;

struct TetCollectParams {
  const float4* spins;
  int L, L3, n_rep;
  float rcpL;
  int rep_global, temp_base;
  float J1;
  const int* temp_of_rep;
  const float* beta;
  int stride;          // every stride-th tetrahedron of a class
  float* features;     // ring [cap][16]
  float* targets;      // ring [cap][12]
  int cap;
  long long head;      // first slot written (mod cap)
};

// Writes the weight image (kImgBytes) of the FP32 master weights.
void launch_mlp_pack(const float* master, unsigned char* image, cudaStream_t st);
// One pass of the learned move over up-tetrahedra of FCC corner f. form 0:
// one lane per tetrahedron (mma.sync network); 2: two lanes per tetrahedron
// (same decisions as 0); 3: the network on tcgen05 (tensor memory), one
// thread per tetrahedron, 128 per CTA (same move, its own rounding of the
// network's accumulations).
void launch_tet_move(const TetMoveParams& p, int f, int form, cudaStream_t st);
// n sweeps (4 corner passes each) of every replica in one launch, one
// thread-block cluster of csize CTAs per replica.
cudaError_t launch_tet_sweep_cluster(const TetMoveParams& p, int n_sweeps, int csize,
                                     cudaStream_t st);
cudaError_t tet_cluster_prepare(int csize, int* max_active);
int tet_chunks(int L3);  // chunks of tetrahedra per corner and replica
// Number of samples one collect call writes: 4 classes x n_rep x ceil(L3 / stride).
long long tet_collect_count(int L3, int n_rep, int stride);
void launch_tet_collect(const TetCollectParams& p, cudaStream_t st);
// Network outputs for n feature rows on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory), 128 rows per CTA; *err is set
// to 1 if a wait for an MMA ran out (the outputs are then not written).
cudaError_t launch_umma_forward(const float* features, int n, const unsigned char* image,
                               float* out, int* err, cudaStream_t st);
// Network outputs for n feature rows (host-visible test path).
void launch_mlp_forward(const float* features, int n, const unsigned char* image, float* out,
                        cudaStream_t st);
// Adds d(sum of per-sample negative log-likelihood)/d(params) of rows
// idx[0..n) (or 0..n if idx is null) to grad[kMlpParams] and the loss sum to
// *loss.
void launch_mlp_gradient(const float* features, const float* targets, const int* idx, int n,
                         const unsigned char* image, float* grad, double* loss, cudaStream_t st);
void launch_adam(float* master, float* m, float* v, const float* grad, int n, float lr,
                 float beta1, float beta2, float eps, float scale, int step, cudaStream_t st);
// idx[i] = Philox-drawn sample indices in [0, n_avail).
void launch_draw_batch(int* idx, int n, long long n_avail, uint32_t seed_lo, uint32_t seed_hi,
                       uint32_t step, cudaStream_t st);

}  // namespace pyro
