// Launch interface of the structure-factor kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace pyro {

struct SqParams {
  int L, G, stride;
  int Lf;              // fold period L / gcd(L, stride)
  int R;               // transform outputs per axis: G if G <= Lf, else Lf
  int residues;        // R == Lf < G: wave number w uses transform index w mod Lf
  const double2* tw4;  // tw4[j] = exp(-2 pi i j / (4 L)), j < 4 L (basis phases)
  int pos4[48];        // basis positions of the 16 sites, units a/4
  double inv_n_norm;   // 1 / (N * replicas averaged)
};

// Scratch bytes per replica of one launch_structure_factor call.
size_t sq_scratch_per_replica(const SqParams& p);
// Raises the DFT kernels' dynamic shared memory limit (outside any capture).
cudaError_t sq_prepare();
// Adds S(q) of n_rep consecutive replicas (divided by N * replicas averaged,
// p.inv_n_norm) to sq[G^3]. roots[j] = exp(-2 pi i j / Lf), j < Lf;
// steps[k] = (stride / gcd(L, stride)) w(k) mod Lf for the transform index
// k < R (w(k) = k - G/2, or k with residues). scratch: n_rep *
// sq_scratch_per_replica(p) bytes.
void launch_structure_factor(const float4* spins, int n_rep, const SqParams& p,
                             const double2* roots, const int* steps, void* scratch, double* sq,
                             cudaStream_t st);

}  // namespace pyro
