// Launch interface of the structure-factor kernels.
#pragma once
#include <cuda_runtime.h>

namespace pyro {

struct SqParams {
  int L, G, stride;
  const double2* tw;   // tw[j] = exp(-2 pi i j / (4 L)), j < 4 L
  int pos4[48];        // basis positions of the 16 sites, units a/4
  double inv_n_norm;   // 1 / (N * replicas averaged)
};

// Adds one replica's S(q) (divided by N * replicas) to sq[G^3]. Scratch:
// s1: 48 L^2 G, s2: 48 L G^2, s3: 48 G^3 complex doubles.
void launch_structure_factor_replica(const float4* rep_spins, const SqParams& p, double2* s1,
                                     double2* s2, double2* s3, double* sq, cudaStream_t st);

}  // namespace pyro
