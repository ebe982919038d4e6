// Launch interface of the compile-time-offset 16-colour pass kernel.
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace pyro {

constexpr int kFarThreads = kPassThreads;  // same segment lists as the generic kernel

// One pass of colour `site` (16-colour systems only) over the segments of p.
void launch_far_pass(const PassParams& p, int site, int n_blocks, bool metro, cudaStream_t st);

}  // namespace pyro
