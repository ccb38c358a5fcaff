// Relevance-mask tools: device kernels.
#pragma once
#include "common.cuh"

namespace sred {

__global__ void k_local_var2d(const float* img, int W, int H, Ellipse e, int take_sqrt, float* out);
__global__ void k_noise_tiles64(const float* img, int W, int t, int nbx, int nb, float* vars);
__global__ void k_sweep_masks(const float* stat, int W, int H, int rw, int rh, const float* thr, float* masks);
__global__ void k_stat_sq_minmax(const float* stat, int W, int H, int rw, int rh, unsigned* mm);

}  // namespace sred
