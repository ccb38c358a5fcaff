// Generalised Anscombe transform (variance stabilisation of the input image)
// and the fit of its parameters.
//
// java/VarianceStabilisingTransform2D_.java:136-151 (getGAT) transforms the
// image; java/GATMinimizer2D.java (userFunction, applyGAT, getMeanAndVarBlock)
// defines the objective its Simplex option minimises: the transformed image
// cut into a 6 x 6 grid of blocks, sum over blocks of (variance - 1)^2 /
// blocks. Both are double-precision code in the reference; this file is
// compiled with -fmad=false so that no multiply-add is fused where Java
// rounds twice.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace sred {

// getGAT: v < 0 under the root -> 0, else (2 / gain) sqrt(gain v + c), in
// double, stored as float; c = (3/8) gain^2 + sigma^2 - gain offset.
__global__ void k_gat(float* __restrict__ img, size_t n, double gain, double c) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    double v = (double)img[i];
    if ((gain * v + c) < 0.0) {
      v = 0.0;
    } else {
      v = (2.0 / gain) * sqrt(gain * v + c);
    }
    img[i] = (float)v;
  }
}

// One block of the objective (GATMinimizer2D.userFunction): the pixels
// transformed as applyGAT does (v <= -c / gain -> 0), stored as float, then
// sum v and sum v*v (the product in float, as Java multiplies two floats) in
// double. Block b's pixels are split into gridDim.y equal runs, one CTA per
// run (so a grid of few blocks still fills the GPU), for each of gridDim.z
// parameter points; out[2 ((p B + b) S + s)] = the run's sum, + 1 its sum of
// squares (B = gridDim.x blocks, S = gridDim.y runs).
__global__ void __launch_bounds__(256)
    k_gat_block_moments(const float* __restrict__ img, int W, int bw, int bh, int nbx, GatPoints pts,
                        double* __restrict__ out) {
  __shared__ double s1[256], s2[256];
  const double gain = pts.gain[blockIdx.z], c = pts.c[blockIdx.z];
  const int b = blockIdx.x, bx = b % nbx, by = b / nbx;
  const int x0 = bx * bw, y0 = by * bh;
  const double lim = -c / gain, scale = 2.0 / gain;
  const int n = bw * bh, run = (n + gridDim.y - 1) / gridDim.y;
  const int t0 = blockIdx.y * run, t1 = min(n, t0 + run);
  double a1 = 0.0, a2 = 0.0;
  for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    const int x = x0 + t % bw, y = y0 + t / bw;
    double v = (double)img[(size_t)y * W + x];
    v = (v <= lim) ? 0.0 : scale * sqrt(gain * v + c);
    const float f = (float)v;
    a1 += (double)f;
    a2 += (double)(f * f);
  }
  s1[threadIdx.x] = a1;
  s2[threadIdx.x] = a2;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s1[threadIdx.x] += s1[threadIdx.x + s];
      s2[threadIdx.x] += s2[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const size_t o = 2 * (((size_t)blockIdx.z * gridDim.x + b) * gridDim.y + blockIdx.y);
    out[o] = s1[0];
    out[o + 1] = s2[0];
  }
}

// One block of GATMinimizer3D.userFunction's grid: the voxels transformed as
// applyGAT does (stored as float), then sum v and sum v*v in double (the
// product of the widened value, as java/Utils.java getMeanAndVarBlock3D
// computes it). Runs of a block per CTA and the output layout as in
// k_gat_block_moments.
__global__ void __launch_bounds__(256)
    k_gat_block_moments3d(const float* __restrict__ vol, int W, int H, int bw, int bh, int bd, int nbx, int nby,
                          GatPoints pts, double* __restrict__ out) {
  __shared__ double s1[256], s2[256];
  const double gain = pts.gain[blockIdx.z], c = pts.c[blockIdx.z];
  const int b = blockIdx.x, bx = b % nbx, by = (b / nbx) % nby, bz = b / (nbx * nby);
  const size_t x0 = (size_t)bx * bw, y0 = (size_t)by * bh, z0 = (size_t)bz * bd;
  const double lim = -c / gain, scale = 2.0 / gain;
  const size_t n = (size_t)bw * bh * bd, run = (n + gridDim.y - 1) / gridDim.y;
  const size_t t0 = blockIdx.y * run, t1 = n < t0 + run ? n : t0 + run;
  double a1 = 0.0, a2 = 0.0;
  for (size_t t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
    const size_t x = x0 + t % bw, y = y0 + (t / bw) % bh, z = z0 + t / ((size_t)bw * bh);
    double v = (double)vol[(z * H + y) * W + x];
    v = (v <= lim) ? 0.0 : scale * sqrt(gain * v + c);
    const double f = (double)(float)v;
    a1 += f;
    a2 += f * f;
  }
  s1[threadIdx.x] = a1;
  s2[threadIdx.x] = a2;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      s1[threadIdx.x] += s1[threadIdx.x + s];
      s2[threadIdx.x] += s2[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const size_t o = 2 * (((size_t)blockIdx.z * gridDim.x + b) * gridDim.y + blockIdx.y);
    out[o] = s1[0];
    out[o + 1] = s2[0];
  }
}

// GATMinimizer3D's grid: width/6, height/6, depth/6 (at least 1), halved
// along the axes with fewer than 2 blocks until all have 2 or the block is a
// single voxel (or, for an axis of length 1, until nothing changes).
void gat3d_grid(int w, int h, int d, int* bw, int* bh, int* bd, int* nbx, int* nby, int* nbz) {
  int a = std::max(w / 6, 1), b = std::max(h / 6, 1), c = std::max(d / 6, 1);
  int nx = w / a, ny = h / b, nz = d / c;
  while (nx < 2 || ny < 2 || nz < 2) {
    const int a0 = a, b0 = b, c0 = c;
    if (nx < 2 && a > 1) a = std::max(a / 2, 1);
    if (ny < 2 && b > 1) b = std::max(b / 2, 1);
    if (nz < 2 && c > 1) c = std::max(c / 2, 1);
    nx = w / a;
    ny = h / b;
    nz = d / c;
    if (a == 1 && b == 1 && c == 1) break;
    // An axis of 1 voxel can never have 2 blocks: the reference's loop then
    // runs forever; stop once nothing changes.
    if (a == a0 && b == b0 && c == c0) break;
  }
  *bw = a;
  *bh = b;
  *bd = c;
  *nbx = nx;
  *nby = ny;
  *nbz = nz;
}

// Block grid of the objective: width / 6 by height / 6 pixels
// (java/GATMinimizer2D.java userFunction). Returns false when the grid has
// fewer than 2 blocks a side (the reference then loops forever).
bool gat_grid(int w, int h, int* bw, int* bh, int* nbx, int* nby) {
  *bw = w / 6;
  *bh = h / 6;
  if (*bw < 1 || *bh < 1) return false;
  *nbx = w / *bw;
  *nby = h / *bh;
  return *nbx >= 2 && *nby >= 2;
}

// The objective from the per-block sums, in the reference's order.
double gat_error(const double* sums, int nblocks, int bw, int bh) {
  double error = 0.0;
  const int bwh = bw * bh;
  for (int b = 0; b < nblocks; b++) {
    double mean = sums[2 * b] / bwh;
    const double var = sums[2 * b + 1] / bwh - mean * mean;
    const double delta = var - 1;
    error += (delta * delta) / (double)nblocks;
  }
  return error;
}

}  // namespace sred
