// 3D (volume) block repetition maps: device kernels and host helpers.
#pragma once
#include "common.cuh"

namespace sred {

constexpr int kMaxK3 = 4096;  // largest ellipsoid block size accepted

// A W x H x D volume ([D][H][W] floats) and the ellipsoid block radii; k is
// the number of voxels of the ellipsoid.
struct Vol3 {
  int W, H, D;
  int rw, rh, rd;
  int k;
  int z0 = 0;  // first slice of a launch over slices [z0, z0 + gridDim.z) of the per-voxel kernels
};

// Host: linear offsets (z W H + y W + x) of the voxels of the ellipsoid
// inscribed in a bw x bh x bd block, z-y-x order (java/Utils.java:1075-1085,
// float arithmetic). Writes at most kMaxK3 offsets; returns the voxel count.
int build_ellipsoid(int bw, int bh, int bd, int W, int H, int* off);

// One thread per voxel; dynamic shared memory: k ints (stats), k ints + k
// floats (block map).
__global__ void k_local_stats3d(const float* img, Vol3 v, const int* off, float* means, float* stds);
// The raw 3D block map (one thread per voxel; the dynamic shared memory it
// needs is chosen here) over slices [v.z0, z1) (z1 < 0: to the last slice).
cudaError_t launch_block_map3d(const float* img, Vol3 v, const int* off, const float* ref, float ref_mean,
                               float ref_std, int metric, const float* means, const float* stds, float* out,
                               cudaStream_t st, int z1 = -1);
__global__ void k_divide_fixed(const float* a, size_t n, float b, float* out);
__global__ void k_divide_fixed64(const double* a, size_t n, double b, double* out);
__global__ void k_block3d_post(float* a, Vol3 v, int metric);
__global__ void k_mask3d(const float* stds, Vol3 v, float thr, float* mask, float* map);
__global__ void k_minmax3d(const float* a, const float* mask, Vol3 v, unsigned* mm);
__global__ void k_remap3d(float* a, const float* mask, Vol3 v, const unsigned* mm);

// 3D global map (the 2D pair engines run on the compacted block lists).
__global__ void k_flags3d(const float* stds, Vol3 v, float thr, int flat_columns, float* mask, uint8_t* flags,
                          unsigned long long* n_mask);
__global__ void k_pack3d(const float* img, Vol3 v, const int* off, const int* gram_pix, int n, float wscale,
                         int mode, float* U, int kp, __nv_bfloat16* A, __nv_bfloat16* B, int kq,
                         BlockParams* params, float* tile_rmax);
__global__ void k_finalize3d(const int* slot, Vol3 v, const double* num, const double* den,
                             const BlockParams* params, int n_flat, int metric, double sk, double n_pixels,
                             const float* mask, int apply_mask, float* out);

}  // namespace sred
