// Quadtree / octree variance stabilisation: device kernels.
#pragma once
#include "common.cuh"

namespace sred {

constexpr int kTreeThreads = 256;

// A node of the tree: origin and extent in voxels (d = 1 for the quadtree).
struct TreeBox {
  int x, y, z, w, h, d;
};

__global__ void k_tree_node_stats(const float* img, int W, int H, int D, const TreeBox* boxes, int three_d,
                                  float scale, double* out);
__global__ void k_tree_robust_mean(const float* img, int W, int H, const TreeBox* boxes, int max_iter, float* out);
__global__ void k_tree_lts(const float* img, int W, int H, const TreeBox* boxes, const float* means, float frac,
                           float* out);

}  // namespace sred
