// Redundancy classification (k-means): device kernels and block layout.
#pragma once
#include "common.cuh"

namespace sred {

constexpr int kKmThreads = 256;                 // threads per block
constexpr int kKmPer = 4;                       // points per thread
constexpr int kKmSpan = kKmThreads * kKmPer;    // points per block
constexpr int kKmMaxK = 64;                     // largest number of classes

__global__ void k_km_gather(const float* map, int W, int H, int border, double* x);
__global__ void k_km_d2(const double* x, size_t n, double c, int first, double* d2, double* partial);
__global__ void k_km_assign(const double* x, size_t n, const double* centers, int k, int* labels,
                            unsigned long long* changed, double* bsum, double* bcnt, double* bwcss);
__global__ void k_km_distvar(const double* x, size_t n, const double* centers, int k, const int* labels,
                             double* bd1, double* bd2);
__global__ void k_km_scatter(const int* labels, const int* rank, int W, int H, int border, float* out);

}  // namespace sred
