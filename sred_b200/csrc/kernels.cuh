// Kernel declarations shared between the device translation units and the
// host orchestration (sred_api.cu).
#pragma once
#include "common.cuh"

namespace sred {

constexpr int kCompactSeg = 2048;

struct RefBlock {
  int k;
  float mean, std;
  float px[kMaxK];
};

// moments.cu
__global__ void k_local_stats(const float* img, int W, int H, Ellipse e, float* means, float* stds);
__global__ void k_noise_tiles(const float* img, int W, int t, int nbx, int nb, float* vars, int* bad);
__global__ void k_flags(const float* stds, const float* mask_in, int W, int H, int rw, int rh, float thr,
                        float* mask, uint8_t* flags, unsigned long long* n_mask);
__global__ void k_count(const uint8_t* flags, size_t n, int2* counts);
__global__ void k_scan(int2* counts, int nseg);
__global__ void k_scatter(const uint8_t* flags, size_t n, const int2* offs, int* gram_pix, int* flat_pix,
                          int* slot);
__global__ void k_pack(const float* img, int W, Ellipse e, const int* gram_pix, int n, float wscale, int mode,
                       float* U, int kp, __nv_bfloat16* A, __nv_bfloat16* B, int kq, BlockParams* params,
                       float* tile_rmax, double* sums);
__global__ void k_finalize(const int* slot, int W, int H, int rw, int rh, const double* num, const double* den,
                           const BlockParams* params, const double* sums, int n_flat, int metric, double sk,
                           double n_pixels, const float* mask, int apply_mask, float* out);
__global__ void k_pack_vectors(const float* u, int n, int K, int mode, float* U, int kp, __nv_bfloat16* A,
                               __nv_bfloat16* B, int kq);
__global__ void k_minmax(const float* a, const float* mask, int W, int H, int bw_, int bh_, size_t plane,
                         unsigned* mm);
__global__ void k_remap(float* a, const float* mask, int W, int H, int bw_, int bh_, size_t plane,
                        const unsigned* mm);
// Per-plane min/max words before k_minmax: {ordered +inf, ordered -inf} per plane
// (a kernel rather than a copy from pageable host memory, which would wait
// for the stream to drain).
__global__ void k_init_minmax(unsigned* mm, int planes);

// block_map.cu
__global__ void k_block_map(const float* img, int W, int H, int frames, Ellipse e, RefBlock rb, int metric,
                            float* out, float* stds_out);
// Dynamic shared memory and launch shape of k_block_map.
size_t block_map_smem(const Ellipse& e);
void block_map_launch_shape(int w, int h, int frames, dim3* grid, dim3* block);
__global__ void k_block_absdiff_post(float* a, int W, int H, int rw, int rh, size_t plane, const unsigned* mm);
__global__ void k_interior_mask(float* mask, int W, int H, int rw, int rh, size_t plane);
__global__ void k_apply_mask(float* a, const float* mask, size_t n);
__global__ void k_invert_masked(float* a, const float* mask, int W, int H, int rw, int rh, size_t plane);

// gat.cu
__global__ void k_gat(float* img, size_t n, double gain, double c);
// Parameter points of one launch of the GAT objective's moments kernels
// (gain and c = 3/8 gain^2 + sigma^2 - gain offset per point).
constexpr int kGatMaxPoints = 4;
struct GatPoints {
  double gain[kGatMaxPoints], c[kGatMaxPoints];
};
__global__ void k_gat_block_moments(const float* img, int W, int bw, int bh, int nbx, GatPoints pts, double* out);
bool gat_grid(int w, int h, int* bw, int* bh, int* nbx, int* nby);
double gat_error(const double* sums, int nblocks, int bw, int bh);
__global__ void k_gat_block_moments3d(const float* vol, int W, int H, int bw, int bh, int bd, int nbx, int nby,
                                      GatPoints pts, double* out);
void gat3d_grid(int w, int h, int d, int* bw, int* bh, int* bd, int* nbx, int* nby, int* nbz);

// shape.cu (k_block_phase is declared in shape.cuh, next to PhaseRef)
__global__ void k_patch_hu(const float* img, int W, int H, Ellipse e, int patch_size, double ref_hu1, float* out,
                           float* stds_out);
__global__ void k_hu_features(const float* img, const float* means, const float* stds, int W, int bw, int bh,
                              int nx, int n, float* feat, float* sig);
__global__ void k_hu_pairs(const float* feat, const float* sig, int n, int W, int rw, int rh, int nx, float* out);
__global__ void k_phase_dft(const float* img, const float* means, const float* stds, int W, int bw, int bh, int nx,
                            int n, double* fr, double* fi);
__global__ void k_gather_interior(const float* a, int W, int rw, int rh, int nx, int n, float* out);
// The all-pairs phase map (shape.cu): one CTA per reference block, on stream st.
void launch_phase_pairs(const double* fr, const double* fi, const float* sig, int n, int bw, int bh, int W, int nx,
                        float* out, cudaStream_t st);

}  // namespace sred
