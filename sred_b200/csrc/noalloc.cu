// Allocation-free block repetition map.
//
// Some callers cannot call cudaMalloc at all: host runtimes that own the
// device allocator and forbid foreign allocations, and real-time loops that
// must not touch the allocator once started. For them this entry point
// computes the same block map as sred_block_map_2d_device without allocating
// anything: the little device scratch it needs (the per-frame min/max words
// of the normalisation and, for NRMSE, the interior mask) lives in one
// file-scope __device__ array of fixed size that every GPU loading this
// library holds until exit. The call synchronises its stream before it
// returns; the caller's buffers are complete then.
//
// Host code must not use the array's name as a device address (there it is
// a host-side stand-in); the device address is obtained once per device with
// cudaGetSymbolAddress, on the first call made while that device is current
// (make that first call before any stream capture). Limits: at most 4096
// frames, for NRMSE frames * w * h <= 1,048,576, and an image tile with halo
// of at most 48 KB of shared memory (blocks whose ellipse needs more, such as
// 3 x 401, are refused); SRED_ERR_ARG beyond any of them.
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"
#include "shape.cuh"

namespace {

constexpr size_t kNoAllocMaskFloats = 1u << 20;  // NRMSE interior mask: frames * w * h <= 1,048,576
constexpr int kNoAllocMaxFrames = 4096;          // normalisation min/max words: 2 per frame
constexpr size_t kNoAllocScratchBytes = kNoAllocMaskFloats * sizeof(float) + 2 * kNoAllocMaxFrames * sizeof(unsigned);
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once).
sred_status scratch_address(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return SRED_ERR_NODEV;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return SRED_ERR_LAUNCH;
    }
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_addr[dev];
  return SRED_OK;
}

int grid_of(size_t n, int threads, int cap) {
  size_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > (size_t)cap) g = cap;
  return (int)g;
}

int block_metric_id(const char* m) {
  if (!m) return -1;
  if (!std::strcmp(m, "Pearson's R")) return sred::kPearson;
  if (!std::strcmp(m, "SSIM")) return sred::kSsim;
  if (!std::strcmp(m, "NRMSE (inverted)")) return sred::kNrmse;
  if (!std::strcmp(m, "Abs. Diff. of StdDevs.")) return sred::kAbsDiff;
  if (!std::strcmp(m, "Cosine")) return sred::kCosine;
  if (!std::strcmp(m, "Hu moments")) return sred::kHu;
  if (!std::strcmp(m, "Phase correlation")) return sred::kPhase;
  if (!std::strcmp(m, "Hu distance")) return sred::kHu7;
  return -1;
}

}  // namespace

extern "C" sred_status sred_block_map_2d_device_noalloc(const char* metric, const float* d_img, int w, int h,
                                                        int frames, const float* ref_pixels, int block_size, int bw,
                                                        int bh, float ref_mean, float ref_std, int normalize_output,
                                                        float* d_out, void* stream) {
  using namespace sred;
  const int m = block_metric_id(metric);
  if (m < 0) return SRED_ERR_UNKNOWN_METRIC;
  if (!d_img || !ref_pixels || !d_out || w <= 0 || h <= 0 || frames < 1) return SRED_ERR_ARG;
  if (bw % 2 == 0 || bh % 2 == 0 || bw < 3 || bh < 3) return SRED_ERR_ARG;
  Ellipse e;
  if (build_ellipse(bw, bh, &e) != block_size || block_size < 2 || block_size > kMaxK) return SRED_ERR_ARG;
  const size_t plane = (size_t)w * h, n = plane * frames;
  // Sizes beyond the fixed scratch are refused, not truncated.
  if (frames > kNoAllocMaxFrames) return SRED_ERR_ARG;
  if (m == kNrmse && n > kNoAllocMaskFloats) return SRED_ERR_ARG;
  const size_t tile_smem = block_map_smem(e);
  if (tile_smem > 48 * 1024) return SRED_ERR_ARG;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SRED_ERR_NODEV;
  unsigned char* scratch = nullptr;
  sred_status st = scratch_address(dev, &scratch);
  if (st != SRED_OK) return st;
  float* d_mask = reinterpret_cast<float*>(scratch);
  unsigned* d_mm = reinterpret_cast<unsigned*>(scratch + kNoAllocMaskFloats * sizeof(float));
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  RefBlock rb;
  rb.k = block_size;
  rb.mean = ref_mean;
  rb.std = ref_std;
  std::memcpy(rb.px, ref_pixels, sizeof(float) * block_size);
  const int rw = e.rw, rh = e.rh;
  if (m == kHu) {
    float patch[kMaxK * 4];  // bw * bh < 4 K for every ellipse of K <= kMaxK
    if (bw * bh > kMaxK * 4) return SRED_ERR_ARG;
    hu_prepare_patch(ref_pixels, bw, bh, patch);
    k_patch_hu<<<dim3((unsigned)((plane + 127) / 128), frames), 128, 0, s>>>(
        d_img, w, h, e, block_size, patch_hu1(patch, bw, bh), d_out, nullptr);
  } else if (m == kHu7) {
    Hu7Ref hr;
    hu7_reference(ref_pixels, e, &hr);
    launch_block_hu7(d_img, w, h, frames, e, hr, d_out, nullptr, s);
  } else if (m == kPhase) {
    if (bw > kPhaseMaxDim || bh > kPhaseMaxDim) return SRED_ERR_ARG;
    PhaseRef pr;
    phase_reference_dft(ref_pixels, ref_std, bw, bh, &pr);
    launch_block_phase(d_img, w, h, frames, e, bw, bh, pr, d_out, nullptr, s);
  } else {
    dim3 grid, blk;
    block_map_launch_shape(w, h, frames, &grid, &blk);
    k_block_map<<<grid, blk, tile_smem, s>>>(d_img, w, h, frames, e, rb, m, d_out, nullptr);
  }
  const dim3 pg(grid_of(plane, 256, 4 * sms), frames);
  const int ig = grid_of((size_t)frames, 256, 64);
  // The relevance constant is 0 here: the mask is the interior for NRMSE
  // (java/CLUtils.java:788-797) and absent otherwise.
  if (m == kNrmse) {
    k_interior_mask<<<pg, 256, 0, s>>>(d_mask, w, h, rw, rh, plane);
    k_apply_mask<<<grid_of(n, 256, 8 * sms), 256, 0, s>>>(d_out, d_mask, n);
    k_init_minmax<<<ig, 256, 0, s>>>(d_mm, frames);
    k_minmax<<<pg, 256, 0, s>>>(d_out, d_mask, w, h, rw, rh, plane, d_mm);
    k_remap<<<pg, 256, 0, s>>>(d_out, d_mask, w, h, rw, rh, plane, d_mm);
    k_invert_masked<<<pg, 256, 0, s>>>(d_out, d_mask, w, h, rw, rh, plane);
    if (normalize_output) {
      k_init_minmax<<<ig, 256, 0, s>>>(d_mm, frames);
      k_minmax<<<pg, 256, 0, s>>>(d_out, d_mask, w, h, rw, rh, plane, d_mm);
      k_remap<<<pg, 256, 0, s>>>(d_out, d_mask, w, h, rw, rh, plane, d_mm);
    }
  } else {
    if (m == kAbsDiff) {
      k_init_minmax<<<ig, 256, 0, s>>>(d_mm, frames);
      k_minmax<<<pg, 256, 0, s>>>(d_out, nullptr, w, h, rw, rh, plane, d_mm);
      k_block_absdiff_post<<<pg, 256, 0, s>>>(d_out, w, h, rw, rh, plane, d_mm);
    }
    if (normalize_output) {
      k_init_minmax<<<ig, 256, 0, s>>>(d_mm, frames);
      k_minmax<<<pg, 256, 0, s>>>(d_out, nullptr, w, h, rw, rh, plane, d_mm);
      k_remap<<<pg, 256, 0, s>>>(d_out, nullptr, w, h, rw, rh, plane, d_mm);
    }
  }
  if (cudaGetLastError() != cudaSuccess) return SRED_ERR_LAUNCH;
  if (cudaStreamSynchronize(s) != cudaSuccess) return SRED_ERR_LAUNCH;
  return SRED_OK;
}
