// Split-BF16 tcgen05 engine of the global repetition map (sm_100a).
//
// G = A' B'^T on the 5th-generation tensor cores, where each block's FP64 unit
// vector u is split into bf16 hi = bf16(u), lo = bf16(u - hi), and
//   A' = [hi | lo | hi],  B' = [hi | hi | lo]   (K' = round_up(3K, 16))
// so one BF16 MMA chain with FP32 accumulation yields hi.hi + lo.hi + hi.lo,
// an FP32-accurate <u_p, u_q> (the dropped lo.lo term is below 2^-16).
//
// CTA = 1 per SM, persistent over work items (128-row block, range of
// 256-column tiles). Warp roles:
//   warp 16     TMA producer: the item's A tile (resident, all K' chunks), a
//               ring of B stages (one 256 x 64 bf16 chunk each, SWIZZLE_128B)
//               and a ring of four column-parameter slots (4 KB per tile)
//   warp 17     MMA issuer (one thread): on claiming one of two TMEM
//               accumulators (2 x 256 columns) it issues tcgen05.mma
//               M=128 N=256 K=16 and tcgen05.commit to release B stages and
//               to publish the finished accumulator. It shares an SM
//               sub-partition with four busy epilogue warps, so its loop is
//               kept to a few instructions per MMA: no divisions, operand
//               descriptors advanced by adds, K steps unrolled.
//   warps 0-15  epilogue: tcgen05.ld of the accumulator (warp w reads TMEM
//               lanes 32(w%4).. and columns 64(w/4)..), the fused per-pair
//               metric (epilogue.cuh), row sums in registers; FP64 atomics
//               per row per item. The N x N matrix is never stored. Epilogue
//               warps synchronise only through mbarriers, so they drift and
//               overlap each other's TMEM-load latency.
// Every mbarrier wait is bounded by wall time; on expiry the kernel records a
// status code, stops issuing work, waits (bounded) for its own copies in
// flight, frees TMEM and returns. No TMA multicast is used.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "epilogue.cuh"

namespace sred {

namespace {

constexpr int kBM = 128;          // rows per tile (TMEM lanes)
constexpr int kBN = 256;          // columns per tile
constexpr int kChunk = 64;        // bf16 elements per K chunk (128 B, one SWIZZLE_128B atom row)
constexpr int kAChunkBytes = kBM * kChunk * 2;   // 16 KB
constexpr int kBStageBytes = kBN * kChunk * 2;   // 32 KB
constexpr int kMaxStages = 16;
constexpr int kEpiWarps = 16;                       // 4 per SM sub-partition
constexpr int kColsPerWarp = kBN / (kEpiWarps / 4);  // 64: each warp reads 32 lanes x 64 columns
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr int kSoaBytes = kColSoaFloats * 4;         // one tile's column parameters
constexpr int kParSlots = 4;                         // column-parameter ring depth
constexpr unsigned long long kTimeoutNs = 4000000000ull;  // 4 s per wait

enum { ST_OK = 0, ST_TIMEOUT_PRODUCER = 1, ST_TIMEOUT_MMA = 2, ST_TIMEOUT_EPI = 3, ST_TIMEOUT_DRAIN = 4 };

struct TcArgs {
  int kq, nkc, stages;
  int nfull, tail;              // tile-ring mode: 64-column chunks and a 32-column tail (0 or 1)
  uint32_t a_bytes, b_bytes;    // tile-ring mode: A tile and one B tile in shared memory
  int rb0;                      // first 128-row block of this launch
  int n_rb, n_ct, ct_per_item, n_items;
  const BlockParams* params;
  const float* colsoa;
  const float* tile_rmax;
  EpiConsts ec;
  double* num;
  double* den;
  int* status;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with the given parity. Returns false (and
// records `code`) if the wait exceeded kTimeoutNs or another role of any CTA
// already gave up. Drain waits (for copies or MMAs this CTA issued) pass
// abort = false: they keep waiting, within the same bound, after another
// role has given up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* status, int code,
                                          bool abort = true) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  for (uint32_t i = 1;; i++) {
    if (mbar_test(bar, parity)) return true;
    if ((i & 255u) == 0) {
      if (abort && *reinterpret_cast<volatile int*>(status) != ST_OK) return false;
      if (globaltimer() - t0 > kTimeoutNs) {
        atomicCAS(status, ST_OK, code);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
          "r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(bar), "r"(x), "r"(y)
      : "memory");
}

// Plain bulk copy (no tensor map): 16-byte aligned addresses, size a multiple of 16.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
               : "memory");
}

// Shared-memory matrix descriptor: K-major, SWIZZLE_128B (128-byte rows),
// 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>(1) << 16;           // leading byte offset (unused for swizzled K-major)
  d |= static_cast<uint64_t>(1024 >> 4) << 32;   // stride byte offset
  d |= static_cast<uint64_t>(1) << 46;           // descriptor version (sm_100)
  d |= static_cast<uint64_t>(2) << 61;           // SWIZZLE_128B
  return d;
}

// Same for SWIZZLE_64B (64-byte rows, 8-row groups 512 B apart): the 32-column
// tail of K' in the tile-ring mode.
__device__ __forceinline__ uint64_t desc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>(1) << 16;
  d |= static_cast<uint64_t>(512 >> 4) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(4) << 61;  // SWIZZLE_64B
  return d;
}

// Instruction descriptor, kind::f16: D = F32, A = B = BF16, both K-major, M = 128, N = 256.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(kBN >> 3) << 17) |
                            (static_cast<uint32_t>(kBM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Issue a load of 32 lanes x 16 columns of 32-bit accumulator (no wait).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}

// Wait for every TMEM load this thread issued; the register operands tie
// later uses of v to the wait, so none is scheduled before it.
__device__ __forceinline__ void tmem_wait(uint32_t (&v)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7]),
                 "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]), "+r"(v[13]), "+r"(v[14]),
                 "+r"(v[15])
               :
               : "memory");
}

// 16 pairs: accumulator columns c0..c0+15 of this thread's row against the
// columns' parameters in the shared-memory slot (structure of arrays).
template <int METRIC, int CMODE, bool FULL, bool DIAG>
__device__ __forceinline__ void epi_chunk(const uint32_t (&v)[16], const float* __restrict__ soa, int c0, int col0,
                                          int row, const RowState& rs, const EpiConsts& ec, float& sn, float& sd) {
#pragma unroll
  for (int j = 0; j < 16; j += 4) {
    const int q = c0 + j;
    const float4 a4 = *reinterpret_cast<const float4*>(soa + q);
    const float4 r4 = *reinterpret_cast<const float4*>(soa + kBN + q);
    float4 s4 = make_float4(0.f, 0.f, 0.f, 0.f), m4 = s4;
    if (METRIC != kPearson && METRIC != kDebugDot) s4 = *reinterpret_cast<const float4*>(soa + 2 * kBN + q);
    if (METRIC == kSsim) m4 = *reinterpret_cast<const float4*>(soa + 3 * kBN + q);
    const float av[4] = {a4.x, a4.y, a4.z, a4.w};
    const float rv[4] = {r4.x, r4.y, r4.z, r4.w};
    const float sv[4] = {s4.x, s4.y, s4.z, s4.w};
    const float mv[4] = {m4.x, m4.y, m4.z, m4.w};
#pragma unroll
    for (int u = 0; u < 4; u++) {
      BlockParams cq;
      cq.a = av[u];
      cq.r = rv[u];
      cq.sigma = sv[u];
      cq.mu = mv[u];
      float G = __uint_as_float(v[j + u]);
      if (DIAG && col0 + q + u == row && rs.r > 0.0f) G = 1.0f;
      if (FULL || col0 + q + u < ec.n) epi_pair<METRIC, CMODE>(G, rs, cq, ec, sn, sd);
    }
  }
}

// Packed Pearson fast path (full, off-diagonal tiles, CMODE kCFirst or
// kCSecond): 16 pairs as eight f32x2 pairs.
template <int CMODE>
__device__ __forceinline__ void epi_chunk_pearson2(const uint32_t (&v)[16], const float* __restrict__ soa, int c0,
                                                   const PearsonRow2& r2, F2& sn, F2& sd) {
#pragma unroll
  for (int j = 0; j < 16; j += 4) {
    const float4 a4 = *reinterpret_cast<const float4*>(soa + c0 + j);
    const float4 r4 = *reinterpret_cast<const float4*>(soa + kBN + c0 + j);
    pearson_pair2<CMODE>(f2(__uint_as_float(v[j]), __uint_as_float(v[j + 1])), f2(a4.x, a4.y), f2(r4.x, r4.y), r2,
                         sn, sd);
    pearson_pair2<CMODE>(f2(__uint_as_float(v[j + 2]), __uint_as_float(v[j + 3])), f2(a4.z, a4.w),
                         f2(r4.z, r4.w), r2, sn, sd);
  }
}

// Packed SSIM path (full, off-diagonal tiles): 16 pairs as eight f32x2 pairs.
__device__ __forceinline__ void epi_chunk_ssim2(const uint32_t (&v)[16], const float* __restrict__ soa, int c0,
                                                const SsimRow2& r2, F2& sn, F2& sd) {
#pragma unroll
  for (int j = 0; j < 16; j += 4) {
    const float4 a4 = *reinterpret_cast<const float4*>(soa + c0 + j);
    const float4 s4 = *reinterpret_cast<const float4*>(soa + 2 * kBN + c0 + j);
    const float4 m4 = *reinterpret_cast<const float4*>(soa + 3 * kBN + c0 + j);
    ssim_pair2(f2(__uint_as_float(v[j]), __uint_as_float(v[j + 1])), f2(a4.x, a4.y), f2(s4.x, s4.y),
               f2(m4.x, m4.y), r2, sn, sd);
    ssim_pair2(f2(__uint_as_float(v[j + 2]), __uint_as_float(v[j + 3])), f2(a4.z, a4.w), f2(s4.z, s4.w),
               f2(m4.z, m4.w), r2, sn, sd);
  }
}

__device__ __forceinline__ void epi_tile_ssim2(uint32_t taddr, const float* __restrict__ soa, int cbase,
                                               const SsimRow2& r2, float& sn_out, float& sd_out) {
  uint32_t v0[16], v1[16];
  F2 sn = f2(0.0f, 0.0f), sd = sn;
  tmem_ld16(taddr, v0);
  tmem_wait(v0);
  tmem_ld16(taddr + 16, v1);
  epi_chunk_ssim2(v0, soa, cbase, r2, sn, sd);
  tmem_wait(v1);
  tmem_ld16(taddr + 32, v0);
  epi_chunk_ssim2(v1, soa, cbase + 16, r2, sn, sd);
  tmem_wait(v0);
  tmem_ld16(taddr + 48, v1);
  epi_chunk_ssim2(v0, soa, cbase + 32, r2, sn, sd);
  tmem_wait(v1);
  epi_chunk_ssim2(v1, soa, cbase + 48, r2, sn, sd);
  float a, b;
  f2_split(sn, a, b);
  sn_out += a + b;
  f2_split(sd, a, b);
  sd_out += a + b;
}

template <int CMODE>
__device__ __forceinline__ void epi_tile_pearson2(uint32_t taddr, const float* __restrict__ soa, int cbase,
                                                  const PearsonRow2& r2, float& sn_out, float& sd_out) {
  uint32_t v0[16], v1[16];
  F2 sn = f2(0.0f, 0.0f), sd = sn;
  tmem_ld16(taddr, v0);
  tmem_wait(v0);
  tmem_ld16(taddr + 16, v1);
  epi_chunk_pearson2<CMODE>(v0, soa, cbase, r2, sn, sd);
  tmem_wait(v1);
  tmem_ld16(taddr + 32, v0);
  epi_chunk_pearson2<CMODE>(v1, soa, cbase + 16, r2, sn, sd);
  tmem_wait(v0);
  tmem_ld16(taddr + 48, v1);
  epi_chunk_pearson2<CMODE>(v0, soa, cbase + 32, r2, sn, sd);
  tmem_wait(v1);
  epi_chunk_pearson2<CMODE>(v1, soa, cbase + 48, r2, sn, sd);
  float a, b;
  f2_split(sn, a, b);
  sn_out += a + b;
  f2_split(sd, a, b);
  sd_out += a + b;
}

// One warp's 64 columns of a tile in four 16-column chunks: each chunk's TMEM
// load is in flight while the previous chunk is evaluated.
template <int METRIC, int CMODE, bool FULL, bool DIAG>
__device__ __forceinline__ void epi_tile(uint32_t taddr, const float* __restrict__ soa, int cbase, int col0, int row,
                                         const RowState& rs, const EpiConsts& ec, float& sn, float& sd) {
  uint32_t v0[16], v1[16];
  tmem_ld16(taddr, v0);
  tmem_wait(v0);
  tmem_ld16(taddr + 16, v1);
  epi_chunk<METRIC, CMODE, FULL, DIAG>(v0, soa, cbase, col0, row, rs, ec, sn, sd);
  tmem_wait(v1);
  tmem_ld16(taddr + 32, v0);
  epi_chunk<METRIC, CMODE, FULL, DIAG>(v1, soa, cbase + 16, col0, row, rs, ec, sn, sd);
  tmem_wait(v0);
  tmem_ld16(taddr + 48, v1);
  epi_chunk<METRIC, CMODE, FULL, DIAG>(v0, soa, cbase + 32, col0, row, rs, ec, sn, sd);
  tmem_wait(v1);
  epi_chunk<METRIC, CMODE, FULL, DIAG>(v1, soa, cbase + 48, col0, row, rs, ec, sn, sd);
}

// TR (tile ring, K' <= 160): the B operand moves one whole 256-column tile at
// a time through two buffers, and the single tcgen05.commit per tile both
// publishes the accumulator and frees the tile's B buffer (the producer waits
// on the accumulator barrier). Each mbarrier operation that follows a commit
// stalls the MMA stream for ~100 cycles, so one commit-then-wait per tile
// instead of one per K chunk is worth ~30% of MMA throughput. K' = 64 c + 32 t:
// c SWIZZLE_128B chunks and an optional SWIZZLE_64B tail.
// !TR (chunk ring): B moves in 64-column chunks through S stages, one commit
// per chunk; used when two whole tiles do not fit in shared memory.
template <int METRIC, bool TR>
__global__ void __launch_bounds__(kThreads, 1)
    k_gram_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              const __grid_constant__ CUtensorMap tmA64, const __grid_constant__ CUtensorMap tmB64, TcArgs g) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* sbase = smem_raw + (base - raw);
  const int S = g.stages, nkc = g.nkc;
  const uint32_t sA = base;  // TR: a_bytes; else nkc x 16 KB
  const uint32_t sB = sA + (TR ? g.a_bytes : nkc * kAChunkBytes);   // TR: 2 x b_bytes; else S x 32 KB
  const uint32_t sP = sB + (TR ? 2 * g.b_bytes : S * kBStageBytes);  // kParSlots column-parameter slots
  const float* slots = reinterpret_cast<const float*>(sbase + (sP - base));
  uint64_t* bars = reinterpret_cast<uint64_t*>(sbase + (sP - base) + kParSlots * kSoaBytes);
  // barrier layout: full[S], empty[S], acc_full[2], acc_empty[2], par_full[4], par_empty[4],
  //                 a_full, a_empty, done
  const uint32_t b_full = smem_u32(bars), b_empty = b_full + 8 * S, b_accf = b_empty + 8 * S,
                 b_acce = b_accf + 16, b_parf = b_acce + 16, b_pare = b_parf + 8 * kParSlots,
                 b_afull = b_pare + 8 * kParSlots, b_aempty = b_afull + 8, b_done = b_aempty + 8;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2 * S + 4 + 2 * kParSlots + 3);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(b_full + 8 * s, 1);
      mbar_init(b_empty + 8 * s, 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(b_accf + 8 * b, 1);
      mbar_init(b_acce + 8 * b, kEpiWarps);
    }
    for (int p = 0; p < kParSlots; p++) {
      mbar_init(b_parf + 8 * p, 1);
      mbar_init(b_pare + 8 * p, kEpiWarps);
    }
    mbar_init(b_afull, 1);
    mbar_init(b_aempty, 1);
    mbar_init(b_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kEpiWarps + 1) {  // MMA warp owns the TMEM allocation
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * kBN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == kEpiWarps) {
    // ---------------------------------------------------------------- TMA
    if (lane == 0) {
      uint32_t it = 0, item_i = 0, ptile = 0;
      uint32_t s = 0, eph = 0;  // B ring: stage, parity of the round being refilled
      bool ok = true, a_issued = false;
      for (int item = blockIdx.x; ok && item < g.n_items; item += gridDim.x, item_i++) {
        const int rb = g.rb0 + item % g.n_rb, seg = item / g.n_rb;
        const int ct0 = seg * g.ct_per_item, ct1 = min(ct0 + g.ct_per_item, g.n_ct);
        if (!mbar_wait(b_aempty, (item_i & 1) ^ 1, g.status, ST_TIMEOUT_PRODUCER)) { ok = false; break; }
        if (TR) {
          mbar_expect_tx(b_afull, g.a_bytes);
          for (int c = 0; c < g.nfull; c++) tma_load_2d(sA + c * kAChunkBytes, &tmA, b_afull, c * kChunk, rb * kBM);
          if (g.tail) tma_load_2d(sA + g.nfull * kAChunkBytes, &tmA64, b_afull, g.nfull * kChunk, rb * kBM);
        } else {
          mbar_expect_tx(b_afull, nkc * kAChunkBytes);
          for (int kc = 0; kc < nkc; kc++) tma_load_2d(sA + kc * kAChunkBytes, &tmA, b_afull, kc * kChunk, rb * kBM);
        }
        a_issued = true;
        for (int ct = ct0; ok && ct < ct1; ct++, ptile++) {
          // the tile's column parameters, into the slot the epilogue released four tiles ago
          const uint32_t ps = ptile & (kParSlots - 1);
          if (!mbar_wait(b_pare + 8 * ps, ((ptile / kParSlots) & 1) ^ 1, g.status, ST_TIMEOUT_PRODUCER)) {
            ok = false;
            break;
          }
          // TR: B buffer ptile & 1 is free once the accumulator of tile ptile - 2
          // is published. Both waits come before any copy of this tile is issued.
          if (TR && !mbar_wait(b_accf + 8 * (ptile & 1), ((ptile >> 1) & 1) ^ 1, g.status, ST_TIMEOUT_PRODUCER)) {
            ok = false;
            break;
          }
          mbar_expect_tx(b_parf + 8 * ps, kSoaBytes);
          bulk_load(sP + ps * kSoaBytes, g.colsoa + (size_t)ct * kColSoaFloats, kSoaBytes, b_parf + 8 * ps);
          if (TR) {
            const uint32_t b = ptile & 1;
            const uint32_t dst = sB + b * g.b_bytes;
            mbar_expect_tx(b_full + 8 * b, g.b_bytes);
            for (int c = 0; c < g.nfull; c++)
              tma_load_2d(dst + c * kBStageBytes, &tmB, b_full + 8 * b, c * kChunk, ct * kBN);
            if (g.tail) tma_load_2d(dst + g.nfull * kBStageBytes, &tmB64, b_full + 8 * b, g.nfull * kChunk, ct * kBN);
            it++;
            continue;
          }
          for (int kc = 0; kc < nkc; kc++, it++) {
            if (!mbar_wait(b_empty + 8 * s, eph ^ 1, g.status, ST_TIMEOUT_PRODUCER)) { ok = false; break; }
            mbar_expect_tx(b_full + 8 * s, kBStageBytes);
            tma_load_2d(sB + s * kBStageBytes, &tmB, b_full + 8 * s, kc * kChunk, ct * kBN);
            if (++s == (uint32_t)S) {
              s = 0;
              eph ^= 1;
            }
          }
        }
      }
      // Drain: every issued copy has landed before the CTA may exit (TR: `it`
      // counts whole-tile loads through S = 2 buffers).
      for (uint32_t k = (it > (uint32_t)S ? it - S : 0); k < it; k++)
        mbar_wait(b_full + 8 * (k % S), (k / S) & 1, g.status, ST_TIMEOUT_DRAIN, false);
      for (uint32_t k = (ptile > (uint32_t)kParSlots ? ptile - kParSlots : 0); k < ptile; k++)
        mbar_wait(b_parf + 8 * (k % kParSlots), (k / kParSlots) & 1, g.status, ST_TIMEOUT_DRAIN, false);
      // item_i - 1 is the last item whose A tile was issued (a failed wait
      // leaves item_i at the item it was waiting for)
      if (a_issued) mbar_wait(b_afull, (item_i - 1) & 1, g.status, ST_TIMEOUT_DRAIN, false);
    }
    __syncwarp();
  } else if (warp == kEpiWarps + 1) {
    // ---------------------------------------------------------------- MMA
    if (lane == 0) {
      uint32_t tile = 0, item_i = 0;
      uint32_t s = 0, fph = 0;  // B ring: stage, parity of the round being consumed
      // Operand descriptors: the start-address field counts 16-byte units, so
      // a K step of 16 bf16 (32 B) adds 2 and a chunk or stage adds its size / 16.
      const uint64_t a_desc0 = desc_sw128(sA), b_desc0 = desc_sw128(sB);
      const int last_nks = (g.kq - (nkc - 1) * kChunk) / 16;
      bool ok = true;
      for (int item = blockIdx.x; ok && item < g.n_items; item += gridDim.x, item_i++) {
        const int seg = item / g.n_rb;
        const int ct0 = seg * g.ct_per_item, ct1 = min(ct0 + g.ct_per_item, g.n_ct);
        if (!mbar_wait(b_afull, item_i & 1, g.status, ST_TIMEOUT_MMA)) { ok = false; break; }
        tc_fence_after();
        for (int ct = ct0; ok && ct < ct1; ct++, tile++) {
          const uint32_t b = tile & 1;
          if (!mbar_wait(b_acce + 8 * b, ((tile >> 1) & 1) ^ 1, g.status, ST_TIMEOUT_MMA)) { ok = false; break; }
          tc_fence_after();
          const uint32_t d = tmem + b * kBN;
          if (TR) {
            if (!mbar_wait(b_full + 8 * b, (tile >> 1) & 1, g.status, ST_TIMEOUT_MMA)) { ok = false; break; }
            tc_fence_after();
            const uint64_t db0 = b_desc0 + (uint64_t)((b * g.b_bytes) >> 4);
            for (int c = 0; c < g.nfull; c++) {
#pragma unroll
              for (int ks = 0; ks < kChunk / 16; ks++)
                mma_bf16(d, a_desc0 + (uint64_t)(c * (kAChunkBytes >> 4) + 2 * ks),
                         db0 + (uint64_t)(c * (kBStageBytes >> 4) + 2 * ks), (c | ks) != 0);
            }
            if (g.tail) {
              const uint64_t da = desc_sw64(sA + g.nfull * kAChunkBytes);
              const uint64_t db = desc_sw64(sB + b * g.b_bytes + g.nfull * kBStageBytes);
              mma_bf16(d, da, db, g.nfull != 0);
              mma_bf16(d, da + 2, db + 2, 1);
            }
            mma_commit(b_accf + 8 * b);
            continue;
          }
          uint64_t da = a_desc0;
          for (int kc = 0; kc < nkc; kc++) {
            if (!mbar_wait(b_full + 8 * s, fph, g.status, ST_TIMEOUT_MMA)) { ok = false; break; }
            tc_fence_after();
            const uint64_t db = b_desc0 + (uint64_t)(s * (kBStageBytes >> 4));
            if (kc + 1 < nkc) {
#pragma unroll
              for (int ks = 0; ks < kChunk / 16; ks++) mma_bf16(d, da + 2 * ks, db + 2 * ks, (kc | ks) != 0);
            } else {
#pragma unroll
              for (int ks = 0; ks < kChunk / 16; ks++)
                if (ks < last_nks) mma_bf16(d, da + 2 * ks, db + 2 * ks, (kc | ks) != 0);
            }
            mma_commit(b_empty + 8 * s);
            da += kAChunkBytes >> 4;
            if (++s == (uint32_t)S) {
              s = 0;
              fph ^= 1;
            }
          }
          if (ok) mma_commit(b_accf + 8 * b);
        }
        if (ok) mma_commit(b_aempty);
      }
      // All MMAs this thread issued are complete before TMEM is released and
      // the CTA exits.
      mma_commit(b_done);
      mbar_wait(b_done, 0, g.status, ST_TIMEOUT_DRAIN, false);
    }
    __syncwarp();
  } else {
    // ---------------------------------------------------------------- epilogue
    const int quarter = warp & 3, group = warp >> 2;
    const int cbase = group * kColsPerWarp;
    uint32_t tile = 0;
    bool ok = true;
    for (int item = blockIdx.x; ok && item < g.n_items; item += gridDim.x) {
      const int rb = g.rb0 + item % g.n_rb, seg = item / g.n_rb;
      const int ct0 = seg * g.ct_per_item, ct1 = min(ct0 + g.ct_per_item, g.n_ct);
      const int row = rb * kBM + quarter * 32 + lane;
      const RowState rs = make_row(g.params[row], g.ec);
      const PearsonRow2 r2 = make_pearson_row2(rs);
      const SsimRow2 s2 = make_ssim_row2(rs, g.ec);
      const float rmax_r = g.tile_rmax[rb];
      double acc_n = 0.0, acc_d = 0.0;
      for (int ct = ct0; ok && ct < ct1; ct++, tile++) {
        const uint32_t b = tile & 1, par = (tile >> 1) & 1;
        const uint32_t ps = tile & (kParSlots - 1), pph = (tile / kParSlots) & 1;
        if (!mbar_wait(b_parf + 8 * ps, pph, g.status, ST_TIMEOUT_EPI) ||
            !mbar_wait(b_accf + 8 * b, par, g.status, ST_TIMEOUT_EPI)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const float* soa = slots + ps * kColSoaFloats;
        const int col0 = ct * kBN;
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + b * kBN + cbase;
        const int cm = METRIC == kPearson ? c_mode(kEps * rmax_r * soa[4 * kBN]) : kCFirst;
        const bool full = col0 + kBN <= g.ec.n;
        const bool diag = (ct == (rb >> 1));
        float sn = 0.0f, sd = 0.0f;
        if (METRIC == kPearson && full && !diag && cm == kCFirst)
          epi_tile_pearson2<kCFirst>(taddr, soa, cbase, r2, sn, sd);
        else if (METRIC == kPearson && full && !diag && cm == kCSecond)
          epi_tile_pearson2<kCSecond>(taddr, soa, cbase, r2, sn, sd);
        else if (METRIC == kSsim && full && !diag)
          epi_tile_ssim2(taddr, soa, cbase, s2, sn, sd);
        else if (full && !diag && cm == kCFirst)
          epi_tile<METRIC, kCFirst, true, false>(taddr, soa, cbase, col0, row, rs, g.ec, sn, sd);
        else if (full && !diag && cm == kCSecond)
          epi_tile<METRIC, kCSecond, true, false>(taddr, soa, cbase, col0, row, rs, g.ec, sn, sd);
        else if (cm == kCFirst)
          epi_tile<METRIC, kCFirst, false, true>(taddr, soa, cbase, col0, row, rs, g.ec, sn, sd);
        else if (cm == kCSecond)
          epi_tile<METRIC, kCSecond, false, true>(taddr, soa, cbase, col0, row, rs, g.ec, sn, sd);
        else
          epi_tile<METRIC, kCExact, false, true>(taddr, soa, cbase, col0, row, rs, g.ec, sn, sd);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(b_acce + 8 * b);
          mbar_arrive(b_pare + 8 * ps);
        }
        acc_n += (double)sn;
        acc_d += (double)sd;
      }
      if (ok && row < g.ec.n) {
        atomicAdd(g.num + row, acc_n);
        atomicAdd(g.den + row, acc_d);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kEpiWarps + 1) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * kBN) : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// box_cols 64 (128-byte rows, SWIZZLE_128B) or 32 (64-byte rows, SWIZZLE_64B).
bool make_map(CUtensorMap* m, const __nv_bfloat16* ptr, int kq, int rows, int box_rows, int box_cols = kChunk) {
  auto enc = get_encode();
  if (!enc) return false;
  cuuint64_t dims[2] = {(cuuint64_t)kq, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)kq * 2};
  cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16*>(ptr), dims, strides, box,
                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   box_cols == kChunk ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

cudaError_t launch_gram_tc(const __nv_bfloat16* A, const __nv_bfloat16* B, int kq, int n_pad,
                           const BlockParams* params, const float* colsoa, const float* tile_rmax, EpiConsts ec,
                           double* num, double* den, int num_sms, int* status, cudaStream_t st, int rb_begin,
                           int rb_end) {
  if (kq % 16 != 0 || n_pad % kBN != 0) return cudaErrorInvalidValue;
  TcArgs g;
  g.kq = kq;
  g.nkc = (kq + kChunk - 1) / kChunk;
  g.n_ct = (ec.n + kBN - 1) / kBN;
  const size_t budget = 227 * 1024;
  g.nfull = kq / kChunk;
  g.tail = (kq % kChunk) ? 1 : 0;
  g.a_bytes = (uint32_t)kBM * kq * 2;
  g.b_bytes = (uint32_t)kBN * kq * 2;
  const size_t tr_smem = 1024 + (size_t)g.a_bytes + 2 * (size_t)g.b_bytes + kParSlots * kSoaBytes + 8 * 64;
  const bool tr = (kq % (kChunk / 2) == 0) && tr_smem <= budget;
  size_t smem;
  if (tr) {
    g.stages = 2;
    smem = tr_smem;
  } else {
    const size_t fixed = 1024 + (size_t)g.nkc * kAChunkBytes + kParSlots * kSoaBytes + 8 * 64;
    if (fixed + 2 * kBStageBytes > budget) return cudaErrorInvalidValue;
    g.stages = (int)std::min<size_t>(kMaxStages, (budget - fixed) / kBStageBytes);
    smem = fixed + (size_t)g.stages * kBStageBytes;
  }
  // Only row blocks that hold valid rows are work; split the column range so
  // that every SM gets several items.
  int n_rb_valid = (ec.n + kBM - 1) / kBM;
  if (rb_end < 0) rb_end = n_rb_valid;
  rb_end = std::min(rb_end, n_rb_valid);
  if (rb_begin < 0 || rb_begin >= rb_end) return cudaSuccess;  // no rows in this range
  g.rb0 = rb_begin;
  n_rb_valid = rb_end - rb_begin;
  int segs = (4 * num_sms + n_rb_valid - 1) / n_rb_valid;
  segs = std::max(1, std::min(segs, g.n_ct));
  g.ct_per_item = (g.n_ct + segs - 1) / segs;
  segs = (g.n_ct + g.ct_per_item - 1) / g.ct_per_item;
  g.n_rb = n_rb_valid;
  g.n_items = g.n_rb * segs;
  g.params = params;
  g.colsoa = colsoa;
  g.tile_rmax = tile_rmax;
  g.ec = ec;
  g.num = num;
  g.den = den;
  g.status = status;
  CUtensorMap mA, mB, mA64, mB64;
  if (!make_map(&mA, A, kq, n_pad, kBM) || !make_map(&mB, B, kq, n_pad, kBN)) return cudaErrorInvalidValue;
  mA64 = mA;
  mB64 = mB;
  if (tr && g.tail && (!make_map(&mA64, A, kq, n_pad, kBM, kChunk / 2) || !make_map(&mB64, B, kq, n_pad, kBN, kChunk / 2)))
    return cudaErrorInvalidValue;
  const int grid = std::min(g.n_items, num_sms);
  cudaError_t e;
#define SRED_TC(M)                                                                                         \
  if (tr) {                                                                                                \
    e = cudaFuncSetAttribute(k_gram_tc<M, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
    if (e != cudaSuccess) return e;                                                                        \
    k_gram_tc<M, true><<<grid, kThreads, smem, st>>>(mA, mB, mA64, mB64, g);                               \
  } else {                                                                                                 \
    e = cudaFuncSetAttribute(k_gram_tc<M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);  \
    if (e != cudaSuccess) return e;                                                                        \
    k_gram_tc<M, false><<<grid, kThreads, smem, st>>>(mA, mB, mA64, mB64, g);                              \
  }
  switch (ec.metric) {
    case kPearson: SRED_TC(kPearson); break;
    case kSsim: SRED_TC(kSsim); break;
    case kDebugDot: SRED_TC(kDebugDot); break;
    default: return cudaErrorInvalidValue;
  }
#undef SRED_TC
  return cudaGetLastError();
}

}  // namespace sred
