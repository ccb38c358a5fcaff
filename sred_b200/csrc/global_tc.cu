// Split-BF16 tcgen05 engine of the global repetition map (sm_100a).
//
// G = A' B'^T on the 5th-generation tensor cores, where each block's FP64 unit
// vector u is split into bf16 parts (common.cuh: store_split), so one BF16
// MMA chain with FP32 accumulation yields an FP32-accurate <u_p, u_q>.
//
// Symmetric schedule. Every per-pair term of the global map (weight, Pearson,
// global SSIM, NRMSE, Abs-diff; epilogue.cuh) is symmetric in (p, q), so each
// unordered pair is evaluated once: only tiles of the upper triangle are
// scheduled (a 128-row block rb against a BN-column tile ct with
// 128 rb <= BN ct + BN - 1), pairs below the diagonal are masked in the
// diagonal tiles, and each pair's numerator and denominator terms are added to
// the sums of both blocks (the self pair once).
//
// Work item = (column tile ct, a run of up to L row blocks). The item's B tile
// (BN x K') and column parameters stay in shared memory for the whole item;
// the A tiles of its row blocks stream through (two whole tiles when they fit,
// else a ring of 64-column chunks). Items are ordered panel-major (decode_item):
// all CTAs work on the same row blocks at a time and share their A tiles in
// L2, and a panel's B tiles stay in L2 while the runs pass over them; the
// producer prefetches A two row blocks ahead and the next item's B into L2.
// Each CTA walks its items twice: first their full tiles, then their masked
// ones (diagonal and ragged tiles, about 0.2% of all), so that the masked
// epilogue form sits in a loop of its own (with it in the main loop the full
// tiles ran 3% slower).
// The launch shape (BN = 256 or 128, whole-tile or chunk-ring A, L) is the
// default of plan_gram_tc or a tuned TcChoice. CTA = 1 per SM, persistent.
// Warp roles:
//   warp 16     TMA producer (one thread)
//   warp 17     MMA issuer (one thread): tcgen05.mma M=128 N=BN K=16 into one
//               of two TMEM accumulators, tcgen05.commit to publish it
//   warps 0-15  epilogue: warp w reads TMEM lanes 32(w%4).. and BN/4 columns
//               from BN/4 (w/4) with tcgen05.ld.16x256b, which gives each
//               thread 4 rows x (BN/16) columns of the warp's slab. The fused
//               per-pair metric runs on f32x2 pairs of neighbouring columns.
//               Column sums of the item accumulate in per-thread shared
//               memory slots (BN/16 values per thread and sum, read and
//               written once per 16-column chunk of each tile) and leave once
//               per item after a butterfly over the 8 lanes that share
//               columns; row sums of a tile leave
//               once per tile after a butterfly over the 4 lanes that share
//               rows and a combine of the 4 column-group warps in shared
//               memory: one FP64 atomic add per row per tile.
// Every mbarrier wait is bounded by wall time (a host-set limit); on expiry the
// kernel records a status code, stops issuing work, waits (bounded) for its own
// copies in flight, frees TMEM and returns. No TMA multicast is used.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "epilogue.cuh"

namespace sred {

namespace {

constexpr int kBM = 128;                          // rows per tile (TMEM lanes)
constexpr int kChunk = 64;                        // bf16 per K chunk (128 B: one SWIZZLE_128B atom row)
constexpr int kAChunkBytes = kBM * kChunk * 2;    // 16 KB
constexpr int kMaxStages = 16;
constexpr int kEpiWarps = 16;                     // 4 per SM sub-partition
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr int kEpiThreads = kEpiWarps * 32;
constexpr int kRSlots = 2;                        // row-parameter ring depth
constexpr int kRowR = 8 * kBM;                    // offset of r in a row-parameter slot
constexpr int kRowMax = kRowR + kBM;              // offset of max r
constexpr int kRowFloats = kRowSoaFloats;         // one 128-row block's parameters
constexpr int kRowPartBytes = 2 * 4 * kBM * 8;    // [2 buffers][4 column groups][128 rows] float2
constexpr int kMaxRun = 32;                       // row blocks per run (work item), at most
constexpr int kBarBytes = 512;
constexpr size_t kSmemBudget = 227 * 1024;

enum { ST_OK = 0, ST_TIMEOUT_PRODUCER = 1, ST_TIMEOUT_MMA = 2, ST_TIMEOUT_EPI = 3, ST_TIMEOUT_DRAIN = 4 };

template <int BN>
struct Cfg {
  static constexpr int kColW = BN / 4;              // columns per epilogue warp
  static constexpr int kCH = kColW / 16;            // 16-column chunks per warp and tile
  static constexpr int kM = BN / kBM;               // row blocks per column tile
  static constexpr int kCSoa = col_soa_floats(BN);  // floats per column tile's parameters
  static constexpr int kBChunkBytes = BN * kChunk * 2;
  static constexpr int kColAccBytes = kEpiThreads * 8 * kCH * 4;  // per thread: 2 sums x 4 columns x chunks
};

struct TcArgs {
  int kq, nkc, stages;          // K', K chunks per tile (nfull + tail), chunk-ring depth
  int nfull, tail;              // whole-tile mode: 64-column chunks and a 32-column tail (0 or 1)
  uint32_t a_bytes, b_bytes;    // whole A tile and whole B tile (64-column chunks + 32-column tail)
  int n_rb, n_ct;               // row blocks holding valid rows, column tiles
  int L, h;                     // row blocks per item (a run), L / (BN / 128)
  int n_runs;                   // runs of L row blocks
  int panel, n_panels;          // column tiles per panel (panel-major item order), panels
  long long item0, item1;       // items of this launch
  const float* colsoa;          // per column tile, permuted (col_soa_pos)
  const float* rowsoa;          // per 128-row block, natural order
  EpiConsts ec;
  double* num;
  double* den;
  int* status;
  unsigned long long timeout_ns;
  long long withhold;           // test hook: the producer never issues this tile's loads (-1: none)
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
// records `code`) if the wait exceeded the limit or another role of any CTA
// already gave up. Drain waits (for copies or MMAs this CTA issued) pass
// abort = false: they keep waiting, within the same bound, after another
// role has given up. The single-thread roles (producer, MMA issuer) wait
// mostly for the epilogue; they back off with nanosleep (up to 0.5 us) so
// that their polling does not take issue slots from the epilogue warps of
// their SM sub-partition.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const TcArgs& g, int code,
                                          bool abort = true, bool backoff = false) {
  if (mbar_test(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  uint32_t ns = 32;
  for (uint32_t i = 1;; i++) {
    if (backoff) {
      __nanosleep(ns);
      ns = ns < 512 ? 2 * ns : 512;
    }
    if (mbar_test(bar, parity)) return true;
    if ((i & (backoff ? 7u : 255u)) == 0) {
      if (abort && *reinterpret_cast<volatile int*>(g.status) != ST_OK) return false;
      if (globaltimer() - t0 > g.timeout_ns) {
        atomicCAS(g.status, ST_OK, code);
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

// L2 prefetch of one tensor-map box (no shared memory, no completion).
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int x, int y) {
  asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];" ::"l"(reinterpret_cast<uint64_t>(map)),
               "r"(x), "r"(y)
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
// tail of K' in the whole-tile mode.
__device__ __forceinline__ uint64_t desc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4);
  d |= static_cast<uint64_t>(1) << 16;
  d |= static_cast<uint64_t>(512 >> 4) << 32;
  d |= static_cast<uint64_t>(1) << 46;
  d |= static_cast<uint64_t>(4) << 61;  // SWIZZLE_64B
  return d;
}

// Instruction descriptor, kind::f16: D = F32, A = B = BF16, both K-major, M = 128, N = BN.
template <int BN>
constexpr uint32_t idesc() {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(BN >> 3) << 17) |
         (static_cast<uint32_t>(kBM >> 4) << 24);
}

template <int BN>
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc<BN>()), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Issue a load of 16 lanes x 16 columns of 32-bit accumulator (no wait).
// Thread t receives lanes t/4 and t/4 + 8, columns 2(t%4), 2(t%4) + 1 of
// each 8-column half: v[0..1] (lane t/4, cols 0-7), v[2..3] (lane t/4 + 8),
// v[4..5] and v[6..7] the same for columns 8-15.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.16x256b.x2.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr)
               : "memory");
}

// Wait for every TMEM load this thread issued; the register operands tie
// later uses of v to the wait, so none is scheduled before it.
__device__ __forceinline__ void tmem_wait8(uint32_t (&v)[8]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7])
               :
               : "memory");
}

// ---------------------------------------------------------------------------
// Epilogue arithmetic on f32x2 pairs (two neighbouring columns of one row).
// ---------------------------------------------------------------------------

// Row constants, both halves equal (only the fields a metric uses survive).
struct RowC {
  F2 a, ne, r;                 // weight argument, -eps/sigma, 1/sigma (diagnostic terms)
  F2 mu2, sg2, mumu, s2, sg;   // 2 mu, 2 sigma, mu^2, sigma^2 + c2, sigma
};

template <int METRIC>
__device__ __forceinline__ RowC make_rowc(const float* __restrict__ rs, int row, const EpiConsts& ec) {
  RowC c;
  const float4 lo = *reinterpret_cast<const float4*>(rs + 8 * row);  // a, a, -eps r, -eps r
  c.a = f2(lo.x, lo.y);
  if (METRIC == kPearson) c.ne = f2(lo.z, lo.w);
  if (METRIC == kDebugDot) {
    const float r = rs[kRowR + row];
    c.r = f2(r, r);
  }
  if (METRIC == kSsim || METRIC == kNrmse || METRIC == kNrmseW) {
    const float4 hi = *reinterpret_cast<const float4*>(rs + 8 * row + 4);  // sigma, sigma, mu, mu
    c.sg = f2(hi.x, hi.y);
    c.sg2 = add2(c.sg, c.sg);
    if (METRIC == kSsim) {
      const F2 m = f2(hi.z, hi.w);
      c.mu2 = add2(m, m);
      c.mumu = mul2(m, m);
      c.s2 = fma2(c.sg, c.sg, f2(ec.c2, ec.c2));
    }
  }
  return c;
}

// Numerator factor x and weight w of two pairs; the numerator term is x w for
// the weighted metrics and x for unweighted NRMSE (2D) and the diagnostic dot
// product (whose "weight" is r_p + r_q). Same arithmetic as pair_terms.
template <int METRIC, int CMODE>
__device__ __forceinline__ void terms2(F2 G, const RowC& rc, F2 qa, F2 qr, F2 qs, F2 qm, const EpiConsts& ec,
                                       F2& x, F2& w) {
  const F2 one = f2(1.0f, 1.0f);
  if (METRIC == kDebugDot) {
    x = mul2(G, mul2(rc.a, qa));
    w = add2(rc.r, qr);
    return;
  }
  const F2 d = sub2(rc.a, qa);
  float m0, m1;
  f2_split(mul2(d, d), m0, m1);
  w = f2(ex2_approx(-m0), ex2_approx(-m1));
  float x0, x1;
  if (METRIC == kPearson) {
    F2 gc;
    if (CMODE == kCFirst) {
      gc = fma2(mul2(G, rc.ne), qr, G);  // G (1 - t)
    } else if (CMODE == kCSecond) {
      const F2 nt = mul2(rc.ne, qr);     // -t
      gc = mul2(G, fma2(nt, add2(nt, one), one));  // G (1 - t + t^2)
    } else {
      float d0, d1;
      f2_split(sub2(one, mul2(rc.ne, qr)), d0, d1);  // 1 + t
      gc = mul2(G, f2(rcp_approx(d0), rcp_approx(d1)));
    }
    f2_split(gc, x0, x1);
    x = f2(fmaxf(x0, 0.0f), fmaxf(x1, 0.0f));
  } else if (METRIC == kSsim) {
    const F2 c1 = f2(ec.c1, ec.c1), c2 = f2(ec.c2, ec.c2);
    const F2 num = mul2(fma2(rc.mu2, qm, c1), fma2(mul2(rc.sg2, qs), G, c2));
    const F2 den = mul2(fma2(rc.mumu, mul2(qm, qm), c1), fma2(qs, qs, rc.s2));
    float e0, e1, q0, q1;
    f2_split(den, e0, e1);
    f2_split(mul2(num, f2(rcp_approx(e0), rcp_approx(e1))), q0, q1);
    x = f2(fmaxf(q0, 0.0f), fmaxf(q1, 0.0f));
  } else {  // kNrmse, kNrmseW: ((K-1)/K)((s_p - s_q)^2 + 2 s_p s_q (1 - G))
    const F2 sc = f2(ec.nrmse_scale, ec.nrmse_scale);
    const F2 ds = sub2(rc.sg, qs);
    f2_split(mul2(sc, fma2(ds, ds, mul2(mul2(rc.sg2, qs), sub2(one, G)))), x0, x1);
    x = f2(sqrtf(fmaxf(x0, 0.0f)), sqrtf(fmaxf(x1, 0.0f)));
  }
}

template <int METRIC>
constexpr bool weighted_num() {
  return METRIC == kPearson || METRIC == kSsim || METRIC == kNrmseW;
}

// Exact squared distance of two FP32 unit vectors (NRMSE near-identical pairs).
__device__ __noinline__ float exact_diff2(const float* __restrict__ up, const float* __restrict__ uq, int K) {
  float acc = 0.0f;
  for (int i = 0; i < K; i++) {
    const float d = up[i] - uq[i];
    acc = fmaf(d, d, acc);
  }
  return acc;
}

__device__ __forceinline__ void f2_add_half(F2& v, int half, float x) {
  float lo, hi;
  f2_split(v, lo, hi);
  if (half) hi += x;
  else lo += x;
  v = f2(lo, hi);
}

template <int METRIC>
constexpr bool nrmse_tc() {
  return METRIC == kNrmse || METRIC == kNrmseW;
}

// One 32-row x BN/4-column slab of a tile for this warp: BN/64 chunks of 16
// columns, each read for both 16-lane halves of the warp's 32 TMEM lanes.
// rs: the tile's row parameters; cs: this warp's column parameters (permuted);
// cacc: this thread's column accumulators in shared memory, float4 j at
// cacc[j * kEpiThreads] for j = 2c + {0: num, 1: den}, each holding the
// thread's four columns of chunk c (2(t%4) + {0, 1}, 8 + 2(t%4) + {0, 1});
// p0: block index of tile row 0; q0: block index of the slab's first column.
// The tile's row sums are returned in rsum[2k + {0: num, 1: den}] for rows
// 32(w%4) + t/4 + 8k.
// Row passes of the epilogue: the metrics with many row constants (SSIM,
// NRMSE) take the 4 rows in two passes of 2 so that their constants fit in
// registers; the column accumulators are then read and written once per pass.
template <int METRIC>
constexpr int row_passes() {
  return (METRIC == kSsim || METRIC == kNrmse || METRIC == kNrmseW) ? 2 : 1;
}

template <int METRIC, int BN, int CMODE, bool MASKED>
__device__ __forceinline__ void sym_tile(uint32_t taddr, const float* __restrict__ rs, const float* __restrict__ cs,
                                         float4* __restrict__ cacc, int p0, int q0, const EpiConsts& ec,
                                         float (&rsum)[8]) {
  constexpr int CH = Cfg<BN>::kCH;
  constexpr int NP = row_passes<METRIC>(), R = 4 / NP;  // passes, rows per pass
  constexpr int HP = R / 2;                              // 16-lane halves per pass
  const int lane = threadIdx.x & 31, rsub = lane >> 2, csub = lane & 3;
  const int quarter = (threadIdx.x >> 5) & 3;
#pragma unroll 1
  for (int pass = 0; pass < NP; pass++) {
    RowC rc[R];
    F2 rn[R], rd[R];
    int prow[R];
    bool force[R];
#pragma unroll
    for (int kr = 0; kr < R; kr++) {
      const int row = quarter * 32 + rsub + 8 * (pass * R + kr);
      rc[kr] = make_rowc<METRIC>(rs, row, ec);
      rn[kr] = rd[kr] = f2(0.0f, 0.0f);
      prow[kr] = p0 + row;
      force[kr] = MASKED && rs[kRowR + row] > 0.0f;
    }
    // TMEM reads, one (chunk, half) step at a time; the next step's load is
    // issued before the current step is evaluated.
    const uint32_t tp = taddr + ((uint32_t)(16 * pass * HP) << 16);
    uint32_t buf[2][8];
    tmem_ld8(tp, buf[0]);
    tmem_wait8(buf[0]);
#pragma unroll
    for (int c = 0; c < CH; c++) {
      const float4 cnv = cacc[(2 * c) * kEpiThreads], cdv = cacc[(2 * c + 1) * kEpiThreads];
      F2 cn[2] = {f2(cnv.x, cnv.y), f2(cnv.z, cnv.w)};
      F2 cd[2] = {f2(cdv.x, cdv.y), f2(cdv.z, cdv.w)};
      const int cb = 16 * c + 4 * csub;
      const float4 a4 = *reinterpret_cast<const float4*>(cs + cb);
      float4 r4 = make_float4(0.f, 0.f, 0.f, 0.f), s4 = r4, m4 = r4;
      if (METRIC == kPearson || METRIC == kDebugDot) r4 = *reinterpret_cast<const float4*>(cs + BN + cb);
      if (METRIC == kSsim || METRIC == kNrmse || METRIC == kNrmseW)
        s4 = *reinterpret_cast<const float4*>(cs + 2 * BN + cb);
      if (METRIC == kSsim) m4 = *reinterpret_cast<const float4*>(cs + 3 * BN + cb);
#pragma unroll
      for (int hh = 0; hh < HP; hh++) {
        const int step = c * HP + hh;
        uint32_t(&cur)[8] = buf[step & 1];
        uint32_t(&nxt)[8] = buf[(step + 1) & 1];
        if (step + 1 < CH * HP) {
          const int nc = (step + 1) / HP, nh = (step + 1) % HP;
          tmem_ld8(tp + ((uint32_t)(16 * nh) << 16) + 16 * nc, nxt);
        }
        uint32_t near = 0;  // NRMSE: sign bits of (1 - delta) - G, any set = a near-identical pair
#pragma unroll
        for (int rep = 0; rep < 2; rep++) {
          const F2 qa = rep ? f2(a4.z, a4.w) : f2(a4.x, a4.y);
          const F2 qr = rep ? f2(r4.z, r4.w) : f2(r4.x, r4.y);
          const F2 qs = rep ? f2(s4.z, s4.w) : f2(s4.x, s4.y);
          const F2 qm = rep ? f2(m4.z, m4.w) : f2(m4.x, m4.y);
          const int qlo = q0 + 16 * c + 8 * rep + 2 * csub;
#pragma unroll
          for (int kk = 0; kk < 2; kk++) {
            const int kr = 2 * hh + kk;
            float g0 = __uint_as_float(cur[4 * rep + 2 * kk]), g1 = __uint_as_float(cur[4 * rep + 2 * kk + 1]);
            const int p = prow[kr];
            if (MASKED) {
              if (force[kr] && qlo == p) g0 = 1.0f;
              if (force[kr] && qlo + 1 == p) g1 = 1.0f;
            }
            F2 x, w;
            terms2<METRIC, CMODE>(f2(g0, g1), rc[kr], qa, qr, qs, qm, ec, x, w);
            if (nrmse_tc<METRIC>()) {
              float t0, t1;
              f2_split(sub2(f2(ec.nrmse_near, ec.nrmse_near), f2(g0, g1)), t0, t1);
              asm("lop3.b32 %0, %0, %1, %2, 0xFE;" : "+r"(near) : "r"(__float_as_uint(t0)), "r"(__float_as_uint(t1)));
            }
            if (!MASKED) {
              if (weighted_num<METRIC>()) {
                rn[kr] = fma2(x, w, rn[kr]);
                cn[rep] = fma2(x, w, cn[rep]);
              } else {
                rn[kr] = add2(rn[kr], x);
                cn[rep] = add2(cn[rep], x);
              }
              rd[kr] = add2(rd[kr], w);
              cd[rep] = add2(cd[rep], w);
            } else {
              float x0, x1, w0, w1;
              f2_split(weighted_num<METRIC>() ? mul2(x, w) : x, x0, x1);
              f2_split(w, w0, w1);
              const bool pv = p < ec.n;
              const bool r0 = pv && qlo >= p && qlo < ec.n, r1 = pv && qlo + 1 >= p && qlo + 1 < ec.n;
              const bool c0 = r0 && qlo != p, c1 = r1 && qlo + 1 != p;
              rn[kr] = add2(rn[kr], f2(r0 ? x0 : 0.0f, r1 ? x1 : 0.0f));
              rd[kr] = add2(rd[kr], f2(r0 ? w0 : 0.0f, r1 ? w1 : 0.0f));
              cn[rep] = add2(cn[rep], f2(c0 ? x0 : 0.0f, c1 ? x1 : 0.0f));
              cd[rep] = add2(cd[rep], f2(c0 ? w0 : 0.0f, c1 ? w1 : 0.0f));
            }
          }
        }
        if (nrmse_tc<METRIC>() && (int)near < 0) {
          // Near-identical pairs: replace the accumulated term by the one of the
          // exact squared difference (the same arithmetic as terms2 recomputes
          // the term to remove).
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const int rep = j >> 2, kk = (j >> 1) & 1, lh = j & 1;
            const int kr = 2 * hh + kk;
            const float g = __uint_as_float(cur[4 * rep + 2 * kk + lh]);
            const int row = quarter * 32 + rsub + 8 * (pass * R + kr);
            const int p = prow[kr], q = q0 + 16 * c + 8 * rep + 2 * csub + lh;
            const bool rv = !MASKED || (p < ec.n && q >= p && q < ec.n);
            const bool cv = !MASKED || (rv && q != p);
            float ge = g;
            if (MASKED && force[kr] && q == p) ge = 1.0f;
            if (!(ge > ec.nrmse_near) || !rv) continue;
            const float sp = rs[8 * row + 4];
            const int ci = 16 * c + 4 * csub + 2 * rep + lh;  // permuted column slot
            const float sq = cs[2 * BN + ci];
            const float ds = __fsub_rn(sp, sq);
            const float approx = sqrtf(fmaxf(
                __fmul_rn(ec.nrmse_scale, __fmaf_rn(ds, ds, __fmul_rn(__fmul_rn(__fadd_rn(sp, sp), sq), __fsub_rn(1.0f, ge)))),
                0.0f));
            const float D = (q == p) ? 0.0f : exact_diff2(ec.U + (size_t)p * ec.kp, ec.U + (size_t)q * ec.kp, ec.K);
            const float exact = sqrtf(__fmul_rn(ec.nrmse_scale, __fmaf_rn(ds, ds, __fmul_rn(__fmul_rn(sp, sq), D))));
            float corr = exact - approx;
            if (METRIC == kNrmseW) {
              const float d = __fsub_rn(rs[8 * row], cs[ci]);
              corr *= ex2_approx(-__fmul_rn(d, d));
            }
            f2_add_half(rn[kr], lh, corr);
            if (cv) f2_add_half(cn[rep], lh, corr);
          }
        }
        if (step + 1 < CH * HP) tmem_wait8(nxt);
      }
      float4 o;
      f2_split(cn[0], o.x, o.y);
      f2_split(cn[1], o.z, o.w);
      cacc[(2 * c) * kEpiThreads] = o;
      f2_split(cd[0], o.x, o.y);
      f2_split(cd[1], o.z, o.w);
      cacc[(2 * c + 1) * kEpiThreads] = o;
    }
#pragma unroll
    for (int kr = 0; kr < R; kr++) {
      float lo, hi, n, d;
      f2_split(rn[kr], lo, hi);
      n = lo + hi;
      f2_split(rd[kr], lo, hi);
      d = lo + hi;
      if (pass == 0) {  // compile-time indices into rsum (the pass loop is not unrolled)
        rsum[2 * kr] = n;
        rsum[2 * kr + 1] = d;
      } else {
        rsum[2 * (R + kr)] = n;
        rsum[2 * (R + kr) + 1] = d;
      }
    }
  }
}

// Row sums of the 4 lanes that share rows (lanes 4i..4i+3): x[2k + s] holds
// row k's sum s; lane t ends with (num, den) of row k = 2 (t & 1) + ((t >> 1) & 1).
__device__ __forceinline__ float2 reduce_rows4(const float (&x)[8]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const bool b0 = lane & 1, b1 = lane & 2;
  float y[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const float keep = b0 ? x[4 + i] : x[i], send = b0 ? x[i] : x[4 + i];
    y[i] = keep + __shfl_xor_sync(full, send, 1);
  }
  float z[2];
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const float keep = b1 ? y[2 + i] : y[i], send = b1 ? y[i] : y[2 + i];
    z[i] = keep + __shfl_xor_sync(full, send, 2);
  }
  return make_float2(z[0], z[1]);
}

// Column sums of the 8 lanes that share columns (lanes with equal t % 4),
// then one FP64 atomic add per column and sum. x index:
// ((c * 2 + rep) * 2 + lohi) * 2 + sum, column 16c + 8rep + 2(t % 4) + lohi.
template <int NV>
__device__ __forceinline__ void flush_columns(const float (&x)[NV], int q0, const EpiConsts& ec, double* num,
                                              double* den) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, csub = lane & 3;
  const int b1 = (lane >> 2) & 1, b2 = (lane >> 3) & 1, b3 = (lane >> 4) & 1;
  float y[NV / 2], z[NV / 4], u[NV / 8];
#pragma unroll
  for (int i = 0; i < NV / 2; i++) {
    const float keep = b1 ? x[NV / 2 + i] : x[i], send = b1 ? x[i] : x[NV / 2 + i];
    y[i] = keep + __shfl_xor_sync(full, send, 4);
  }
#pragma unroll
  for (int i = 0; i < NV / 4; i++) {
    const float keep = b2 ? y[NV / 4 + i] : y[i], send = b2 ? y[i] : y[NV / 4 + i];
    z[i] = keep + __shfl_xor_sync(full, send, 8);
  }
#pragma unroll
  for (int i = 0; i < NV / 8; i++) {
    const float keep = b3 ? z[NV / 8 + i] : z[i], send = b3 ? z[i] : z[NV / 8 + i];
    u[i] = keep + __shfl_xor_sync(full, send, 16);
  }
#pragma unroll
  for (int j = 0; j < NV / 8; j++) {
    const int i = b1 * (NV / 2) + b2 * (NV / 4) + b3 * (NV / 8) + j;
    const int c = i >> 3, rep = (i >> 2) & 1, lohi = (i >> 1) & 1, s = i & 1;
    const int q = q0 + 16 * c + 8 * rep + 2 * csub + lohi;
    if (q < ec.n) atomicAdd((s ? den : num) + q, (double)u[j]);
  }
}

// Work items. Run j holds row blocks [jL, jL + L); it meets the column tiles
// ct >= j h (h = L / (BN / 128): the first column tile that reaches the run's
// rows), each (run, column tile) an item, clipped to the triangle. The column
// tiles are grouped into panels of g.panel tiles whose B operand fits in L2;
// items go panel by panel, within a panel run by run, within a run by column
// tile. All CTAs then work on the same row blocks at once (their A tiles are
// read from DRAM once per panel and shared in L2), and a panel's B tiles stay
// in L2 while every run passes over them (B is read from DRAM about once).
// With one panel this is the plain run-major order.
//
// Items of runs [0, j) in the panel of column tiles [c0, c1): sum over
// j' < j of c1 - max(c0, j' h).
__host__ __device__ inline long long panel_items_before_run(long long j, int c0, int c1, int h) {
  const long long a = min(j, (long long)(c0 / h) + 1);  // runs with j' h <= c0 take the whole panel
  long long s = a * (c1 - c0);
  if (j > a) s += (j - a) * (long long)c1 - (long long)h * (j * (j - 1) / 2 - a * (a - 1) / 2);
  return s;
}

// Items of runs [0, j) over all column tiles (one panel).
__host__ __device__ inline long long items_before_run(long long j, int n_ct, int h) {
  return j * n_ct - (long long)h * j * (j - 1) / 2;
}

// Runs that reach the panel [c0, c1) (j h <= c1 - 1), at most n_runs.
__host__ __device__ inline int panel_runs(int c1, int h, int n_runs) { return min((c1 - 1) / h + 1, n_runs); }

// Item -> (column tile, row-block range); false for an empty range.
__host__ __device__ inline bool decode_item(long long it, const TcArgs& g, int m, int& ct, int& rb0, int& rb1) {
  long long base = 0;
  int c0 = 0, c1 = 0, J = 0;
  for (int k = 0; k < g.n_panels; k++) {
    c0 = k * g.panel;
    c1 = min(c0 + g.panel, g.n_ct);
    J = panel_runs(c1, g.h, g.n_runs);
    const long long cnt = panel_items_before_run(J, c0, c1, g.h);
    if (it < base + cnt || k == g.n_panels - 1) break;
    base += cnt;
  }
  const long long r = it - base;
  int lo = 0, hi = J - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (panel_items_before_run(mid, c0, c1, g.h) <= r) lo = mid;
    else hi = mid - 1;
  }
  ct = max(c0, lo * g.h) + (int)(r - panel_items_before_run(lo, c0, c1, g.h));
  rb0 = lo * g.L;
  rb1 = min(rb0 + g.L, min((ct + 1) * m, g.n_rb));
  return rb0 < rb1 && ct < c1;
}

// A CTA's walk over its items it = start, start + stride, ...: the first is
// decoded with decode_item's search, each later one by stepping forward run by
// run (a few operations per step instead of a search per item, which matters
// for small maps whose items hold few tiles).
struct ItemCursor {
  long long it;  // current item
  long long r;   // its offset among the items of run j in panel k
  int k, c0, c1, J, j;

  __host__ __device__ __forceinline__ void set_panel(const TcArgs& g, int kk) {
    k = kk;
    c0 = kk * g.panel;
    c1 = min(c0 + g.panel, g.n_ct);
    J = panel_runs(c1, g.h, g.n_runs);
  }
  __host__ __device__ __forceinline__ void init(const TcArgs& g, long long start) {
    it = start;
    long long base = 0;
    set_panel(g, 0);
    while (k < g.n_panels - 1) {
      const long long cnt = panel_items_before_run(J, c0, c1, g.h);
      if (start < base + cnt) break;
      base += cnt;
      set_panel(g, k + 1);
    }
    const long long rr = start - base;
    int lo = 0, hi = J - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (panel_items_before_run(mid, c0, c1, g.h) <= rr) lo = mid;
      else hi = mid - 1;
    }
    j = lo;
    r = rr - panel_items_before_run(lo, c0, c1, g.h);
  }
  __host__ __device__ __forceinline__ void advance(const TcArgs& g, long long d) {
    it += d;
    r += d;
    for (;;) {
      const int cnt = c1 - max(c0, j * g.h);  // >= 1 for every run below J
      if (r < cnt) break;
      r -= cnt;
      if (++j >= J) {
        if (k + 1 >= g.n_panels) break;  // past the last item; the caller stops on it
        set_panel(g, k + 1);
        j = 0;
      }
    }
  }
  // The tiles of the current item that pass `phase` takes: pass 0 the full
  // tiles, pass 1 the masked ones (tiles that reach the diagonal, rb >= ct m,
  // and every tile of a ragged last column tile). Every role walks pass 0 over
  // all of the CTA's items, then pass 1, so the masked epilogue runs in a loop
  // of its own. False for an empty range.
  __host__ __device__ __forceinline__ bool part(const TcArgs& g, int m, int bn, int phase, int& ct, int& lo,
                                                int& hi) const {
    ct = max(c0, j * g.h) + (int)r;
    const int rb0 = j * g.L, rb1 = min(rb0 + g.L, min((ct + 1) * m, g.n_rb));
    const bool full = (long long)(ct + 1) * bn <= g.ec.n;
    const int rbm = full ? min(max(rb0, ct * m), rb1) : rb0;
    lo = phase == 0 ? rb0 : rbm;
    hi = phase == 0 ? rbm : rb1;
    return lo < hi;
  }
};

__device__ __forceinline__ ItemCursor first_item(const TcArgs& g) {
  ItemCursor c;
  c.init(g, g.item0 + blockIdx.x);
  return c;
}

// End of a role: all warps meet, then the MMA warp frees TMEM.
__device__ __forceinline__ void role_exit(uint32_t tmem, int tmem_cols, bool owner) {
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (owner) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
}

// TR (whole-tile mode, when two A tiles and the B tile fit): A moves one
// whole 128-row tile at a time through two buffers, and the single
// tcgen05.commit per tile both publishes the accumulator and frees the tile's
// A buffer (the producer waits on the accumulator barrier). K' = 64 c + 32 t:
// c SWIZZLE_128B chunks and an optional SWIZZLE_64B tail.
// !TR (chunk ring): A moves in 64-column chunks through S stages, one commit
// per chunk.
template <int METRIC, int BN, bool TR>
__global__ void __launch_bounds__(kThreads, 1)
    k_gram_tc(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
              const __grid_constant__ CUtensorMap tmA64, const __grid_constant__ CUtensorMap tmB64, TcArgs g) {
  using C = Cfg<BN>;
  constexpr int CH = C::kCH;
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* sbase = smem_raw + (base - raw);
  const int S = g.stages, nkc = g.nkc;
  const uint32_t sB = base;                                            // resident B tile
  const uint32_t sA = sB + g.b_bytes;                                  // TR: 2 x a_bytes; else S x 16 KB
  const uint32_t sC = sA + (TR ? 2 * g.a_bytes : S * kAChunkBytes);    // 2 column-parameter slots
  const uint32_t sR = sC + 2 * C::kCSoa * 4;                           // kRSlots row-parameter slots
  const uint32_t sP = sR + kRSlots * kRowFloats * 4;                   // row partials
  const uint32_t sQ = sP + kRowPartBytes;                              // column accumulators
  const uint32_t sBar = sQ + C::kColAccBytes;
  const float* cslots = reinterpret_cast<const float*>(sbase + (sC - base));
  const float* rslots = reinterpret_cast<const float*>(sbase + (sR - base));
  float2* rowpart = reinterpret_cast<float2*>(sbase + (sP - base));
  float4* colacc = reinterpret_cast<float4*>(sbase + (sQ - base));
  // barriers: a_full[16], a_empty[16], b_full, b_empty, acc_full[2], acc_empty[2],
  //           c_full[2], c_empty[2], r_full[2], r_empty[2], done; then the TMEM
  //           address and 8 row-partial counters
  const uint32_t b_afull = sBar, b_aempty = b_afull + 8 * kMaxStages, b_bfull = b_aempty + 8 * kMaxStages,
                 b_bempty = b_bfull + 8, b_accf = b_bempty + 8, b_acce = b_accf + 16, b_cfull = b_acce + 16,
                 b_cempty = b_cfull + 16, b_rfull = b_cempty + 16, b_rempty = b_rfull + 8 * kRSlots,
                 b_done = b_rempty + 8 * kRSlots;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sbase + (b_done + 8 - base));
  // per (accumulator buffer, quarter): column-group warps that have written
  // their row partials of the current tile (the fourth combines them)
  unsigned* rowcnt = tmem_slot + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kMaxStages; s++) {
      mbar_init(b_afull + 8 * s, 1);
      mbar_init(b_aempty + 8 * s, 1);
    }
    mbar_init(b_bfull, 1);
    mbar_init(b_bempty, 1);
    for (int b = 0; b < 2; b++) {
      mbar_init(b_accf + 8 * b, 1);
      mbar_init(b_acce + 8 * b, kEpiWarps);
      mbar_init(b_cfull + 8 * b, 1);
      mbar_init(b_cempty + 8 * b, kEpiWarps);
    }
    for (int r = 0; r < kRSlots; r++) {
      mbar_init(b_rfull + 8 * r, 1);
      mbar_init(b_rempty + 8 * r, kEpiWarps);
    }
    for (int i = 0; i < 8; i++) rowcnt[i] = 0;
    mbar_init(b_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == kEpiWarps + 1) {  // MMA warp owns the TMEM allocation
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * BN)
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
      long long tile = 0;
      uint32_t item_i = 0, n_r = 0, n_a = 0;  // items, row-parameter loads, A loads (tiles or chunks) issued
      uint32_t s = 0, eph = 0;                // chunk ring: stage, parity of the round being refilled
      bool ok = true;
      for (int phase = 0; ok && phase < 2; phase++)
      for (ItemCursor cur = first_item(g); ok && cur.it < g.item1; cur.advance(g, gridDim.x)) {
        int ct, rb0, rb1;
        if (!cur.part(g, C::kM, BN, phase, ct, rb0, rb1)) continue;
        const uint32_t cs = item_i & 1;
        // the column-parameter slot the epilogue released two items ago, and the
        // B buffer once the MMAs of the previous item are complete
        if (!mbar_wait(b_cempty + 8 * cs, ((item_i >> 1) & 1) ^ 1, g, ST_TIMEOUT_PRODUCER, true, true)) { ok = false; break; }
        if (item_i > 0 && !mbar_wait(b_bempty, (item_i - 1) & 1, g, ST_TIMEOUT_PRODUCER, true, true)) { ok = false; break; }
        mbar_expect_tx(b_cfull + 8 * cs, C::kCSoa * 4);
        bulk_load(sC + cs * C::kCSoa * 4, g.colsoa + (size_t)ct * C::kCSoa, C::kCSoa * 4, b_cfull + 8 * cs);
        mbar_expect_tx(b_bfull, g.b_bytes);
        for (int c = 0; c < g.nfull; c++) tma_load_2d(sB + c * C::kBChunkBytes, &tmB, b_bfull, c * kChunk, ct * BN);
        if (g.tail) tma_load_2d(sB + g.nfull * C::kBChunkBytes, &tmB64, b_bfull, g.nfull * kChunk, ct * BN);
        item_i++;
        {  // the B tile of this CTA's next item into L2
          int nct, nrb0, nrb1;
          ItemCursor nx = cur;
          nx.advance(g, gridDim.x);
          if (nx.it < g.item1 && nx.part(g, C::kM, BN, phase, nct, nrb0, nrb1) && nct != ct) {
            for (int c = 0; c < g.nfull; c++) tma_prefetch_2d(&tmB, c * kChunk, nct * BN);
            if (g.tail) tma_prefetch_2d(&tmB64, g.nfull * kChunk, nct * BN);
          }
        }
        for (int rb = rb0; ok && rb < rb1; rb++, tile++) {
          if (tile == g.withhold) { ok = false; break; }
          // A two row blocks ahead into L2, so that the copies below hit L2
          if (rb + 2 < rb1) {
            for (int c = 0; c < g.nfull; c++) tma_prefetch_2d(&tmA, c * kChunk, (rb + 2) * kBM);
            if (g.tail) tma_prefetch_2d(&tmA64, g.nfull * kChunk, (rb + 2) * kBM);
          }
          // The A operand first (the MMA waits for it), then the row parameters
          // (the epilogue needs them only once the accumulator is ready).
          if (TR) {
            // A buffer tile & 1 is free once the accumulator of tile - 2 is published
            if (tile >= 2 && !mbar_wait(b_accf + 8 * (tile & 1), ((tile - 2) >> 1) & 1, g, ST_TIMEOUT_PRODUCER, true, true)) {
              ok = false;
              break;
            }
            const uint32_t ab = (uint32_t)(tile & 1);
            const uint32_t dst = sA + ab * g.a_bytes;
            mbar_expect_tx(b_afull + 8 * ab, g.a_bytes);
            for (int c = 0; c < g.nfull; c++) tma_load_2d(dst + c * kAChunkBytes, &tmA, b_afull + 8 * ab, c * kChunk, rb * kBM);
            if (g.tail) tma_load_2d(dst + g.nfull * kAChunkBytes, &tmA64, b_afull + 8 * ab, g.nfull * kChunk, rb * kBM);
            n_a++;
          } else {
            for (int kc = 0; kc < nkc; kc++) {
              if (!mbar_wait(b_aempty + 8 * s, eph ^ 1, g, ST_TIMEOUT_PRODUCER, true, true)) { ok = false; break; }
              if (kc < g.nfull) {
                mbar_expect_tx(b_afull + 8 * s, kAChunkBytes);
                tma_load_2d(sA + s * kAChunkBytes, &tmA, b_afull + 8 * s, kc * kChunk, rb * kBM);
              } else {  // the 32-column tail
                mbar_expect_tx(b_afull + 8 * s, kAChunkBytes / 2);
                tma_load_2d(sA + s * kAChunkBytes, &tmA64, b_afull + 8 * s, kc * kChunk, rb * kBM);
              }
              n_a++;
              if (++s == (uint32_t)S) {
                s = 0;
                eph ^= 1;
              }
            }
            if (!ok) break;
          }
          const uint32_t rsl = (uint32_t)(tile & (kRSlots - 1));
          if (!mbar_wait(b_rempty + 8 * rsl, ((tile / kRSlots) & 1) ^ 1, g, ST_TIMEOUT_PRODUCER, true, true)) { ok = false; break; }
          mbar_expect_tx(b_rfull + 8 * rsl, kRowFloats * 4);
          bulk_load(sR + rsl * kRowFloats * 4, g.rowsoa + (size_t)rb * kRowFloats, kRowFloats * 4, b_rfull + 8 * rsl);
          n_r++;
        }
      }
      // Drain: every issued copy has landed before the CTA may exit.
      if (item_i > 0) {
        mbar_wait(b_bfull, (item_i - 1) & 1, g, ST_TIMEOUT_DRAIN, false);
        for (uint32_t k = (item_i > 2 ? item_i - 2 : 0); k < item_i; k++)
          mbar_wait(b_cfull + 8 * (k & 1), (k >> 1) & 1, g, ST_TIMEOUT_DRAIN, false);
      }
      for (uint32_t k = (n_r > (uint32_t)kRSlots ? n_r - kRSlots : 0); k < n_r; k++)
        mbar_wait(b_rfull + 8 * (k % kRSlots), (k / kRSlots) & 1, g, ST_TIMEOUT_DRAIN, false);
      const uint32_t ring = TR ? 2u : (uint32_t)S;
      for (uint32_t k = (n_a > ring ? n_a - ring : 0); k < n_a; k++)
        mbar_wait(b_afull + 8 * (k % ring), (k / ring) & 1, g, ST_TIMEOUT_DRAIN, false);
    }
    __syncwarp();
    role_exit(tmem, 2 * BN, false);
    return;
  } else if (warp == kEpiWarps + 1) {
    // ---------------------------------------------------------------- MMA
    if (lane == 0) {
      long long tile = 0;
      uint32_t item_i = 0;
      uint32_t s = 0, fph = 0;  // chunk ring: stage, parity of the round being consumed
      // Operand descriptors: the start-address field counts 16-byte units, so
      // a K step of 16 bf16 (32 B) adds 2 and a chunk or stage adds its size / 16.
      const uint64_t a_desc0 = desc_sw128(sA), b_desc0 = desc_sw128(sB);
      bool ok = true;
      for (int phase = 0; ok && phase < 2; phase++)
      for (ItemCursor cur = first_item(g); ok && cur.it < g.item1; cur.advance(g, gridDim.x)) {
        int ct, rb0, rb1;
        if (!cur.part(g, C::kM, BN, phase, ct, rb0, rb1)) continue;
        if (!mbar_wait(b_bfull, item_i & 1, g, ST_TIMEOUT_MMA, true, true)) { ok = false; break; }
        tc_fence_after();
        item_i++;
        for (int rb = rb0; ok && rb < rb1; rb++, tile++) {
          const uint32_t b = (uint32_t)(tile & 1);
          if (!mbar_wait(b_acce + 8 * b, ((tile >> 1) & 1) ^ 1, g, ST_TIMEOUT_MMA, true, true)) { ok = false; break; }
          tc_fence_after();
          const uint32_t d = tmem + b * BN;
          if (TR) {
            if (!mbar_wait(b_afull + 8 * b, (tile >> 1) & 1, g, ST_TIMEOUT_MMA, true, true)) { ok = false; break; }
            tc_fence_after();
            const uint64_t da0 = a_desc0 + (uint64_t)((b * g.a_bytes) >> 4);
            for (int c = 0; c < g.nfull; c++) {
#pragma unroll
              for (int ks = 0; ks < kChunk / 16; ks++)
                mma_bf16<BN>(d, da0 + (uint64_t)(c * (kAChunkBytes >> 4) + 2 * ks),
                             b_desc0 + (uint64_t)(c * (C::kBChunkBytes >> 4) + 2 * ks), (c | ks) != 0);
            }
            if (g.tail) {
              const uint64_t da = desc_sw64(sA + b * g.a_bytes + g.nfull * kAChunkBytes);
              const uint64_t db = desc_sw64(sB + g.nfull * C::kBChunkBytes);
              mma_bf16<BN>(d, da, db, g.nfull != 0);
              mma_bf16<BN>(d, da + 2, db + 2, 1);
            }
            mma_commit(b_accf + 8 * b);
            continue;
          }
          for (int kc = 0; kc < nkc; kc++) {
            if (!mbar_wait(b_afull + 8 * s, fph, g, ST_TIMEOUT_MMA, true, true)) { ok = false; break; }
            tc_fence_after();
            if (kc < g.nfull) {
              const uint64_t da = a_desc0 + (uint64_t)(s * (kAChunkBytes >> 4));
              const uint64_t db = b_desc0 + (uint64_t)(kc * (C::kBChunkBytes >> 4));
#pragma unroll
              for (int ks = 0; ks < kChunk / 16; ks++) mma_bf16<BN>(d, da + 2 * ks, db + 2 * ks, (kc | ks) != 0);
            } else {
              const uint64_t da = desc_sw64(sA + s * kAChunkBytes);
              const uint64_t db = desc_sw64(sB + g.nfull * C::kBChunkBytes);
              mma_bf16<BN>(d, da, db, kc != 0);
              mma_bf16<BN>(d, da + 2, db + 2, 1);
            }
            mma_commit(b_aempty + 8 * s);
            if (++s == (uint32_t)S) {
              s = 0;
              fph ^= 1;
            }
          }
          if (ok) mma_commit(b_accf + 8 * b);
        }
        if (ok) mma_commit(b_bempty);  // the item's B tile is free once these MMAs complete
      }
      // All MMAs this thread issued are complete before TMEM is released and
      // the CTA exits.
      mma_commit(b_done);
      mbar_wait(b_done, 0, g, ST_TIMEOUT_DRAIN, false);
    }
    __syncwarp();
    role_exit(tmem, 2 * BN, true);
    return;
  } else {
    // ---------------------------------------------------------------- epilogue
    const int quarter = warp & 3, group = warp >> 2;
    long long tile = 0;
    uint32_t item_i = 0;
    bool ok = true;
    // One pass over the CTA's items per phase (ItemCursor::part): the full tiles with
    // the unmasked forms, then the masked tiles, each in a loop of its own.
    auto pass = [&](auto phase_tag) {
    constexpr int kPhase = decltype(phase_tag)::value;
    for (ItemCursor cur = first_item(g); ok && cur.it < g.item1; cur.advance(g, gridDim.x)) {
      int ct, rb0, rb1;
      if (!cur.part(g, C::kM, BN, kPhase, ct, rb0, rb1)) continue;
      const uint32_t cs = item_i & 1;
      if (!mbar_wait(b_cfull + 8 * cs, (item_i >> 1) & 1, g, ST_TIMEOUT_EPI)) { ok = false; break; }
      item_i++;
      const float* csl = cslots + cs * C::kCSoa;
      const float rmax_c = csl[4 * BN];
      const int q0 = ct * BN + group * C::kColW;
      float4* cacc = colacc + threadIdx.x;
#pragma unroll
      for (int j = 0; j < 2 * CH; j++) cacc[j * kEpiThreads] = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int rb = rb0; ok && rb < rb1; rb++, tile++) {
        const uint32_t b = (uint32_t)(tile & 1);
        const uint32_t rsl = (uint32_t)(tile & (kRSlots - 1));
        if (!mbar_wait(b_rfull + 8 * rsl, (tile / kRSlots) & 1, g, ST_TIMEOUT_EPI) ||
            !mbar_wait(b_accf + 8 * b, (tile >> 1) & 1, g, ST_TIMEOUT_EPI)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const float* rsp = rslots + rsl * kRowFloats;
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + b * BN + group * C::kColW;
        const int p0 = rb * kBM;
        const float* csw = csl + group * C::kColW;
        float rsum[8];
        if constexpr (kPhase == 1) {
          sym_tile<METRIC, BN, kCExact, true>(taddr, rsp, csw, cacc, p0, q0, g.ec, rsum);
        } else {
          const int cm = METRIC == kPearson ? c_mode(kEps * rsp[kRowMax] * rmax_c) : kCFirst;
          if (cm == kCFirst)
            sym_tile<METRIC, BN, kCFirst, false>(taddr, rsp, csw, cacc, p0, q0, g.ec, rsum);
          else if (METRIC == kPearson && cm == kCSecond)
            sym_tile<METRIC, BN, kCSecond, false>(taddr, rsp, csw, cacc, p0, q0, g.ec, rsum);
          else
            sym_tile<METRIC, BN, kCExact, false>(taddr, rsp, csw, cacc, p0, q0, g.ec, rsum);
        }
        tc_fence_before();
        // Row sums: 4 lanes per row, then the 4 column-group warps of this
        // quarter through shared memory: the last of them to write its
        // partials adds the four (fixed order) and issues one atomic per row
        // and sum. It releases the accumulator only after reading, so no warp
        // overwrites these partials (two tiles later) before they are read.
        const float2 z = reduce_rows4(rsum);
        const int krow = 2 * (lane & 1) + ((lane >> 1) & 1);
        float2* rp = rowpart + b * (4 * kBM);
        rp[group * kBM + quarter * 32 + (lane >> 2) + 8 * krow] = z;
        __syncwarp();
        unsigned last = 0;
        if (lane == 0) {
          // acquire-release at CTA scope: publishes this warp's partials and,
          // for the fourth warp, makes the other three warps' partials visible
          unsigned prev;
          asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], 1;"
                       : "=r"(prev)
                       : "r"(smem_u32(rowcnt + b * 4 + quarter))
                       : "memory");
          last = (prev & 3u) == 3u;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) {
          __syncwarp();
          const int row = quarter * 32 + lane;
          float sn = 0.0f, sd = 0.0f;
#pragma unroll
          for (int gg = 0; gg < 4; gg++) {
            const float2 v = rp[gg * kBM + row];
            sn += v.x;
            sd += v.y;
          }
          const int p = p0 + row;
          if (p < g.ec.n) {
            atomicAdd(g.num + p, (double)sn);
            atomicAdd(g.den + p, (double)sd);
          }
        }
        __syncwarp();
        if (lane == 0) {
          mbar_arrive(b_acce + 8 * b);
          mbar_arrive(b_rempty + 8 * rsl);
        }
      }
      if (!ok) break;
      // Column sums of the item.
      float x[8 * CH];
#pragma unroll
      for (int c = 0; c < CH; c++) {
        const float4 nv = cacc[(2 * c) * kEpiThreads], dv = cacc[(2 * c + 1) * kEpiThreads];
        const float ns[4] = {nv.x, nv.y, nv.z, nv.w}, ds[4] = {dv.x, dv.y, dv.z, dv.w};
#pragma unroll
        for (int r = 0; r < 2; r++)
#pragma unroll
          for (int lh = 0; lh < 2; lh++) {
            const int i = ((c * 2 + r) * 2 + lh) * 2;
            x[i] = ns[2 * r + lh];
            x[i + 1] = ds[2 * r + lh];
          }
      }
      flush_columns<8 * CH>(x, q0, g.ec, g.num, g.den);
      __syncwarp();
      if (lane == 0) mbar_arrive(b_cempty + 8 * cs);
    }
    };
    pass(std::integral_constant<int, 0>{});
    pass(std::integral_constant<int, 1>{});
    role_exit(tmem, 2 * BN, false);
  }
}

// Column parameters of each BN-column tile, permuted so that thread t of an
// epilogue warp finds its four columns of a 16-column chunk (2(t%4) + {0, 1}
// and 8 + 2(t%4) + {0, 1}) in one float4 (col_soa_pos), with the tile's
// largest 1/sigma; and the row parameters of each 128-row block as the
// epilogue's f32x2 pairs (kRowSoaFloats) with the block's largest 1/sigma.
// Blocks [0, n_ctp): column tiles; [n_ctp, n_ctp + n_rbp): row blocks.
template <int BN>
__global__ void k_sym_soa(const BlockParams* __restrict__ params, int n_ctp, float* __restrict__ colsoa,
                          float* __restrict__ rowsoa) {
  const int i = threadIdx.x;
  __shared__ float wm[8];
  const bool col = blockIdx.x < n_ctp;
  const int width = col ? BN : kBM;
  const int tile = col ? blockIdx.x : blockIdx.x - n_ctp;
  float* o = col ? colsoa + (size_t)tile * col_soa_floats(BN) : rowsoa + (size_t)tile * kRowSoaFloats;
  float r = 0.0f;
  if (i < width) {
    const BlockParams p = params[(size_t)tile * width + i];
    if (col) {
      const int pos = col_soa_pos(i);
      o[pos] = p.a;
      o[width + pos] = p.r;
      o[2 * width + pos] = p.sigma;
      o[3 * width + pos] = p.mu;
    } else {
      const float ne = -kEps * p.r;
      reinterpret_cast<float4*>(o + 8 * i)[0] = make_float4(p.a, p.a, ne, ne);
      reinterpret_cast<float4*>(o + 8 * i)[1] = make_float4(p.sigma, p.sigma, p.mu, p.mu);
      o[kRowR + i] = p.r;
    }
    r = p.r;
  }
  for (int s = 16; s; s >>= 1) r = fmaxf(r, __shfl_xor_sync(0xffffffffu, r, s));
  if ((i & 31) == 0) wm[i >> 5] = r;
  __syncthreads();
  if (i < 4) {
    float m = 0.0f;
    if (i == 0)
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) m = fmaxf(m, wm[w]);
    o[(col ? 4 * width : kRowMax) + i] = m;
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

size_t fixed_smem(int bn) {
  return 1024 + 2 * (size_t)col_soa_floats(bn) * 4 + kRSlots * kRowFloats * 4 + kRowPartBytes +
         (size_t)kEpiThreads * 8 * (bn / 64) * 4 + kBarBytes;
}

}  // namespace

// Launch shape for a column tile width and A mode, if it fits: the whole-tile
// mode needs two A tiles beside the B tile, the chunk ring at least three 16 KB
// A stages (as many as fit, up to kMaxStages).
bool plan_shape(int kq, int bn, bool tr, TcPlan* p) {
  if (kq <= 0 || kq % 32 != 0 || (bn != 256 && bn != 128)) return false;
  const size_t fixed = fixed_smem(bn);
  const size_t a_bytes = (size_t)kBM * kq * 2, b_bytes = (size_t)bn * kq * 2;
  if (tr) {
    if (fixed + 2 * a_bytes + b_bytes > kSmemBudget) return false;
    *p = TcPlan{bn, true, 2, fixed + 2 * a_bytes + b_bytes};
    return true;
  }
  if (fixed + b_bytes + 3 * kAChunkBytes > kSmemBudget) return false;
  const int st = (int)std::min<size_t>(kMaxStages, (kSmemBudget - fixed - b_bytes) / kAChunkBytes);
  *p = TcPlan{bn, false, st, fixed + b_bytes + (size_t)st * kAChunkBytes};
  return true;
}

bool plan_gram_tc(int kq, TcPlan* p) {
  // default: 256-column tiles (whole-tile A when it fits), else 128 (chunk ring)
  return plan_shape(kq, 256, true, p) || plan_shape(kq, 256, false, p) || plan_shape(kq, 128, false, p);
}

int gram_tc_candidates(int kq, TcChoice* out, int cap) {
  int n = 0;
  TcPlan p;
  for (int bn : {256, 128})
    for (int tr : {1, 0})
      if (plan_shape(kq, bn, tr != 0, &p))
        for (int L : {32, 16, 8, 4})
          if (n < cap) out[n++] = TcChoice{bn, tr, L};
  return n;
}

size_t gram_tc_soa_floats(int n_pad) {
  // column tiles of 128 or 256 blocks plus one row-parameter block per 128 rows
  return (size_t)(n_pad / 128) * col_soa_floats(128) + (size_t)(n_pad / 128) * kRowSoaFloats;
}

long long gram_tc_items(int n, int bn, int* L_out, int num_sms, int max_L) {
  const int m = bn / kBM;
  const int n_rb = (n + kBM - 1) / kBM, n_ct = (n + bn - 1) / bn;
  auto items = [&](int L) {
    const int runs = (n_rb + L - 1) / L;
    return items_before_run(runs, n_ct, L / m);
  };
  int L = max_L > 0 && max_L < kMaxRun ? max_L : kMaxRun;
  while (L > 2 && items(L) < 4LL * num_sms) L >>= 1;
  if (L < m) L = m;
  if (L_out) *L_out = L;
  return items(L);
}

cudaError_t launch_gram_tc(const __nv_bfloat16* A, const __nv_bfloat16* B, int kq, int n_pad,
                           const BlockParams* params, float* soa_ws, EpiConsts ec, double* num, double* den,
                           int num_sms, int* status, cudaStream_t st, int shard, int n_shards,
                           const TcDebug* dbg, const TcChoice* choice) {
  TcPlan plan;
  const bool planned = choice && choice->bn ? plan_shape(kq, choice->bn, choice->tr != 0, &plan)
                                            : plan_gram_tc(kq, &plan);
  if (!planned || n_pad % 256 != 0 || n_shards < 1 || shard < 0 || shard >= n_shards) return cudaErrorInvalidValue;
  if (ec.n <= 0) return cudaSuccess;
  const int bn = plan.bn;
  TcArgs g;
  g.kq = kq;
  g.nkc = (kq + kChunk - 1) / kChunk;  // nfull + tail
  g.stages = plan.stages;
  g.nfull = kq / kChunk;
  g.tail = (kq % kChunk) ? 1 : 0;
  g.a_bytes = (uint32_t)kBM * kq * 2;
  g.b_bytes = (uint32_t)bn * kq * 2;
  g.n_rb = (ec.n + kBM - 1) / kBM;
  g.n_ct = (ec.n + bn - 1) / bn;
  int L;
  const long long items = gram_tc_items(ec.n, bn, &L, num_sms, choice ? choice->L : 0);
  g.L = L;
  g.h = L / (bn / kBM);
  g.n_runs = (g.n_rb + L - 1) / L;
  // panels of column tiles whose B tiles (bn x K' bf16 each) fill at most 48 MB of L2
  g.panel = std::max(1, (int)(((size_t)48 << 20) / g.b_bytes));
  g.n_panels = (g.n_ct + g.panel - 1) / g.panel;
  g.item0 = items * shard / n_shards;
  g.item1 = items * (shard + 1) / n_shards;
  const int n_ctp = n_pad / bn, n_rbp = n_pad / kBM;
  float* colsoa = soa_ws;
  float* rowsoa = soa_ws + (size_t)n_ctp * col_soa_floats(bn);
  g.colsoa = colsoa;
  g.rowsoa = rowsoa;
  g.ec = ec;
  g.num = num;
  g.den = den;
  g.status = status;
  g.timeout_ns = dbg && dbg->timeout_ns ? dbg->timeout_ns : 4000000000ull;
  g.withhold = dbg ? dbg->withhold_tile : -1;
  if (bn == 256) k_sym_soa<256><<<n_ctp + n_rbp, 256, 0, st>>>(params, n_ctp, colsoa, rowsoa);
  else k_sym_soa<128><<<n_ctp + n_rbp, 256, 0, st>>>(params, n_ctp, colsoa, rowsoa);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (g.item0 >= g.item1) return cudaSuccess;
  CUtensorMap mA, mB, mA64, mB64;
  if (!make_map(&mA, A, kq, n_pad, kBM) || !make_map(&mB, B, kq, n_pad, bn)) return cudaErrorInvalidValue;
  mA64 = mA;
  mB64 = mB;
  if (g.tail && (!make_map(&mA64, A, kq, n_pad, kBM, kChunk / 2) || !make_map(&mB64, B, kq, n_pad, bn, kChunk / 2)))
    return cudaErrorInvalidValue;
  const int grid = (int)std::min<long long>(g.item1 - g.item0, num_sms);
  const int smem = (int)plan.smem;
#define SRED_TC3(M, BNV, TRV)                                                                            \
  do {                                                                                                   \
    e = cudaFuncSetAttribute(k_gram_tc<M, BNV, TRV>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); \
    if (e != cudaSuccess) return e;                                                                      \
    k_gram_tc<M, BNV, TRV><<<grid, kThreads, smem, st>>>(mA, mB, mA64, mB64, g);                         \
  } while (0)
#define SRED_TC(M)                                   \
  if (bn == 256 && plan.tr) SRED_TC3(M, 256, true);       \
  else if (bn == 256) SRED_TC3(M, 256, false);       \
  else if (plan.tr) SRED_TC3(M, 128, true);          \
  else SRED_TC3(M, 128, false);
  switch (ec.metric) {
    case kPearson: SRED_TC(kPearson); break;
    case kSsim: SRED_TC(kSsim); break;
    case kNrmse: SRED_TC(kNrmse); break;
    case kNrmseW: SRED_TC(kNrmseW); break;
    case kDebugDot: SRED_TC(kDebugDot); break;
    default: return cudaErrorInvalidValue;
  }
#undef SRED_TC
#undef SRED_TC3
  return cudaGetLastError();
}

}  // namespace sred
