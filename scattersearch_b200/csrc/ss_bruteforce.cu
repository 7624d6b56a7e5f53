// Exact k-nearest-neighbour brute force on the tensor cores (tcgen05).
//
// The reference takes its ground truth from external files (load_groundtruth,
// src/util.cpp:72-93); this is the project's own exact k-NN, used for ground
// truth and for graph building.  Three kernels:
//
//   bf_pack_kernel        splits queries and base rows into TF32 hi and lo
//                         parts (x ~ hi + lo to about FP32 accuracy) and
//                         writes them in the 128-byte-swizzled K-major tiles
//                         that the tensor core's shared-memory descriptors
//                         read, so that one bulk copy moves a tile as is.
//   bf_tc_candidates_kernel
//                         128 queries x a split of the base rows per CTA,
//                         warp-specialised: warp 0 streams 32-float k-blocks
//                         of the query tile and of a 256-row base tile into
//                         a two-stage shared-memory ring (cp.async.bulk,
//                         mbarrier completion); one thread of warp 1 issues
//                         tcgen05.mma kind::tf32 in three terms
//                         (lo*hi + hi*lo + hi*hi, FP32 accumulate) into one
//                         of two 128 x 256 TMEM accumulators; warps 2-17 read
//                         the other accumulator with tcgen05.ld (one query
//                         row per thread, a quarter of the columns per
//                         warp) and keep each query's C best
//                         (approximate score, id) in a candidate list, while
//                         the tensor core fills the next tile.
//   bf_rerank_kernel      one warp per query merges the splits' lists, keeps
//                         the C best by approximate score, computes their
//                         distances exactly as the search does (the
//                         reference's FP32 lane model, bit-identical) and
//                         returns the k best by (distance, id).
//
// C exceeds k by a margin of at least 16, so a true neighbour is lost only if
// more than C - k rows score within the three-term TF32 error of it, which
// needs a tie group far larger than the margin; exact ties (e.g. integer-
// valued data, where the three-term products are exact) are ordered by id in
// both passes.
//
// Every wait on an mbarrier is bounded; a wait that runs out sets the error
// word (BruteArgs::err), after which the kernel stops issuing work, waits
// (bounded) for its copies and tensor-core operations in flight, frees its
// TMEM and returns.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <set>
#include <utility>

#include "ss_distance.cuh"
#include "ss_internal.h"

namespace ssb {
namespace {

constexpr int kTM = 128;                 // queries per CTA = accumulator lanes
constexpr int kTN = 256;                 // base rows per tile = accumulator columns
constexpr int kKBlock = 32;              // floats per k-block: one 128-byte row
constexpr int kStages = 2;
constexpr uint32_t kABlock = kTM * 128;  // bytes of one hi (or lo) k-block of queries
constexpr uint32_t kBBlock = kTN * 128;  // bytes of one hi (or lo) k-block of base rows
constexpr uint32_t kStageBytes = 2 * kABlock + 2 * kBBlock;
constexpr int kEpiWarps = 16;                // selection warps: 4 per TMEM lane quadrant
constexpr int kColParts = kEpiWarps / 4;     // column parts of a tile, one list each
constexpr int kTcThreads = 64 + 32 * kEpiWarps;
constexpr uint32_t kTmemCols = 2 * kTN;  // two accumulators
constexpr uint32_t kBarBytes = 8 * (2 * kStages + 5);
constexpr size_t kTcSmem = 1024 + (size_t)kStages * kStageBytes + kBarBytes + 16;
constexpr uint32_t kBfWaitLimit = 1u << 24;

// Instruction descriptor of tcgen05.mma kind::tf32: FP32 accumulator (bits
// 4-5 = 1), A and B TF32 (bits 7-9 and 10-12 = 2), both K-major, N >> 3 at
// bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ uint32_t saddr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of a K-major operand in 128-byte-swizzled
// 8-row atoms (1024 bytes apart): start address >> 4 at bits 0-13, leading
// offset 1 (unused by this layout) at 16-29, stride offset 1024 >> 4 at
// 32-45, descriptor version 1 at 46-47, swizzle mode 2 (128 B) at 61-63.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
// Bounded wait for the phase of parity `parity`; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t spin = 0; spin < kBfWaitLimit; ++spin) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes,
                                          uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
      : "memory");
}
// The mbarrier `bar` receives one arrival once every tensor-core operation
// this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   bar)
               : "memory");
}
// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ uint64_t shfl_u64(uint64_t v, int src) {
  const uint32_t lo = __shfl_sync(kFull, (uint32_t)v, src);
  const uint32_t hi = __shfl_sync(kFull, (uint32_t)(v >> 32), src);
  return ((uint64_t)hi << 32) | lo;
}

// ---------------------------------------------------------------- packing --
// Row `row`, floats [k, k+4) of a matrix packed in tiles of `tile_rows` rows:
// tile t holds, for each k-block, a hi block then a lo block of tile_rows x
// 128 bytes.  Inside a block, rows form 8-row atoms of 1024 bytes, and row r
// of an atom keeps its 16-byte chunk c at chunk position c ^ r.
__global__ void bf_pack_kernel(const float *src, uint32_t rows, uint32_t pitch, uint32_t dim,
                               uint32_t kblocks, uint32_t tile_rows, uint32_t rows_pad,
                               float *dst) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)rows_pad * kblocks * 8) return;
  const uint32_t c = (uint32_t)(i & 7);
  const uint64_t rk = i >> 3;
  const uint32_t kb = (uint32_t)(rk % kblocks);
  const uint32_t row = (uint32_t)(rk / kblocks);
  const uint32_t k = kb * kKBlock + c * 4;
  float x[4] = {0.f, 0.f, 0.f, 0.f};
  if (row < rows) {
    const float *s = src + (size_t)row * pitch;
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (k + e < dim) x[e] = s[k + e];
  }
  float4 h, l;
  float *hp = &h.x, *lp = &l.x;
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const uint32_t hb = to_tf32(x[e]);
    hp[e] = __uint_as_float(hb);
    lp[e] = __uint_as_float(to_tf32(x[e] - __uint_as_float(hb)));
  }
  const uint32_t t = row / tile_rows, r = row % tile_rows;
  const size_t block = ((size_t)t * kblocks + kb) * 2 * (size_t)tile_rows * 32;  // floats
  const size_t off = (size_t)(r >> 3) * 256 + (r & 7) * 32 + ((c ^ (r & 7)) * 4);
  *reinterpret_cast<float4 *>(dst + block + off) = h;
  *reinterpret_cast<float4 *>(dst + block + (size_t)tile_rows * 32 + off) = l;
}

// ------------------------------------------------------------ candidates --
// Sorts a candidate list (cnt used entries) ascending with one warp, writes
// its C best back to the front (kInvalidKey where fewer) and returns the C-th
// key.
template <int CAP, int C>
__device__ __forceinline__ uint64_t compact_list(uint64_t *list, int cnt, int lane) {
  constexpr int IT = CAP / 32;
  uint64_t x[IT];
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    const int e = i * 32 + lane;
    x[i] = e < cnt ? list[e] : kInvalidKey;
  }
  warp_sort<IT>(x, lane);
  __syncwarp();
#pragma unroll
  for (int i = 0; i < C / 32; ++i) list[i * 32 + lane] = x[i];
  __syncwarp();
  return shfl_u64(x[C / 32 - 1], 31);
}

template <int C>
__global__ void __launch_bounds__(kTcThreads, 1) bf_tc_candidates_kernel(BruteArgs a) {
  constexpr int CAP = C + 64 <= 128 ? 128 : 256;
  extern __shared__ unsigned char smem_raw[];
  const uint32_t raw = saddr(smem_raw);
  const uint32_t sbase = (raw + 1023u) & ~1023u;
  unsigned char *gbase = smem_raw + (sbase - raw);
  const uint32_t bar0 = sbase + kStages * kStageBytes;
  uint32_t *slot = reinterpret_cast<uint32_t *>(gbase + kStages * kStageBytes + kBarBytes);
  volatile uint32_t *broken = slot + 1;
  // barriers: full[kStages], empty[kStages], tfull[2], tempty[2], done
  const auto full_bar = [&](uint32_t s) { return bar0 + 8u * s; };
  const auto empty_bar = [&](uint32_t s) { return bar0 + 8u * (kStages + s); };
  const auto tfull_bar = [&](uint32_t b) { return bar0 + 8u * (2 * kStages + b); };
  const auto tempty_bar = [&](uint32_t b) { return bar0 + 8u * (2 * kStages + 2 + b); };
  const uint32_t done_bar = bar0 + 8u * (2 * kStages + 4);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t qt = blockIdx.x, split = blockIdx.y;
  const uint32_t row_lo = split * a.rows_per_split;
  const uint32_t row_hi = min(a.n, row_lo + a.rows_per_split);
  const uint32_t ntiles = row_lo < row_hi ? (row_hi - row_lo + kTN - 1) / kTN : 0;
  const uint32_t KB = a.kblocks;

  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    for (uint32_t b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), kEpiWarps * 32);
    }
    mbar_init(done_bar, 1);
    *broken = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     saddr(slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *slot;

  if (warp == 0) {
    // ---- producer: one thread streams k-blocks of queries and base rows
    if (lane == 0) {
      const unsigned char *qa =
          reinterpret_cast<const unsigned char *>(a.qpack) + (size_t)qt * KB * 2 * kABlock;
      const uint32_t tile0 = row_lo / kTN;
      uint32_t it = 0;
      bool ok = true;
      for (uint32_t t = 0; t < ntiles && ok; ++t) {
        const unsigned char *bt =
            reinterpret_cast<const unsigned char *>(a.bpack) + (size_t)(tile0 + t) * KB * 2 * kBBlock;
        for (uint32_t kb = 0; kb < KB; ++kb, ++it) {
          const uint32_t s = it % kStages, use = it / kStages;
          if (use > 0 && !mbar_wait(empty_bar(s), (use - 1) & 1)) {
            ok = false;
            break;
          }
          const uint32_t dst = sbase + s * kStageBytes;
          mbar_expect_tx(full_bar(s), kStageBytes);
          bulk_load(dst, qa + (size_t)kb * 2 * kABlock, 2 * kABlock, full_bar(s));
          bulk_load(dst + 2 * kABlock, bt + (size_t)kb * 2 * kBBlock, 2 * kBBlock, full_bar(s));
        }
      }
      if (!ok) *broken = 1;
      // every copy issued has landed before the CTA may exit
      for (uint32_t j = it > (uint32_t)kStages ? it - kStages : 0; j < it; ++j)
        if (!mbar_wait(full_bar(j % kStages), (j / kStages) & 1)) *broken = 1;
    }
  } else if (warp == 1) {
    // ---- MMA issuer: one thread
    if (lane == 0) {
      uint32_t it = 0;
      bool ok = true;
      for (uint32_t t = 0; t < ntiles && ok; ++t) {
        const uint32_t b = t & 1, use = t >> 1;
        if (use > 0 && !mbar_wait(tempty_bar(b), (use - 1) & 1)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t d = tmem + b * kTN;
        for (uint32_t kb = 0; kb < KB; ++kb, ++it) {
          const uint32_t s = it % kStages;
          if (!mbar_wait(full_bar(s), (it / kStages) & 1)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = sbase + s * kStageBytes;
#pragma unroll
          for (uint32_t kk = 0; kk < kKBlock / 8; ++kk) {
            const uint32_t off = kk * 32;  // 8 TF32 values per MMA
            const uint64_t ah = sw128_desc(sa + off), al = sw128_desc(sa + kABlock + off);
            const uint64_t bh = sw128_desc(sa + 2 * kABlock + off);
            const uint64_t bl = sw128_desc(sa + 2 * kABlock + kBBlock + off);
            mma_tf32(d, al, bh, (kb | kk) != 0);
            mma_tf32(d, ah, bl, 1);
            mma_tf32(d, ah, bh, 1);
          }
          mma_commit(empty_bar(s));  // stage s is free once these MMAs are done
        }
        if (ok) mma_commit(tfull_bar(b));  // accumulator b is complete
      }
      if (!ok) *broken = 1;
      // no tensor-core operation may still run when TMEM is freed
      mma_commit(done_bar);
      if (!mbar_wait(done_bar, 0)) *broken = 1;
    }
  } else {
    // ---- selection: 16 warps; warp w reads TMEM lanes 32*(w%4).. (its
    // queries) and part (w-2)/4 of each tile's columns
    const int quad = warp & 3, half = (warp - 2) >> 2;  // half: the column part
    const uint32_t row = quad * 32 + lane;
    const uint32_t q = qt * kTM + row;
    const bool qv = q < a.nq;
    uint64_t *list =
        a.cand + ((size_t)(qv ? q : 0) * a.lists + split * kColParts + half) *
                     (size_t)a.list_stride;
    uint64_t thr = kInvalidKey;
    float thr_f = __int_as_float(0x7f800000);  // +inf
    int cnt = 0;
    const uint32_t lane_base = (uint32_t)(quad * 32) << 16;
    bool ok = true;
    for (uint32_t t = 0; t < ntiles; ++t) {
      const uint32_t b = t & 1;
      ok = __all_sync(kFull, mbar_wait(tfull_bar(b), (t >> 1) & 1));
      if (!ok) break;
      tc_fence_after();
      const uint32_t taddr = tmem + lane_base + b * kTN + half * (kTN / kColParts);
      const uint32_t cbase = row_lo + t * kTN + half * (kTN / kColParts);
#pragma unroll 1
      for (int ch = 0; ch < kTN / kColParts / 32; ++ch) {
        uint32_t r[32];
        tmem_ld32(taddr + ch * 32, r);
        tmem_wait_ld();
        if (ch == kTN / kColParts / 32 - 1) {  // this thread's last read of accumulator b
          tc_fence_before();
          mbar_arrive(tempty_bar(b));
        }
        const uint32_t c0 = cbase + ch * 32;
        float xn = 0.f;
        if (a.metric == 0 && c0 + lane < row_hi) xn = __ldg(a.xnorm + c0 + lane);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const float acc = __uint_as_float(r[j]);
          // inner product -> -dot; L2 -> |x|^2 - 2 dot (the query's norm is
          // the same for every row and does not change the ranking)
          const float sc = a.metric == 0 ? __fsub_rn(__shfl_sync(kFull, xn, j), __fmul_rn(2.f, acc))
                                         : -acc;
          const uint32_t id = c0 + j;
          if (sc <= thr_f && id < row_hi && qv) {
            const uint64_t key = ((uint64_t)float_to_key(sc) << 32) | id;
            if (key < thr) list[cnt++] = key;
          }
        }
        __syncwarp();
        unsigned need = __ballot_sync(kFull, cnt > CAP - 32);
        while (need) {
          const int l = __ffs(need) - 1;
          need &= need - 1;
          uint64_t *lp = reinterpret_cast<uint64_t *>(
              shfl_u64(reinterpret_cast<uint64_t>(list), l));
          const int lc = __shfl_sync(kFull, cnt, l);
          const uint64_t nt = compact_list<CAP, C>(lp, lc, lane);
          if (lane == l) {
            cnt = C;
            thr = nt;
            thr_f = key_to_float((uint32_t)(nt >> 32));
          }
        }
      }
    }
    if (!ok) {
      *broken = 1;
    } else {
      // each query's C best of this split's column part, sorted, at the list front
      unsigned have = __ballot_sync(kFull, qv);
      while (have) {
        const int l = __ffs(have) - 1;
        have &= have - 1;
        uint64_t *lp =
            reinterpret_cast<uint64_t *>(shfl_u64(reinterpret_cast<uint64_t>(list), l));
        compact_list<CAP, C>(lp, __shfl_sync(kFull, cnt, l), lane);
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
  if (threadIdx.x == 0 && *broken && a.err) atomicExch(a.err, 1u);
}

// One warp per query: merge the splits' candidates, re-rank the C best with
// exact distances, write the k best.
template <int C, int SC>
__global__ void __launch_bounds__(128) bf_rerank_kernel(BruteArgs a, GraphView g) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t q = blockIdx.x * 4 + warp;
  const int pitch = (int)a.nb * 8;
  float *qs = reinterpret_cast<float *>(smem_raw) + warp * pitch;
  uint32_t *cid = reinterpret_cast<uint32_t *>(reinterpret_cast<float *>(smem_raw) + 4 * pitch) +
                  warp * 2 * C;
  uint32_t *ckey = cid + C;
  if (q >= a.nq) return;
  for (int i = lane; i < pitch; i += 32) qs[i] = a.queries[(size_t)q * pitch + i];
  // merge by approximate score
  constexpr int IT = SC / 32;
  uint64_t x[IT];
  const uint64_t *src = a.cand + (size_t)q * a.lists * a.list_stride;
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    const int e = i * 32 + lane;
    x[i] = e < (int)(a.lists * C) ? src[(size_t)(e / C) * a.list_stride + (e % C)] : kInvalidKey;
  }
  warp_sort<IT>(x, lane);
  // the C best (first C/32 items) -> ids
  int nvalid = 0;
#pragma unroll
  for (int i = 0; i < C / 32; ++i) {
    const bool v = x[i] != kInvalidKey;
    cid[i * 32 + lane] = v ? (uint32_t)x[i] : 0u;
    nvalid += __popc(__ballot_sync(kFull, v));
  }
  __syncwarp();
  eval_candidates<0>(g, qs, cid, ckey, nvalid, lane);
  __syncwarp();
  constexpr int IC = C / 32;
  uint64_t y[IC];
#pragma unroll
  for (int i = 0; i < IC; ++i) {
    const int e = i * 32 + lane;
    y[i] = e < nvalid ? (((uint64_t)ckey[e] << 32) | cid[e]) : kInvalidKey;
  }
  warp_sort<IC>(y, lane);
#pragma unroll
  for (int i = 0; i < IC; ++i) {
    const int e = i * 32 + lane;
    if (e < a.k) {
      const bool v = y[i] != kInvalidKey;
      a.ids[(size_t)q * a.k + e] = v ? (uint32_t)y[i] : kNoneId;
      if (a.dists) a.dists[(size_t)q * a.k + e] = v ? key_to_float((uint32_t)(y[i] >> 32)) : 0.f;
    }
  }
}

// |x|^2 of every base row in FP32 (used only to rank candidates for L2).
__global__ void bf_norms_kernel(const float *base, uint32_t n, uint32_t pitch, float *out) {
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const float *r = base + (size_t)warp * pitch;
  float s = 0.f;
  for (uint32_t i = lane; i < pitch; i += 32) s = fmaf(r[i], r[i], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
  if (lane == 0) out[warp] = s;
}

// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum, once per (device, kernel).  One fixed value for every launch: a
// per-launch size set from several host threads could race with another
// thread's launch of the same kernel.
cudaError_t allow_max_smem_bf(const void *fn) {
  static std::mutex mu;
  static std::set<std::pair<int, const void *>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({dev, fn})) return cudaSuccess;
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  if (e == cudaSuccess) done.insert({dev, fn});
  return e;
}

template <int C>
cudaError_t launch_candidates(const BruteArgs &a, cudaStream_t s) {
  static_assert(kTcSmem <= 227 * 1024, "candidate kernel exceeds shared memory");
  cudaError_t e = allow_max_smem_bf((const void *)bf_tc_candidates_kernel<C>);
  if (e != cudaSuccess) return e;
  dim3 grid((a.nq + kTM - 1) / kTM, a.splits);
  bf_tc_candidates_kernel<C><<<grid, kTcThreads, kTcSmem, s>>>(a);
  return cudaGetLastError();
}

template <int C, int SC>
cudaError_t launch_rerank(const BruteArgs &a, const GraphView &g, cudaStream_t s) {
  const size_t smem = (size_t)4 * a.nb * 8 * 4 + (size_t)4 * 2 * C * 4;
  cudaError_t e = allow_max_smem_bf((const void *)bf_rerank_kernel<C, SC>);
  if (e != cudaSuccess) return e;
  bf_rerank_kernel<C, SC><<<(a.nq + 3) / 4, 128, smem, s>>>(a, g);
  return cudaGetLastError();
}

template <int C>
cudaError_t launch_rerank_c(const BruteArgs &a, const GraphView &g, cudaStream_t s) {
  switch (a.lists * C) {
    case 64: return launch_rerank<C, 64>(a, g, s);
    case 128: return launch_rerank<C, 128>(a, g, s);
    case 256: return launch_rerank<C, 256>(a, g, s);
    case 512: return launch_rerank<C, 512>(a, g, s);
    case 1024: return launch_rerank<C, 1024>(a, g, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

BrutePlan plan_bruteforce(uint32_t n, uint32_t nq, int k, int sm_count) {
  BrutePlan p{};
  p.C = k + 16 <= 32 ? 32 : (k + 16 <= 64 ? 64 : 128);
  p.list_cap = p.C + 64 <= 128 ? 128 : 256;
  const uint32_t tiles = (nq + kTM - 1) / kTM;
  // kColParts lists per split (one per column part); at most 1024 candidates
  // to merge
  const uint32_t max_splits = 1024u / kColParts / (uint32_t)p.C;
  uint32_t splits = 1;
  while (splits < max_splits && tiles * splits < 4u * (uint32_t)sm_count) splits <<= 1;
  // never more splits than 256-row tiles of the base
  while (splits > 1 && (uint64_t)splits * kTN > n) splits >>= 1;
  p.splits = splits;
  p.lists = kColParts * splits;
  uint32_t rps = (n + splits - 1) / splits;
  p.rows_per_split = (rps + kTN - 1) / kTN * kTN;
  p.kblocks = 0;
  return p;
}

uint32_t bruteforce_kblocks(uint32_t dim) { return (dim + kKBlock - 1) / kKBlock; }
size_t bruteforce_pack_bytes(uint32_t rows, uint32_t dim, bool base_side) {
  const uint32_t tr = base_side ? kTN : kTM;
  const size_t rows_pad = ((size_t)rows + tr - 1) / tr * tr;
  return rows_pad * bruteforce_kblocks(dim) * kKBlock * 2 * 4;
}

cudaError_t launch_pack(const float *src, uint32_t rows, uint32_t pitch, uint32_t dim,
                        bool base_side, float *dst, cudaStream_t s) {
  if (rows == 0) return cudaSuccess;
  const uint32_t tr = base_side ? kTN : kTM;
  const uint32_t rows_pad = (rows + tr - 1) / tr * tr;
  const uint32_t kb = bruteforce_kblocks(dim);
  const uint64_t chunks = (uint64_t)rows_pad * kb * 8;
  const uint32_t blocks = (uint32_t)((chunks + 255) / 256);
  bf_pack_kernel<<<blocks, 256, 0, s>>>(src, rows, pitch, dim, kb, tr, rows_pad, dst);
  return cudaGetLastError();
}

cudaError_t launch_norms(const float *base, uint32_t n, uint32_t pitch, float *out,
                         cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  const uint32_t blocks = (uint32_t)(((uint64_t)n * 32 + 255) / 256);
  bf_norms_kernel<<<blocks, 256, 0, s>>>(base, n, pitch, out);
  return cudaGetLastError();
}

cudaError_t launch_bruteforce(const BruteArgs &a, const GraphView &g, cudaStream_t s) {
  if (a.nq == 0) return cudaSuccess;
  cudaError_t e;
  switch (a.C) {
    case 32: e = launch_candidates<32>(a, s); break;
    case 64: e = launch_candidates<64>(a, s); break;
    case 128: e = launch_candidates<128>(a, s); break;
    default: return cudaErrorInvalidValue;
  }
  if (e != cudaSuccess) return e;
  switch (a.C) {
    case 32: return launch_rerank_c<32>(a, g, s);
    case 64: return launch_rerank_c<64>(a, g, s);
    default: return launch_rerank_c<128>(a, g, s);
  }
}

}  // namespace ssb
