// Graph beam-search kernels for sm_100a.
//
// Semantics follow ANNSearch::SearchArraySimulation (src/annsearch.cpp:182-259)
// in its equivalent batch-merge form; see the per-function comments for the
// exact rules and their reference lines.  The arithmetic of every distance is
// the reference's AVX model (src/distance.cpp:19-56, :115-149): 8 lane
// partials, the odd 8-block first when the padded dimension is 8 mod 16, one
// rounding per subtract, multiply and add (no FMA), lanes summed left to
// right.  That makes the GPU results bit-identical to the reference built
// without fast-math.
//
// Three kernels:
//   warp_search_kernel   one warp owns one query (pool, visited hash and
//                        candidate buffers in shared memory); a CTA holds
//                        several independent query teams; teams pull queries
//                        from a device work counter until the batch is empty
//                        (persistent) or take them by index (static).  Base
//                        rows reach each team through a row stage filled by
//                        the tensor-memory-access engine: four rows per
//                        gather4 copy when a row has at most 256 floats, one
//                        bulk copy per row otherwise; the stage is a team's
//                        own, or one taken from a pool the CTA's teams
//                        share.  Stages deeper than 16
//                        rows (one copy round trip per hop) are a separate
//                        instantiation (DEEP), used for launches small
//                        enough to keep every query resident.
//   intra_search_kernel  one CTA owns one query; each step expands the W best
//                        unexplored entries at once, one per warp.
//   scatter_search_kernel  ScatterSearch's own intra-query search: one CTA
//                        per query, a pool per warp from its own entry point,
//                        one shared visited set, optional election and early
//                        termination.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <set>
#include <utility>

#include "scattersearch.h"
#include "ss_distance.cuh"
#include "ss_internal.h"

namespace ssb {
namespace {

constexpr uint32_t kExplored = 0x80000000u;
// Most rows staged in shared memory per pass of the warp kernel (one per
// lane pair), and the iteration limit of a wait for them (a stage load takes
// microseconds; the limit is far above that and only ends a wait that would
// never finish).
constexpr int kStageRows = 16;
// Deepest whole-row stage: a hop has at most 32 fresh candidates (degree
// <= 32 with one adjacency chunk), so a 32-row stage takes every row of a
// hop in one copy round trip; its rows are computed in groups of 16.
constexpr int kMaxStageRows = 32;
constexpr uint32_t kStageWaitLimit = 1u << 24;

// Number of a[0..n) with a[i] <= key (a ascending).
__device__ __forceinline__ int count_le(const uint32_t *a, int n, uint32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= key) lo = mid + 1; else hi = mid;
  }
  return lo;
}
// Number of a[0..n) with a[i] < key (a ascending).
__device__ __forceinline__ int count_lt(const uint32_t *a, int n, uint32_t key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// --------------------------------------------------------- visited set ---
// Exact visited set: open-addressing hash of ids in shared memory (linear
// probing).  When it reaches `limit` entries, further ids go to a per-team
// bitset in global memory (n bits), so nothing is ever forgotten; lookups
// then check both.  The bitset is cleared again before the team's next query.
struct Visited {
  uint32_t *tab;
  uint32_t mask, log2cap, limit, count;
  uint32_t *bits;  // global, may be null when spilling is impossible
  bool spilled;
};

__device__ __forceinline__ uint32_t hash_slot(uint32_t id, uint32_t log2cap) {
  return (id * 0x9E3779B1u) >> (32 - log2cap);
}

// Inserts `id`; true if it was not present.  Distinct lanes may race on the
// same id: the atomicCAS lets exactly one of them see it as new.
__device__ __forceinline__ bool hash_insert(uint32_t *tab, uint32_t mask, uint32_t log2cap,
                                            uint32_t id) {
  uint32_t s = hash_slot(id, log2cap);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t cur = tab[s];
    if (cur == id) return false;
    if (cur == kNoneId) {
      const uint32_t old = atomicCAS(&tab[s], kNoneId, id);
      if (old == kNoneId) return true;
      if (old == id) return false;
    }
    s = (s + 1) & mask;
  }
  return false;  // unreachable: the table never fills past `limit`
}

__device__ __forceinline__ bool hash_contains(const uint32_t *tab, uint32_t mask, uint32_t log2cap,
                                              uint32_t id) {
  uint32_t s = hash_slot(id, log2cap);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t cur = tab[s];
    if (cur == id) return true;
    if (cur == kNoneId) return false;
    s = (s + 1) & mask;
  }
  return false;
}

// Marks `id` visited; true if it was new.
__device__ __forceinline__ bool visit(Visited &v, uint32_t id) {
  if (!v.spilled) return hash_insert(v.tab, v.mask, v.log2cap, id);
  if (hash_contains(v.tab, v.mask, v.log2cap, id)) return false;
  const uint32_t bit = 1u << (id & 31u);
  return (atomicOr(v.bits + (id >> 5), bit) & bit) == 0u;
}

// Read-only membership test.
__device__ __forceinline__ bool visited_test(const Visited &v, uint32_t id) {
  if (hash_contains(v.tab, v.mask, v.log2cap, id)) return true;
  if (!v.spilled) return false;
  const uint32_t bit = 1u << (id & 31u);
  return (*(volatile uint32_t *)(v.bits + (id >> 5)) & bit) != 0u;
}

// ------------------------------------------------------- warp per query ---
// Visited set of the warp kernel: a two-choice bucketed hash in shared memory
// that may forget ids but never reports an unvisited id as visited.  Bucket =
// 8 slots of 16 bits (one 16-byte row, read with a single LDS.128).  An id is
// mixed by two multiplications with odd constants modulo 2^B (2^B >= n);
// each product is a bijection of [0, 2^B), so its high bits (the bucket) plus
// its low bits (the 16-bit tag) identify the id exactly.  Tags of the second
// choice carry bit 15, so a tag names both the id and the choice; 0xFFFF
// marks an empty slot.  When both buckets of an id are full, a slot of the
// first bucket chosen by the id is overwritten: the evicted id is forgotten.
//
// Forgetting does not change results.  The acceptance threshold
// pool[size-1] never increases during a search (accepted candidates are
// below it, and truncation to L only lowers it).  A forgotten id that is met
// again is evaluated again, to the same distance bits, and then either
//   - it is in the pool: the pool holds it under exactly that key, so the
//     acceptance step finds it in the key's run and drops it; or
//   - it is not: it was rejected (distance >= the threshold then) or pushed
//     out by L entries at or below its distance, so its distance is >= the
//     current threshold and it is rejected again.
// So a forgetful table only costs extra distance evaluations, and the pool
// check runs only after the first eviction of a query (`lossy`).
struct QHash {
  uint4 *bkt;
  uint32_t *evb;  // bit per bucket: the bucket has evicted an id this query
  uint32_t rbits, rmask, bmask;
  bool lossy;  // an id was evicted (or not recorded) during this query
};

// Words of the per-bucket eviction bits of a table of 2^bbits buckets.
__host__ __device__ __forceinline__ uint32_t evict_words(uint32_t bbits) {
  return bbits >= 5 ? (1u << (bbits - 5)) : 1u;
}

// True when a bucket of the probe has evicted an id this query: only then
// can an id the table does not hold have been visited.  An id is recorded
// in one of its two buckets (into an empty slot, or over an evicted one,
// which sets that bucket's bit), and leaves the table only by eviction.
__device__ __forceinline__ bool probe_lossy(const QHash &h, uint32_t b1, uint32_t b2) {
  return ((h.evb[b1 >> 5] >> (b1 & 31u)) | (h.evb[b2 >> 5] >> (b2 & 31u))) & 1u;
}

constexpr uint32_t kMix1 = 0x9E3779B1u;
constexpr uint32_t kMix2 = 0x7FEB352Du;
constexpr uint32_t kMix3 = 0x2C1B3C6Du;

__device__ __forceinline__ void qh_keys(const QHash &h, uint32_t id, uint32_t &b1, uint32_t &t1,
                                        uint32_t &b2, uint32_t &t2) {
  const uint32_t f1 = (id * kMix1) & h.bmask;
  const uint32_t f2 = (id * kMix2) & h.bmask;
  b1 = f1 >> h.rbits;
  t1 = f1 & h.rmask;
  b2 = f2 >> h.rbits;
  t2 = (f2 & h.rmask) | 0x8000u;
}

// Nonzero iff one of the two 16-bit halves of x is zero: x - 1 per half sets
// bit 15 of a half and leaves it clear in ~x only when that half is zero,
// and a borrow into the upper half only comes from a zero lower half.
__device__ __forceinline__ uint32_t has_zero_half(uint32_t x) {
  return (x - 0x00010001u) & ~x & 0x80008000u;
}

__device__ __forceinline__ bool bucket_has(uint4 v, uint32_t t) {
  const uint32_t tt = t | (t << 16);
  return (has_zero_half(v.x ^ tt) | has_zero_half(v.y ^ tt) | has_zero_half(v.z ^ tt) |
          has_zero_half(v.w ^ tt)) != 0u;
}

// 8-bit mask of the empty slots of a bucket: bit p stands for slot p ^ 6
// (slot s = 16-bit half s of the bucket).  A tag holds at most 14 remainder
// bits and the choice flag in bit 15, so bit 14 is set only in the empty
// marker 0xFFFF; the four words' bit-14/30 flags are shifted into one byte.
__device__ __forceinline__ uint32_t bucket_empty(uint4 v) {
  const uint32_t m = (v.x & 0x40004000u) | ((v.y & 0x40004000u) >> 2) |
                     ((v.z & 0x40004000u) >> 4) | ((v.w & 0x40004000u) >> 6);
  return ((m >> 8) & 0x55u) | ((m >> 23) & 0xAAu);
}

// Slot of the (r+1)-th empty slot in an empty mask from bucket_empty.
__device__ __forceinline__ uint32_t nth_empty_slot(uint32_t e, int r) {
  for (int i = 0; i < r; ++i) e &= e - 1u;
  return (uint32_t)(__ffs(e) - 1) ^ 6u;
}

// 16-byte shared-memory load that is never cached in registers or reordered
// across other shared-memory accesses (buckets change under concurrent CAS).
__device__ __forceinline__ uint4 lds128(const uint4 *p) {
  uint4 v;
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "r"(a)
               : "memory");
  return v;
}

// One lane's probe of the table: both candidate buckets of an id as they
// were read, and the id's tags in them.
struct QProbe {
  uint32_t b1, t1, b2, t2;
  uint4 v1, v2;
};

// Read-only lookup; true when `id` is in the table.
__device__ __forceinline__ bool qh_lookup(const QHash &h, uint32_t id, QProbe &pr) {
  qh_keys(h, id, pr.b1, pr.t1, pr.b2, pr.t2);
  pr.v1 = lds128(h.bkt + pr.b1);
  pr.v2 = lds128(h.bkt + pr.b2);
  return bucket_has(pr.v1, pr.t1) || bucket_has(pr.v2, pr.t2);
}

// Records the ids of the `ins` lanes (distinct ids, none found by their
// qh_lookup, whose bucket reads are still current).  Each id goes to the
// emptier of its two buckets; lanes that picked the same bucket take its
// empty slots in lane order, and a lane left without one overwrites a slot
// chosen by its id, so the table forgets an id.  Plain 16-bit stores, no
// atomics.  All 32 lanes call it.
__device__ __forceinline__ void qh_record(QHash &h, const QProbe &pr, uint32_t id, bool ins,
                                          int lane) {
  const uint32_t e1 = bucket_empty(pr.v1), e2 = bucket_empty(pr.v2);
  const bool use1 = __popc(e1) >= __popc(e2);
  const uint32_t b = use1 ? pr.b1 : pr.b2, t = use1 ? pr.t1 : pr.t2, e = use1 ? e1 : e2;
  const unsigned grp = __match_any_sync(kFull, ins ? b : (0x80000000u | (uint32_t)lane));
  const int r = __popc(grp & ((1u << lane) - 1u));
  unsigned short *slots = reinterpret_cast<unsigned short *>(h.bkt);
  bool ev = false;
  if (ins) {
    uint32_t sl;
    if (r < __popc(e)) {
      sl = nth_empty_slot(e, r);
    } else {
      sl = (id * kMix3) >> 29;
      ev = true;
      atomicOr(h.evb + (b >> 5), 1u << (b & 31u));
    }
    slots[b * 8 + sl] = (unsigned short)t;
  }
  if (__any_sync(kFull, ev)) h.lossy = true;
}

// Starts an L2 prefetch of the base rows of cid[0..nc), one 128-byte line
// per lane and instruction (a row starts on a 32-byte boundary, so it spans
// bytes/128 + 1 lines at most), so later copy passes find their rows in L2.
// Plain per-line prefetches: a bulk prefetch per row was measured to cost
// about 100 cycles of issue each, over 1,000 cycles a hop.
__device__ __forceinline__ void prefetch_rows(const GraphView &g, const uint32_t *cid, int nc,
                                              int lane) {
  const uint32_t bytes = g.nb * 32u;
  const uint32_t lines = bytes / 128u + 1u;
  const uint32_t total = (uint32_t)nc * lines;
  for (uint32_t j = lane; j < total; j += 32) {
    const uint32_t r = j / lines, l = j - r * lines;
    const char *row = reinterpret_cast<const char *>(g.base + (size_t)cid[r] * (size_t)(g.nb * 8));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(row + min(l * 128u, bytes - 1u)) : "memory");
  }
}

// Starts an L2 prefetch of the base rows of cid[0..nc) through the row map,
// four rows per gather4 prefetch (group j = rows 4j..4j+3, taken by lane
// j mod 32; a short last group repeats its first row).  One instruction per
// four rows, against about 77 line prefetches for 11 rows of 800 bytes.
__device__ __forceinline__ void prefetch_rows_gather(const CUtensorMap *rows, const uint32_t *cid,
                                                     int nc, int lane) {
  const int groups = (nc + 3) >> 2;
  for (int j = lane; j < groups; j += 32) {
    const int r = 4 * j;
    const uint32_t i0 = cid[r];
    const uint32_t i1 = r + 1 < nc ? cid[r + 1] : i0;
    const uint32_t i2 = r + 2 < nc ? cid[r + 2] : i0;
    const uint32_t i3 = r + 3 < nc ? cid[r + 3] : i0;
    asm volatile(
        "cp.async.bulk.prefetch.tensor.2d.L2.global.tile::gather4 [%0, {%1, %2, %3, %4, %5}];" ::"l"(
            rows),
        "r"(0), "r"(i0), "r"(i1), "r"(i2), "r"(i3)
        : "memory");
  }
}

// Branch-free binary searches over ascending arrays (warp-uniform trip
// counts, so lanes never diverge).  `top` = largest power of two <= n.
__device__ __forceinline__ int count_le_bf(const uint32_t *a, int n, int top, uint32_t key) {
  int pos = 0;
  for (int step = top; step > 0; step >>= 1) {
    const int np = pos + step;
    const uint32_t v = a[min(np, n) - 1];
    pos = (np <= n && v <= key) ? np : pos;
  }
  return pos;
}

__device__ __forceinline__ int floor_pow2(int n) { return n > 0 ? 1 << (31 - __clz(n)) : 0; }

// Per-team shared memory of the warp kernel.  The row stage comes first so
// that it starts on a 128-byte boundary (every team's region is a multiple of
// 128 bytes).
struct WarpSmem {
  float *stage;                    // stage_rows base rows (nb*8 floats each), filled by TMA
  uint64_t *bar;                   // mbarrier of the stage
  float *q;
  uint32_t *pk, *pid;              // pool keys / ids (bit 31 of id = explored)
  uint32_t *cid, *ckey;            // this hop's fresh candidates, adjacency order
  uint32_t *ak, *aid, *acle;       // accepted candidates (key, id, pool rank), adjacency order
  uint4 *bkt;                      // visited hash buckets
  uint32_t *evb;                   // per-bucket eviction bits (evict_words)
};

__device__ __forceinline__ WarpSmem carve_warp(uint32_t *base, const SmemPlan &p) {
  WarpSmem s;
  if (p.shared_stages == 0) {
    s.stage = reinterpret_cast<float *>(base);
    base += p.stage_words;
    s.bar = reinterpret_cast<uint64_t *>(base);
    base += 4;
  } else {  // the CTA's stage pool holds the stages and their mbarriers
    s.stage = nullptr;
    s.bar = nullptr;
  }
  s.q = reinterpret_cast<float *>(base);
  base += p.q_words;
  s.pk = base;
  base += p.pool_cap;
  s.pid = base;
  base += p.pool_cap;
  uint32_t **bufs[5] = {&s.cid, &s.ckey, &s.ak, &s.aid, &s.acle};
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    *bufs[i] = base;
    base += p.cand_cap;
  }
  s.bkt = reinterpret_cast<uint4 *>(base);
  s.evb = base + (1u << p.hash_log2) * 4;
  return s;
}

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Bounded wait for phase `parity` of a shared-memory mbarrier; false when the
// iteration limit ran out first.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (uint32_t spin = 0; spin < kStageWaitLimit; ++spin) {
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

// Row stage of one team: base rows are copied whole into shared memory by
// the tensor-memory-access (TMA) engine, completing on the team's mbarrier.
// A row requested as one 16-byte-aligned block reaches DRAM as one burst per
// row, which a random gather needs to approach the HBM copy rate; rows read
// by many lanes a sector at a time do not.  With a row map (rows of at most
// 256 floats), one cp.async.bulk.tensor ... tile::gather4 copies four rows,
// named by their indices, into four consecutive stage rows; otherwise one
// cp.async.bulk copies each row.  Issuing a copy costs the team's warp about
// 60-110 cycles per instruction, so four rows per instruction cut the issue
// time of a 12-row pass from about 760 to 320 cycles (measured, 8 teams per
// SM).
struct RowStage {
  uint32_t bar;     // shared address of the mbarrier
  uint32_t phase;   // parity of the phase being filled
  bool broken;      // a wait timed out: the stage may still be written to
  float *buf;       // the stage's rows
  int slot;         // pool slot held (shared stages), -1 when none
  const CUtensorMap *rows;  // 2-D map of the base rows (gather4 copies), or null
};

// Stage pool of a CTA whose teams share row stages (SmemPlan::shared_stages
// > 0): `count` stages, each with its mbarrier and the parity of its next
// phase, and a bit mask of free stages.  A team takes a stage just before it
// starts copying rows and gives it back once the distances of its last pass
// are computed, so a stage is held only over copy latency and distance
// arithmetic and the CTA needs fewer stages than teams.
struct StagePool {
  float *stages;      // count x stage_words floats
  uint32_t bar0;      // shared address of the first mbarrier (8 bytes apart)
  uint32_t *phases;   // count words
  uint32_t *mask;     // bit i set = stage i free
  uint32_t count, stage_words;
};

// Words of the CTA-wide stage pool region (0 with private stages).
__host__ __device__ __forceinline__ uint32_t stage_pool_words(const SmemPlan &p) {
  if (p.shared_stages == 0) return 0;
  const uint32_t w = p.shared_stages * p.stage_words + 2 * p.shared_stages + p.shared_stages + 1;
  return (w + 31u) & ~31u;
}

__device__ __forceinline__ StagePool carve_pool(uint32_t *base, const SmemPlan &p) {
  StagePool sp;
  sp.count = p.shared_stages;
  sp.stage_words = p.stage_words;
  sp.stages = reinterpret_cast<float *>(base);
  uint32_t *b = base + p.shared_stages * p.stage_words;  // 8-byte aligned (stage_words % 32 == 0)
  sp.bar0 = (uint32_t)__cvta_generic_to_shared(b);
  sp.phases = b + 2 * p.shared_stages;
  sp.mask = sp.phases + p.shared_stages;
  return sp;
}

// Takes a free stage of the pool for this team (no-op with a private stage
// or when one is held).  Lane 0 claims a free bit with compare-and-swap,
// spinning (bounded) while every stage is in use.  False when the limit ran
// out; the team then holds nothing.
__device__ __forceinline__ bool stage_acquire(RowStage &st, const StagePool &sp, int lane) {
  if (sp.count == 0 || st.slot >= 0) return true;
  int got = -1;
  uint32_t phase = 0;
  if (lane == 0) {
    volatile uint32_t *vm = sp.mask;
    for (uint32_t spin = 0; spin < kStageWaitLimit && got < 0; ++spin) {
      const uint32_t m = *vm;
      if (m == 0u) {
        __nanosleep(32);
        continue;
      }
      const int i = __ffs(m) - 1;
      if (atomicCAS(sp.mask, m, m & ~(1u << i)) == m) got = i;
    }
    if (got >= 0) {
      __threadfence_block();
      phase = *(volatile uint32_t *)(sp.phases + got);
    }
  }
  got = __shfl_sync(kFull, got, 0);
  phase = __shfl_sync(kFull, phase, 0);
  if (got < 0) return false;
  st.slot = got;
  st.buf = sp.stages + (size_t)got * sp.stage_words;
  st.bar = sp.bar0 + 8u * (uint32_t)got;
  st.phase = phase;
  return true;
}

// Gives a pool stage back once its copies have landed and its rows are
// read (no-op with a private stage).
__device__ __forceinline__ void stage_release(RowStage &st, const StagePool &sp, int lane) {
  if (sp.count == 0 || st.slot < 0) return;
  __syncwarp();
  if (lane == 0) {
    // this team's reads of the stage come before any later copy into it
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    *(volatile uint32_t *)(sp.phases + st.slot) = st.phase;
    __threadfence_block();
    atomicOr(sp.mask, 1u << st.slot);
  }
  st.slot = -1;
}

// Blocks (8 floats each) of the first half-row of a split stage: the odd
// tail block (processed first, distance.cpp:42-45) plus the leading blocks.
__host__ __device__ __forceinline__ uint32_t split_first(uint32_t nb) { return (nb + 1) / 2; }

// Starts copying part `part` of the base rows of cid[0..m) (m <= the stage's
// rows) into the stage: part 2 is the whole row (memory order); with a split
// stage, part 0 is the first half of the blocks in processing order (the odd
// tail block, then blocks 0, 1, ...) and part 1 the rest.  All 32 lanes call
// it; cid must be visible to every lane.
__device__ __forceinline__ void stage_issue(const GraphView &g, const WarpSmem &s, const RowStage &st,
                                            const uint32_t *cid, int m, int part, uint32_t row_words,
                                            int lane) {
  const uint32_t nb = g.nb, A = split_first(nb);
  const bool odd = nb & 1u;
  uint32_t bytes, src_block, dst_block = 0, nblocks;
  if (part == 2) {
    nblocks = nb;
    src_block = 0;
  } else if (part == 0) {
    nblocks = odd ? A - 1 : A;
    src_block = 0;
    dst_block = odd ? 1 : 0;
  } else {
    nblocks = nb - A;
    src_block = odd ? A - 1 : A;
  }
  bytes = (nblocks + (part == 0 && odd ? 1u : 0u)) * 32u;
  // earlier reads of the stage (generic proxy) come before the copies that
  // overwrite it (async proxy)
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (part == 2 && st.rows != nullptr) {
    // gather4: lane l copies rows 4l..4l+3 into stage rows 4l..4l+3; a group
    // past row m-1 repeats its first row (the stage holds a multiple of 4
    // rows, and a repeated row is an L2 hit)
    const int groups = (m + 3) >> 2;
    if (lane == 0)
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(st.bar),
                   "r"(bytes * 4u * (uint32_t)groups)
                   : "memory");
    __syncwarp();
    if (lane < groups) {
      const int r = 4 * lane;
      const uint32_t i0 = cid[r];
      const uint32_t i1 = r + 1 < m ? cid[r + 1] : i0;
      const uint32_t i2 = r + 2 < m ? cid[r + 2] : i0;
      const uint32_t i3 = r + 3 < m ? cid[r + 3] : i0;
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
          " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(st.buf + r * row_words)),
          "l"(st.rows), "r"(0), "r"(i0), "r"(i1), "r"(i2), "r"(i3), "r"(st.bar)
          : "memory");
    }
    return;
  }
  if (lane == 0)
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(st.bar),
                 "r"(bytes * (uint32_t)m)
                 : "memory");
  __syncwarp();
  if (lane < m) {
    const float *row = g.base + (size_t)cid[lane] * (size_t)(nb * 8);
    float *dst = st.buf + lane * row_words;
    if (nblocks > 0)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(dst + dst_block * 8)),
          "l"(row + src_block * 8), "r"(nblocks * 32u), "r"(st.bar)
          : "memory");
    if (part == 0 && odd)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_addr(dst)),
          "l"(row + (nb - 1) * 8), "r"(32u), "r"(st.bar)
          : "memory");
  }
}

// Waits for the copies of stage_issue.  Returns false on a timed-out wait.
__device__ __forceinline__ bool stage_wait(RowStage &st) {
  const bool ok = mbar_wait(st.bar, st.phase);
  st.phase ^= 1u;
  if (!ok) st.broken = true;
  return __all_sync(kFull, ok);
}

// Lane-pair accumulation over processing steps [T0, T1) of the reference
// model (step t = block block_at(t, nb)) from a staged row: lane h (0/1) of
// the pair owns reference lanes 4h..4h+3.  WHOLE: the staged row is in
// memory order (block b at b); otherwise the staged part holds steps
// T0..T1-1 in order.
template <int NB, bool WHOLE>
__device__ __forceinline__ void staged_accumulate(const GraphView &g, const float *qs,
                                                  const float *row, int h, int T0, int T1,
                                                  float &a0, float &a1, float &a2, float &a3) {
  const int nb = NB > 0 ? NB : (int)g.nb;
  const float4 *r4 = reinterpret_cast<const float4 *>(row) + h;
  const float4 *q4 = reinterpret_cast<const float4 *>(qs) + h;
  const bool l2 = g.metric == 0;
  if constexpr (NB > 0) {
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      if (t < T0 || t >= T1) continue;
      const int b = block_at(t, NB);
      const int sb = WHOLE ? b : t - T0;
      if (l2) acc_l2(a0, a1, a2, a3, q4[2 * b], r4[2 * sb]);
      else acc_ip(a0, a1, a2, a3, q4[2 * b], r4[2 * sb]);
    }
  } else {
#pragma unroll 4
    for (int t = T0; t < T1; ++t) {
      const int b = block_at(t, nb);
      const int sb = WHOLE ? b : t - T0;
      if (l2) acc_l2(a0, a1, a2, a3, q4[2 * b], r4[2 * sb]);
      else acc_ip(a0, a1, a2, a3, q4[2 * b], r4[2 * sb]);
    }
  }
}

// Horizontal sum u0 + u1 + ... + u7 of a lane pair's partials, left to right
// (distance.cpp:53); both lanes return the distance.
__device__ __forceinline__ float pair_finish(const GraphView &g, int h, float a0, float a1, float a2,
                                             float a3) {
  const float o0 = __shfl_xor_sync(kFull, a0, 1);
  const float o1 = __shfl_xor_sync(kFull, a1, 1);
  const float o2 = __shfl_xor_sync(kFull, a2, 1);
  const float o3 = __shfl_xor_sync(kFull, a3, 1);
  const float l0 = h ? o0 : a0, l1 = h ? o1 : a1, l2v = h ? o2 : a2, l3 = h ? o3 : a3;
  const float u0 = h ? a0 : o0, u1 = h ? a1 : o1, u2 = h ? a2 : o2, u3 = h ? a3 : o3;
  float r = __fadd_rn(l0, l1);
  r = __fadd_rn(r, l2v);
  r = __fadd_rn(r, l3);
  r = __fadd_rn(r, u0);
  r = __fadd_rn(r, u1);
  r = __fadd_rn(r, u2);
  r = __fadd_rn(r, u3);
  return g.metric == 0 ? r : -r;
}

// Keys of cid[0..nc) into ckey[0..nc) in passes of `srows` rows (<= 16),
// one distance per lane pair.  With a whole-row stage, rows beyond the first
// pass are sent to L2 first; with a split stage every row is, and each pass
// loads the first halves, accumulates, then loads the second halves (L2
// hits) into the same buffer.  When `first_issued`, the first load (part 0,
// or the whole rows) was already started with stage_issue.  Returns false
// when a stage wait timed out.
template <int NB, bool DEEP>
__device__ __forceinline__ bool eval_staged(const GraphView &g, const WarpSmem &s, RowStage &st,
                                            const StagePool &sp, const SmemPlan &p,
                                            const uint32_t *cid, uint32_t *ckey, int nc,
                                            bool first_issued, int lane) {
  if (!stage_acquire(st, sp, lane)) return false;
  const int srows = (int)p.stage_rows;
  const bool split = p.stage_split > 1;
  const int nb = NB > 0 ? NB : (int)g.nb;
  const int A = (int)split_first((uint32_t)nb);
  if (split) prefetch_rows(g, cid, nc, lane);
  else if (nc > srows && st.rows) prefetch_rows_gather(st.rows, cid + srows, nc - srows, lane);
  else if (nc > srows) prefetch_rows(g, cid + srows, nc - srows, lane);
  const int h = lane & 1, c = lane >> 1;
  for (int p0 = 0; p0 < nc; p0 += srows) {
    const int m = min(srows, nc - p0);
    if constexpr (DEEP) {  // stages deeper than 16 rows: one wait, 16-row groups
      if (!split) {
        if (p0 > 0 || !first_issued)
          stage_issue(g, s, st, cid + p0, m, 2, p.stage_row_words, lane);
        if (!stage_wait(st)) return false;
        for (int g0 = 0; g0 < m; g0 += 16) {
          const int mg = min(16, m - g0);
          const float *rowg = st.buf + (g0 + (c < mg ? c : 0)) * p.stage_row_words;
          float b0 = 0.f, b1 = 0.f, b2 = 0.f, b3 = 0.f;
          staged_accumulate<NB, true>(g, s.q, rowg, h, 0, nb, b0, b1, b2, b3);
          const float dg = pair_finish(g, h, b0, b1, b2, b3);
          if (h == 0 && c < mg) ckey[p0 + g0 + c] = float_to_key(dg);
        }
        __syncwarp();
        continue;
      }
    }
    const float *row = st.buf + (c < m ? c : 0) * p.stage_row_words;
    float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
    if (!split) {
      if (p0 > 0 || !first_issued) stage_issue(g, s, st, cid + p0, m, 2, p.stage_row_words, lane);
      if (!stage_wait(st)) return false;
      staged_accumulate<NB, true>(g, s.q, row, h, 0, nb, a0, a1, a2, a3);
      // the last pass's rows are read: a shared stage goes back before the
      // lane-pair sums (stage_release waits for every lane's reads)
      if (p0 + srows >= nc) stage_release(st, sp, lane);
    } else {
      if (p0 > 0 || !first_issued) stage_issue(g, s, st, cid + p0, m, 0, p.stage_row_words, lane);
      if (!stage_wait(st)) return false;
      staged_accumulate<NB, false>(g, s.q, row, h, 0, A, a0, a1, a2, a3);
      __syncwarp();
      stage_issue(g, s, st, cid + p0, m, 1, p.stage_row_words, lane);
      if (!stage_wait(st)) return false;
      staged_accumulate<NB, false>(g, s.q, row, h, A, nb, a0, a1, a2, a3);
    }
    const float d = pair_finish(g, h, a0, a1, a2, a3);
    if (h == 0 && c < m) ckey[p0 + c] = float_to_key(d);
    __syncwarp();
  }
  stage_release(st, sp, lane);
  return true;
}

// Loads this lane's share of a node's adjacency row.
template <int RCH>
__device__ __forceinline__ void load_row(const GraphView &g, uint32_t node, int lane,
                                         uint32_t (&row)[RCH]) {
  const uint32_t *nrow = g.adj + (size_t)node * g.rstride;
#pragma unroll
  for (int c = 0; c < RCH; ++c) {
    const int m = c * 32 + lane;
    row[c] = m < (int)g.rstride ? __ldg(nrow + m) : kNoneId;
  }
}

// Starts an L2 prefetch of a node's adjacency row (one lane issues it).
__device__ __forceinline__ void prefetch_adj_l2(const GraphView &g, uint32_t node) {
  const uint32_t *nrow = g.adj + (size_t)node * g.rstride;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(nrow), "r"(g.rstride * 4u)
               : "memory");
}

// Rank of each accepted candidate among the accepted ones by (key, adjacency
// position): lane-held candidate i = t*32 + lane.  The pool position of
// candidate i after the merge is its rank plus its pool rank acle[i].
template <int RCH>
__device__ __forceinline__ void accepted_positions(const WarpSmem &s, int na, int lane,
                                                   uint32_t (&nkey)[RCH], uint32_t (&nid)[RCH],
                                                   int (&npos)[RCH], int L) {
  int rank[RCH];
#pragma unroll
  for (int t = 0; t < RCH; ++t) {
    const int i = t * 32 + lane;
    nkey[t] = i < na ? s.ak[i] : 0xFFFFFFFFu;
    nid[t] = i < na ? s.aid[i] : 0u;
    rank[t] = 0;
  }
#pragma unroll 4
  for (int j = 0; j < na; ++j) {
    const uint32_t kj = s.ak[j];
#pragma unroll
    for (int t = 0; t < RCH; ++t) {
      const int i = t * 32 + lane;
      rank[t] += (kj < nkey[t]) || (kj == nkey[t] && j < i);
    }
  }
#pragma unroll
  for (int t = 0; t < RCH; ++t) {
    const int i = t * 32 + lane;
    npos[t] = i < na ? rank[t] + (int)s.acle[i] : L;
  }
}

// Step 4 of a hop: candidates cid/ckey[0..nc) (adjacency order) with key
// below the hop's threshold are accepted, in order, into ak/aid/acle with
// their pool rank (entries <= key).  With check_dups, a candidate whose id is
// already in the pool under the same key is dropped, and so is one whose id
// was accepted from an earlier 32-id chunk of the same row: a table that
// forgets can lose an id recorded earlier in the same hop, so a row that
// repeats an id across chunks would otherwise offer it twice, where the
// reference's visited flags skip the second occurrence (annsearch.cpp:229-231).
// Both copies have the same key, so the first one is accepted iff the second
// would be.  `chunk_dups` asks for the same check among the candidates of one
// 32-candidate chunk; only a list that can hold repeats needs it (rows wider
// than 32, entries copied from another pool).  Returns the count.
template <int RCH>
__device__ __forceinline__ int accept_candidates(const WarpSmem &s, int nc, int size, uint32_t thr,
                                                 bool check_dups, int lane,
                                                 bool chunk_dups = false) {
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const int top = floor_pow2(size);
  int na = 0;
#pragma unroll
  for (int c = 0; c < RCH; ++c) {
    const int e = c * 32 + lane;
    const uint32_t key = e < nc ? s.ckey[e] : 0xFFFFFFFFu;
    bool acc = e < nc && key < thr;
    int cle = 0;
    uint32_t id = 0;
    if (c > 0 && check_dups) __syncwarp();  // earlier chunks' aid/ak stores are visible
    if (acc) {
      id = s.cid[e];
      cle = count_le_bf(s.pk, size, top, key);
      if (check_dups) {
        for (int j = cle - 1; j >= 0 && s.pk[j] == key; --j) {
          if ((s.pid[j] & ~kExplored) == id) {
            acc = false;
            break;
          }
        }
        for (int j = 0; c > 0 && acc && j < na; ++j) {
          if (s.aid[j] == id && s.ak[j] == key) acc = false;
        }
      }
    }
    if (chunk_dups) {
      // copies of one id in this 32-candidate chunk (the fresh ids of a row's
      // chunks are compacted, so they need not sit in different chunks
      // here): the first in adjacency order stays
      const unsigned am0 = __ballot_sync(kFull, acc);
      const unsigned same = __match_any_sync(kFull, acc ? id : kNoneId);
      if (acc && (same & am0 & lanemask_lt)) acc = false;
    }
    const unsigned am = __ballot_sync(kFull, acc);
    if (acc) {
      const int pos = na + __popc(am & lanemask_lt);
      s.ak[pos] = key;
      s.aid[pos] = id;
      s.acle[pos] = (uint32_t)cle;
    }
    na += __popc(am);
  }
  return na;
}

// Step 5 of a hop: stable in-place merge of the na accepted candidates
// (slots npos, from accepted_positions) into the pool of `size` entries,
// truncated to L.  Old entries at and after p0 move up by the number of new
// keys below them, in 128-entry windows from the top down, 4 entries per
// lane, each window fully read before it is written; then the new entries go
// to their slots.  `size` becomes min(L, size + na).
template <int RCH>
__device__ __forceinline__ void merge_accepted(const WarpSmem &s, int &size, int na, int p0, int L,
                                               const uint32_t (&nkey)[RCH],
                                               const uint32_t (&nid)[RCH], const int (&npos)[RCH],
                                               int lane) {
  for (int w = ((size - 1) >> 7) << 7; w + 128 > p0 && w >= 0; w -= 128) {
    const int j0 = w + 4 * lane;
    const bool any = j0 + 3 >= p0 && j0 < size;
    uint4 kk = make_uint4(0, 0, 0, 0), ii = make_uint4(0, 0, 0, 0);
    if (any) {
      kk = *reinterpret_cast<const uint4 *>(s.pk + j0);
      ii = *reinterpret_cast<const uint4 *>(s.pid + j0);
    }
    int c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll 4
    for (int i = 0; i < na; ++i) {
      const uint32_t sv = s.ak[i];
      c0 += kk.x > sv;
      c1 += kk.y > sv;
      c2 += kk.z > sv;
      c3 += kk.w > sv;
    }
    __syncwarp();
    if (any) {
      const uint32_t ks[4] = {kk.x, kk.y, kk.z, kk.w};
      const uint32_t is[4] = {ii.x, ii.y, ii.z, ii.w};
      const int cs[4] = {c0, c1, c2, c3};
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int j = j0 + t;
        const int dst = j + cs[t];
        if (j >= p0 && j < size && dst < L) {
          s.pk[dst] = ks[t];
          s.pid[dst] = is[t];
        }
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int c = 0; c < RCH; ++c) {
    if (npos[c] < L) {
      s.pk[npos[c]] = nkey[c];
      s.pid[npos[c]] = nid[c];
    }
  }
  __syncwarp();
  size = min(L, size + na);
}

// Visited marks of a row's ids (0 for padding), read through L2: byte
// marks[id] holds the epoch of the team's query that last visited id.  A
// null `marks` reads nothing.
template <int RCH>
__device__ __forceinline__ void load_marks(const uint8_t *marks, const uint32_t (&row)[RCH],
                                           uint32_t (&mk)[RCH]) {
#pragma unroll
  for (int c = 0; c < RCH; ++c)
    mk[c] = (marks != nullptr && row[c] != kNoneId) ? (uint32_t)__ldcg(marks + row[c]) : 0u;
}

// The marks to read for the next row: none while the table has forgotten
// nothing this query (every id it does not hold is then fresh), unless rows
// span several 32-id chunks (a chunk's records may evict an id that a later
// chunk of the same row repeats).
template <int RCH>
__device__ __forceinline__ const uint8_t *mark_src(const uint8_t *marks, const QHash &vis) {
  return (RCH > 1 || vis.lossy) ? marks : nullptr;
}

// One query, one warp.  Each hop (batch-merge form of annsearch.cpp:218-253):
//   1. expand pool slot k, the first unexplored one (known from the previous
//      hop); u is the unexplored slot after it;
//   2. read k's adjacency row; drop ids already visited and mark the rest
//      visited, the first occurrence in adjacency order winning (:229-231);
//   3. compute their distances (:236) from rows staged in shared memory;
//   4. accept d < pool[size-1] taken at the start of the hop (:238); each
//      accepted key's rank in the pool (entries <= key) plus its rank among
//      the accepted ones by (d, adjacency position) is its new slot;
//   5. stable-merge the accepted candidates into the pool, older entries
//      first on ties, truncated to L (InsertIntoPool upper-bound insert,
//      util.h:56-75; :242-243).
// After step 4 the next expansion is known: u, unless the best accepted
// candidate lands before it.  u's adjacency row is loaded at the start of
// the hop and its visited marks after step 2, so when u is next both are in
// registers; otherwise the next node's row loads during step 5 and its marks
// after it.
//
// Visited ids: the shared-memory table (QHash) may forget ids, and a
// forgotten id met again is evaluated again (results unchanged, bytes
// wasted: 1.4 evaluations per distinct id at 2048 slots and L = 400).  With
// `marks` (this team's byte per base row, `epoch` = this query's value) an
// id the table does not hold is looked up there too, so no id is evaluated
// twice.  The next row's marks are loaded as soon as the next node is known
// (u's during the hop), so their memory round trip overlaps other work, and
// they are read only for ids whose buckets have evicted (probe_lossy).
template <int NB, int RCH, bool DEEP>
__device__ void warp_search_one(const GraphView &g, const float *__restrict__ qsrc, int K, int L,
                                uint32_t *out_ids, float *out_dists, uint32_t *out_ndc,
                                uint32_t *out_hops, int32_t *out_status, const WarpSmem &s,
                                const SmemPlan &p, RowStage &st, const StagePool &sp,
                                uint32_t max_hops, uint8_t *marks, uint32_t epoch, int lane) {
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const int qw = (int)g.nb * 8;
  for (int i = lane; i < qw; i += 32) s.q[i] = i < (int)g.dim ? qsrc[i] : 0.f;
  const uint32_t nbk = 1u << p.hash_log2;
  for (uint32_t i = lane; i < nbk; i += 32) s.bkt[i] = make_uint4(~0u, ~0u, ~0u, ~0u);
  for (uint32_t i = lane; i < evict_words(p.hash_log2); i += 32) s.evb[i] = 0u;
  __syncwarp();

  QHash vis;
  vis.bkt = s.bkt;
  vis.evb = s.evb;
  vis.rbits = p.qh_rbits;
  vis.rmask = (1u << p.qh_rbits) - 1u;
  vis.bmask = (p.hash_log2 + p.qh_rbits >= 32) ? ~0u : ((1u << (p.hash_log2 + p.qh_rbits)) - 1u);
  vis.lossy = false;

  uint32_t ndc = 0, hops = 0;
  int32_t status = kStatusOk;

  // The loop's first pass builds the initial pool: the first min(L, deg(ep))
  // neighbours of the entry point, all marked visited, sorted by distance
  // (annsearch.cpp:185-215), exact ties in adjacency order.  It runs as a
  // hop into an empty pool (every candidate accepted with pool rank 0) from
  // no slot, except that an id the row repeats enters the pool once per copy,
  // as the reference's initial pool takes the row as it is.  Each later pass
  // is one hop.
  int size = 0;
  uint32_t pref_node = g.ep;
  uint32_t pref_row[RCH], pref_mark[RCH];
  load_row<RCH>(g, g.ep, lane, pref_row);
  load_marks<RCH>(mark_src<RCH>(marks, vis), pref_row, pref_mark);

  bool first = true;
  int k = 0;  // slot expanded by the hop (none in the first pass)
#pragma unroll 1
  while (k >= 0) {
    const bool init = first;  // this pass builds the initial pool
    first = false;
    if (!init && hops >= max_hops) {
      status = kStatusHopLimit;
      break;
    }
    // 1. u: the first unexplored slot after k
    int u = -1;
    for (int b0 = k + 1; b0 < size; b0 += 32) {
      const int idx = b0 + lane;
      const bool un = idx < size && !(s.pid[idx] & kExplored);
      const unsigned bm = __ballot_sync(kFull, un);
      if (bm) {
        u = b0 + __ffs(bm) - 1;
        break;
      }
    }
    const uint32_t node = init ? g.ep : s.pid[k];
    const uint32_t thr = init ? 0xFFFFFFFFu : s.pk[size - 1];
    const uint32_t unode = u >= 0 ? s.pid[u] : kNoneId;
    __syncwarp();
    if (!init) {
      if (lane == 0) s.pid[k] = node | kExplored;
      ++hops;
    }
    // node's row and marks were loaded when it was chosen (pref_node is
    // always node; the reload only guards that)
    if (node != pref_node) {
      load_row<RCH>(g, node, lane, pref_row);
      load_marks<RCH>(mark_src<RCH>(marks, vis), pref_row, pref_mark);
    }
    const uint32_t(&row)[RCH] = pref_row;
    const uint32_t(&rmark)[RCH] = pref_mark;
    // u is the next node unless an accepted candidate lands before it: its
    // row loads now, its marks once this hop's marks are stored (below)
    uint32_t spec_row[RCH], spec_mark[RCH];
#pragma unroll
    for (int c = 0; c < RCH; ++c) {
      spec_row[c] = kNoneId;
      spec_mark[c] = 0u;
    }
    if (unode != kNoneId) load_row<RCH>(g, unode, lane, spec_row);

    // 2. in-row dedupe, visited filter, compaction in m order (the initial
    //    pool: the row's first L entries as they are).  The row copies of
    //    the first stage load start as soon as the fresh ids are known; the
    //    table is updated while they are in flight.
    int nc = 0;
    const int srows = (int)p.stage_rows;
    bool issued = false;
#pragma unroll
    for (int c = 0; c < RCH; ++c) {
      const bool valid = row[c] != kNoneId && (!init || c * 32 + lane < L);
      // copies of one id in the row: the first in adjacency order counts
      // (a graph whose rows repeat no id skips the match)
      const unsigned peers = g.row_dups ? __match_any_sync(kFull, row[c]) : (1u << lane);
      const bool leader = valid && (peers & lanemask_lt) == 0u;
      QProbe pr{};
      // every valid lane probes the table, so the probe overlaps the
      // match above instead of waiting for it; only leaders count
      bool seen = valid ? qh_lookup(vis, row[c], pr) : true;
      // the marks are read only where a bucket of the id has evicted, and
      // the warp waits for them only when some lane needs them
      if (marks != nullptr) {
        const bool need = !seen && probe_lossy(vis, pr.b1, pr.b2);
        if (__any_sync(kFull, need)) seen = seen || (need && rmark[c] == epoch);
      }
      const bool fresh = init ? valid : leader && !seen;
      const unsigned fm = __ballot_sync(kFull, fresh);
      if (fresh) s.cid[nc + __popc(fm & lanemask_lt)] = row[c];
      nc += __popc(fm);
      if (RCH == 1 && nc > 0) {
        __syncwarp();
        if (stage_acquire(st, sp, lane)) {
          stage_issue(g, s, st, s.cid, min(nc, srows), p.stage_split > 1 ? 0 : 2,
                      p.stage_row_words, lane);
          issued = true;
        }
      }
      qh_record(vis, pr, row[c], leader && !seen, lane);
      if (marks != nullptr && leader && !seen) __stcg(marks + row[c], (uint8_t)epoch);
      __syncwarp();
    }
    if (unode != kNoneId) load_marks<RCH>(mark_src<RCH>(marks, vis), spec_row, spec_mark);
    if (nc == 0) {
      pref_node = unode;
#pragma unroll
      for (int c = 0; c < RCH; ++c) {
        pref_row[c] = spec_row[c];
        pref_mark[c] = spec_mark[c];
      }
      k = u;
      continue;
    }
    __syncwarp();

    // 3. distances of the staged rows
    if (!eval_staged<NB, DEEP>(g, s, st, sp, p, s.cid, s.ckey, nc, issued, lane)) {
      status = kStatusStageTimeout;
      break;
    }
    ndc += nc;

    // 4. acceptance in adjacency order, with each key's pool rank; after an
    //    eviction, a candidate already in the pool (same id under the same
    //    key) is dropped
    const int na = accept_candidates<RCH>(s, nc, size, thr, !init && vis.lossy, lane,
                                          !init && RCH > 1 && vis.lossy && g.row_dups);
    if (na == 0) {
      pref_node = unode;
#pragma unroll
      for (int c = 0; c < RCH; ++c) {
        pref_row[c] = spec_row[c];
        pref_mark[c] = spec_mark[c];
      }
      k = u;
      continue;
    }
    __syncwarp();
    uint32_t nkey[RCH], nid[RCH];
    int npos[RCH];
    accepted_positions<RCH>(s, na, lane, nkey, nid, npos, L);

    // Next expansion: the best accepted candidate lands at p0 (the smallest
    // new slot); old slot u stays ahead of it iff u < p0.  Its adjacency row
    // loads during the merge.
    int pmin = npos[0];
#pragma unroll
    for (int c = 1; c < RCH; ++c) pmin = min(pmin, npos[c]);
    const int p0 = (int)__reduce_min_sync(kFull, (uint32_t)pmin);
    {
      uint32_t cand = kNoneId;
#pragma unroll
      for (int c = 0; c < RCH; ++c)
        if (npos[c] == p0) cand = nid[c];
      const uint32_t best = __reduce_min_sync(kFull, cand);  // the one lane holding p0
      const uint32_t nxt = (u >= 0 && u < p0) ? unode : best;
      pref_node = nxt;
      if (nxt == unode) {
#pragma unroll
        for (int c = 0; c < RCH; ++c) {
          pref_row[c] = spec_row[c];
          pref_mark[c] = spec_mark[c];
        }
      } else {
        load_row<RCH>(g, nxt, lane, pref_row);
      }
      k = (u >= 0 && u < p0) ? u : p0;
    }

    // 5. stable merge into the pool (older entries first on ties)
    merge_accepted<RCH>(s, size, na, p0, L, nkey, nid, npos, lane);
    if (pref_node != unode) load_marks<RCH>(mark_src<RCH>(marks, vis), pref_row, pref_mark);
  }

  // Results: slots the pool never filled keep the reference's value-
  // initialised Neighbor (id 0, distance 0), annsearch.cpp:193, :254-257.
  for (int i = lane; i < K; i += 32) {
    const bool have = i < size;
    out_ids[i] = have ? (s.pid[i] & ~kExplored) : 0u;
    if (out_dists) out_dists[i] = have ? key_to_float(s.pk[i]) : 0.f;
  }
  if (lane == 0) {
    if (out_ndc) *out_ndc = ndc;
    if (out_hops) *out_hops = hops;
    if (out_status) *out_status = status;
  }
  __syncwarp();
}

// At most 128 registers a thread (two 256-thread CTAs' worth per SM).
// `rows` is the 2-D tensor map of the base rows (nb*8 floats x n), used when
// p.gather is set.
template <int NB, int RCH, bool DEEP>
__global__ void __launch_bounds__(256, 2) warp_search_kernel(GraphView g, BatchArgs a, SmemPlan p,
                                                              const __grid_constant__ CUtensorMap rows) {
  extern __shared__ __align__(128) uint32_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  const StagePool sp = carve_pool(smem, p);
  const WarpSmem s = carve_warp(smem + stage_pool_words(p) + (size_t)warp * p.words_per_team, p);
  RowStage st;
  st.phase = 0;
  st.broken = false;
  st.rows = p.gather ? &rows : nullptr;
  if (p.shared_stages == 0) {  // a private stage, always held
    st.bar = smem_addr(s.bar);
    st.buf = s.stage;
    st.slot = 0;
    if (lane == 0) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(st.bar) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
  } else {  // the CTA's stage pool
    st.bar = 0;
    st.buf = nullptr;
    st.slot = -1;
    if (threadIdx.x == 0) {
      for (uint32_t i = 0; i < sp.count; ++i) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(sp.bar0 + 8u * i) : "memory");
        sp.phases[i] = 0u;
      }
      *sp.mask = sp.count >= 32 ? ~0u : ((1u << sp.count) - 1u);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
  }
  const uint32_t slot = blockIdx.x * wpb + warp;
  const uint32_t nslots = gridDim.x * wpb;
  uint32_t q = slot;
  for (;;) {
    if (a.work_counter) {
      uint32_t t = 0;
      if (lane == 0) t = atomicAdd(a.work_counter, 1u);
      q = __shfl_sync(kFull, t, 0);
    }
    if (q >= a.nq) break;
    const int K = a.Ks ? a.Ks[q] : a.K0;
    const int L = a.Ls ? a.Ls[q] : a.L0;
    const int64_t off = a.out_off ? a.out_off[q] : (int64_t)q * a.K0;
    if (K < 1 || K > L || L > (int)p.pool_cap) {
      if (lane == 0 && a.status) a.status[q] = kStatusBadArgs;
    } else {
      // this slot's visited marks: a new epoch per query; when the byte
      // epoch wraps, the slot's marks are cleared first
      uint8_t *marks = nullptr;
      uint32_t epoch = 0;
      if (a.marks != nullptr) {
        marks = a.marks + (size_t)slot * a.mark_stride;
        uint32_t e = 0;
        if (lane == 0) e = a.mark_epoch[slot] + 1u;
        e = __shfl_sync(kFull, e, 0);
        if (e > 255u) {
          uint4 *m4 = reinterpret_cast<uint4 *>(marks);
          for (uint32_t i = lane; i < a.mark_stride / 16u; i += 32) __stcg(m4 + i, make_uint4(0, 0, 0, 0));
          e = 1u;
        }
        if (lane == 0) a.mark_epoch[slot] = e;
        __syncwarp();
        epoch = e;
      }
      warp_search_one<NB, RCH, DEEP>(g, a.queries + (size_t)q * a.qstride, K, L, a.ids + off,
                               a.dists ? a.dists + off : nullptr, a.ndc ? a.ndc + q : nullptr,
                               a.hops ? a.hops + q : nullptr, a.status ? a.status + q : nullptr, s,
                               p, st, sp, a.max_hops, marks, epoch, lane);
      // a stage copy that never completed leaves this team's stage unusable:
      // wait once more (bounded) for it and take no further queries
      if (st.broken) {
        mbar_wait(st.bar, st.phase ^ 1u);
        break;
      }
    }
    if (!a.work_counter) q += nslots;
  }
}

// ------------------------------------------------------- CTA per query ---
// W warps share one query.  Each step (the several-candidates-per-step form,
// structured like ModifiedDeltaStepping, annsearch.cpp:1632-1691, with the
// acceptance and termination rules of SearchArraySimulation):
//   A. warp 0 picks the first W unexplored slots; the acceptance threshold is
//      pool[size-1] at this point;
//   B. warp w reads the adjacency row of pick w, dedupes it, and keeps ids
//      that were not visited before this step;
//   C. ids seen by several warps in the same step are resolved in (w, m)
//      order through a step-local table with atomicMin claims, so the first
//      occurrence wins exactly as a sequential scan would;
//   D. winners are marked visited and evaluated; accepted ones are sorted per
//      warp by (key, m);
//   E. the pool and all W sorted lists are merged by rank (ties: old pool,
//      then lower w, then lower m) into the second pool buffer.
// With W = 1 this is exactly the warp kernel's search.
struct CtaSmem {
  float *q;
  uint32_t *pk[2], *pid[2];
  uint32_t *hash;
  uint32_t *st_id, *st_claim;           // step-local dedupe table
  uint32_t *wc_id, *wc_key, *wc_slot;   // per-warp candidates [W][cand_cap]
  uint32_t *ws_key, *ws_id;             // per-warp sorted accepted [W][cand_cap]
  int *wn;                              // per-warp accepted counts [W]
  int *misc;                            // [0] npicks, [1..W] picks, [W+1] pmin
};

constexpr int kStepTableFactor = 2;

__device__ __forceinline__ uint32_t st_find_or_insert(uint32_t *tab, uint32_t mask, uint32_t log2cap,
                                                      uint32_t id) {
  uint32_t s = hash_slot(id, log2cap);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t cur = tab[s];
    if (cur == id) return s;
    if (cur == kNoneId) {
      const uint32_t old = atomicCAS(&tab[s], kNoneId, id);
      if (old == kNoneId || old == id) return s;
    }
    s = (s + 1) & mask;
  }
  return 0xFFFFFFFFu;  // unreachable: the table holds twice the step's candidates
}

template <int NB, int RCH>
__global__ void __launch_bounds__(512) intra_search_kernel(GraphView g, BatchArgs a, SmemPlan p,
                                                           int W) {
  extern __shared__ __align__(128) uint32_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nthr = blockDim.x;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const uint32_t q_idx = blockIdx.x;
  if (q_idx >= a.nq) return;
  const int K = a.Ks ? a.Ks[q_idx] : a.K0;
  const int L = a.Ls ? a.Ls[q_idx] : a.L0;
  const int64_t off = a.out_off ? a.out_off[q_idx] : (int64_t)q_idx * a.K0;
  if (K < 1 || K > L || L > (int)p.pool_cap) {
    if (threadIdx.x == 0 && a.status) a.status[q_idx] = kStatusBadArgs;
    return;
  }
  const int cc = (int)p.cand_cap;
  const uint32_t st_cap = p.step_cap;
  const uint32_t st_log2 = p.step_log2;

  CtaSmem s;
  {
    uint32_t *b = smem;
    s.q = reinterpret_cast<float *>(b); b += p.q_words;
    s.pk[0] = b; b += p.pool_cap;
    s.pid[0] = b; b += p.pool_cap;
    s.pk[1] = b; b += p.pool_cap;
    s.pid[1] = b; b += p.pool_cap;
    s.hash = b; b += p.hash_cap;
    s.st_id = b; b += st_cap;
    s.st_claim = b; b += st_cap;
    s.wc_id = b; b += W * cc;
    s.wc_key = b; b += W * cc;
    s.wc_slot = b; b += W * cc;
    s.ws_key = b; b += W * cc;
    s.ws_id = b; b += W * cc;
    s.wn = reinterpret_cast<int *>(b); b += 32;
    s.misc = reinterpret_cast<int *>(b);
  }
  uint32_t *spill = a.spill_bits ? a.spill_bits + (size_t)q_idx * a.spill_words : nullptr;

  const float *qsrc = a.queries + (size_t)q_idx * a.qstride;
  const int qw = (int)g.nb * 8;
  for (int i = threadIdx.x; i < qw; i += nthr) s.q[i] = i < (int)g.dim ? qsrc[i] : 0.f;
  for (uint32_t i = threadIdx.x; i < p.hash_cap; i += nthr) s.hash[i] = kNoneId;
  for (uint32_t i = threadIdx.x; i < st_cap; i += nthr) {
    s.st_id[i] = kNoneId;
    s.st_claim[i] = 0xFFFFFFFFu;
  }
  __syncthreads();

  Visited vis;
  vis.tab = s.hash;
  vis.mask = p.hash_cap - 1;
  vis.log2cap = p.hash_log2;
  vis.limit = p.hash_limit;
  vis.count = 0;
  vis.bits = spill;
  vis.spilled = false;

  uint32_t ndc = 0, hops = 0;
  int32_t status = kStatusOk;
  int cur = 0;  // active pool buffer
  int size = 0;

  // Initial pool (warp 0), identical to the warp kernel's.
  if (warp == 0) {
    const uint32_t *erow = g.adj + (size_t)g.ep * g.rstride;
    uint32_t *cid = s.wc_id, *ckey = s.wc_key;
#pragma unroll
    for (int c = 0; c < RCH; ++c) {
      const int m = c * 32 + lane;
      const uint32_t id = m < (int)g.rstride ? __ldg(erow + m) : kNoneId;
      const bool valid = id != kNoneId && m < L;
      if (valid) {
        cid[m] = id;
        visit(vis, id);
      }
      size += __popc(__ballot_sync(kFull, valid));
    }
    __syncwarp();
    eval_candidates<NB>(g, s.q, cid, ckey, size, lane);
    __syncwarp();
    uint64_t x[RCH];
#pragma unroll
    for (int i = 0; i < RCH; ++i) {
      const int e = i * 32 + lane;
      x[i] = e < size ? (((uint64_t)ckey[e] << 32) | (uint32_t)e) : kInvalidKey;
    }
    warp_sort<RCH>(x, lane);
#pragma unroll
    for (int i = 0; i < RCH; ++i) {
      const int e = i * 32 + lane;
      if (e < size) {
        s.pk[0][e] = (uint32_t)(x[i] >> 32);
        s.pid[0][e] = cid[(uint32_t)x[i]];
      }
    }
    if (lane == 0) s.misc[0] = size;
  }
  __syncthreads();
  size = s.misc[0];
  vis.count = size;
  ndc += size;

  int cursor = 0;
  for (;;) {
    uint32_t *pk = s.pk[cur], *pid = s.pid[cur];
    // A. picks
    if (warp == 0) {
      int np = 0, last = -1;
      for (int b0 = cursor; b0 < size && np < W; b0 += 32) {
        const int idx = b0 + lane;
        const bool un = idx < size && !(pid[idx] & kExplored);
        const unsigned bm = __ballot_sync(kFull, un);
        if (un) {
          const int r = np + __popc(bm & lanemask_lt);
          if (r < W) {
            s.misc[1 + r] = idx;
            last = idx;
          }
        }
        np += __popc(bm);
      }
      np = min(np, W);
      // highest picked index: max over lanes of `last`
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) last = max(last, __shfl_xor_sync(kFull, last, o));
      if (lane == 0) {
        s.misc[0] = np;
        s.misc[W + 2] = last;
      }
    }
    __syncthreads();
    const int np = s.misc[0];
    if (np == 0) break;
    if (hops >= a.max_hops) {
      status = kStatusHopLimit;
      break;
    }
    // Spill decision for this step, identical in every thread: the step can
    // add at most W * cand_cap entries.
    if (!vis.spilled && vis.count + (uint32_t)(W * cc) > p.hash_limit) {
      if (!spill) {
        status = kStatusVisitedFull;
        break;
      }
      vis.spilled = true;
    }
    const uint32_t thr = pk[size - 1];
    cursor = s.misc[W + 2] + 1;
    hops += np;

    // B. per-warp adjacency row: in-row dedupe + not-yet-visited filter
    int nfresh = 0;
    uint32_t my_node = 0;
    if (warp < np) {
      my_node = pid[s.misc[1 + warp]];
      const uint32_t *nrow = g.adj + (size_t)my_node * g.rstride;
#pragma unroll
      for (int c = 0; c < RCH; ++c) {
        const int m = c * 32 + lane;
        const uint32_t id = m < (int)g.rstride ? __ldg(nrow + m) : kNoneId;
        const bool valid = id != kNoneId;
        const unsigned peers = __match_any_sync(kFull, id);
        const bool leader = valid && (peers & lanemask_lt) == 0u;
        const bool fresh = leader && !visited_test(vis, id);
        const unsigned fm = __ballot_sync(kFull, fresh);
        if (fresh) {
          const int pos = nfresh + __popc(fm & lanemask_lt);
          s.wc_id[warp * cc + pos] = id;
          // C. claim in (w, m) order
          const uint32_t slot = st_find_or_insert(s.st_id, st_cap - 1, st_log2, id);
          s.wc_slot[warp * cc + pos] = slot;
          atomicMin(&s.st_claim[slot], (uint32_t)(warp * cc + m));
          s.wc_key[warp * cc + pos] = (uint32_t)m;  // remember m until claims settle
        }
        nfresh += __popc(fm);
      }
    }
    __syncthreads();
    // mark explored (after every warp has read its node id)
    if (threadIdx.x < (unsigned)np) {
      const int kk = s.misc[1 + threadIdx.x];
      pid[kk] |= kExplored;
    }

    // D. winners: visited insert, distance, acceptance, per-warp sort
    int nwin = 0;
    if (warp < np) {
      for (int c0 = 0; c0 < nfresh; c0 += 32) {
        const int e = c0 + lane;
        bool win = false;
        uint32_t id = 0;
        if (e < nfresh) {
          const uint32_t m = s.wc_key[warp * cc + e];
          const uint32_t slot = s.wc_slot[warp * cc + e];
          id = s.wc_id[warp * cc + e];
          win = s.st_claim[slot] == (uint32_t)(warp * cc + (int)m);
        }
        const unsigned wm = __ballot_sync(kFull, win);
        if (win) {
          visit(vis, id);
          // compact winners in place (positions only move down)
          s.ws_id[warp * cc + nwin + __popc(wm & lanemask_lt)] = id;
        }
        nwin += __popc(wm);
      }
    }
    // every warp applies the same count update so vis.count stays uniform
    __syncthreads();
    if (warp < np && lane == 0) s.wn[warp] = nwin;
    __syncthreads();
    {
      int tot = 0;
      for (int w = 0; w < np; ++w) tot += s.wn[w];
      if (!vis.spilled) vis.count += tot;
      ndc += tot;
    }
    // reset the step table slots used this step (claims and ids)
    if (warp < np) {
      for (int e = lane; e < nfresh; e += 32) {
        const uint32_t slot = s.wc_slot[warp * cc + e];
        s.st_id[slot] = kNoneId;
        s.st_claim[slot] = 0xFFFFFFFFu;
      }
    }
    int nacc = 0;
    if (warp < np) {
      // distances of the winners (ws_id[warp][0..nwin)) into wc_key
      eval_candidates<NB>(g, s.q, s.ws_id + warp * cc, s.wc_key + warp * cc, nwin, lane);
      __syncwarp();
      uint64_t x[RCH];
#pragma unroll
      for (int i = 0; i < RCH; ++i) {
        const int e = i * 32 + lane;
        const bool acc = e < nwin && s.wc_key[warp * cc + e] < thr;
        x[i] = acc ? (((uint64_t)s.wc_key[warp * cc + e] << 32) | (uint32_t)e) : kInvalidKey;
        nacc += __popc(__ballot_sync(kFull, acc));
      }
      warp_sort<RCH>(x, lane);
      uint32_t sid[RCH];
#pragma unroll
      for (int i = 0; i < RCH; ++i) {
        const int e = i * 32 + lane;
        if (e < nacc) sid[i] = s.ws_id[warp * cc + (uint32_t)x[i]];
      }
      __syncwarp();
#pragma unroll
      for (int i = 0; i < RCH; ++i) {
        const int e = i * 32 + lane;
        if (e < nacc) {
          s.ws_key[warp * cc + e] = (uint32_t)(x[i] >> 32);
          s.ws_id[warp * cc + e] = sid[i];
        }
      }
    }
    __syncthreads();
    if (warp < np && lane == 0) s.wn[warp] = nacc;
    __syncthreads();
    int total = 0;
    for (int w = 0; w < np; ++w) total += s.wn[w];
    if (total == 0) continue;

    // E. rank merge into the other buffer.  New entries first, all (list w,
    //    element e) pairs in parallel: the rank r of each among the new keys
    //    (ties: lower w, then lower e) and its slot r + (old entries <= key).
    //    The new keys, in rank order, go to wc_key (free again at this
    //    point), so each old entry then finds its shift -- the new keys
    //    strictly below it -- with one search.
    uint32_t *npk = s.pk[cur ^ 1], *npid = s.pid[cur ^ 1];
    uint32_t *allnew = s.wc_key;  // W * cand_cap >= total entries
    if (threadIdx.x == 0) s.misc[W + 1] = 0x7FFFFFFF;
    __syncthreads();
    int local_min = 0x7FFFFFFF;
    for (int t = threadIdx.x; t < total; t += nthr) {
      int w = 0, e = t;
      while (e >= s.wn[w]) {
        e -= s.wn[w];
        ++w;
      }
      const uint32_t key = s.ws_key[w * cc + e];
      int r = e;
      for (int v = 0; v < np; ++v) {
        if (v == w) continue;
        r += (v < w) ? count_le(s.ws_key + v * cc, s.wn[v], key)
                     : count_lt(s.ws_key + v * cc, s.wn[v], key);
      }
      allnew[r] = key;
      const int pos = r + count_le(pk, size, key);
      if (pos < L) {
        const uint32_t nid = s.ws_id[w * cc + e];
        npk[pos] = key;
        npid[pos] = nid;
        // a new entry near the head is a likely pick of the next step
        if (pos < cursor + W) prefetch_adj_l2(g, nid);
      }
      local_min = min(local_min, pos);
    }
    __syncthreads();
    // old entries, after the new keys strictly below them
    for (int j = threadIdx.x; j < size; j += nthr) {
      const uint32_t key = pk[j];
      const int pos = j + count_lt(allnew, total, key);
      if (pos < L) {
        npk[pos] = key;
        npid[pos] = pid[j];
      }
    }
    if (local_min != 0x7FFFFFFF) atomicMin(&s.misc[W + 1], local_min);
    __syncthreads();
    size = min(L, size + total);
    cursor = min(cursor, s.misc[W + 1]);
    cur ^= 1;
  }

  // results
  {
    const uint32_t *pk = s.pk[cur], *pid = s.pid[cur];
    uint32_t *oid = a.ids + off;
    float *od = a.dists ? a.dists + off : nullptr;
    for (int i = threadIdx.x; i < K; i += nthr) {
      const bool have = i < size;
      oid[i] = have ? (pid[i] & ~kExplored) : 0u;
      if (od) od[i] = have ? key_to_float(pk[i]) : 0.f;
    }
  }
  if (vis.spilled && spill) {
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < a.spill_words; w += nthr) spill[w] = 0u;
  }
  if (threadIdx.x == 0) {
    if (a.ndc) a.ndc[q_idx] = ndc;
    if (a.hops) a.hops[q_idx] = hops;
    if (a.status) a.status[q_idx] = status;
  }
}

// ------------------------------------------- scatter: independent pools ---
// ScatterSearch's intra-query search (MultiThreadSearchArraySimulation,
// src/annsearch.cpp:532-699, and its election variant
// MultiThreadSearchArraySimulationWithET, :839-1025 with
// SearchUntilBestThreadStop, :1368-1455).  One CTA per query, one warp per
// reference thread.  Each warp starts from its own entry point and runs the
// plain best-first loop on its own pool of L; all warps share one exact
// visited set, so whichever warp meets an id first owns it (as with the
// reference's shared bitset, results depend on the warps' timing and are
// judged by recall).  At the end the pools' top K are merged, duplicates
// dropped.
//   plain  the pool starts with every neighbour of the entry point and is
//          padded to L with random unvisited ids (:552-575);
//   ET     the pool starts with the neighbours only; at the warp's 50th
//          expansion it votes with its K-th distance; once all have voted,
//          warps whose best entry is worse than the winning vote stop.
//          Those, like the others that finish early, copy every unexplored
//          entry of one "good" warp's pool, then a few entries of a second
//          good warp, and continue from their own pool; the winner finishing
//          stops every warp (:858-999, :1368-1455).
// Entry points and pads come from a counter-based hash of (seed, query, warp)
// instead of rand(); the election's ties go to the lower warp; and entries are
// read out of another warp's pool under that pool's sequence counter, where
// the reference reads the other thread's pool unsynchronised.
// One rule is not carried over: the reference's thief also marks the stolen
// entries explored in the good thread's pool (:1390).  On CPU threads that
// is a race the owner mostly wins (it keeps expanding from the front of its
// pool while the thief walks in from the end); on warps in lockstep the thief
// marks the whole pool within one hop, the winner then has nothing left,
// finishes and stops every warp, and recall fell below a single plain search
// (0.947 against 0.982 on 50k x 96 unit vectors, L = 100, 4 warps).  Stolen
// entries are therefore copied and left to their owner as well.
constexpr int kMaxScatter = SS_SCATTER_MAX_WARPS;
constexpr int kElectionHop = 50;

struct ScatterCtl {
  unsigned long long best;  // (K-th key at the election hop) << 32 | warp
  int decided;              // warps that voted
  int finish;               // the elected warp finished: all stop
  int vis_count;            // entries reserved in the visited hash
  int vis_spilled;          // hash full: new ids go to the global bitset
  int status;
  unsigned ndc, hops;
  unsigned ndc_max, ndc_min;      // one warp's most / fewest distance evaluations
  int good[kMaxScatter];          // 1: pool head better than the winning vote
  int reached[kMaxScatter];       // voted
  unsigned version[kMaxScatter];  // pool sequence counters (odd while changing)
  int size[kMaxScatter];          // pool sizes
};

// Shared state that other warps change is read by lane 0 and broadcast, so
// every lane of a warp takes the same branch (warp-wide collectives follow).
__device__ __forceinline__ int uniform_load(const int *p, int lane) {
  int v = 0;
  if (lane == 0) v = *(const volatile int *)p;
  return __shfl_sync(kFull, v, 0);
}
__device__ __forceinline__ unsigned uniform_load(const unsigned *p, int lane) {
  unsigned v = 0;
  if (lane == 0) v = *(const volatile unsigned *)p;
  return __shfl_sync(kFull, v, 0);
}
__device__ __forceinline__ unsigned long long uniform_load(const unsigned long long *p, int lane) {
  unsigned long long v = 0;
  if (lane == 0) v = *(const volatile unsigned long long *)p;
  const unsigned lo = __shfl_sync(kFull, (unsigned)v, 0);
  const unsigned hi = __shfl_sync(kFull, (unsigned)(v >> 32), 0);
  return ((unsigned long long)hi << 32) | lo;
}

__device__ __forceinline__ uint32_t scatter_rng(uint64_t seed, uint32_t q, uint32_t w,
                                                uint32_t i) {
  uint64_t x = seed ^ ((uint64_t)q << 32) ^ ((uint64_t)w << 20) ^ (uint64_t)i;
  x += 0x9E3779B97F4A7C15ull;  // splitmix64 finaliser
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return (uint32_t)((x ^ (x >> 31)) >> 32);
}

// Reserves room for up to `m` new ids in the shared visited hash; switches
// this warp (and, through ctl, the others) to spilling once the hash is full.
__device__ __forceinline__ void scatter_reserve(Visited &v, ScatterCtl *ctl, int m, int lane) {
  if (v.spilled) return;
  int r = 0;
  if (lane == 0) r = atomicAdd(&ctl->vis_count, m);
  r = __shfl_sync(kFull, r, 0);
  if ((uint32_t)(r + m) > v.limit) {
    if (lane == 0) atomicExch(&ctl->vis_spilled, 1);
    v.spilled = true;
  } else if (uniform_load(&ctl->vis_spilled, lane)) {
    v.spilled = true;
  }
}

// Copies unexplored entries of warp t's pool in slots [b-31, b] (b counts
// down from the pool's end; slot 0 is never taken), as SearchUntilBestThreadStop
// walks a good thread's pool from its end (annsearch.cpp:1384-1396 steals,
// :1402-1413 peeks), into this warp's cid/ckey.  The window is read under
// t's sequence counter (a consistent copy, up to 4 attempts); at most `limit`
// entries are taken, the ones nearest the pool's end first.  The entries stay
// unexplored in t's pool: see the kernel's comment on stealing.  Returns how
// many went to cid/ckey (0 also when every attempt saw the pool change).
__device__ __forceinline__ int scatter_take_window(const WarpSmem &src, ScatterCtl *ctl, int t,
                                                   const WarpSmem &dst, int b, int limit, int lane) {
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const int j = b - lane;
  uint32_t id = 0, key = 0;
  bool un = false, valid = false;
  for (int attempt = 0; attempt < 4 && !valid; ++attempt) {
    const unsigned v0 = uniform_load(&ctl->version[t], lane);
    if (v0 & 1u) continue;
    __threadfence_block();
    un = false;
    if (j >= 1) {
      id = *(volatile uint32_t *)&src.pid[j];
      key = *(volatile uint32_t *)&src.pk[j];
      un = !(id & kExplored);
    }
    __threadfence_block();
    valid = uniform_load(&ctl->version[t], lane) == v0;
  }
  if (!valid) return 0;
  const unsigned um = __ballot_sync(kFull, un);
  const bool take = un && __popc(um & lanemask_lt) < limit;
  const unsigned tm = __ballot_sync(kFull, take);
  if (take) {
    const int pos = __popc(tm & lanemask_lt);
    dst.cid[pos] = id;
    dst.ckey[pos] = key;
  }
  __syncwarp();
  return __popc(tm);
}

template <int NB, int RCH, int PITEMS>
__global__ void __launch_bounds__(512) scatter_search_kernel(GraphView g, BatchArgs a, SmemPlan p,
                                                             int W, int et, uint64_t seed) {
  extern __shared__ __align__(128) uint32_t smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  const uint32_t q_idx = blockIdx.x;
  if (q_idx >= a.nq) return;
  const int K = a.Ks ? a.Ks[q_idx] : a.K0;
  const int L = a.Ls ? a.Ls[q_idx] : a.L0;
  const int64_t off = a.out_off ? a.out_off[q_idx] : (int64_t)q_idx * a.K0;
  if (K < 1 || K > L || L > (int)p.pool_cap) {
    if (threadIdx.x == 0 && a.status) a.status[q_idx] = kStatusBadArgs;
    return;
  }
  // shared: query, visited hash, control block; then one pool region per warp
  float *qs = reinterpret_cast<float *>(smem);
  uint32_t *tab = smem + p.q_words;
  ScatterCtl *ctl = reinterpret_cast<ScatterCtl *>(tab + p.hash_cap);
  uint32_t *wbase = tab + p.hash_cap + p.step_cap;  // step_cap: words of ScatterCtl
  auto carve = [&](int w) {
    WarpSmem s{};
    uint32_t *b = wbase + (size_t)w * p.words_per_team;
    s.q = qs;
    s.pk = b;
    b += p.pool_cap;
    s.pid = b;
    b += p.pool_cap;
    s.cid = b;
    b += p.cand_cap;
    s.ckey = b;
    b += p.cand_cap;
    s.ak = b;
    b += p.cand_cap;
    s.aid = b;
    b += p.cand_cap;
    s.acle = b;
    return s;
  };
  const WarpSmem s = carve(warp);
  const float *qsrc = a.queries + (size_t)q_idx * a.qstride;
  const int qw = (int)g.nb * 8;
  for (int i = threadIdx.x; i < qw; i += blockDim.x) qs[i] = i < (int)g.dim ? qsrc[i] : 0.f;
  for (uint32_t i = threadIdx.x; i < p.hash_cap; i += blockDim.x) tab[i] = kNoneId;
  if (threadIdx.x == 0) {
    ctl->best = ~0ull;
    ctl->decided = 0;
    ctl->finish = 0;
    ctl->vis_count = 0;
    ctl->vis_spilled = 0;
    ctl->status = kStatusOk;
    ctl->ndc = 0;
    ctl->hops = 0;
    ctl->ndc_max = 0;
    ctl->ndc_min = 0xFFFFFFFFu;
  }
  if (threadIdx.x < kMaxScatter) {
    ctl->good[threadIdx.x] = 0;
    ctl->reached[threadIdx.x] = 0;
    ctl->version[threadIdx.x] = 0;
    ctl->size[threadIdx.x] = 0;
  }
  __syncthreads();

  Visited vis;
  vis.tab = tab;
  vis.mask = p.hash_cap - 1;
  vis.log2cap = p.hash_log2;
  vis.limit = p.hash_limit;
  vis.count = 0;
  vis.bits = a.spill_bits ? a.spill_bits + (size_t)q_idx * a.spill_words : nullptr;
  vis.spilled = false;
  uint32_t ndc = 0, hops = 0;
  int32_t status = kStatusOk;

  // --- initial pool
  int size = 0;
  {
    const uint32_t ep = scatter_rng(seed, q_idx, warp, 0) % g.n;
    uint32_t row[RCH];
    load_row<RCH>(g, ep, lane, row);
    scatter_reserve(vis, ctl, (int)g.rstride, lane);
#pragma unroll
    for (int c = 0; c < RCH; ++c) {
      const int m = c * 32 + lane;
      const bool valid = row[c] != kNoneId && m < L;
      if (valid) {
        s.pid[m] = row[c];
        visit(vis, row[c]);
      }
      size += __popc(__ballot_sync(kFull, valid));
    }
    if (!et) {
      // pad to L with random ids nobody has visited (claimed atomically)
      scatter_reserve(vis, ctl, L - size, lane);
      for (uint32_t round = 0; size < L && round < 64; ++round) {
        const int need = L - size;
        uint32_t id = scatter_rng(seed, q_idx, warp, 1 + round * 32 + lane) % g.n;
        bool got = false;
        if (lane < need) {
          for (uint32_t probe = 0; probe < 64 && !got; ++probe) {
            got = visit(vis, id);
            if (!got) id = id + 1 == g.n ? 0 : id + 1;
          }
        }
        const unsigned gm = __ballot_sync(kFull, got);
        if (got) s.pid[size + __popc(gm & lanemask_lt)] = id;
        size += __popc(gm);
      }
    }
    if (vis.spilled && !vis.bits) status = kStatusVisitedFull;
    __syncwarp();
    eval_candidates<NB>(g, qs, s.pid, s.pk, size, lane);
    ndc += size;
    __syncwarp();
    // sort by (key, position)
    uint64_t x[PITEMS];
#pragma unroll
    for (int i = 0; i < PITEMS; ++i) {
      const int e = i * 32 + lane;
      x[i] = e < size ? (((uint64_t)s.pk[e] << 32) | (uint32_t)e) : kInvalidKey;
    }
    warp_sort<PITEMS>(x, lane);
    uint32_t sid[PITEMS];
#pragma unroll
    for (int i = 0; i < PITEMS; ++i) {
      const int e = i * 32 + lane;
      sid[i] = e < size ? s.pid[(uint32_t)x[i]] : 0u;
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < PITEMS; ++i) {
      const int e = i * 32 + lane;
      if (e < size) {
        s.pk[e] = (uint32_t)(x[i] >> 32);
        s.pid[e] = sid[i];
      }
    }
    __syncwarp();
    if (lane == 0) ctl->size[warp] = size;
  }

  // --- best-first loop, then (ET) stealing rounds
  bool voted = false, need_identify = true, dup_check = false;
  const bool is_et = et != 0;
  for (int phase = 0; phase < 2 && status == kStatusOk; ++phase) {
    if (phase == 1) {
      // ET: a warp that is not the winner continues while the winner runs
      // (SearchUntilBestThreadStop, annsearch.cpp:1368-1455): it copies every
      // unexplored entry of one good warp (up to 10 random draws), then a few
      // of a second random good warp, and goes on from its own pool.
      if (!is_et || uniform_load(&ctl->finish, lane)) break;
      const unsigned long long best = uniform_load(&ctl->best, lane);
      if (best != ~0ull && (int)(best & 0xFFFFFFFFu) == warp) break;
      need_identify = false;  // the stealing loop has no election (:1417-1454)
      dup_check = true;
      int target = -1;
      for (int round = 0; round < 10 && target < 0; ++round) {
        if (uniform_load(&ctl->finish, lane)) break;
        const int t = (int)(scatter_rng(seed, q_idx, warp, 100000u + round) % (uint32_t)W);
        if (t != warp && uniform_load(&ctl->reached[t], lane) && uniform_load(&ctl->good[t], lane))
          target = t;
      }
      const int peek = (int)(scatter_rng(seed, q_idx, warp, 100010u) % (uint32_t)W);
      int taken = 0;
      for (int round = 0; round < 2; ++round) {
        const int t = round == 0 ? target : peek;
        if (t < 0 || t == warp) continue;
        if (round == 1 && !(uniform_load(&ctl->reached[t], lane) && uniform_load(&ctl->good[t], lane)))
          continue;
        const WarpSmem src = carve(t);
        const int tsize = uniform_load(&ctl->size[t], lane);
        // the first round takes all; the peek takes entries until 21 were
        // taken in both rounds together, at least one (:1402-1412)
        int left = round == 0 ? L : max(1, 21 - taken);
        for (int b = tsize - 1; b >= 1 && left > 0 && size > 0; b -= 32) {
          const int got = scatter_take_window(src, ctl, t, s, b, left, lane);
          taken += got;
          left -= got;
          if (got == 0) continue;
          const uint32_t thr = s.pk[size - 1];
          const int na = accept_candidates<RCH>(s, got, size, thr, true, lane, true);
          if (na == 0) continue;
          __syncwarp();
          uint32_t nkey[RCH], nid[RCH];
          int npos[RCH];
          accepted_positions<RCH>(s, na, lane, nkey, nid, npos, size);
          int pmin = npos[0];
#pragma unroll
          for (int c = 1; c < RCH; ++c) pmin = min(pmin, npos[c]);
          const int p0 = (int)__reduce_min_sync(kFull, (uint32_t)pmin);
          if (lane == 0) atomicAdd(&ctl->version[warp], 1u);
          __threadfence_block();
          int sz = size;
          merge_accepted<RCH>(s, sz, na, p0, size, nkey, nid, npos, lane);  // size kept
          __threadfence_block();
          if (lane == 0) atomicAdd(&ctl->version[warp], 1u);
        }
      }
    }
    for (;;) {
      if (is_et) {
        if (uniform_load(&ctl->finish, lane)) break;
        if (hops == (uint32_t)kElectionHop && !voted) {
          voted = true;
          const uint32_t kth = size >= K ? s.pk[K - 1] : 0xFFFFFFFFu;
          if (lane == 0) {
            atomicMin(&ctl->best, ((unsigned long long)kth << 32) | (unsigned)warp);
            ctl->reached[warp] = 1;
            __threadfence_block();
            atomicAdd(&ctl->decided, 1);
          }
          __syncwarp();
        }
        if (need_identify && uniform_load(&ctl->decided, lane) == W) {
          need_identify = false;
          const unsigned long long best = uniform_load(&ctl->best, lane);
          const uint32_t bk = (uint32_t)(best >> 32);
          if (size > 0 && bk < s.pk[0]) break;                      // a losing warp stops
          if (size > 0 && bk > s.pk[0] && lane == 0) ctl->good[warp] = 1;
        }
      }
      // first unexplored slot
      int k = -1;
      for (int b0 = 0; b0 < size; b0 += 32) {
        const int idx = b0 + lane;
        const bool un = idx < size && !(s.pid[idx] & kExplored);
        const unsigned bm = __ballot_sync(kFull, un);
        if (bm) {
          k = b0 + __ffs(bm) - 1;
          break;
        }
      }
      if (k < 0) break;
      if (hops >= a.max_hops) {
        status = kStatusHopLimit;
        break;
      }
      // the next unexplored slot's adjacency row is likely the next hop's:
      // send it to L2 now
      for (int b0 = k + 1; b0 < size; b0 += 32) {
        const int idx = b0 + lane;
        const bool un = idx < size && !(s.pid[idx] & kExplored);
        const unsigned bm = __ballot_sync(kFull, un);
        if (bm) {
          const int u = b0 + __ffs(bm) - 1;
          const uint32_t unode = s.pid[u] & ~kExplored;
          if (lane == 0) prefetch_adj_l2(g, unode);
          break;
        }
      }
      // A stealing warp may mark slot k explored after the ballot above (the
      // entry is then its to expand), so the slot is read once, by lane 0,
      // and skipped when taken; the node id never carries the explored bit.
      const uint32_t raw = uniform_load(&s.pid[k], lane);
      if (raw & kExplored) continue;
      const uint32_t node = raw;
      const uint32_t thr = s.pk[size - 1];
      __syncwarp();
      if (lane == 0) s.pid[k] = node | kExplored;
      ++hops;
      uint32_t row[RCH];
      load_row<RCH>(g, node, lane, row);
      scatter_reserve(vis, ctl, (int)g.rstride, lane);
      if (vis.spilled && !vis.bits) {
        status = kStatusVisitedFull;
        break;
      }
      int nc = 0;
#pragma unroll
      for (int c = 0; c < RCH; ++c) {
        const bool valid = row[c] != kNoneId;
        const unsigned peers = __match_any_sync(kFull, row[c]);
        const bool leader = valid && (peers & lanemask_lt) == 0u;
        const bool fresh = leader && visit(vis, row[c]);
        const unsigned fm = __ballot_sync(kFull, fresh);
        if (fresh) s.cid[nc + __popc(fm & lanemask_lt)] = row[c];
        nc += __popc(fm);
      }
      if (nc == 0) continue;
      __syncwarp();
      // the candidate rows go to L2 first: the distance loads read each row
      // in groups of 8 blocks, and the groups after the first (and the
      // second 16-row pass) then find their lines there
      prefetch_rows(g, s.cid, nc, lane);
      eval_candidates<NB>(g, qs, s.cid, s.ckey, nc, lane);
      ndc += nc;
      __syncwarp();
      const int na = accept_candidates<RCH>(s, nc, size, thr, dup_check, lane);
      if (na == 0) continue;
      __syncwarp();
      uint32_t nkey[RCH], nid[RCH];
      int npos[RCH];
      accepted_positions<RCH>(s, na, lane, nkey, nid, npos, L);
      int pmin = npos[0];
#pragma unroll
      for (int c = 1; c < RCH; ++c) pmin = min(pmin, npos[c]);
      const int p0 = (int)__reduce_min_sync(kFull, (uint32_t)pmin);
      if (lane == 0) atomicAdd(&ctl->version[warp], 1u);
      __threadfence_block();
      merge_accepted<RCH>(s, size, na, p0, L, nkey, nid, npos, lane);
      __threadfence_block();
      if (lane == 0) {
        ctl->size[warp] = size;
        atomicAdd(&ctl->version[warp], 1u);
      }
    }
    if (phase == 0 && is_et) {
      // the winner finishing stops everyone
      const unsigned long long best = uniform_load(&ctl->best, lane);
      if (best != ~0ull && (int)(best & 0xFFFFFFFFu) == warp && lane == 0)
        atomicExch(&ctl->finish, 1);
    }
  }
  if (lane == 0) {
    atomicAdd(&ctl->ndc, ndc);
    atomicAdd(&ctl->hops, hops);
    atomicMax(&ctl->ndc_max, ndc);
    atomicMin(&ctl->ndc_min, ndc);
    if (status != kStatusOk) atomicExch(&ctl->status, status);
  }
  __syncthreads();

  // --- merge: the K best of all pools, one copy per id (warp 0; lane w
  // follows pool w)
  if (warp == 0) {
    uint32_t *oid = a.ids + off;
    float *od = a.dists ? a.dists + off : nullptr;
    const WarpSmem mine = carve(lane < W ? lane : 0);
    const int msize = lane < W ? ctl->size[lane] : 0;
    int head = 0, out = 0;
    uint32_t last = kNoneId;
    while (out < K) {
      const uint64_t v = head < msize ? (((uint64_t)mine.pk[head] << 32) |
                                         (mine.pid[head] & ~kExplored))
                                      : kInvalidKey;
      uint64_t mn = v;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const uint64_t other = shfl_xor_u64(mn, o);
        mn = other < mn ? other : mn;
      }
      if (mn == kInvalidKey) break;
      const unsigned who = __ballot_sync(kFull, v == mn);
      if (lane == __ffs(who) - 1) ++head;
      const uint32_t id = (uint32_t)mn;
      if (id != last) {
        if (lane == 0) {
          oid[out] = id;
          if (od) od[out] = key_to_float((uint32_t)(mn >> 32));
        }
        ++out;
        last = id;
      }
    }
    for (int i = out + lane; i < K; i += 32) {
      oid[i] = 0u;
      if (od) od[i] = 0.f;
    }
  }
  if (ctl->vis_spilled && vis.bits) {
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < a.spill_words; w += blockDim.x) vis.bits[w] = 0u;
  }
  if (threadIdx.x == 0) {
    if (a.ndc) a.ndc[q_idx] = ctl->ndc;
    if (a.hops) a.hops[q_idx] = ctl->hops;
    if (a.ndc_max) a.ndc_max[q_idx] = ctl->ndc_max;
    if (a.ndc_min) a.ndc_min[q_idx] = ctl->ndc_min;
    if (a.status) a.status[q_idx] = ctl->status;
  }
}

// ----------------------------------------------------------- dispatch ---
using WarpFn = void (*)(GraphView, BatchArgs, SmemPlan, CUtensorMap);
using IntraFn = void (*)(GraphView, BatchArgs, SmemPlan, int);

template <int RCH, bool DEEP>
WarpFn warp_fn_for_nb(uint32_t nb) {
  switch (nb) {
    case 8: return warp_search_kernel<8, RCH, DEEP>;
    case 12: return warp_search_kernel<12, RCH, DEEP>;
    case 16: return warp_search_kernel<16, RCH, DEEP>;
    case 25: return warp_search_kernel<25, RCH, DEEP>;
    default: return warp_search_kernel<0, RCH, DEEP>;
  }
}
template <int RCH>
IntraFn intra_fn_for_nb(uint32_t nb) {
  switch (nb) {
    case 8: return intra_search_kernel<8, RCH>;
    case 12: return intra_search_kernel<12, RCH>;
    case 16: return intra_search_kernel<16, RCH>;
    case 25: return intra_search_kernel<25, RCH>;
    default: return intra_search_kernel<0, RCH>;
  }
}

using ScatterFn = void (*)(GraphView, BatchArgs, SmemPlan, int, int, uint64_t);

template <int RCH>
ScatterFn scatter_fn_for_pool(uint32_t pool_cap) {
  switch (pool_cap) {
    case 32: return scatter_search_kernel<0, RCH, 1>;
    case 64: return scatter_search_kernel<0, RCH, 2>;
    case 128: return scatter_search_kernel<0, RCH, 4>;
    case 256: return scatter_search_kernel<0, RCH, 8>;
    default: return scatter_search_kernel<0, RCH, 16>;
  }
}
ScatterFn scatter_fn(const GraphView &g, uint32_t pool_cap) {
  const uint32_t rch = (g.rstride + 31) / 32;
  if (rch <= 1) return scatter_fn_for_pool<1>(pool_cap);
  if (rch <= 2) return scatter_fn_for_pool<2>(pool_cap);
  return scatter_fn_for_pool<4>(pool_cap);
}

// The DEEP instantiations (stages of more than 16 rows) are separate kernels,
// so the code of the common 16-row kernel is unchanged by them.
WarpFn warp_fn(const GraphView &g, const SmemPlan &p) {
  const uint32_t rch = (g.rstride + 31) / 32;
  const bool deep = p.stage_rows > (uint32_t)kStageRows;
  if (rch <= 1) return deep ? warp_fn_for_nb<1, true>(g.nb) : warp_fn_for_nb<1, false>(g.nb);
  if (rch <= 2) return deep ? warp_fn_for_nb<2, true>(g.nb) : warp_fn_for_nb<2, false>(g.nb);
  return deep ? warp_fn_for_nb<4, true>(g.nb) : warp_fn_for_nb<4, false>(g.nb);
}
IntraFn intra_fn(const GraphView &g) {
  const uint32_t rch = (g.rstride + 31) / 32;
  if (rch <= 1) return intra_fn_for_nb<1>(g.nb);
  if (rch <= 2) return intra_fn_for_nb<2>(g.nb);
  return intra_fn_for_nb<4>(g.nb);
}

uint32_t round_up(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }
uint32_t pow2_at_least(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}
uint32_t log2_of(uint32_t p) {
  uint32_t l = 0;
  while ((1u << l) < p) ++l;
  return l;
}

}  // namespace

SmemPlan plan_warp_smem(const GraphView &g, int L_max, int hash_cap_override, int stage_rows) {
  SmemPlan p{};
  p.q_words = g.nb * 8;
  p.pool_cap = round_up((uint32_t)L_max, 32);
  p.cand_cap = round_up(g.rstride, 32);
  // Visited table: buckets of 8 tags.  It may forget (see QHash), so its
  // size trades shared memory (teams resident per SM) against repeated
  // distance evaluations; the default, 2 slots per unit of L and at least
  // 1024, measured fastest on the 1.2M x 200 workload at L = 200 and 400.
  uint32_t slots = hash_cap_override > 0 ? pow2_at_least((uint32_t)hash_cap_override)
                                         : pow2_at_least((uint32_t)L_max * 2u);
  if (slots < 1024 && hash_cap_override <= 0) slots = 1024;
  if (slots < 512) slots = 512;
  if (slots > 65536) slots = 65536;
  uint32_t bbits = log2_of(slots / 8);
  uint32_t nbits = 1;
  while (nbits < 32 && (1ull << nbits) < (unsigned long long)g.n) ++nbits;
  // tags hold at most 14 remainder bits (bit 15 = second choice, 0xFFFF = empty)
  if (nbits > bbits + 14) bbits = nbits - 14;
  p.hash_log2 = bbits;
  p.qh_rbits = nbits > bbits ? nbits - bbits : 0;
  p.hash_cap = (1u << bbits) * 8;
  p.hash_limit = p.hash_cap;
  // Row stage: 16 whole rows.  Rows so wide that 16 of them would pass 64 KB
  // (over 4 KB each) are staged in two halves, keeping 16 rows per pass at
  // the cost of one L2 round trip per pass (measured slower than whole rows
  // at 200 dims: 546k against 640k queries/s at L = 400), and fewer rows
  // only beyond that.
  uint32_t rows = stage_rows > 0 ? (uint32_t)std::min(stage_rows, kMaxStageRows) : kStageRows;
  p.stage_split = kStageRows * g.nb * 32u > 65536u ? 2 : 1;
  if (p.stage_split > 1) rows = std::min(rows, (uint32_t)kStageRows);  // split rows: 16 at most
  p.stage_row_words = (p.stage_split > 1 ? split_first(g.nb) : g.nb) * 8;
  p.stage_rows = rows;
  while (p.stage_rows > 1 && p.stage_rows * p.stage_row_words * 4u > 65536u) p.stage_rows >>= 1;
  p.stage_words = p.stage_rows * p.stage_row_words;
  p.shared_stages = 0;
  // gather4 copies (four whole rows each) need rows of at most 256 floats (a
  // tensor-map box) and a stage of a multiple of 4 rows
  p.gather = (p.stage_split == 1 && g.nb * 8u <= 256u && p.stage_rows % 4u == 0u) ? 1u : 0u;
  p.words_per_team = p.stage_words + 4 + p.q_words + 2 * p.pool_cap + 5 * p.cand_cap +
                     (1u << bbits) * 4 + evict_words(bbits);
  p.words_per_team = round_up(p.words_per_team, 32);  // 128-byte aligned stages
  return p;
}

void share_stages(SmemPlan &p, int stages) {
  const uint32_t rest = p.q_words + 2 * p.pool_cap + 5 * p.cand_cap + (1u << p.hash_log2) * 4 +
                        evict_words(p.hash_log2);
  if (stages > 0) {
    p.shared_stages = (uint32_t)std::min(stages, 32);
    p.words_per_team = round_up(rest, 32);
  } else {
    p.shared_stages = 0;
    p.words_per_team = round_up(p.stage_words + 4 + rest, 32);
  }
}

size_t warp_search_smem_bytes(const SmemPlan &p, int warps_per_block) {
  return ((size_t)stage_pool_words(p) + (size_t)p.words_per_team * warps_per_block) * 4;
}

SmemPlan plan_intra_smem(const GraphView &g, int L_max, int width, int hash_cap_override) {
  SmemPlan p{};
  p.q_words = g.nb * 8;
  p.pool_cap = round_up((uint32_t)L_max, 32);
  p.cand_cap = round_up(g.rstride, 32);
  uint32_t hc = hash_cap_override > 0 ? pow2_at_least((uint32_t)hash_cap_override)
                                      : pow2_at_least((uint32_t)L_max * 16u * (uint32_t)width);
  if (hc < 1024) hc = 1024;
  if (hc > 16384) hc = 16384;
  p.hash_cap = hc;
  p.hash_log2 = log2_of(hc);
  p.hash_limit = hc - hc / 4;
  const uint32_t st_cap = pow2_at_least((uint32_t)(kStepTableFactor * width) * p.cand_cap);
  p.step_cap = st_cap;
  p.step_log2 = log2_of(st_cap);
  p.words_per_team = p.q_words + 4 * p.pool_cap + p.hash_cap + 2 * st_cap +
                     5 * (uint32_t)width * p.cand_cap + 32 + 64;
  p.words_per_team = round_up(p.words_per_team, 4);
  return p;
}

namespace {
// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum, once per (device, kernel).  Every launch then only has to fit that
// maximum, so concurrent callers planning different sizes never lower the
// limit under one another's launch.
cudaError_t allow_max_smem(const void *fn) {
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
}  // namespace

SmemPlan plan_scatter_smem(const GraphView &g, int L_max, int width) {
  SmemPlan p{};
  p.q_words = g.nb * 8;
  p.pool_cap = pow2_at_least(std::max<uint32_t>(32u, (uint32_t)L_max));
  p.cand_cap = round_up(g.rstride, 32);
  p.words_per_team = 2 * p.pool_cap + 5 * p.cand_cap;  // per warp
  p.step_cap = round_up((uint32_t)((sizeof(ScatterCtl) + 3) / 4), 32);
  uint32_t cap = pow2_at_least(std::max<uint32_t>(2048u, (uint32_t)L_max * (uint32_t)width * 8u));
  if (cap > 32768) cap = 32768;
  const uint32_t budget_words = (227u * 1024u) / 4u;
  const uint32_t fixed = p.q_words + p.step_cap + (uint32_t)width * p.words_per_team;
  while (cap > 1024 && fixed + cap > budget_words) cap >>= 1;
  p.hash_cap = cap;
  p.hash_log2 = log2_of(cap);
  const uint32_t reserve = (uint32_t)width * p.cand_cap;
  p.hash_limit = std::min(cap - cap / 4, cap > reserve ? cap - reserve : 0u);
  return p;
}

size_t scatter_smem_bytes(const SmemPlan &p, int width) {
  return (size_t)(p.q_words + p.hash_cap + p.step_cap + (uint32_t)width * p.words_per_team) * 4;
}

cudaError_t launch_scatter_search(const GraphView &g, const BatchArgs &a, const SmemPlan &p,
                                  int width, int et, uint64_t seed, cudaStream_t stream) {
  ScatterFn fn = scatter_fn(g, p.pool_cap);
  cudaError_t e = allow_max_smem((const void *)fn);
  if (e != cudaSuccess) return e;
  if (a.nq == 0) return cudaSuccess;
  fn<<<a.nq, width * 32, scatter_smem_bytes(p, width), stream>>>(g, a, p, width, et, seed);
  return cudaGetLastError();
}

int warp_search_occupancy(const GraphView &g, const SmemPlan &p, int warps_per_block) {
  WarpFn fn = warp_fn(g, p);
  const size_t smem = warp_search_smem_bytes(p, warps_per_block);
  if (allow_max_smem((const void *)fn) != cudaSuccess) return 0;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, (const void *)fn, warps_per_block * 32,
                                                    smem) != cudaSuccess)
    return 0;
  return blocks;
}

namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                   const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                   const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// The driver's cuTensorMapEncodeTiled, looked up once through the runtime
// (no link against the driver library); null when unavailable.
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}
}  // namespace

// Tensor map of the base rows for gather4 copies: a 2-D float32 tensor of
// n rows of nb*8 floats (the padded row, stride nb*32 bytes), box = one whole
// row.  Host-only (no device call); false when the rows do not qualify.
bool encode_row_map(const GraphView &g, CUtensorMap *m) {
  if (g.nb * 8u > 256u || g.n == 0 || (reinterpret_cast<uintptr_t>(g.base) & 15u) != 0) return false;
  EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)g.nb * 8u, (cuuint64_t)g.n};
  const cuuint64_t strides[1] = {(cuuint64_t)g.nb * 32u};
  const cuuint32_t box[2] = {g.nb * 8u, 1u};
  const cuuint32_t estr[2] = {1u, 1u};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(g.base), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

cudaError_t launch_warp_search(const GraphView &g, const BatchArgs &a, const SmemPlan &p,
                               int warps_per_block, int blocks, cudaStream_t stream) {
  WarpFn fn = warp_fn(g, p);
  const size_t smem = warp_search_smem_bytes(p, warps_per_block);
  cudaError_t e = allow_max_smem((const void *)fn);
  if (e != cudaSuccess) return e;
  if (blocks <= 0) blocks = (int)((a.nq + warps_per_block - 1) / warps_per_block);
  if (blocks <= 0) return cudaSuccess;
  // gather4 staging when the plan allows it and the rows encode as a map
  // (the map is re-encoded per launch: a few microseconds of host work)
  SmemPlan q = p;
  CUtensorMap rows;
  std::memset(&rows, 0, sizeof(rows));
  if (q.gather && (q.stage_split != 1 || q.stage_rows % 4u != 0u || !encode_row_map(g, &rows)))
    q.gather = 0;
  fn<<<blocks, warps_per_block * 32, smem, stream>>>(g, a, q, rows);
  return cudaGetLastError();
}

cudaError_t launch_intra_search(const GraphView &g, const BatchArgs &a, const SmemPlan &p,
                                int width, cudaStream_t stream) {
  IntraFn fn = intra_fn(g);
  const size_t smem = (size_t)p.words_per_team * 4;
  cudaError_t e = allow_max_smem((const void *)fn);
  if (e != cudaSuccess) return e;
  if (a.nq == 0) return cudaSuccess;
  fn<<<a.nq, width * 32, smem, stream>>>(g, a, p, width);
  return cudaGetLastError();
}

namespace {
// One thread per adjacency row: any id met twice before the padding.
__global__ void __launch_bounds__(256) row_repeats_kernel(const uint32_t *__restrict__ adj,
                                                          uint32_t n, uint32_t rstride,
                                                          uint32_t *flag) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const uint32_t *row = adj + (size_t)r * rstride;
  for (uint32_t i = 1; i < rstride; ++i) {
    const uint32_t a = __ldg(row + i);
    if (a == kNoneId) break;
    for (uint32_t j = 0; j < i; ++j) {
      if (__ldg(row + j) == a) {
        atomicExch(flag, 1u);
        return;
      }
    }
  }
}
}  // namespace

cudaError_t launch_row_repeats(const uint32_t *adj, uint32_t n, uint32_t rstride, uint32_t *flag,
                               cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  row_repeats_kernel<<<(n + 255) / 256, 256, 0, stream>>>(adj, n, rstride, flag);
  return cudaGetLastError();
}

// ------------------------------------------------ allocation-free launch ---
// Scratch of ss_search_batch_noalloc: one file-scope device array per GPU
// that loads the library, held until the process exits.  Layout (4-byte
// words): [0] work-queue head, [1] first failed query, [2, 1 + kStatusKinds)
// failed queries per status code, [64, 64 + max queries) per-query status.
// Every call shares it, so calls whose work overlaps on the GPU race; each
// call resets the parts it uses before its search runs.
namespace {
constexpr size_t kNoallocWords = kNoallocScratchBytes / 4;
constexpr size_t kNoallocStatusAt = 64;
static_assert(kNoallocStatusAt + kNoallocMaxQueries <= kNoallocWords,
              "scratch too small for its status words");
static_assert(1 + kStatusKinds <= kNoallocStatusAt, "counters overlap the status words");

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoallocWords];

// Counts the failed queries of a batch per status code into
// failed[1..kStatusKinds) (zeroed beforehand) and lowers failed[0] (set to
// 0xFFFFFFFF beforehand) to the smallest failed query index.  A code outside
// the known ones counts as invalid arguments.
__global__ void __launch_bounds__(256) count_failed_kernel(const int32_t *status, uint32_t nq,
                                                           uint32_t *failed) {
  uint32_t c[kStatusKinds] = {};
  uint32_t first = 0xFFFFFFFFu;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) {
    const int32_t s = status[i];
    if (s != kStatusOk) {
      first = min(first, i);
#pragma unroll
      for (int k = 1; k < kStatusKinds; ++k)
        c[k] += (s == k) || (k == kStatusBadArgs && (s < 0 || s >= kStatusKinds));
    }
  }
  first = __reduce_min_sync(kFull, first);
  const bool lead = (threadIdx.x & 31) == 0;
  if (lead && first != 0xFFFFFFFFu) atomicMin(failed, first);
#pragma unroll
  for (int k = 1; k < kStatusKinds; ++k) {
    const uint32_t t = __reduce_add_sync(kFull, c[k]);
    if (lead && t) atomicAdd(failed + k, t);
  }
}
}  // namespace

cudaError_t noalloc_scratch(NoallocScratch *out) {
  // Host code cannot use the array's name as a device address (on the host
  // it names a host-side stand-in), so its device address is resolved once
  // per device, with that device current, and cached.
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static uint32_t *addr[kMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  uint32_t *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return e;
      addr[dev] = static_cast<uint32_t *>(p);
    }
    base = addr[dev];
  }
  out->counter = base;
  out->failed = base + 1;
  out->status = reinterpret_cast<int32_t *>(base + kNoallocStatusAt);
  return cudaSuccess;
}

cudaError_t launch_count_failed(const int32_t *status, uint32_t nq, uint32_t *failed,
                                cudaStream_t stream) {
  if (nq == 0) return cudaSuccess;
  const uint32_t blocks = std::min<uint32_t>((nq + 255) / 256, 148);
  count_failed_kernel<<<blocks, 256, 0, stream>>>(status, nq, failed);
  return cudaGetLastError();
}

}  // namespace ssb
