// Internal interface between the host API (ss_api.cpp) and the search
// kernels (ss_search.cu).  Not installed; the public surface is
// include/scattersearch.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

struct ss_index;

namespace ssb {

constexpr uint32_t kNoneId = 0xFFFFFFFFu;

// Device view of one index: base rows padded to nb*8 floats, fixed-stride
// adjacency padded with kNoneId.
struct GraphView {
  const float *base;     // n x (nb*8) floats
  const uint32_t *adj;   // n x rstride
  uint32_t n, dim, nb, rstride, ep;
  int metric;            // 0 = L2, 1 = inner product
  uint32_t row_dups;     // 1 = some adjacency row repeats an id (in-row checks needed)
};

// One batched launch.  Per-query K/L come from Ks/Ls when non-null, else
// K0/L0.  Results of query q start at out_off[q] (or q*K0).
struct BatchArgs {
  const float *queries;  // nq x qstride floats
  uint32_t qstride, nq;
  const int32_t *Ks, *Ls;
  int32_t K0, L0;
  const int64_t *out_off;
  uint32_t *ids;
  float *dists;          // may be null
  uint32_t *ndc, *hops;  // may be null
  uint32_t *ndc_max, *ndc_min;  // scatter kernel: per query, one warp's most / fewest
                                // distance evaluations (may be null)
  int32_t *status;       // nq entries, may be null
  uint32_t *work_counter;  // persistent work queue head; null = static schedule
  uint32_t *spill_bits;    // per-slot visited bitsets, spill_words each
  uint32_t spill_words;
  uint32_t max_hops;
  // warp kernel: exact visited marks per team slot (blockIdx * teams + team):
  // one byte per base row holding the epoch of the slot's query that
  // visited it, mark_stride bytes per slot; mark_epoch[slot] = the slot's
  // last epoch.  Null = the shared-memory table alone.
  uint8_t *marks;
  uint32_t *mark_epoch;
  uint32_t mark_stride;
};

// Per-team shared-memory plan (sizes in 4-byte words, all multiples of 4).
struct SmemPlan {
  uint32_t q_words;     // nb*8
  uint32_t pool_cap;    // >= max L of the launch, multiple of 32
  uint32_t cand_cap;    // candidates per step (multiple of 32)
  uint32_t hash_cap;    // slots, power of two
  uint32_t hash_log2;   // intra kernel: log2(slots); warp kernel: log2(buckets of 8)
  uint32_t hash_limit;  // entries before spilling to the global bitset
  uint32_t qh_rbits;    // warp kernel: tag remainder bits of the visited hash
  uint32_t step_cap;    // CTA kernel: step-local dedupe table (power of two)
  uint32_t step_log2;
  uint32_t stage_rows;  // warp kernel: rows of the shared-memory row stage
  uint32_t stage_split; // warp kernel: 1 = whole rows, 2 = rows staged in two halves
  uint32_t stage_row_words;  // warp kernel: floats per staged row
  uint32_t stage_words; // warp kernel: size of the row stage
  uint32_t shared_stages;  // warp kernel: row stages shared by a CTA's teams (0 = one per team)
  uint32_t gather;      // warp kernel: whole rows staged by gather4 copies (set at launch)
  uint32_t words_per_team;
};

// Query status codes written to BatchArgs::status.
enum : int32_t {
  kStatusOk = 0,
  kStatusBadArgs = 1,
  kStatusHopLimit = 2,
  kStatusVisitedFull = 3,
  kStatusStageTimeout = 4,  // a shared-memory row stage was not filled within its wait limit
  kStatusKinds = 5          // number of status codes
};

// Plans shared memory for a warp-per-query launch.
// stage_rows: rows of the row stage (0 = 16, the most one pass computes).
SmemPlan plan_warp_smem(const GraphView &g, int L_max, int hash_cap_override, int stage_rows = 0);
// Lets the teams of a CTA share `stages` row stages (0: a private stage per
// team); updates words_per_team.
void share_stages(SmemPlan &p, int stages);
// Dynamic shared memory of a warp-kernel CTA of `warps_per_block` teams.
size_t warp_search_smem_bytes(const SmemPlan &p, int warps_per_block);
// Plans shared memory for a CTA-per-query launch with `width` expansion warps.
SmemPlan plan_intra_smem(const GraphView &g, int L_max, int width, int hash_cap_override);

// Launch helpers.  Return cudaSuccess or the launch error.
//   warps_per_block: teams per CTA; blocks: grid size (0 = one per team
//   needed for nq with a static schedule).
// Sets *flag (device word, zeroed by the caller) to 1 when some row of the
// adjacency (n rows of rstride ids, kNoneId padding) repeats an id.
cudaError_t launch_row_repeats(const uint32_t *adj, uint32_t n, uint32_t rstride, uint32_t *flag,
                               cudaStream_t stream);

// Stages whole rows with gather4 copies when p.gather is set and the base
// rows encode as a tensor map (rows of at most 256 floats, 16-byte aligned
// base); otherwise with one bulk copy per row.
cudaError_t launch_warp_search(const GraphView &g, const BatchArgs &a, const SmemPlan &p,
                               int warps_per_block, int blocks, cudaStream_t stream);
cudaError_t launch_intra_search(const GraphView &g, const BatchArgs &a, const SmemPlan &p,
                                int width, cudaStream_t stream);

// ScatterSearch's intra-query search: one CTA of `width` warps per query,
// each warp with its own pool (et: election and early termination).
SmemPlan plan_scatter_smem(const GraphView &g, int L_max, int width);
size_t scatter_smem_bytes(const SmemPlan &p, int width);
cudaError_t launch_scatter_search(const GraphView &g, const BatchArgs &a, const SmemPlan &p,
                                  int width, int et, uint64_t seed, cudaStream_t stream);

// Resident CTAs per SM for the warp kernel with this plan (0 if it cannot run).
int warp_search_occupancy(const GraphView &g, const SmemPlan &p, int warps_per_block);

// Scratch of the allocation-free batched search: a static device array of
// kNoallocScratchBytes per GPU (sizes mirrored by SS_NOALLOC_* in
// include/scattersearch.h): 256 bytes of counters, then one status word per
// query.
constexpr uint32_t kNoallocMaxQueries = 65536;
constexpr size_t kNoallocScratchBytes = 256 + size_t(4) * kNoallocMaxQueries;
struct NoallocScratch {
  uint32_t *counter;  // persistent work-queue head
  uint32_t *failed;   // kStatusKinds words: [c] = queries with status c (c >= 1),
                      // [0] = index of the first failed query (0xFFFFFFFF: none)
  int32_t *status;    // kNoallocMaxQueries entries
};
// Device addresses of the scratch on the current device.  The first call on
// a device resolves them (cudaGetSymbolAddress); later calls only read a
// cache.
cudaError_t noalloc_scratch(NoallocScratch *out);
// Counts the failed queries of status[0..nq) per status code into
// failed[1..kStatusKinds) and lowers failed[0] to the smallest failed index
// (failed[] as in NoallocScratch, set up by the caller beforehand).
cudaError_t launch_count_failed(const int32_t *status, uint32_t nq, uint32_t *failed,
                                cudaStream_t stream);

// ---- brute-force k-NN (ss_bruteforce.cu) --------------------------------
struct BruteArgs {
  const float *base;      // n x (nb*8), padded rows (exact re-rank)
  uint32_t n, nb;
  const float *queries;   // nq x (nb*8), padded with zeros (exact re-rank)
  uint32_t nq;
  const float *qpack;     // queries in packed tensor-core tiles (launch_pack)
  const float *bpack;     // base rows in packed tensor-core tiles
  uint32_t kblocks;       // 32-float k-blocks per row
  const float *xnorm;     // n squared norms (L2 only)
  int metric;
  int k, C;               // results per query; candidates kept per list (32/64/128)
  uint32_t splits, rows_per_split;
  uint32_t lists, list_stride;  // candidate lists per query (BrutePlan::lists); entries per list
  uint64_t *cand;         // nq x lists x list_stride scratch
  uint32_t *ids;          // nq x k
  float *dists;           // nq x k, may be null
  uint32_t *err;          // set to 1 when a bounded wait ran out; may be null
};
struct BrutePlan {
  int C;
  uint32_t list_cap;      // entries per candidate list
  uint32_t splits, rows_per_split;
  uint32_t lists;         // candidate lists per query (a fixed number per split)
  uint32_t kblocks;
};
// Largest k the brute force accepts (candidates kept = k + 16 <= 128).
constexpr int kBruteMaxK = 112;
BrutePlan plan_bruteforce(uint32_t n, uint32_t nq, int k, int sm_count);
uint32_t bruteforce_kblocks(uint32_t dim);
// Bytes of `rows` rows of width `dim` in packed tensor-core tiles (base side:
// 256-row tiles; query side: 128-row tiles).
size_t bruteforce_pack_bytes(uint32_t rows, uint32_t dim, bool base_side);
cudaError_t launch_pack(const float *src, uint32_t rows, uint32_t pitch, uint32_t dim,
                        bool base_side, float *dst, cudaStream_t s);
cudaError_t launch_norms(const float *base, uint32_t n, uint32_t pitch, float *out,
                         cudaStream_t s);
cudaError_t launch_bruteforce(const BruteArgs &a, const GraphView &g, cudaStream_t s);

// ---- host-side hooks of the C ABI layer (ss_api.cpp) used by the serving
// loop (ss_server.cpp).  `ss_index` is the opaque handle of
// include/scattersearch.h.
int index_device(const ::ss_index *h);
uint32_t index_dim(const ::ss_index *h);
bool index_ready(const ::ss_index *h);
// Records `msg` as the handle's last error and returns `code`.
int index_error(::ss_index *h, int code, const char *msg);
// Enqueues one batched search of nq device-resident queries with per-query K
// and L (device arrays) on `stream`; results of query i start at d_off[i].
// d_status (nq words) and d_counter (1 word) are scratch owned by the caller.
int server_launch(::ss_index *h, const float *d_q, uint32_t nq, const int32_t *d_K,
                  const int32_t *d_L, const int64_t *d_off, int L_max, uint32_t *d_ids,
                  float *d_dists, int32_t *d_status, uint32_t *d_counter, cudaStream_t stream);

}  // namespace ssb
