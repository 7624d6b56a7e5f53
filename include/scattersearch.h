/*
 * scattersearch.h -- C ABI of the B200 graph search library
 * (libscattersearch_b200.so).
 *
 * The reference (ScatterSearch) is a C++ class, ANNSearch
 * (include/annsearch.h:37-84), used in-process by its benchmark drivers.  Each
 * entry point below replaces one member of that class or one loop of its
 * drivers; the comment on each names the reference code it replaces.
 * include/scattersearch/annsearch.hpp wraps these calls in a header-only C++
 * class with the reference's member names, so reference-style drivers compile
 * against it unchanged.
 *
 * Conventions
 *   - Every call returns an ss_status (0 = SS_OK).  On failure the message is
 *     available from ss_last_error(handle) (or ss_last_error(NULL) for calls
 *     that failed before a handle existed).  No C++ exception crosses the ABI.
 *   - Host pointers are plain caller-owned buffers.  Calls with a _device
 *     suffix take device pointers and a cudaStream_t passed as void*.
 *   - A handle may be shared by several host threads: concurrent ss_search /
 *     ss_search_batch calls on one handle are safe (each call borrows its own
 *     stream and staging buffers).  Graph loading must not overlap searches.
 *   - Metric values follow the reference's enum Metric {L2, INNER_PRODUCT}
 *     (include/annsearch.h:22-26).  Inner-product distances are returned
 *     negated, as distance_ip_avx does (src/distance.cpp:148).
 *   - Result slots the search never filled (only possible on tiny or
 *     disconnected graphs) hold id 0 and distance 0, the value-initialised
 *     Neighbor of src/annsearch.cpp:193.
 */
#ifndef SCATTERSEARCH_H
#define SCATTERSEARCH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ss_index ss_index;

enum ss_metric { SS_METRIC_L2 = 0, SS_METRIC_INNER_PRODUCT = 1 };

enum ss_status {
  SS_OK = 0,
  SS_ERR_INVALID_ARGUMENT = 1, /* bad size, K > L, null pointer, ...           */
  SS_ERR_IO = 2,               /* file could not be opened or read            */
  SS_ERR_FORMAT = 3,           /* malformed .nsg / .fbin / ground-truth file  */
  SS_ERR_NO_GRAPH = 4,         /* search before a graph was loaded            */
  SS_ERR_CUDA = 5,             /* CUDA runtime error (message has details)    */
  SS_ERR_OUT_OF_MEMORY = 6,    /* device or host allocation failed            */
  SS_ERR_UNSUPPORTED = 7,      /* parameter outside the compiled limits       */
  SS_ERR_SEARCH_LIMIT = 8,     /* a query hit the device hop limit            */
  SS_ERR_BUSY = 9,             /* the server's request queue is full          */
  SS_ERR_TIMEOUT = 10          /* a wait for a request ran out of time        */
};

/* Largest beam width (pool size L) and graph degree the kernels accept. */
#define SS_MAX_L 4096
#define SS_MAX_DEGREE 128
/* Largest number of expansions per step of ss_search_intra. */
#define SS_MAX_INTRA_WIDTH 16

/* ---- index lifetime ---------------------------------------------------- */

/* Replaces ANNSearch::ANNSearch(unsigned dim, unsigned num, float *base,
 * Metric m) (include/annsearch.h:40, src/annsearch.cpp:11-58).  Unlike the
 * reference, which borrows `base`, the rows are copied into device memory
 * (zero-padded to a multiple of 8 floats); the caller may free `base_host`
 * after the call.  device: CUDA ordinal, or -1 for the current device. */
int ss_create(uint32_t dim, uint32_t num, const float *base_host, int metric, int device,
              ss_index **out);

/* Same, with `base_dev` already on the device (num x dim floats, row-major,
 * 16-byte aligned).  The rows are copied; the caller keeps ownership. */
int ss_create_from_device(uint32_t dim, uint32_t num, const float *base_dev, int metric,
                          int device, ss_index **out);

/* Replaces ANNSearch::~ANNSearch (src/annsearch.cpp:60-62).  Frees every
 * device allocation of the handle.  NULL is ignored. */
void ss_destroy(ss_index *h);

/* ---- graph ----------------------------------------------------------- */

/* Replaces ANNSearch::LoadGraph (src/annsearch.cpp:64-80).  Reads the NSG
 * file format: u32 width (ignored), u32 entry point, then per node u32 k and
 * k u32 neighbour ids, until end of file.  Unlike the reference, a missing
 * file, a truncated record, a node count different from `num`, or an id
 * >= num is reported (SS_ERR_IO / SS_ERR_FORMAT) instead of ignored. */
int ss_load_graph(ss_index *h, const char *path);

/* Sets the graph from memory; replaces assigning the public members
 * `graph` and `default_ep` (include/annsearch.h:77, :82).  adj is n x
 * rstride uint32 on the host; each row is a prefix of neighbour ids followed
 * by 0xFFFFFFFF padding.  n must equal the index's num. */
int ss_set_graph(ss_index *h, const uint32_t *adj, uint32_t n, uint32_t rstride,
                 uint32_t entry_point);

/* Reads back the graph shape: node count, largest degree, entry point
 * (default_ep, include/annsearch.h:77) and the padded row stride used on the
 * device.  Any output pointer may be NULL. */
int ss_graph_info(const ss_index *h, uint32_t *n, uint32_t *max_degree, uint32_t *entry_point,
                  uint32_t *rstride);

/* Copies the device adjacency back to the host (n x rstride uint32). */
int ss_get_graph(ss_index *h, uint32_t *adj, uint32_t rstride);

/* ---- search ------------------------------------------------------------ */

/* Replaces ANNSearch::SearchArraySimulation(query, query_id, K, L, flags,
 * indices) (src/annsearch.cpp:182-259): best-first search from the entry
 * point with a pool of L, returning the K nearest in ascending distance.
 * The visited set lives on the device, so the reference's caller-owned
 * `flags` bitset has no counterpart.  One query per launch: this is the
 * plain per-query GPU path.  ids: K uint32; dists: K floats (may be NULL).
 * Requires 1 <= K <= L <= SS_MAX_L. */
int ss_search(ss_index *h, const float *query, int K, int L, uint32_t *ids, float *dists);

/* Replaces the drivers' query loop around SearchArraySimulation
 * (tests/search.cpp:75-85; race-free per-thread visited sets as in
 * tests/intraxinter.cpp:74-86).  All nq queries go to one persistent kernel
 * that pulls queries from a device work queue; results are identical to nq
 * calls of ss_search.  queries: nq x dim; ids/dists: nq x K. */
int ss_search_batch(ss_index *h, const float *queries, uint32_t nq, int K, int L, uint32_t *ids,
                    float *dists);

/* Batched search with per-query K and L (Ks[i], Ls[i]); query i's results
 * start at offset sum(Ks[0..i)) of ids/dists.  Results are identical to
 * ss_search(query i, Ks[i], Ls[i]). */
int ss_search_batch_uneven(ss_index *h, const float *queries, uint32_t nq, const int32_t *Ks,
                           const int32_t *Ls, uint32_t *ids, float *dists);

/* Device-resident batched search on `stream` (a cudaStream_t, NULL for the
 * legacy default stream); asynchronous: returns after enqueueing.
 * queries: nq x dim floats on the device.  Either (Ks, Ls, out_off) are
 * device arrays of length nq, or they are NULL and K, L apply to all queries
 * with query i's results at i*K.  ndc / hops (device, nq uint32, may be NULL)
 * receive each query's distance evaluations and expansions.  Validation of
 * per-query K/L happens on the device: a query with invalid K/L or one that
 * hits the hop limit leaves its status nonzero, readable with
 * ss_batch_status. */
int ss_search_batch_device(ss_index *h, const float *queries, uint32_t nq, const int32_t *Ks,
                           const int32_t *Ls, const int64_t *out_off, int K, int L, int L_max,
                           uint32_t *ids, float *dists, uint32_t *ndc, uint32_t *hops,
                           void *stream);

/* Graph-captured batched search.  No counterpart in the reference.
 * ss_plan_create records one ss_search_batch_device launch (uniform K and
 * L; queries, ids and dists are fixed device buffers; dists may be NULL) --
 * the work-queue reset, the status reset and the persistent search kernel --
 * into a CUDA graph; ss_plan_launch replays it on `stream` with one graph
 * launch.  The plan owns its status words, work-queue head and visited
 * marks (ss_set_visited_marks; allocated and cleared at creation):
 * ss_plan_status reports the failed queries of its last synchronised
 * replay, and replays of one plan must not overlap on the GPU (order them
 * on one stream, or use one plan per stream).  Buffers must stay valid while
 * the plan exists; rewrite the query buffer between replays to search new
 * queries. */
typedef struct ss_plan ss_plan;
int ss_plan_create(ss_index *h, const float *queries, uint32_t nq, int K, int L, uint32_t *ids,
                   float *dists, ss_plan **out);
/* Same for a batch with per-query K and L: Ks, Ls and out_off are device
 * arrays of nq entries, as for ss_search_batch_device; L_max bounds Ls. */
int ss_plan_create_uneven(ss_index *h, const float *queries, uint32_t nq, const int32_t *Ks,
                          const int32_t *Ls, const int64_t *out_off, int K, int L, int L_max,
                          uint32_t *ids, float *dists, ss_plan **out);
int ss_plan_launch(ss_plan *p, void *stream);
int ss_plan_status(ss_plan *p, uint32_t *failed_queries);
void ss_plan_destroy(ss_plan *p);

/* After a synchronised ss_search_batch_device: number of queries of the last
 * device batch on this handle whose status was nonzero. */
int ss_batch_status(ss_index *h, uint32_t *failed_queries);

/* Allocation-free batched search.  No counterpart in the reference, which
 * runs on the host.  It exists for callers that must not allocate device
 * memory: a process whose device memory belongs to a host framework's pool
 * allocator with a fixed budget, or a latency-critical serving loop where the
 * device-wide synchronisation of cudaMalloc/cudaFree would stall other work.
 * Same search and results as ss_search_batch_device with uniform K and L
 * (queries, ids, dists are device pointers; dists may be NULL), but it calls
 * no cudaMalloc, cudaFree or allocating library routine: its scratch (work
 * queue head, failure count, per-query status) is one static device array of
 * SS_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until the
 * process exits.
 *   - Limit: nq <= SS_NOALLOC_MAX_QUERIES; a larger batch fails with
 *     SS_ERR_UNSUPPORTED before any work is enqueued.
 *   - The first call on a device sets the scratch up (it resolves the
 *     array's device address), so make that first call before any stream
 *     capture begins.
 *   - Every call, from any handle in the process, shares the one array per
 *     device and each call clears the parts it uses: calls whose work
 *     overlaps on the GPU (other streams, other threads) race and must be
 *     serialised by the caller.
 *   - Enqueued on `stream` (a cudaStream_t, NULL for the legacy default
 *     stream); the call returns once the search has finished.  Failed
 *     queries are reported as ss_search_batch reports them:
 *     SS_ERR_SEARCH_LIMIT for the hop limit or a full visited table,
 *     SS_ERR_TIMEOUT for a row-copy wait that ran out, SS_ERR_INVALID_ARGUMENT
 *     otherwise; ss_last_error names the count and the first failed query. */
#define SS_NOALLOC_MAX_QUERIES 65536
#define SS_NOALLOC_SCRATCH_BYTES (256u + 4u * SS_NOALLOC_MAX_QUERIES)
int ss_search_batch_noalloc(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                            uint32_t *ids, float *dists, void *stream);

/* Several expansions per step for one query, keeping the plain search's
 * rules: one CTA of `num_threads` warps (1..SS_MAX_INTRA_WIDTH) expands the
 * num_threads best unexplored pool entries at once (the structure of the
 * reference's ModifiedDeltaStepping, src/annsearch.cpp:1586-1731, with the
 * acceptance, merge and termination rules of SearchArraySimulation).
 * num_threads == 1 returns exactly the ss_search result; larger widths trade
 * extra distance evaluations for fewer dependent steps, which lowers the
 * latency of small batches.  ScatterSearch's own intra-query search is
 * ss_search_scatter_batch below. */
int ss_search_intra(ss_index *h, const float *query, int K, int L, int num_threads, uint32_t *ids,
                    float *dists);

/* Batch of queries, each searched by its own CTA of num_threads warps
 * (config: small batches, several candidates expanded per step). */
int ss_search_intra_batch(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                          int num_threads, uint32_t *ids, float *dists);

/* Device-pointer form of ss_search_intra_batch (asynchronous on `stream`). */
int ss_search_intra_batch_device(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                                 int num_threads, uint32_t *ids, float *dists, uint32_t *ndc,
                                 uint32_t *hops, void *stream);

/* ScatterSearch's intra-query search itself: replaces
 * ANNSearch::MultiThreadSearchArraySimulation (src/annsearch.cpp:532-699)
 * and, with early_termination, MultiThreadSearchArraySimulationWithET
 * (:839-1025, SearchUntilBestThreadStop :1368-1455).  One CTA per query;
 * each of its num_threads warps (1..SS_SCATTER_MAX_WARPS) plays one
 * reference thread: its own entry point and pool of L, one visited set
 * shared by all, the pools' top K merged at the end.  Without early
 * termination a pool is padded to L with random unvisited ids; with it, the
 * warps vote at their 50th expansion, losers stop and continue from
 * entries copied out of better warps' pools, and the winner's finish stops
 * all.  Entry points and pads come from `seed` (the reference uses rand()).
 * As with the reference's shared bitset, which warp reaches an id first
 * decides where it lands, so results may differ between runs; they are
 * measured by recall, not compared id for id.  L <= 512. */
#define SS_SCATTER_MAX_WARPS 16
int ss_search_scatter_batch(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                            int num_threads, int early_termination, uint64_t seed, uint32_t *ids,
                            float *dists);

/* ss_search_scatter_batch that also returns the counters the reference's
 * engine keeps for these searches (src/annsearch.cpp:683-695, :1011-1020),
 * per query, in host arrays of nq entries (each may be NULL): distance
 * evaluations summed over the warps (dist_comps), the most and the fewest
 * of one warp (max_dist_comps; max / min is its ub_ratio), and expansions
 * summed over the warps (hop_count, kept by the form without election). */
int ss_search_scatter_batch_stats(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                                  int num_threads, int early_termination, uint64_t seed,
                                  uint32_t *ids, float *dists, uint32_t *ndc_sum,
                                  uint32_t *ndc_max, uint32_t *ndc_min, uint32_t *hops_sum);

/* Device-pointer form (asynchronous on `stream`); ndc / hops (nq uint32,
 * may be NULL) receive each query's distance evaluations and expansions
 * summed over its warps. */
int ss_search_scatter_batch_device(ss_index *h, const float *queries, uint32_t nq, int K, int L,
                                   int num_threads, int early_termination, uint64_t seed,
                                   uint32_t *ids, float *dists, uint32_t *ndc, uint32_t *hops,
                                   void *stream);

/* Launch tuning of the batched warp-per-query kernel, normally chosen by the
 * autotuner (scattersearch_b200.autotune) per (dim, degree, L); no
 * counterpart in the reference, whose only knobs are #defines and argv.
 * warps_per_block: query teams per CTA (1, 2, 4 or 8; 0 = the count that
 * keeps the most teams resident); hash_cap: visited-table slots per query
 * (0 = automatic: 2 x L rounded up to a power of two, at least 1024; the
 * table may forget visited ids, which costs repeated distance evaluations
 * but never changes results);
 * blocks_per_sm_cap: limit on resident CTAs per SM (0 = occupancy limit). */
int ss_set_tuning(ss_index *h, int warps_per_block, int hash_cap, int blocks_per_sm_cap);
/* Launches whose queries can all be resident on the GPU at once in a
 * latency layout (one 32-row stage per team, a visited table of about
 * 20 x L slots, the CTA size that keeps the most teams resident) take that
 * layout and ignore this tuning and the stage layout below: about 1000
 * queries at dim 200 and L = 100, 590 at L = 400.  The serving loop's
 * launches take it for batches of at most 128 requests.  Results are the
 * same either way. */

/* Row stages of the batched kernel.  stage_rows: base rows one stage holds
 * (1-32, 0 = 16); a hop with more fresh candidates than that copies and
 * evaluates them in several passes, and a smaller stage leaves room for more
 * query teams per SM.  stages_per_block: row stages shared by the query
 * teams of one CTA (0 = each team has its own; n > 0 = a pool of n stages
 * per CTA, used when the CTA has more than n teams).  A team holds a stage
 * only while its rows are copied in and its distances computed.  Results
 * never depend on either. */
int ss_set_stage_layout(ss_index *h, int stage_rows, int stages_per_block);

/* How the batched kernel fills its row stages.  SS_ROW_COPY_AUTO: four rows
 * per tensor-map gather copy (cp.async.bulk.tensor tile::gather4) when a row
 * has at most 256 floats and a stage holds a multiple of 4 rows, else one
 * bulk copy per row; SS_ROW_COPY_BULK: always one bulk copy per row.
 * Results never depend on it. */
enum { SS_ROW_COPY_AUTO = 0, SS_ROW_COPY_BULK = 1 };
int ss_set_row_copy(ss_index *h, int mode);

/* Visited ids of the batched kernel.  Each query team keeps a small table
 * in shared memory that may forget ids (a forgotten id met again is
 * evaluated again: the same results, more bytes read).
 * SS_VISITED_MARKS_AUTO: persistent batched launches (ss_search_batch*,
 * plans) also give each team slot one byte per base row in device memory
 * (n bytes x the launch's team slots, allocated once per search context
 * when it takes at most a quarter of the free memory and 16 GB), so no id
 * is evaluated twice.  SS_VISITED_MARKS_OFF: the shared-memory table alone.
 * Results never depend on it. */
enum { SS_VISITED_MARKS_AUTO = 0, SS_VISITED_MARKS_OFF = 1 };
int ss_set_visited_marks(ss_index *h, int mode);

/* ---- exact brute force -------------------------------------------------- */

/* Exact k nearest base rows of each query by brute force (no graph needed);
 * replaces the reference's external ground-truth files (load_groundtruth,
 * src/util.cpp:72-93) and gives the graph builder exact k-NN lists.
 * Inner products run on the tensor cores (TF32 in three terms, FP32
 * accumulation) to select candidates; the candidates are then re-ranked with
 * the search's exact distance (the reference's FP32 lane model), so ids and
 * distances are those of an exact scan, ties broken by smaller id.
 * ids/dists: nq x k (dists may be NULL); rows beyond the index size get id
 * 0xFFFFFFFF.  1 <= k <= 112. */
int ss_bruteforce(ss_index *h, const float *queries, uint32_t nq, int k, uint32_t *ids,
                  float *dists);

/* Device-pointer form (queries nq x dim on the device), asynchronous on
 * `stream`. */
int ss_bruteforce_device(ss_index *h, const float *queries, uint32_t nq, int k, uint32_t *ids,
                         float *dists, void *stream);

/* ---- serving ------------------------------------------------------------ */

/* Online search service over one index.  Replaces the reference's online
 * driver (tests/online_parallel_search.cpp:91-160: a generator thread pushes
 * queries into a mutex-guarded deque, one consumer searches them one at a
 * time).  Here requests arrive one at a time (ss_server_submit) and are
 * batched continuously: a dispatcher thread launches everything pending (up
 * to max_batch requests, each with its own K and L) as soon as one of its
 * launch slots is free, so requests that arrive while others run on the GPU
 * are admitted as slots free up and their launches overlap on the device.
 * The number of slots is bounded by free device memory at creation.  Index,
 * queries, pools and visited tables stay on the device; each result is
 * exactly the ss_search result for that query, whatever it was batched
 * with. */
typedef struct ss_server ss_server;

typedef struct ss_server_config {
  uint32_t max_batch;     /* most requests per launch (1..4096); 0 = 256               */
  uint32_t max_inflight;  /* most launches on the GPU at once (1..16); 0 = 4           */
  uint32_t max_pending;   /* requests held at once (queued, running or finished but not
                             yet collected by ss_server_wait); beyond it submit says
                             SS_ERR_BUSY; 0 = 16384                                   */
  int32_t K_max;          /* largest K a request may ask for; 0 = 100                   */
  int32_t L_max;          /* largest L a request may ask for; 0 = 512                   */
  float memory_fraction;  /* share of free device memory the slots may take; 0 = 0.25  */
} ss_server_config;

typedef struct ss_server_stats {
  uint64_t submitted, completed, failed, batches;
  double mean_batch;                  /* requests per launch                      */
  double p50_us, p99_us, p999_us;     /* arrival-to-result latency, completed ones */
  double max_us;
  uint32_t slots;                     /* launch slots the memory budget allowed   */
} ss_server_stats;

/* Starts the dispatcher.  cfg may be NULL (all defaults).  The index must
 * have a graph and outlive the server. */
int ss_server_create(ss_index *h, const ss_server_config *cfg, ss_server **out);

/* Queues one request (query: dim floats on the host, copied into the
 * server's preallocated request ring; nothing is allocated per request).
 * Returns SS_ERR_BUSY when max_pending requests are already held.  Tickets
 * are nonzero. */
int ss_server_submit(ss_server *s, const float *query, int K, int L, uint64_t *ticket);

/* Waits up to timeout_ms (< 0: no limit) for a request, copies its K ids and
 * distances (dists may be NULL) and its latency in microseconds (may be
 * NULL), and forgets the ticket. */
int ss_server_wait(ss_server *s, uint64_t ticket, int timeout_ms, uint32_t *ids, float *dists,
                   double *latency_us);

/* Load replay: submits request i at arrival_us[i] microseconds after the call
 * starts (a generator thread; arrival_us ascending), waits for all, and
 * writes results at offset Ks[0] + ... + Ks[i-1] of ids/dists and each
 * latency (from its arrival time) to latency_us[i]. */
int ss_server_replay(ss_server *s, const float *queries, uint32_t nq, const int32_t *Ks,
                     const int32_t *Ls, const double *arrival_us, uint32_t *ids, float *dists,
                     double *latency_us);

/* Counters and latency percentiles since creation (or the last reset). */
int ss_server_get_stats(ss_server *s, ss_server_stats *out, int reset);

/* Finishes the launches in flight, drops queued requests, frees the slots. */
void ss_server_destroy(ss_server *s);

/* ---- host I/O (util.cpp) ---------------------------------------------- */

/* Replaces load_fbin (src/util.cpp:40-70): u32 num, u32 dim, then num x dim
 * f32.  *data is malloc'd with 8 floats of zeroed slack after the rows, as
 * the reference allocates; free it with ss_free.  Short files are reported. */
int ss_load_fbin(const char *path, float **data, uint32_t *num, uint32_t *dim);

/* Replaces load_groundtruth (src/util.cpp:72-93): u32 nq, u32 K, then
 * nq x K u32.  *ids is malloc'd; free with ss_free. */
int ss_load_groundtruth(const char *path, uint32_t **ids, uint32_t *nq, uint32_t *k);

void ss_free(void *p);

/* ---- diagnostics ----------------------------------------------------- */

/* Message of the last failed call on `h` (or on this thread when h is
 * NULL).  The string stays valid until the next failing call. */
const char *ss_last_error(const ss_index *h);

/* Library version string, e.g. "scattersearch_b200 0.1 sm_100a". */
const char *ss_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SCATTERSEARCH_H */
