/*
 * ss_oracle.c -- CPU restatement of ScatterSearch's graph search path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this library, and only as the checker.
 * The product (scattersearch_b200/) never links or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference itself, compiled in place from its sources into oracle/_ref/
 * (oracle/Makefile), and against the golden fixtures under tests/golden/ that
 * tests/golden/make_golden.py produced from that compiled reference.
 *
 * Reference semantics restated (reference paths):
 *   distance_l2sqr_avx   src/distance.cpp:19-56
 *   distance_ip_avx      src/distance.cpp:115-149
 *   InsertIntoPool       include/util.h:41-78   (upper-bound insert: ties keep
 *                        the older entry first)
 *   SearchArraySimulation src/annsearch.cpp:182-259
 *
 * The search is written in "batch-merge" form rather than the reference's
 * insert-one-at-a-time loop.  The two are equivalent:
 *   - the reference always expands the first unexplored slot below
 *     min(L, size) (its k / nk bookkeeping, annsearch.cpp:218-253);
 *   - a candidate is accepted iff d < pool[size-1] taken at the START of the
 *     hop: the live threshold only shrinks inside a hop, and any candidate it
 *     rejects would also fall past slot L in the merge below (annsearch.cpp:238);
 *   - the new pool is the stable merge of the old pool and the accepted
 *     candidates (old entries first on equal distance, candidates in adjacency
 *     order), truncated to min(L, size + accepted) (util.h:56-75,
 *     annsearch.cpp:242-243).
 * One place the reference leaves the order open: std::sort of the initial
 * pool (annsearch.cpp:215) is not stable.  Exactly tied initial distances are
 * ordered here by adjacency position.
 *
 * Adjacency layout shared with the GPU path: n x rstride uint32, each row a
 * prefix of neighbour ids followed by 0xFFFFFFFF padding.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SSO_NONE 0xFFFFFFFFu
#define SSO_L2 0
#define SSO_IP 1

/* 8-lane distance model of distance.cpp:19-56 / :115-149.  D = dim rounded up
 * to 8; when D % 16 == 8 the last 8-block is accumulated first (:42-45), then
 * the 8-blocks in order (:47-51), each lane a separate mul and add with no
 * fusion, then lanes summed left to right (:53).  Lanes past `dim` read 0. */
float sso_distance(const float *a, const float *b, unsigned dim, int metric) {
  unsigned nb = (dim + 7u) / 8u;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (unsigned t = 0; t < nb; ++t) {
    unsigned blk = (nb & 1u) ? (t == 0 ? nb - 1 : t - 1) : t;
    for (unsigned j = 0; j < 8; ++j) {
      unsigned i = blk * 8 + j;
      float x = i < dim ? a[i] : 0.0f;
      float y = i < dim ? b[i] : 0.0f;
      float p;
      if (metric == SSO_L2) {
        float df = x - y;
        p = df * df;
      } else {
        p = x * y;
      }
      acc[j] = acc[j] + p;
    }
  }
  float r = acc[0];
  for (unsigned j = 1; j < 8; ++j) r = r + acc[j];
  return metric == SSO_L2 ? r : -r;
}

typedef struct {
  float d;
  uint32_t id;
  uint32_t explored;
} sso_ent;

/* Stable insertion sort by distance (ties keep input order). */
static void sort_stable(sso_ent *e, unsigned n) {
  for (unsigned i = 1; i < n; ++i) {
    sso_ent v = e[i];
    unsigned j = i;
    while (j > 0 && e[j - 1].d > v.d) {
      e[j] = e[j - 1];
      --j;
    }
    e[j] = v;
  }
}

/* Stable merge of pool[0,s) and cand[0,nc) into out, old first on ties,
 * keeping at most cap entries.  Returns the merged length. */
static unsigned merge_pool(const sso_ent *pool, unsigned s, const sso_ent *cand, unsigned nc,
                           sso_ent *out, unsigned cap) {
  unsigned i = 0, j = 0, o = 0;
  while (o < cap && (i < s || j < nc)) {
    if (j >= nc || (i < s && pool[i].d <= cand[j].d)) out[o++] = pool[i++];
    else out[o++] = cand[j++];
  }
  return o;
}

typedef struct {
  const float *base;
  uint32_t n, dim;
  const uint32_t *adj;
  uint32_t rstride, ep;
  int metric;
} sso_index;

/* Best-first search for one query, expanding up to W best unexplored entries
 * per step.  W == 1 is exactly SearchArraySimulation (annsearch.cpp:182-259).
 * For W > 1 (the several-candidates-per-step form, structured like
 * ModifiedDeltaStepping annsearch.cpp:1632-1691) the acceptance threshold,
 * stable merge and truncation rules are the W == 1 ones, and candidates are
 * ordered by (expansion slot w, adjacency position m); the first occurrence of
 * an id in that order is the one evaluated.
 * visited: n bytes, all zero on entry, left dirty.  Returns 0. */
static int search_one(const sso_index *ix, const float *q, int K, int L, int W, uint32_t *ids,
                      float *dists, uint8_t *visited, uint32_t *ndc_out, uint32_t *hops_out,
                      sso_ent *pool, sso_ent *tmp, sso_ent *cand) {
  uint32_t ndc = 0, hops = 0;
  const uint32_t *row = ix->adj + (size_t)ix->ep * ix->rstride;
  unsigned s = 0;
  /* initial pool: first min(L, deg(ep)) neighbours of ep, all marked visited
   * (annsearch.cpp:188-192), distances, sort (:207-215) */
  for (unsigned m = 0; m < ix->rstride && row[m] != SSO_NONE && s < (unsigned)L; ++m) {
    uint32_t id = row[m];
    visited[id] = 1;
    pool[s].id = id;
    pool[s].d = sso_distance(ix->base + (size_t)id * ix->dim, q, ix->dim, ix->metric);
    pool[s].explored = 0;
    ++s;
    ++ndc;
  }
  sort_stable(pool, s);
  for (;;) {
    unsigned picks[64];
    unsigned np = 0;
    for (unsigned k = 0; k < s && np < (unsigned)W; ++k)
      if (!pool[k].explored) picks[np++] = k;
    if (np == 0) break;
    float thr = pool[s - 1].d;
    unsigned nc = 0;
    for (unsigned w = 0; w < np; ++w) {
      pool[picks[w]].explored = 1;
      ++hops;
      const uint32_t *nr = ix->adj + (size_t)pool[picks[w]].id * ix->rstride;
      for (unsigned m = 0; m < ix->rstride && nr[m] != SSO_NONE; ++m) {
        uint32_t id = nr[m];
        if (visited[id]) continue;
        visited[id] = 1;
        float d = sso_distance(q, ix->base + (size_t)id * ix->dim, ix->dim, ix->metric);
        ++ndc;
        if (d >= thr) continue;
        cand[nc].d = d;
        cand[nc].id = id;
        cand[nc].explored = 0;
        ++nc;
      }
    }
    sort_stable(cand, nc);
    unsigned ns = merge_pool(pool, s, cand, nc, tmp, (unsigned)L);
    memcpy(pool, tmp, ns * sizeof(sso_ent));
    s = ns;
  }
  for (int i = 0; i < K; ++i) {
    /* slots the pool never reached hold the value-initialised Neighbor
     * (id 0, distance 0) of annsearch.cpp:193 */
    ids[i] = (unsigned)i < s ? pool[i].id : 0u;
    if (dists) dists[i] = (unsigned)i < s ? pool[i].d : 0.0f;
  }
  if (ndc_out) *ndc_out = ndc;
  if (hops_out) *hops_out = hops;
  return 0;
}

/* Searches nq queries (row-major nq x dim).  Per-query K and L (arrays of
 * length nq, or NULL to use K0 / L0).  ids/dists are written at out_off[i]
 * (or i*K0 when out_off is NULL).  W: expansions per step (1 = plain).
 * nthreads > 1 parallelises across queries with OpenMP.  Returns 0, or -1 on
 * bad arguments. */
int sso_search_batch(const float *base, uint32_t n, uint32_t dim, int metric, const uint32_t *adj,
                     uint32_t rstride, uint32_t ep, const float *queries, uint32_t nq,
                     const int32_t *Ks, const int32_t *Ls, int K0, int L0, int W,
                     const int64_t *out_off, uint32_t *ids, float *dists, uint32_t *ndc,
                     uint32_t *hops, int nthreads) {
  if (W < 1 || W > 64 || ep >= n) return -1;
  sso_index ix = {base, n, dim, adj, rstride, ep, metric};
  int Lmax = L0;
  if (Ls)
    for (uint32_t i = 0; i < nq; ++i) Lmax = Ls[i] > Lmax ? Ls[i] : Lmax;
  int bad = 0;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1) reduction(| : bad)
  {
    uint8_t *visited = (uint8_t *)calloc(n, 1);
    sso_ent *pool = (sso_ent *)malloc(sizeof(sso_ent) * (size_t)(Lmax + 1));
    sso_ent *tmp = (sso_ent *)malloc(sizeof(sso_ent) * (size_t)(Lmax + 1));
    sso_ent *cand = (sso_ent *)malloc(sizeof(sso_ent) * (size_t)rstride * (size_t)W);
#pragma omp for schedule(dynamic, 4)
    for (long i = 0; i < (long)nq; ++i) {
      int K = Ks ? Ks[i] : K0, L = Ls ? Ls[i] : L0;
      int64_t off = out_off ? out_off[i] : (int64_t)i * K0;
      if (K < 1 || K > L) {
        bad = 1;
        continue;
      }
      search_one(&ix, queries + (size_t)i * dim, K, L, W, ids + off, dists ? dists + off : NULL,
                 visited, ndc ? ndc + i : NULL, hops ? hops + i : NULL, pool, tmp, cand);
      memset(visited, 0, n);
    }
    free(visited);
    free(pool);
    free(tmp);
    free(cand);
  }
  return bad ? -1 : 0;
}

/* Exact brute force top-k under the same distance model (ties by id). */
int sso_bruteforce(const float *base, uint32_t n, uint32_t dim, int metric, const float *queries,
                   uint32_t nq, int k, uint32_t *ids, float *dists, int nthreads) {
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(dynamic, 1)
  for (long i = 0; i < (long)nq; ++i) {
    sso_ent *best = (sso_ent *)malloc(sizeof(sso_ent) * (size_t)(k + 1));
    int cnt = 0;
    const float *q = queries + (size_t)i * dim;
    for (uint32_t j = 0; j < n; ++j) {
      float d = sso_distance(q, base + (size_t)j * dim, dim, metric);
      if (cnt == k && d >= best[k - 1].d) continue;
      int p = cnt < k ? cnt++ : k - 1;
      while (p > 0 && best[p - 1].d > d) {
        best[p] = best[p - 1];
        --p;
      }
      best[p].d = d;
      best[p].id = j;
    }
    for (int t = 0; t < k; ++t) {
      ids[(size_t)i * k + t] = t < cnt ? best[t].id : SSO_NONE;
      if (dists) dists[(size_t)i * k + t] = t < cnt ? best[t].d : 0.0f;
    }
    free(best);
  }
  return 0;
}

/* Exact k-NN in double precision: the float64 ground truth the benchmark
 * configurations pin recall against (L2: sum of squared differences; inner
 * product: minus the dot product; both accumulated in double).  Ties are
 * broken by the smaller id.  ids: nq x k (SSO_NONE past n). */
int sso_bruteforce_f64(const float *base, uint32_t n, uint32_t dim, int metric,
                       const float *queries, uint32_t nq, int k, uint32_t *ids, double *dists,
                       int nthreads) {
  if (k <= 0) return -1;
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(dynamic, 1)
  for (long i = 0; i < (long)nq; ++i) {
    double *bd = (double *)malloc(sizeof(double) * (size_t)k);
    uint32_t *bi = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)k);
    int cnt = 0;
    const float *q = queries + (size_t)i * dim;
    for (uint32_t j = 0; j < n; ++j) {
      const float *x = base + (size_t)j * dim;
      double s = 0.0;
      if (metric == SSO_L2) {
        for (uint32_t t = 0; t < dim; ++t) {
          const double d = (double)q[t] - (double)x[t];
          s += d * d;
        }
      } else {
        for (uint32_t t = 0; t < dim; ++t) s += (double)q[t] * (double)x[t];
        s = -s;
      }
      /* j ascends, so an equal distance never displaces an earlier id */
      if (cnt == k && s >= bd[k - 1]) continue;
      int p = cnt < k ? cnt++ : k - 1;
      while (p > 0 && bd[p - 1] > s) {
        bd[p] = bd[p - 1];
        bi[p] = bi[p - 1];
        --p;
      }
      bd[p] = s;
      bi[p] = j;
    }
    for (int t = 0; t < k; ++t) {
      ids[(size_t)i * k + t] = t < cnt ? bi[t] : SSO_NONE;
      if (dists) dists[(size_t)i * k + t] = t < cnt ? bd[t] : 0.0;
    }
    free(bd);
    free(bi);
  }
  return 0;
}

/* ---- ScatterSearch without election, restated for the recall check ------
 * MultiThreadSearchArraySimulation (src/annsearch.cpp:532-699): T pools of
 * L, each seeded with every neighbour of its own random entry point and
 * padded to L with random unvisited ids (:552-575), all sharing one visited
 * set; each pool runs the plain best-first rules; the answer is the K best
 * of all pools, one copy per id (:646-668).  The reference's threads race on
 * a shared bitset without atomics, so its result depends on their timing;
 * this restatement fixes one schedule: the pools are set up in order and
 * then take one expansion each in turn, with an exact visited set.  Entry
 * points and pads come from a seeded counter hash.  ids: nq x K; ndc (may be
 * NULL): distance evaluations per query, all pools together. */
typedef struct { uint32_t id; float d; int explored; } sso_sent;

static uint64_t sso_mix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

static int sso_sent_cmp(const void *a, const void *b) {
  const sso_sent *x = (const sso_sent *)a, *y = (const sso_sent *)b;
  if (x->d < y->d) return -1;
  if (x->d > y->d) return 1;
  return x->id < y->id ? -1 : (x->id > y->id ? 1 : 0);
}

/* one expansion of pool p (size *sz, capacity L); returns 0 when nothing
 * is left to expand */
static int sso_scatter_hop(const float *base, uint32_t dim, int metric, const uint32_t *adj,
                           uint32_t rstride, const float *q, sso_sent *p, int *sz, int L,
                           unsigned char *vis, sso_sent *cand, sso_sent *tmp, uint32_t *ndc) {
  int k = 0;
  while (k < *sz && p[k].explored) ++k;
  if (k >= *sz) return 0;
  p[k].explored = 1;
  const uint32_t *row = adj + (size_t)p[k].id * rstride;
  const float thr = p[*sz - 1].d;
  int nc = 0;
  for (uint32_t m = 0; m < rstride && row[m] != SSO_NONE; ++m) {
    const uint32_t id = row[m];
    if (vis[id]) continue;
    vis[id] = 1;
    const float d = sso_distance(q, base + (size_t)id * dim, dim, metric);
    ++*ndc;
    if (d < thr) {
      /* stable insertion by distance (adjacency order on ties) */
      int j = nc++;
      while (j > 0 && cand[j - 1].d > d) { cand[j] = cand[j - 1]; --j; }
      cand[j].id = id; cand[j].d = d; cand[j].explored = 0;
    }
  }
  /* merge, old entries first on equal distance, truncated to L */
  int a = 0, o = 0, n = 0;
  while (n < L && (o < *sz || a < nc)) {
    if (a < nc && (o >= *sz || cand[a].d < p[o].d)) tmp[n++] = cand[a++];
    else tmp[n++] = p[o++];
  }
  memcpy(p, tmp, sizeof(sso_sent) * (size_t)n);
  *sz = n;
  return 1;
}

int sso_scatter_plain(const float *base, uint32_t n, uint32_t dim, int metric,
                      const uint32_t *adj, uint32_t rstride, const float *queries, uint32_t nq,
                      int K, int L, int T, uint64_t seed, uint32_t *ids, uint32_t *ndc,
                      int nthreads) {
  if (K < 1 || L < K || T < 1 || n == 0) return -1;
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
  {
    unsigned char *vis = (unsigned char *)calloc(n, 1);
    sso_sent *pools = (sso_sent *)malloc(sizeof(sso_sent) * (size_t)T * (size_t)L);
    int *sz = (int *)malloc(sizeof(int) * (size_t)T);
    int *live = (int *)malloc(sizeof(int) * (size_t)T);
    sso_sent *cand = (sso_sent *)malloc(sizeof(sso_sent) * (size_t)(rstride + 1));
    sso_sent *tmp = (sso_sent *)malloc(sizeof(sso_sent) * (size_t)(L + rstride + 1));
    sso_sent *all = (sso_sent *)malloc(sizeof(sso_sent) * (size_t)T * (size_t)L);
#pragma omp for schedule(dynamic, 1)
    for (long qi = 0; qi < (long)nq; ++qi) {
      const float *q = queries + (size_t)qi * dim;
      uint32_t evals = 0;
      uint64_t ctr = 0;
      for (int t = 0; t < T; ++t) {
        sso_sent *p = pools + (size_t)t * L;
        const uint32_t ep = (uint32_t)(sso_mix(seed ^ ((uint64_t)qi << 32) ^ ((uint64_t)t << 20) ^ ctr++) % n);
        int s = 0;
        const uint32_t *row = adj + (size_t)ep * rstride;
        for (uint32_t m = 0; m < rstride && row[m] != SSO_NONE && s < L; ++m) {
          p[s++].id = row[m];
          vis[row[m]] = 1;
        }
        while (s < L) {
          uint32_t id = (uint32_t)(sso_mix(seed ^ ((uint64_t)qi << 32) ^ ((uint64_t)t << 20) ^ ctr++) % n);
          uint32_t probes = 0;
          while (vis[id] && probes++ < n) id = id + 1 == n ? 0 : id + 1;
          if (vis[id]) break;
          vis[id] = 1;
          p[s++].id = id;
        }
        for (int j = 0; j < s; ++j) {
          p[j].d = sso_distance(base + (size_t)p[j].id * dim, q, dim, metric);
          p[j].explored = 0;
        }
        evals += (uint32_t)s;
        /* stable sort by distance */
        for (int j = 1; j < s; ++j) {
          sso_sent x = p[j];
          int i = j;
          while (i > 0 && p[i - 1].d > x.d) { p[i] = p[i - 1]; --i; }
          p[i] = x;
        }
        sz[t] = s;
        live[t] = s > 0;
      }
      for (int any = 1; any;) {
        any = 0;
        for (int t = 0; t < T; ++t) {
          if (!live[t]) continue;
          live[t] = sso_scatter_hop(base, dim, metric, adj, rstride, q, pools + (size_t)t * L,
                                    &sz[t], L, vis, cand, tmp, &evals);
          any |= live[t];
        }
      }
      int na = 0;
      for (int t = 0; t < T; ++t)
        for (int j = 0; j < sz[t]; ++j) all[na++] = pools[(size_t)t * L + j];
      qsort(all, (size_t)na, sizeof(sso_sent), sso_sent_cmp);
      int out = 0;
      for (int j = 0; j < na && out < K; ++j)
        if (j == 0 || all[j].id != all[j - 1].id) ids[(size_t)qi * K + out++] = all[j].id;
      for (; out < K; ++out) ids[(size_t)qi * K + out] = SSO_NONE;
      if (ndc) ndc[qi] = evals;
      memset(vis, 0, n);  /* the next query starts unvisited */
    }
    free(vis); free(pools); free(sz); free(live); free(cand); free(tmp); free(all);
  }
  return 0;
}
