// Exact k-nearest-neighbour brute force on the tensor cores.
//
// The reference takes its ground truth from external files (load_groundtruth,
// src/util.cpp:72-93); this is the project's own exact k-NN, used for ground
// truth and for graph building.  Two kernels:
//
//   bf_candidates_kernel  64 queries x (a split of the base rows) per CTA.
//                         Each 64x64 tile of inner products is computed with
//                         TF32 mma.sync in three terms (a_hi*b_hi + a_hi*b_lo
//                         + a_lo*b_hi, FP32 accumulate), which carries about
//                         FP32 accuracy; the tile's scores go through a per-
//                         query candidate list in shared memory that keeps
//                         the C best (approximate score, id).
//   bf_rerank_kernel      one warp per query merges the splits' lists, keeps
//                         the C best by approximate score, computes their
//                         distances exactly as the search does (the
//                         reference's FP32 lane model, bit-identical) and
//                         returns the k best by (distance, id).
//
// C exceeds k by a margin of at least 16, so a true neighbour is lost only if
// more than C - k rows score within the TF32 error of it, which needs a tie
// group far larger than the margin; exact ties (e.g. integer-valued data,
// where the three-term products are exact) are ordered by id in both passes.
#include <cuda_runtime.h>
#include <stdint.h>

#include "ss_distance.cuh"
#include "ss_internal.h"

namespace ssb {
namespace {

constexpr int kBQ = 64;   // queries per CTA
constexpr int kBN = 64;   // base rows per tile
constexpr int kBK = 32;   // dims per smem chunk
constexpr int kPadK = kBK + 4;

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
      "{%8, %9}, {%0, %1, %2, %3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Sorts a query's candidate list (cnt used entries of cap) ascending and
// keeps the C best; returns the new threshold (the C-th key, or ~0 while
// fewer than C are held).  One warp.
template <int CAP, int C>
__device__ __forceinline__ uint64_t compact_list(uint64_t *list, int &cnt, int lane) {
  constexpr int ITEMS = CAP / 32;
  uint64_t x[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) {
    const int e = i * 32 + lane;
    x[i] = e < cnt ? list[e] : kInvalidKey;
  }
  warp_sort<ITEMS>(x, lane);
  __syncwarp();
#pragma unroll
  for (int i = 0; i < ITEMS; ++i) list[i * 32 + lane] = x[i];
  __syncwarp();
  cnt = min(cnt, C);
  return cnt == C ? list[C - 1] : kInvalidKey;
}

// Candidates of 64 queries over base rows [row_lo, row_hi): out[q][split][0..C).
template <int C>
__global__ void __launch_bounds__(128) bf_candidates_kernel(BruteArgs a) {
  constexpr int CAP = C + 64 <= 128 ? 128 : 256;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *Qs = reinterpret_cast<float *>(smem_raw);                  // [kBQ][kPadK]
  float *Xs = Qs + kBQ * kPadK;                                      // [kBN][kPadK]
  float *S = Xs + kBN * kPadK;                                       // [kBQ][kBN + 1]
  uint64_t *lists = reinterpret_cast<uint64_t *>(S + kBQ * (kBN + 1));  // [kBQ][CAP]
  __shared__ uint64_t thr[kBQ];
  __shared__ int cnt[kBQ];

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const uint32_t q0 = blockIdx.x * kBQ;
  const uint32_t split = blockIdx.y;
  const uint32_t row_lo = split * a.rows_per_split;
  const uint32_t row_hi = min(a.n, row_lo + a.rows_per_split);
  const int pitch = (int)a.nb * 8;
  if (tid < kBQ) {
    thr[tid] = kInvalidKey;
    cnt[tid] = 0;
  }
  __syncthreads();

  for (uint32_t n0 = row_lo; n0 < row_hi; n0 += kBN) {
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[j][c] = 0.f;

    for (int k0 = 0; k0 < pitch; k0 += kBK) {
      __syncthreads();
      // 64 x 32 floats of queries and of base rows: 4 float4 per thread each
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int e = i * 128 + tid;  // float4 index in the 64 x 8 grid
        const int r = e >> 3, c4 = (e & 7) * 4;
        const int k = k0 + c4;
        float4 qv = make_float4(0.f, 0.f, 0.f, 0.f), xv = qv;
        if (q0 + r < a.nq && k < pitch)
          qv = __ldg(reinterpret_cast<const float4 *>(a.queries + (size_t)(q0 + r) * pitch + k));
        if (n0 + r < row_hi && k < pitch)
          xv = __ldg(reinterpret_cast<const float4 *>(a.base + (size_t)(n0 + r) * pitch + k));
        *reinterpret_cast<float4 *>(Qs + r * kPadK + c4) = qv;
        *reinterpret_cast<float4 *>(Xs + r * kPadK + c4) = xv;
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < kBK; kk += 8) {
        uint32_t ah[4], al[4];
        const float *qa = Qs + (warp * 16 + g) * kPadK + kk + t;
        split_tf32(qa[0], ah[0], al[0]);
        split_tf32(qa[8 * kPadK], ah[1], al[1]);
        split_tf32(qa[4], ah[2], al[2]);
        split_tf32(qa[8 * kPadK + 4], ah[3], al[3]);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const float *xb = Xs + (j * 8 + g) * kPadK + kk + t;
          uint32_t bh0, bl0, bh1, bl1;
          split_tf32(xb[0], bh0, bl0);
          split_tf32(xb[4], bh1, bl1);
          mma_tf32(acc[j], al, bh0, bh1);
          mma_tf32(acc[j], ah, bl0, bl1);
          mma_tf32(acc[j], ah, bh0, bh1);
        }
      }
    }
    // scores: inner product -> -dot; L2 -> |x|^2 - 2 dot (the query's norm is
    // the same for every row and does not change the ranking)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int row = warp * 16 + g + (c >= 2 ? 8 : 0);
        const int col = j * 8 + 2 * t + (c & 1);
        const uint32_t id = n0 + col;
        float sc;
        if (a.metric == 0) {
          sc = id < row_hi ? __fsub_rn(a.xnorm[id], __fmul_rn(2.f, acc[j][c])) : 0.f;
        } else {
          sc = -acc[j][c];
        }
        S[row * (kBN + 1) + col] = sc;
      }
    }
    __syncthreads();
    // selection: warp w owns queries 16w .. 16w+15
    for (int r = 0; r < 16; ++r) {
      const int qi = warp * 16 + r;
      if (q0 + qi >= a.nq) break;
      uint64_t *list = lists + (size_t)qi * CAP;
      int count = cnt[qi];
      uint64_t th = thr[qi];
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int col = half * 32 + lane;
        const uint32_t id = n0 + col;
        const uint64_t key = ((uint64_t)float_to_key(S[qi * (kBN + 1) + col]) << 32) | id;
        bool ok = id < row_hi && key < th;
        unsigned m = __ballot_sync(kFull, ok);
        if (count + __popc(m) > CAP) {
          th = compact_list<CAP, C>(list, count, lane);
          ok = ok && key < th;
          m = __ballot_sync(kFull, ok);
        }
        if (ok) list[count + __popc(m & ((1u << lane) - 1u))] = key;
        count += __popc(m);
        __syncwarp();
      }
      if (lane == 0) {
        cnt[qi] = count;
        thr[qi] = th;
      }
      __syncwarp();
    }
    __syncthreads();
  }
  // final: each query's C best of this split
  for (int r = 0; r < 16; ++r) {
    const int qi = warp * 16 + r;
    if (q0 + qi >= a.nq) break;
    uint64_t *list = lists + (size_t)qi * CAP;
    int count = cnt[qi];
    compact_list<CAP, C>(list, count, lane);
    uint64_t *out = a.cand + ((size_t)(q0 + qi) * a.splits + split) * C;
    for (int e = lane; e < C; e += 32) out[e] = e < count ? list[e] : kInvalidKey;
  }
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
  const uint64_t *src = a.cand + (size_t)q * a.splits * C;
#pragma unroll
  for (int i = 0; i < IT; ++i) {
    const int e = i * 32 + lane;
    x[i] = e < (int)(a.splits * C) ? src[e] : kInvalidKey;
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

template <int C>
size_t candidates_smem() {
  constexpr int CAP = C + 64 <= 128 ? 128 : 256;
  return (size_t)(2 * kBQ * kPadK + kBQ * (kBN + 1)) * 4 + (size_t)kBQ * CAP * 8;
}

template <int C>
cudaError_t launch_candidates(const BruteArgs &a, cudaStream_t s) {
  const size_t smem = candidates_smem<C>();
  cudaError_t e = cudaFuncSetAttribute((const void *)bf_candidates_kernel<C>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  dim3 grid((a.nq + kBQ - 1) / kBQ, a.splits);
  bf_candidates_kernel<C><<<grid, 128, smem, s>>>(a);
  return cudaGetLastError();
}

template <int C, int SC>
cudaError_t launch_rerank(const BruteArgs &a, const GraphView &g, cudaStream_t s) {
  const size_t smem = (size_t)4 * a.nb * 8 * 4 + (size_t)4 * 2 * C * 4;
  cudaError_t e = cudaFuncSetAttribute((const void *)bf_rerank_kernel<C, SC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  bf_rerank_kernel<C, SC><<<(a.nq + 3) / 4, 128, smem, s>>>(a, g);
  return cudaGetLastError();
}

template <int C>
cudaError_t launch_rerank_c(const BruteArgs &a, const GraphView &g, cudaStream_t s) {
  switch (a.splits * C) {
    case 32: return launch_rerank<C, 32>(a, g, s);
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
  const uint32_t tiles = (nq + kBQ - 1) / kBQ;
  uint32_t splits = 1;
  const uint32_t max_splits = 1024u / (uint32_t)p.C;
  while (splits < max_splits && tiles * splits < 2u * (uint32_t)sm_count) splits <<= 1;
  // never more splits than 64-row tiles of the base
  while (splits > 1 && (uint64_t)splits * kBN > n) splits >>= 1;
  p.splits = splits;
  uint32_t rps = (n + splits - 1) / splits;
  p.rows_per_split = (rps + kBN - 1) / kBN * kBN;
  return p;
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
