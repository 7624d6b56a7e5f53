// Distance primitives shared by the search kernels (ss_search.cu) and the
// brute-force k-NN kernels (ss_bruteforce.cu).
//
// Every distance follows the reference's AVX model (src/distance.cpp:19-56,
// :115-149): 8 lane partials over the row's 8-float blocks, the odd block
// first when the padded dimension is 8 mod 16, one rounding per subtract,
// multiply and add (never fused), lanes summed left to right.  That makes
// GPU distances bit-identical to the reference built without fast-math.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "ss_internal.h"

namespace ssb {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint64_t kInvalidKey = ~0ull;

// ---------------------------------------------------------------- keys ---
// Order-preserving map float -> uint32 (ascending).  -0 is folded onto +0 so
// that equal floats get equal keys.  NaN inputs are not supported.
__device__ __forceinline__ uint32_t float_to_key(float d) {
  uint32_t u = __float_as_uint(d);
  if (u == 0x80000000u) u = 0u;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_to_float(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  return __uint_as_float(u);
}

__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int m) {
  const uint32_t lo = __shfl_xor_sync(kFull, (uint32_t)v, m);
  const uint32_t hi = __shfl_xor_sync(kFull, (uint32_t)(v >> 32), m);
  return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ float4 ldg_f4(const float4 *p) { return __ldg(p); }

// ----------------------------------------------------------- distances ---
// Block visiting order of distance.cpp:42-51: with an odd number of 8-blocks
// the last block comes first, then blocks 0, 1, ...
__device__ __forceinline__ int block_at(int t, int nb) {
  return (nb & 1) ? (t == 0 ? nb - 1 : t - 1) : t;
}

// One 8-float block's contribution to four of the eight lane partials
// (reference lanes 4h..4h+3 of distance.cpp:47-51): a_j += (q_j - v_j)^2
// (L2) or a_j += q_j * v_j (inner product), each operation rounded once.
// Scalar instructions on purpose: the paired FP32 forms (sub/mul/add.rn.f32x2)
// were measured on this GPU to return distances that differ from these in
// the last bit, which would break bit-exact parity with the reference.
__device__ __forceinline__ void acc_l2(float &a0, float &a1, float &a2, float &a3, float4 q,
                                       float4 v) {
  float d;
  d = __fsub_rn(q.x, v.x); a0 = __fadd_rn(a0, __fmul_rn(d, d));
  d = __fsub_rn(q.y, v.y); a1 = __fadd_rn(a1, __fmul_rn(d, d));
  d = __fsub_rn(q.z, v.z); a2 = __fadd_rn(a2, __fmul_rn(d, d));
  d = __fsub_rn(q.w, v.w); a3 = __fadd_rn(a3, __fmul_rn(d, d));
}
__device__ __forceinline__ void acc_ip(float &a0, float &a1, float &a2, float &a3, float4 q,
                                       float4 v) {
  a0 = __fadd_rn(a0, __fmul_rn(q.x, v.x));
  a1 = __fadd_rn(a1, __fmul_rn(q.y, v.y));
  a2 = __fadd_rn(a2, __fmul_rn(q.z, v.z));
  a3 = __fadd_rn(a3, __fmul_rn(q.w, v.w));
}

// Distance between the shared-memory query and base row `id`, computed by a
// lane pair: lane h (0/1) of the pair owns reference lanes 4h..4h+3 and loads
// one float4 per 8-block.  Both lanes of the pair return the full distance.
// All 32 lanes must call this (it shuffles); `act` false lanes load nothing.
template <int NB>
__device__ __forceinline__ float pair_distance(const GraphView &g, const float *qs, uint32_t id,
                                               bool act, int h) {
  const int nb = NB > 0 ? NB : (int)g.nb;
  const float4 *row = reinterpret_cast<const float4 *>(g.base + (size_t)id * (size_t)(nb * 8)) + h;
  const float4 *q4 = reinterpret_cast<const float4 *>(qs) + h;
  float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
  const bool l2 = g.metric == 0;
  if constexpr (NB > 0) {
    float4 v[NB];
#pragma unroll
    for (int t = 0; t < NB; ++t) {
      v[t] = act ? ldg_f4(row + 2 * block_at(t, NB)) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (l2) {
#pragma unroll
      for (int t = 0; t < NB; ++t) acc_l2(a0, a1, a2, a3, q4[2 * block_at(t, NB)], v[t]);
    } else {
#pragma unroll
      for (int t = 0; t < NB; ++t) acc_ip(a0, a1, a2, a3, q4[2 * block_at(t, NB)], v[t]);
    }
  } else {
    // groups of 8 blocks, double-buffered: the next group's loads are in
    // flight while this group accumulates (same order of operations)
    float4 v[8], w[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      v[u] = (act && u < nb) ? ldg_f4(row + 2 * block_at(u, nb)) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int t0 = 0; t0 < nb; t0 += 8) {
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int t = t0 + 8 + u;
        w[u] = (act && t < nb) ? ldg_f4(row + 2 * block_at(t, nb)) : make_float4(0.f, 0.f, 0.f, 0.f);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int t = t0 + u;
        if (t < nb) {
          if (l2) acc_l2(a0, a1, a2, a3, q4[2 * block_at(t, nb)], v[u]);
          else acc_ip(a0, a1, a2, a3, q4[2 * block_at(t, nb)], v[u]);
        }
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) v[u] = w[u];
    }
  }
  // Horizontal sum u0 + u1 + ... + u7, left to right (distance.cpp:53).
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
  return l2 ? r : -r;
}

// Keys of cand_id[0..nc) into cand_key[0..nc); 16 candidates per pass.
template <int NB>
__device__ __forceinline__ void eval_candidates(const GraphView &g, const float *qs,
                                                const uint32_t *cand_id, uint32_t *cand_key, int nc,
                                                int lane) {
  const int h = lane & 1;
  for (int p = 0; p < nc; p += 16) {
    const int j = p + (lane >> 1);
    const bool act = j < nc;
    const uint32_t id = act ? cand_id[j] : 0u;
    const float d = pair_distance<NB>(g, qs, id, act, h);
    if (act && h == 0) cand_key[j] = float_to_key(d);
  }
}

// -------------------------------------------------------------- sorting ---
// Ascending bitonic sort of 32*ITEMS 64-bit keys held one per lane per item;
// element index e = item*32 + lane.
template <int ITEMS>
__device__ __forceinline__ void warp_sort(uint64_t (&x)[ITEMS], int lane) {
  constexpr int N = 32 * ITEMS;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
        const int js = j >> 5;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
          const int pi = i ^ js;
          if (pi > i) {
            const bool up = ((i * 32 + lane) & k) == 0;
            const uint64_t a = x[i], b = x[pi];
            if ((a > b) == up) {
              x[i] = b;
              x[pi] = a;
            }
          }
        }
      } else {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
          const uint64_t o = shfl_xor_u64(x[i], j);
          const bool up = ((i * 32 + lane) & k) == 0;
          const bool lower = (lane & j) == 0;
          x[i] = (lower == up) ? (x[i] < o ? x[i] : o) : (x[i] < o ? o : x[i]);
        }
      }
    }
  }
}

}  // namespace ssb
