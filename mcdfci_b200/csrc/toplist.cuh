// Per-warp top-M list of (key, payload) pairs kept in registers, sorted
// descending: element i is held by lane i % 32 in register i / 32.  Keys are
// unsigned; 0 marks an empty element.  Used by the column kernel (per-column
// candidates) and by the leader kernel (the k coordinates to pick).
#pragma once

#include "device_common.cuh"

namespace mcd {

template <int R>
struct TopList {
  unsigned long long k[R];
  unsigned p[R];
};

template <int R>
__device__ __forceinline__ void toplist_clear(TopList<R>& L) {
#pragma unroll
  for (int j = 0; j < R; ++j) {
    L.k[j] = 0ull;
    L.p[j] = 0u;
  }
}

// Compare-exchange with lane ^ stride; this lane keeps the larger key if
// keep_max.  Equal keys stay where they are on both sides.
__device__ __forceinline__ void cmpx_lane(unsigned long long& k, unsigned& p, int stride, bool keep_max) {
  const unsigned long long ok = __shfl_xor_sync(~0u, k, stride);
  const unsigned op = __shfl_xor_sync(~0u, p, stride);
  const bool take = keep_max ? (ok > k) : (ok < k);
  if (take) {
    k = ok;
    p = op;
  }
}

// Bitonic sort of one value per lane, ascending over lanes.
__device__ __forceinline__ void sort32_ascending(unsigned long long& k, unsigned& p) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      const bool up = (lane & size) == 0;
      const bool lower = (lane & stride) == 0;
      cmpx_lane(k, p, stride, lower != up);
    }
  }
}

// Sorts a bitonic list of M = 32R elements into descending order.
template <int R>
__device__ __forceinline__ void bitonic_merge_desc(TopList<R>& L) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int sr = R / 2; sr > 0; sr >>= 1) {  // strides of 32*sr elements: across registers
#pragma unroll
    for (int j = 0; j < R; ++j) {
      const int jp = j ^ sr;
      if (jp > j && L.k[jp] > L.k[j]) {
        const unsigned long long tk = L.k[j];
        const unsigned tp = L.p[j];
        L.k[j] = L.k[jp];
        L.p[j] = L.p[jp];
        L.k[jp] = tk;
        L.p[jp] = tp;
      }
    }
  }
#pragma unroll
  for (int stride = 16; stride > 0; stride >>= 1) {
    const bool lower = (lane & stride) == 0;
#pragma unroll
    for (int j = 0; j < R; ++j) cmpx_lane(L.k[j], L.p[j], stride, lower);
  }
}

// Offers one (key, payload) per lane (key 0: nothing).  Keeps the list the
// top M of everything offered so far.
template <int R>
__device__ __forceinline__ void toplist_offer(TopList<R>& L, unsigned long long key, unsigned pay) {
  const unsigned long long theta = __shfl_sync(~0u, L.k[R - 1], 31);
  if (!__any_sync(~0u, key > theta)) return;
  sort32_ascending(key, pay);
  // The top M of (descending list) u (ascending 32) is max(list[i], new[i - (M-32)]).
  if (key > L.k[R - 1]) {
    L.k[R - 1] = key;
    L.p[R - 1] = pay;
  }
  bitonic_merge_desc<R>(L);
}

// Merges another descending list of the same length, read from memory, into L.
template <int R>
__device__ __forceinline__ void toplist_merge(TopList<R>& L, const unsigned long long* ok, const unsigned* op) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    // Element i = 32j + lane pairs with the other list's element M-1-i.
    const int i = (R - 1 - j) * 32 + (31 - lane);
    const unsigned long long k2 = ok[i];
    if (k2 > L.k[j]) {
      L.k[j] = k2;
      L.p[j] = op[i];
    }
  }
  bitonic_merge_desc<R>(L);
}

template <int R>
__device__ __forceinline__ void toplist_store(const TopList<R>& L, unsigned long long* k, unsigned* p) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    k[j * 32 + lane] = L.k[j];
    p[j * 32 + lane] = L.p[j];
  }
}

// Tree merge of the lists of all warps of the CTA through shared memory
// (skey / spay: nwarps * 32R entries).  The result is in warp 0's registers
// and at skey[0..32R).
template <int R>
__device__ __forceinline__ void toplist_cta_merge(TopList<R>& T, unsigned long long* skey, unsigned* spay) {
  constexpr int M = 32 * R;
  const int warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  toplist_store<R>(T, skey + warp * M, spay + warp * M);
  __syncthreads();
  for (int half = nw / 2; half > 0; half >>= 1) {
    if (warp < half) toplist_merge<R>(T, skey + (warp + half) * M, spay + (warp + half) * M);
    __syncthreads();
    if (warp < half) toplist_store<R>(T, skey + warp * M, spay + warp * M);
    __syncthreads();
  }
}

}  // namespace mcd
