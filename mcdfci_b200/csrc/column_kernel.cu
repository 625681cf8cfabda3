// Column kernel: Hamiltonian column generation fused with the hash-table
// z-update, one thread-block cluster per picked determinant.
//
// Replaces, per iteration, HamiltonianMolecule::get_column (src/hamiltonian.h:
// 412-424, called at src/solver.h:717-739) and stage 1 of
// WaveFunctionCuckoo::update_z_and_get_sub (src/wavefunction.h:468-552): for
// every connected determinant D' of column c (value H = <D'|H|D_c>):
//
//   dz = H * dx_c
//   if |dz * scale| > z_threshold: upsert z[D'] += dz   (insert {x=0, z=dz} if absent)
//   else:                          z[D'] += dz only if D' is present
//   new_z_c += H * x[D'];  dot += dz * x[D']
//   candidate score |x[D'] * xss + z[D']| (value right after this update)
//
// and keeps, per column, the `estimate` (m) candidates with the largest score,
// as the reference's per-thread priority queue does (src/wavefunction.h:544-551).
//
// Work decomposition.  The connected determinants of any determinant in a
// fixed (n_alpha, n_beta) sector form the same index space, so entry e of a
// column is decoded arithmetically from the occupied/virtual orbital lists:
//   e = 0                       diagonal
//   [off1, off2)  alpha singles  (i occ, a vir)
//   [off2, off3)  beta singles
//   [off3, off4)  alpha-alpha doubles  (occupied pair, virtual pair)
//   [off4, off5)  beta-beta doubles
//   [off5, total) alpha-beta doubles   (ia, ib, aa, ab), ab fastest so that
//                 consecutive threads read consecutive integral-table entries
// Cluster rank r of the column's C CTAs takes the r-th contiguous slice.
//
// Candidates.  Each warp streams its entries through a buffer of cap_w slots in
// shared memory with a running threshold (keys <= the m-th best so far are
// dropped; the buffer is compacted to its top m when it would overflow).  The
// thresholds of all warps of the cluster are shared through a 64-bit maximum
// in CTA 0's shared memory (distributed shared memory), so later warps drop
// most entries at once.  At the end, warp 0 of each CTA merges its CTA's warp
// lists, and warp 0 of CTA 0 merges the CTA lists of the cluster.
#include <cooperative_groups.h>

#include "device_common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace mcd {
namespace {

constexpr int kNT = 256;
constexpr int kW = kNT / 32;

struct Prelude {
  uint64_t a, b;
  int na, nb, va, vb, nocc;
  int ca_occ, cb_occ, ca_vir, cb_vir;
  int off2, off3, off4, off5, total;
  unsigned char occA[64], occB[64], virA[64], virB[64], occso[128];
};

// Built by one full warp.
__device__ void build_prelude(Prelude& P, Det d, int norb) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  int na = 0, nb = 0, va = 0, vb = 0;
  for (int half = 0; half < 2; ++half) {
    const int p = lane + 32 * half;
    const bool inr = p < norb;
    const bool oa = inr && ((d.a >> p) & 1ull);
    const bool ob = inr && ((d.b >> p) & 1ull);
    const bool xa = inr && !oa, xb = inr && !ob;
    unsigned m = __ballot_sync(~0u, oa);
    if (oa) P.occA[na + __popc(m & lt)] = (unsigned char)p;
    na += __popc(m);
    m = __ballot_sync(~0u, ob);
    if (ob) P.occB[nb + __popc(m & lt)] = (unsigned char)p;
    nb += __popc(m);
    m = __ballot_sync(~0u, xa);
    if (xa) P.virA[va + __popc(m & lt)] = (unsigned char)p;
    va += __popc(m);
    m = __ballot_sync(~0u, xb);
    if (xb) P.virB[vb + __popc(m & lt)] = (unsigned char)p;
    vb += __popc(m);
  }
  int nocc = 0;
  for (int j = 0; j < 4; ++j) {
    const int s = lane + 32 * j;
    const int p = s >> 1;
    const bool o = p < norb && ((((s & 1) ? d.b : d.a) >> p) & 1ull);
    const unsigned m = __ballot_sync(~0u, o);
    if (o) P.occso[nocc + __popc(m & lt)] = (unsigned char)s;
    nocc += __popc(m);
  }
  if (lane == 0) {
    P.a = d.a;
    P.b = d.b;
    P.na = na;
    P.nb = nb;
    P.va = va;
    P.vb = vb;
    P.nocc = nocc;
    P.ca_occ = na * (na - 1) / 2;
    P.cb_occ = nb * (nb - 1) / 2;
    P.ca_vir = va * (va - 1) / 2;
    P.cb_vir = vb * (vb - 1) / 2;
    P.off2 = 1 + na * va;
    P.off3 = P.off2 + nb * vb;
    P.off4 = P.off3 + P.ca_occ * P.ca_vir;
    P.off5 = P.off4 + P.cb_occ * P.cb_vir;
    P.total = P.off5 + na * nb * va * vb;
  }
  __syncwarp();
}

// Pair index t -> (i, j), i < j, with t = j(j-1)/2 + i.
__device__ __forceinline__ void pair_decode(int t, int& i, int& j) {
  int jj = static_cast<int>((1.0f + sqrtf(8.0f * static_cast<float>(t) + 1.0f)) * 0.5f);
  while (jj * (jj - 1) / 2 > t) --jj;
  while ((jj + 1) * jj / 2 <= t) ++jj;
  j = jj;
  i = t - jj * (jj - 1) / 2;
}

// Single p->r of spin s (0 alpha, 1 beta): h_pr + sum over occupied
// spin-orbitals k (interleaved order) of <pk||rk>, as
// get_single_excitation sums it (src/hamiltonian.h:343-347).
__device__ __forceinline__ double single_value(const HamDev& h, const Prelude& P, int s, int p, int r) {
  const int n = h.norb;
  const size_t base = (static_cast<size_t>(s) * n + p) * n + r;
  const double* st = h.st + base * h.nso;
  double v = __ldg(h.sh + base);
  for (int x = 0; x < P.nocc; ++x) v += __ldg(st + P.occso[x]);
  return v;
}

// Entry e of the column of P's determinant: (a2, b2) and the signed value.
// Returns false when the reference stores no such excitation.
__device__ __forceinline__ bool gen_entry(const HamDev& h, const Prelude& P, int e, double hdiag,
                                          uint64_t& a2, uint64_t& b2, double& v) {
  const uint64_t a = P.a, b = P.b;
  const int n = h.norb;
  if (e == 0) {
    a2 = a;
    b2 = b;
    v = hdiag;
    return true;
  }
  if (e < P.off2) {
    const int t = e - 1;
    const int i = t / P.va, ri = t - i * P.va;
    const int p = P.occA[i], r = P.virA[ri];
    if (!((__ldg(h.spres + p) >> r) & 1ull)) return false;
    double val = single_value(h, P, 0, p, r);
    if (sign_alpha(a, b, p, r)) val = -val;
    a2 = a ^ (1ull << p) ^ (1ull << r);
    b2 = b;
    v = val;
    return true;
  }
  if (e < P.off3) {
    const int t = e - P.off2;
    const int i = t / P.vb, ri = t - i * P.vb;
    const int p = P.occB[i], r = P.virB[ri];
    if (!((__ldg(h.spres + n + p) >> r) & 1ull)) return false;
    double val = single_value(h, P, 1, p, r);
    if (sign_beta(a, b, p, r)) val = -val;
    a2 = a;
    b2 = b ^ (1ull << p) ^ (1ull << r);
    v = val;
    return true;
  }
  if (e < P.off4) {
    const int t = e - P.off3;
    const int op = t / P.ca_vir, vp = t - op * P.ca_vir;
    int i, j, ri, sj;
    pair_decode(op, i, j);
    pair_decode(vp, ri, sj);
    const int p = P.occA[i], q = P.occA[j], r = P.virA[ri], s = P.virA[sj];
    double val = __ldg(h.vss + static_cast<size_t>(pair_index(p, q)) * h.npair + pair_index(r, s));
    if (val == 0.0) return false;
    if (sign_aa(a, b, p, q, r, s)) val = -val;
    a2 = a ^ (1ull << p) ^ (1ull << q) ^ (1ull << r) ^ (1ull << s);
    b2 = b;
    v = val;
    return true;
  }
  if (e < P.off5) {
    const int t = e - P.off4;
    const int op = t / P.cb_vir, vp = t - op * P.cb_vir;
    int i, j, ri, sj;
    pair_decode(op, i, j);
    pair_decode(vp, ri, sj);
    const int p = P.occB[i], q = P.occB[j], r = P.virB[ri], s = P.virB[sj];
    const size_t np = static_cast<size_t>(h.npair);
    double val = __ldg(h.vss + (np + pair_index(p, q)) * np + pair_index(r, s));
    if (val == 0.0) return false;
    if (sign_bb(a, b, p, q, r, s)) val = -val;
    a2 = a;
    b2 = b ^ (1ull << p) ^ (1ull << q) ^ (1ull << r) ^ (1ull << s);
    v = val;
    return true;
  }
  int t = e - P.off5;
  const int sbi = t % P.vb;
  t /= P.vb;
  const int rai = t % P.va;
  t /= P.va;
  const int pbi = t % P.nb;
  const int pai = t / P.nb;
  const int pa = P.occA[pai], pb = P.occB[pbi], ra = P.virA[rai], sb = P.virB[sbi];
  double val = __ldg(h.wab + ((static_cast<size_t>(pa) * n + pb) * n + ra) * n + sb);
  if (val == 0.0) return false;
  if (sign_ab(a, b, pa, ra, pb, sb)) val = -val;
  a2 = a ^ (1ull << pa) ^ (1ull << ra);
  b2 = b ^ (1ull << pb) ^ (1ull << sb);
  v = val;
  return true;
}

// ---------------------------------------------------------------------------
// Per-warp top-M list of (key, slot) kept in registers, sorted descending:
// element i is held by lane i % 32 in register i / 32.  Keys are the bit
// pattern of the non-negative score plus one (so unsigned order is value
// order); 0 marks an empty element.
template <int R>
struct TopList {
  unsigned long long k[R];
  unsigned p[R];
};

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

// Offers one (key, slot) per lane (key 0: nothing).  Keeps the list the
// top M of everything offered so far.
template <int R>
__device__ __forceinline__ void toplist_offer(TopList<R>& L, unsigned long long key, unsigned slot) {
  const unsigned long long theta = __shfl_sync(~0u, L.k[R - 1], 31);
  if (!__any_sync(~0u, key > theta)) return;
  sort32_ascending(key, slot);
  // The top M of (descending list) u (ascending 32) is max(list[i], new[i - (M-32)]).
  if (key > L.k[R - 1]) {
    L.k[R - 1] = key;
    L.p[R - 1] = slot;
  }
  bitonic_merge_desc<R>(L);
}

// Merges another descending list, read from memory, into L.
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

template <int R>
__device__ __forceinline__ void toplist_load(TopList<R>& L, const unsigned long long* k, const unsigned* p) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    L.k[j] = k[j * 32 + lane];
    L.p[j] = p[j * 32 + lane];
  }
}

__device__ __forceinline__ double score_of(double x, double z, dd xss) {
  if (x == 0.0) return fabs(z);
  const dd t = dd_add_d(dd_mul_d(xss, x), z);
  return fabs(t.hi + t.lo);
}

// ---------------------------------------------------------------------------

template <int R>
__global__ void __launch_bounds__(kNT, 3) column_kernel(ColumnLaunch L) {
  constexpr int M = 32 * R;
  cg::cluster_group cluster = cg::this_cluster();
  const int C = L.cluster;
  const int rank = static_cast<int>(cluster.block_rank());
  const int col = blockIdx.x / C;
  IterState* S = L.st;
  const int kcur = S->k_cur;
  if (col >= kcur) return;  // every CTA of this cluster has the same column

  __shared__ Prelude P;
  __shared__ unsigned long long s_key[kW][M];
  __shared__ unsigned s_pay[kW][M];
  __shared__ double w_newz[kW], w_dot[kW];
  __shared__ unsigned w_emit[kW], w_upd[kW], w_ins[kW];
  __shared__ double cta_newz, cta_dot;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) build_prelude(P, S->det[col], L.ham.norb);
  __syncthreads();

  const double dxc = S->dx[col];
  const double hd = S->hdiag[col];
  const dd xss = S->xss;
  const dd scale = S->scale;
  const dd zt{S->zt, 0.0};
  const unsigned dslot = static_cast<unsigned>(S->slot[col]);
  const int total = P.total;
  const int per = (total + C - 1) / C;
  const int beg = min(total, rank * per);
  const int end = min(total, beg + per);
  const int nrounds = (end - beg + kNT - 1) / kNT;

  TopList<R> T;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    T.k[j] = 0ull;
    T.p[j] = 0u;
  }
  double acc_newz = 0.0, acc_dot = 0.0;
  unsigned emit = 0, upd = 0, ins = 0;

  for (int r = 0; r < nrounds; ++r) {
    const int e = beg + r * kNT + threadIdx.x;
    unsigned long long key = 0ull;
    unsigned slotu = 0u;
    if (e < end) {
      uint64_t a2, b2;
      double v;
      if (gen_entry(L.ham, P, e, hd, a2, b2, v)) {
        ++emit;
        const double dz = v * dxc;
        const bool above = dd_gt(dd_abs(dd_mul_d(scale, dz)), zt);
        long long slot;
        if (e == 0) {
          slot = dslot;
        } else if (above) {
          bool inserted;
          slot = table_upsert(L.tab, a2, b2, inserted);
          ins += inserted ? 1u : 0u;
        } else {
          slot = table_find(L.tab, a2, b2);
        }
        if (slot >= 0) {
          Slot* sp = L.tab.slots + slot;
          const double x = sp->x;
          const double znew = atomicAdd(&sp->z, dz) + dz;
          ++upd;
          acc_newz += v * x;
          acc_dot += dz * x;
          key = static_cast<unsigned long long>(__double_as_longlong(score_of(x, znew, xss))) + 1ull;
          slotu = static_cast<unsigned>(slot);
        }
      }
    }
    toplist_offer<R>(T, key, slotu);
  }

  acc_newz = warp_sum(acc_newz);
  acc_dot = warp_sum(acc_dot);
  emit = __reduce_add_sync(~0u, emit);
  upd = __reduce_add_sync(~0u, upd);
  ins = __reduce_add_sync(~0u, ins);
  toplist_store<R>(T, s_key[warp], s_pay[warp]);
  if (lane == 0) {
    w_newz[warp] = acc_newz;
    w_dot[warp] = acc_dot;
    w_emit[warp] = emit;
    w_upd[warp] = upd;
    w_ins[warp] = ins;
  }
  __syncthreads();
  // Tree merge of the warp lists inside the CTA; the result lands in s_key[0].
#pragma unroll
  for (int half = kW / 2; half > 0; half >>= 1) {
    if (warp < half) toplist_merge<R>(T, s_key[warp + half], s_pay[warp + half]);
    __syncthreads();
    if (warp < half) toplist_store<R>(T, s_key[warp], s_pay[warp]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double nz = 0.0, dt = 0.0;
    unsigned long long e2 = 0, u2 = 0, i2 = 0;
    for (int w = 0; w < kW; ++w) {
      nz += w_newz[w];
      dt += w_dot[w];
      e2 += w_emit[w];
      u2 += w_upd[w];
      i2 += w_ins[w];
    }
    cta_newz = nz;
    cta_dot = dt;
    if (e2) {
      atomicAdd(&S->emitted, e2);
      atomicAdd(&S->emitted_total, e2);
    }
    if (u2) {
      atomicAdd(&S->updates, u2);
      atomicAdd(&S->updates_total, u2);
    }
    if (i2) atomicAdd(&S->z_size, i2);
  }
  cluster.sync();

  if (rank == 0) {
    // Warp w of CTA 0 merges the lists of CTAs w, w+kW (distributed shared memory).
    TopList<R> U;
#pragma unroll
    for (int j = 0; j < R; ++j) {
      U.k[j] = 0ull;
      U.p[j] = 0u;
    }
    for (int rr = warp; rr < C; rr += kW) {
      const unsigned long long* rk = cluster.map_shared_rank(&s_key[0][0], rr);
      const unsigned* rp = cluster.map_shared_rank(&s_pay[0][0], rr);
      toplist_merge<R>(U, rk, rp);
    }
    // Own CTA-list sits in s_key[0]; every warp is done reading it before
    // s_key[w] is overwritten.
    __syncthreads();
    toplist_store<R>(U, s_key[warp], s_pay[warp]);
    __syncthreads();
#pragma unroll
    for (int half = kW / 2; half > 0; half >>= 1) {
      if (warp < half) toplist_merge<R>(U, s_key[warp + half], s_pay[warp + half]);
      __syncthreads();
      if (warp < half) toplist_store<R>(U, s_key[warp], s_pay[warp]);
      __syncthreads();
    }
    if (warp == 0) {
      int n = 0;
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int i = j * 32 + lane;
        const bool ok = i < L.m && U.k[j] != 0ull;
        if (ok) {
          L.cand_score[static_cast<size_t>(col) * L.m + i] = __longlong_as_double(static_cast<long long>(U.k[j] - 1ull));
          L.cand_slot[static_cast<size_t>(col) * L.m + i] = U.p[j];
        }
        n += __popc(__ballot_sync(~0u, ok));
      }
      if (lane == 0) {
        double nz = 0.0, dt = 0.0;
        for (int rr = 0; rr < C; ++rr) {
          nz += *cluster.map_shared_rank(&cta_newz, rr);
          dt += *cluster.map_shared_rank(&cta_dot, rr);
        }
        S->newz[col] = nz;
        S->dot[col] = dt;
        S->cand_n[col] = n;
      }
    }
  }
  cluster.sync();
}

__global__ void __launch_bounds__(kNT) debug_column_kernel(HamDev h, Det d, double hd, uint64_t* ao,
                                                           uint64_t* bo, double* vo, int cap, int* nout) {
  __shared__ Prelude P;
  if ((threadIdx.x >> 5) == 0) build_prelude(P, d, h.norb);
  __syncthreads();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < P.total; e += gridDim.x * blockDim.x) {
    uint64_t a2, b2;
    double v;
    if (gen_entry(h, P, e, hd, a2, b2, v)) {
      const int pos = atomicAdd(nout, 1);
      if (pos < cap) {
        ao[pos] = a2;
        bo[pos] = b2;
        vo[pos] = v;
      }
    }
  }
}

template <int R>
cudaLaunchConfig_t column_config(const ColumnLaunch& a, cudaStream_t s, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.k_grid * a.cluster, 1, 1);
  cfg.blockDim = dim3(kNT, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = a.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <int R>
cudaError_t launch_column_r(const ColumnLaunch& a, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(column_kernel<R>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = column_config<R>(a, s, attr);
  return cudaLaunchKernelEx(&cfg, column_kernel<R>, a);
}

template <int R>
int max_active_clusters_r(int cluster) {
  ColumnLaunch a{};
  a.k_grid = 64;
  a.cluster = cluster;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = column_config<R>(a, 0, attr);
  cudaFuncSetAttribute(column_kernel<R>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, column_kernel<R>, &cfg) != cudaSuccess) return -1;
  return n;
}

}  // namespace

int column_entries(int norb, int na, int nb) {
  const long long va = norb - na, vb = norb - nb;
  const long long t = 1 + na * va + nb * vb + (long long)na * (na - 1) / 2 * (va * (va - 1) / 2) +
                      (long long)nb * (nb - 1) / 2 * (vb * (vb - 1) / 2) + (long long)na * nb * va * vb;
  return t > 0x7fffffffLL ? -1 : static_cast<int>(t);
}

cudaError_t launch_column(const ColumnLaunch& a, cudaStream_t s) {
  if (a.m <= 32) return launch_column_r<1>(a, s);
  if (a.m <= 64) return launch_column_r<2>(a, s);
  return launch_column_r<4>(a, s);
}

int column_max_active_clusters(int cluster, int m) {
  if (m <= 32) return max_active_clusters_r<1>(cluster);
  if (m <= 64) return max_active_clusters_r<2>(cluster);
  return max_active_clusters_r<4>(cluster);
}

cudaError_t debug_column(const HamDev& h, Det d, double hdiag, uint64_t* a_out, uint64_t* b_out,
                         double* v_out, int cap, int* n_out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(n_out, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  debug_column_kernel<<<64, kNT, 0, s>>>(h, d, hdiag, a_out, b_out, v_out, cap, n_out);
  return cudaGetLastError();
}

}  // namespace mcd
