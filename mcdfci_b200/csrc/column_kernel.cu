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
// Warp-level top-m buffer.  Keys are the bit patterns of non-negative doubles,
// so unsigned order is value order.

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(~0u, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// Keeps the m largest keys of buf[0..cnt) (equal keys: earlier positions
// first), compacted in place.  Returns the new count and sets thr to the
// smallest kept key.  cnt <= 5*32.
__device__ int warp_keep_top(unsigned long long* key, long long* pay, int cnt, int m,
                             unsigned long long& thr) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  unsigned long long k[5];
  long long pl[5];
  bool ok[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    const int idx = j * 32 + lane;
    ok[j] = idx < cnt;
    k[j] = ok[j] ? key[idx] : 0ull;
    pl[j] = ok[j] ? pay[idx] : 0ll;
  }
  __syncwarp();
  unsigned long long K = 0;
  bool exact = false;
  for (int bit = 63; bit >= 0; --bit) {
    const unsigned long long c = K | (1ull << bit);
    unsigned n = 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) n += (ok[j] && k[j] >= c) ? 1u : 0u;
    n = __reduce_add_sync(~0u, n);
    if (n >= static_cast<unsigned>(m)) {
      K = c;
      if (n == static_cast<unsigned>(m)) {
        exact = true;
        break;
      }
    }
  }
  bool keep[5];
  if (exact) {
#pragma unroll
    for (int j = 0; j < 5; ++j) keep[j] = ok[j] && k[j] >= K;
  } else {
    unsigned ngt = 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) ngt += (ok[j] && k[j] > K) ? 1u : 0u;
    ngt = __reduce_add_sync(~0u, ngt);
    const int need = m - static_cast<int>(ngt);
    int prior = 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      const bool eq = ok[j] && k[j] == K;
      const unsigned em = __ballot_sync(~0u, eq);
      const int rank = prior + __popc(em & lt);
      keep[j] = (ok[j] && k[j] > K) || (eq && rank < need);
      prior += __popc(em);
    }
  }
  int pos = 0;
  unsigned long long mn = ~0ull;
#pragma unroll
  for (int j = 0; j < 5; ++j) {
    const unsigned km = __ballot_sync(~0u, keep[j]);
    if (keep[j]) {
      const int dst = pos + __popc(km & lt);
      key[dst] = k[j];
      pay[dst] = pl[j];
      mn = k[j] < mn ? k[j] : mn;
    }
    pos += __popc(km);
  }
  thr = warp_min_u64(mn);
  __syncwarp();
  return pos;
}

struct WarpBuf {
  unsigned long long* key;
  long long* pay;
  int cnt;
  int m;
  int cap;
  bool have;               // thr valid
  unsigned long long thr;  // keys <= thr are dropped
};

// Each lane offers one (key, payload) when `valid`.  Whole warp calls.
__device__ __forceinline__ void warp_offer(WarpBuf& B, bool valid, unsigned long long k, long long p,
                                           bool have_ext, unsigned long long thr_ext) {
  bool have = B.have || have_ext;
  unsigned long long thr = B.have ? B.thr : 0ull;
  if (have_ext && (!B.have || thr_ext > thr)) thr = thr_ext;
  bool pass = valid && (!have || k > thr);
  unsigned bal = __ballot_sync(~0u, pass);
  int n = __popc(bal);
  if (B.cnt + n > B.cap) {
    B.cnt = warp_keep_top(B.key, B.pay, B.cnt, B.m, B.thr);
    B.have = true;
    if (!have_ext || B.thr > thr_ext) thr = B.thr; else thr = thr_ext;
    pass = valid && k > thr;
    bal = __ballot_sync(~0u, pass);
    n = __popc(bal);
  }
  if (pass) {
    const int dst = B.cnt + __popc(bal & lanemask_lt());
    B.key[dst] = k;
    B.pay[dst] = p;
  }
  B.cnt += n;
  __syncwarp();
}

__device__ __forceinline__ void warp_finish(WarpBuf& B) {
  if (B.cnt > B.m) {
    B.cnt = warp_keep_top(B.key, B.pay, B.cnt, B.m, B.thr);
    B.have = true;
  }
}

__device__ __forceinline__ double score_of(double x, double z, dd xss) {
  if (x == 0.0) return fabs(z);
  const dd t = dd_add_d(dd_mul_d(xss, x), z);
  return fabs(t.hi + t.lo);
}

// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(kNT) column_kernel(ColumnLaunch L) {
  cg::cluster_group cluster = cg::this_cluster();
  const int C = L.cluster;
  const int rank = static_cast<int>(cluster.block_rank());
  const int col = blockIdx.x / C;
  IterState* S = L.st;
  const int kcur = S->k_cur;
  if (col >= kcur) return;  // every CTA of this cluster has the same column

  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ Prelude P;
  __shared__ double w_newz[kW], w_dot[kW];
  __shared__ unsigned w_emit[kW], w_upd[kW], w_ins[kW];
  __shared__ int w_cnt[kW];
  __shared__ unsigned long long theta;  // cluster threshold + 1 (0: none yet), used in rank 0
  __shared__ double cta_newz, cta_dot;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned long long* keys0 = reinterpret_cast<unsigned long long*>(smem);
  long long* pays0 = reinterpret_cast<long long*>(smem + static_cast<size_t>(kW) * L.cap_w * 8);

  if (threadIdx.x == 0) theta = 0ull;
  if (warp == 0) build_prelude(P, S->det[col], L.ham.norb);
  cluster.sync();
  unsigned long long* theta0 = cluster.map_shared_rank(&theta, 0);

  const double dxc = S->dx[col];
  const double hd = S->hdiag[col];
  const dd xss = S->xss;
  const dd scale = S->scale;
  const dd zt{S->zt, 0.0};
  const long long dslot = S->slot[col];
  const int total = P.total;
  const int per = (total + C - 1) / C;
  const int beg = min(total, rank * per);
  const int end = min(total, beg + per);
  const int nrounds = (end - beg + kNT - 1) / kNT;

  WarpBuf B{keys0 + warp * L.cap_w, pays0 + warp * L.cap_w, 0, L.m, L.cap_w, false, 0ull};
  double acc_newz = 0.0, acc_dot = 0.0;
  unsigned emit = 0, upd = 0, ins = 0;
  unsigned long long cthr = 0ull;

  for (int r = 0; r < nrounds; ++r) {
    const int e = beg + r * kNT + threadIdx.x;
    bool cand = false;
    unsigned long long key = 0ull;
    long long slot = -1;
    if (e < end) {
      uint64_t a2, b2;
      double v;
      if (gen_entry(L.ham, P, e, hd, a2, b2, v)) {
        ++emit;
        const double dz = v * dxc;
        const bool above = dd_gt(dd_abs(dd_mul_d(scale, dz)), zt);
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
          key = static_cast<unsigned long long>(__double_as_longlong(score_of(x, znew, xss)));
          cand = true;
        }
      }
    }
    if ((r & 3) == 0) {
      unsigned long long t = 0ull;
      if (lane == 0) t = *reinterpret_cast<volatile unsigned long long*>(theta0);
      cthr = __shfl_sync(~0u, t, 0);
    }
    const bool had = B.have;
    const unsigned long long old = B.thr;
    warp_offer(B, cand, key, slot, cthr != 0ull, cthr - 1ull);
    if (B.have && (!had || B.thr != old) && lane == 0) atomicMax(theta0, B.thr + 1ull);
  }

  warp_finish(B);
  acc_newz = warp_sum(acc_newz);
  acc_dot = warp_sum(acc_dot);
  emit = __reduce_add_sync(~0u, emit);
  upd = __reduce_add_sync(~0u, upd);
  ins = __reduce_add_sync(~0u, ins);
  if (lane == 0) {
    w_newz[warp] = acc_newz;
    w_dot[warp] = acc_dot;
    w_emit[warp] = emit;
    w_upd[warp] = upd;
    w_ins[warp] = ins;
    w_cnt[warp] = B.cnt;
  }
  __syncthreads();

  if (warp == 0) {
    for (int w = 1; w < kW; ++w) {
      const int n = w_cnt[w];
      const unsigned long long* k2 = keys0 + w * L.cap_w;
      const long long* p2 = pays0 + w * L.cap_w;
      for (int c0 = 0; c0 < n; c0 += 32) {
        const int idx = c0 + lane;
        const bool ok = idx < n;
        warp_offer(B, ok, ok ? k2[idx] : 0ull, ok ? p2[idx] : -1ll, false, 0ull);
      }
    }
    warp_finish(B);
    if (lane == 0) {
      w_cnt[0] = B.cnt;
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
  }
  cluster.sync();

  if (rank == 0 && warp == 0) {
    for (int rr = 1; rr < C; ++rr) {
      const int n = *cluster.map_shared_rank(&w_cnt[0], rr);
      const unsigned long long* k2 = cluster.map_shared_rank(keys0, rr);
      const long long* p2 = cluster.map_shared_rank(pays0, rr);
      for (int c0 = 0; c0 < n; c0 += 32) {
        const int idx = c0 + lane;
        const bool ok = idx < n;
        warp_offer(B, ok, ok ? k2[idx] : 0ull, ok ? p2[idx] : -1ll, false, 0ull);
      }
    }
    warp_finish(B);
    for (int j = lane; j < B.cnt; j += 32) {
      L.cand_score[static_cast<size_t>(col) * L.m + j] = __longlong_as_double(static_cast<long long>(B.key[j]));
      L.cand_slot[static_cast<size_t>(col) * L.m + j] = B.pay[j];
    }
    if (lane == 0) {
      double nz = 0.0, dt = 0.0;
      for (int rr = 0; rr < C; ++rr) {
        nz += *cluster.map_shared_rank(&cta_newz, rr);
        dt += *cluster.map_shared_rank(&cta_dot, rr);
      }
      S->newz[col] = nz;
      S->dot[col] = dt;
      S->cand_n[col] = B.cnt;
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

}  // namespace

int column_entries(int norb, int na, int nb) {
  const long long va = norb - na, vb = norb - nb;
  const long long t = 1 + na * va + nb * vb + (long long)na * (na - 1) / 2 * (va * (va - 1) / 2) +
                      (long long)nb * (nb - 1) / 2 * (vb * (vb - 1) / 2) + (long long)na * nb * va * vb;
  return t > 0x7fffffffLL ? -1 : static_cast<int>(t);
}

size_t column_smem_bytes(int m, int nthreads) {
  const int cap = ((m + 31) / 32) * 32 + 32;
  return static_cast<size_t>(nthreads / 32) * cap * 16;
}

cudaError_t launch_column(const ColumnLaunch& a, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(column_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.k_grid * a.cluster, 1, 1);
  cfg.blockDim = dim3(kNT, 1, 1);
  cfg.dynamicSmemBytes = column_smem_bytes(a.m, kNT);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = a.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, column_kernel, a);
}

cudaError_t debug_column(const HamDev& h, Det d, double hdiag, uint64_t* a_out, uint64_t* b_out,
                         double* v_out, int cap, int* n_out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(n_out, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  debug_column_kernel<<<64, kNT, 0, s>>>(h, d, hdiag, a_out, b_out, v_out, cap, n_out);
  return cudaGetLastError();
}

}  // namespace mcd
