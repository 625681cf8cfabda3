// Column kernel: Hamiltonian column generation fused with the hash-table
// z-update; G CTAs per picked determinant.
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
// CTA g of the column's G CTAs takes the g-th contiguous slice, about three
// rounds of one entry per thread; CTAs are independent, so the grid runs in as
// many waves as the GPU needs.  Each thread starts the hash probe of its entry
// before it reads the integral value, so an entry costs two memory round
// trips: (table value, home slot key), then (z atomic, x).
//
// Candidates.  Each warp keeps a sorted top-M list (M = 32, 64 or 128 >= m)
// in registers: per round it sorts the 32 new keys with a bitonic network,
// takes the element-wise maximum with the list reversed (the top M of the
// union) and re-sorts with a bitonic merge; rounds whose keys cannot enter the
// list are skipped.  The warp lists of a CTA merge as a tree in shared memory;
// the CTA lists go to global memory, and the last CTA of the column to finish
// (atomic ticket) merges them and writes the column's m candidates, new z and
// dot products (summed in a fixed order).
#include "device_common.cuh"
#include <algorithm>

#include "kernels.h"
#include "toplist.cuh"

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
// Returns kNone when the reference stores no such excitation, kKeep for the
// diagonal and singles (kept whatever their value, as get_single_excitation
// does), and kIfNonzero for doubles, which the reference stores only with a
// non-zero table value.  Leaving that test to the caller lets it start the
// hash probe before the table value arrives.
enum : int { kNone = 0, kKeep = 1, kIfNonzero = 2 };

__device__ __forceinline__ int gen_entry(const HamDev& h, const Prelude& P, int e, double hdiag,
                                         uint64_t& a2, uint64_t& b2, double& v) {
  const uint64_t a = P.a, b = P.b;
  const int n = h.norb;
  if (e == 0) {
    a2 = a;
    b2 = b;
    v = hdiag;
    return kKeep;
  }
  if (e < P.off2) {
    const int t = e - 1;
    const int i = t / P.va, ri = t - i * P.va;
    const int p = P.occA[i], r = P.virA[ri];
    if (!((__ldg(h.spres + p) >> r) & 1ull)) return kNone;
    double val = single_value(h, P, 0, p, r);
    if (sign_alpha(a, b, p, r)) val = -val;
    a2 = a ^ (1ull << p) ^ (1ull << r);
    b2 = b;
    v = val;
    return kKeep;
  }
  if (e < P.off3) {
    const int t = e - P.off2;
    const int i = t / P.vb, ri = t - i * P.vb;
    const int p = P.occB[i], r = P.virB[ri];
    if (!((__ldg(h.spres + n + p) >> r) & 1ull)) return kNone;
    double val = single_value(h, P, 1, p, r);
    if (sign_beta(a, b, p, r)) val = -val;
    a2 = a;
    b2 = b ^ (1ull << p) ^ (1ull << r);
    v = val;
    return kKeep;
  }
  if (e < P.off4) {
    const int t = e - P.off3;
    const int op = t / P.ca_vir, vp = t - op * P.ca_vir;
    int i, j, ri, sj;
    pair_decode(op, i, j);
    pair_decode(vp, ri, sj);
    const int p = P.occA[i], q = P.occA[j], r = P.virA[ri], s = P.virA[sj];
    const double val = __ldg(h.vss + static_cast<size_t>(pair_index(p, q)) * h.npair + pair_index(r, s));
    v = sign_aa(a, b, p, q, r, s) ? -val : val;
    a2 = a ^ (1ull << p) ^ (1ull << q) ^ (1ull << r) ^ (1ull << s);
    b2 = b;
    return kIfNonzero;
  }
  if (e < P.off5) {
    const int t = e - P.off4;
    const int op = t / P.cb_vir, vp = t - op * P.cb_vir;
    int i, j, ri, sj;
    pair_decode(op, i, j);
    pair_decode(vp, ri, sj);
    const int p = P.occB[i], q = P.occB[j], r = P.virB[ri], s = P.virB[sj];
    const size_t np = static_cast<size_t>(h.npair);
    const double val = __ldg(h.vss + (np + pair_index(p, q)) * np + pair_index(r, s));
    v = sign_bb(a, b, p, q, r, s) ? -val : val;
    a2 = a;
    b2 = b ^ (1ull << p) ^ (1ull << q) ^ (1ull << r) ^ (1ull << s);
    return kIfNonzero;
  }
  int t = e - P.off5;
  const int sbi = t % P.vb;
  t /= P.vb;
  const int rai = t % P.va;
  t /= P.va;
  const int pbi = t % P.nb;
  const int pai = t / P.nb;
  const int pa = P.occA[pai], pb = P.occB[pbi], ra = P.virA[rai], sb = P.virB[sbi];
  const double val = __ldg(h.wab + ((static_cast<size_t>(pa) * n + pb) * n + ra) * n + sb);
  v = sign_ab(a, b, pa, ra, pb, sb) ? -val : val;
  a2 = a ^ (1ull << pa) ^ (1ull << ra);
  b2 = b ^ (1ull << pb) ^ (1ull << sb);
  return kIfNonzero;
}

// |dz scale| > zt, the insertion rule (src/wavefunction.h:517-528): a double
// product decides unless it lies within 1e-14 of zt, where the
// double-double product does.
__device__ __forceinline__ bool above_threshold(dd scale, double dz, double zt) {
  const double sd = fabs(scale.hi * dz);
  if (sd > zt * (1.0 + 1e-14)) return true;
  if (sd < zt * (1.0 - 1e-14)) return false;
  return dd_gt(dd_abs(dd_mul_d(scale, dz)), dd{zt, 0.0});
}

// ---------------------------------------------------------------------------

// Reads a descending list stored in global memory by another CTA (through
// L2, bypassing L1), reversed into ascending order for the bitonic merge.
template <int R>
__device__ __forceinline__ void toplist_load_global(TopList<R>& T, const unsigned long long* ok,
                                                    const unsigned* op) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int i = (R - 1 - j) * 32 + (31 - lane);
    T.k[j] = __ldcg(ok + i);
    T.p[j] = __ldcg(op + i);
  }
}

// Merge a list held in ascending order (as toplist_load_global leaves it)
// into the descending list L.
template <int R>
__device__ __forceinline__ void toplist_merge_loaded(TopList<R>& L, const TopList<R>& T) {
#pragma unroll
  for (int j = 0; j < R; ++j) {
    if (T.k[j] > L.k[j]) {
      L.k[j] = T.k[j];
      L.p[j] = T.p[j];
    }
  }
  bitonic_merge_desc<R>(L);
}

template <int R>
__device__ __forceinline__ void toplist_merge_global(TopList<R>& L, const unsigned long long* ok,
                                                     const unsigned* op) {
  TopList<R> T;
  toplist_load_global<R>(T, ok, op);
  toplist_merge_loaded<R>(L, T);
}

// One CTA's share of one column: CTA `blk` of the launch described by L
// (column blk / groups, slice blk % groups).
template <int R>
__device__ __forceinline__ void column_body(const ColumnLaunch& L, int blk) {
  constexpr int M = 32 * R;
  const int G = L.groups;
  const int col = blk / G;
  const int g = blk - col * G;
  IterState* S = L.st;
  const int kcur = S->k_cur;
  if (col >= kcur) return;

  __shared__ Prelude P;
  __shared__ unsigned long long s_key[kW][M];
  __shared__ unsigned s_pay[kW][M];
  __shared__ double w_newz[kW], w_dot[kW];
  __shared__ unsigned w_emit[kW], w_upd[kW], w_ins[kW];
  __shared__ int s_last;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool timed = L.sect != nullptr && threadIdx.x == 0;
  const long long c_start = timed ? clock64() : 0;
  // The column's scalars are read while warp 0 decodes the determinant.
  const double dxc = S->dx[col];
  const double hd = S->hdiag[col];
  const dd xss = S->xss;
  const dd scale = S->scale;
  const dd zt{S->zt, 0.0};
  const unsigned dslot = static_cast<unsigned>(S->slot[col]);
  if (warp == 0) build_prelude(P, S->det[col], L.ham.norb);
  __syncthreads();
  const int total = P.total;
  const int per = (total + G - 1) / G;
  const int beg = min(total, g * per);
  const int end = min(total, beg + per);
  const int nrounds = (end - beg + kNT - 1) / kNT;

  TopList<R> T;
  toplist_clear<R>(T);
  double acc_newz = 0.0, acc_dot = 0.0;
  unsigned emit = 0, upd = 0, ins = 0;

  unsigned long long t_gen = 0, t_probe = 0, t_upd = 0, t_off = 0;
  const long long c_rounds = timed ? clock64() : 0;
  for (int r = 0; r < nrounds; ++r) {
    long long q0 = timed ? clock64() : 0;
    const int e = beg + r * kNT + threadIdx.x;
    unsigned long long key = 0ull;
    unsigned slotu = 0u;
    if (e < end) {
      uint64_t a2, b2;
      double v;
      const int kind = gen_entry(L.ham, P, e, hd, a2, b2, v);
      if (kind != kNone) {
        // Start the probe at the home slot before the integral value is used
        // (the diagonal entry's slot is the picked determinant's own).
        const uint64_t home = e == 0 ? static_cast<uint64_t>(dslot) : det_hash(a2, b2) & L.tab.mask;
        uint64_t ka = 0, kb = 0;
        load_key(L.tab.slots + home, ka, kb);
        long long q1 = 0;
        if (timed) {
          q1 = clock64();
          t_gen += q1 - q0;
        }
        if (kind == kKeep || v != 0.0) {
          ++emit;
          const double dz = v * dxc;
          bool inserted;
          const long long slot =
              table_probe_from(L.tab, a2, b2, home, ka, kb, above_threshold(scale, dz, zt.hi), inserted);
          ins += inserted ? 1u : 0u;
          long long q2 = 0;
          if (timed) {
            q2 = clock64();
            t_probe += q2 - q1;
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
            if (timed) t_upd += clock64() - q2;
          }
        }
      }
    }
    const long long q3 = timed ? clock64() : 0;
    toplist_offer<R>(T, key, slotu);
    if (timed) t_off += clock64() - q3;
  }
  const long long c_post = timed ? clock64() : 0;
  if (timed) {
    atomicAdd(L.sect + 0, t_gen);
    atomicAdd(L.sect + 1, t_probe);
    atomicAdd(L.sect + 2, t_upd);
    atomicAdd(L.sect + 3, t_off);
    atomicAdd(L.sect + 4, static_cast<unsigned long long>(nrounds));
    atomicAdd(L.sect + 5, static_cast<unsigned long long>(c_rounds - c_start));
    atomicAdd(L.sect + 8, 1ull);
  }

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
  }
  toplist_cta_merge<R>(T, &s_key[0][0], &s_pay[0][0]);

  // This CTA's list and partial sums to global memory, then a ticket: the
  // last CTA of the column merges all of them.
  const size_t part = static_cast<size_t>(col) * G + g;
  if (warp == 0) toplist_store<R>(T, L.part_key + part * M, L.part_slot + part * M);
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
    // The counters travel with the sums (exact in a double) and are added
    // once per column by its last CTA, not by every CTA into the same words.
    double* ps = L.part_sum + kPartSum * part;
    ps[0] = nz;
    ps[1] = dt;
    ps[2] = static_cast<double>(e2);
    ps[3] = static_cast<double>(u2);
    ps[4] = static_cast<double>(i2);
  }
  // Only warp 0 wrote what the column's last CTA reads (the list and the
  // partial sums); its fence orders those writes before the ticket.
  if (warp == 0) __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(L.done + col, 1u) == static_cast<unsigned>(G - 1));
  __syncthreads();
  const long long c_merge = timed ? clock64() : 0;
  if (timed) atomicAdd(L.sect + 6, static_cast<unsigned long long>(c_merge - c_post));
  if (!s_last) return;
  __threadfence();

  // Last CTA of the column: merge the G CTA lists (warp w takes w, w+kW, ...).
  TopList<R> U;
  toplist_clear<R>(U);
  const size_t base = static_cast<size_t>(col) * G;
  {
    // A warp's first kPre lists are all requested before the first merge, so
    // their L2 round trips overlap; the merge order stays w, w+kW, ...
    constexpr int kPre = 3;
    TopList<R> T[kPre];
#pragma unroll
    for (int t = 0; t < kPre; ++t) {
      const int gg = warp + t * kW;
      if (gg < G) toplist_load_global<R>(T[t], L.part_key + (base + gg) * M, L.part_slot + (base + gg) * M);
    }
#pragma unroll
    for (int t = 0; t < kPre; ++t)
      if (warp + t * kW < G) toplist_merge_loaded<R>(U, T[t]);
    for (int gg = warp + kPre * kW; gg < G; gg += kW)
      toplist_merge_global<R>(U, L.part_key + (base + gg) * M, L.part_slot + (base + gg) * M);
  }
  toplist_cta_merge<R>(U, &s_key[0][0], &s_pay[0][0]);
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
    // Column sums in a fixed order: lane-strided partials, then a fixed tree.
    double nz = 0.0, dt = 0.0;
    unsigned long long ce = 0, cu = 0, ci = 0;
    for (int gg = lane; gg < G; gg += 32) {
      const double* ps = L.part_sum + kPartSum * (base + gg);
      nz += __ldcg(ps);
      dt += __ldcg(ps + 1);
      ce += static_cast<unsigned long long>(__ldcg(ps + 2));
      cu += static_cast<unsigned long long>(__ldcg(ps + 3));
      ci += static_cast<unsigned long long>(__ldcg(ps + 4));
    }
    nz = warp_sum(nz);
    dt = warp_sum(dt);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ce += __shfl_xor_sync(~0u, ce, o);
      cu += __shfl_xor_sync(~0u, cu, o);
      ci += __shfl_xor_sync(~0u, ci, o);
    }
    if (lane == 0) {
      if (ce) {
        atomicAdd(&S->emitted, ce);
        atomicAdd(&S->emitted_total, ce);
      }
      if (cu) {
        atomicAdd(&S->updates, cu);
        atomicAdd(&S->updates_total, cu);
      }
      if (ci) atomicAdd(&S->z_size, ci);
      S->newz[col] = nz;
      S->dot[col] = dt;
      S->cand_n[col] = n;
      L.done[col] = 0u;
    }
  }
  if (timed) {
    atomicAdd(L.sect + 7, static_cast<unsigned long long>(clock64() - c_merge));
    atomicAdd(L.sect + 9, 1ull);
  }
}

template <int R>
__global__ void __launch_bounds__(kNT, 3) column_kernel(ColumnLaunch L) {
  column_body<R>(L, blockIdx.x);
}

// Several instances in one grid: CTAs [cta_begin[i], cta_begin[i+1]) belong
// to instance i and keep the layout of its own launch.
template <int R>
__global__ void __launch_bounds__(kNT, 3) column_kernel_batch(ColumnBatch B) {
  int lo = 0, hi = B.n;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (B.cta_begin[mid] <= static_cast<int>(blockIdx.x))
      lo = mid;
    else
      hi = mid;
  }
  column_body<R>(B.L[lo], static_cast<int>(blockIdx.x) - B.cta_begin[lo]);
}

__global__ void __launch_bounds__(kNT) debug_column_kernel(HamDev h, Det d, double hd, uint64_t* ao,
                                                           uint64_t* bo, double* vo, int cap, int* nout) {
  __shared__ Prelude P;
  if ((threadIdx.x >> 5) == 0) build_prelude(P, d, h.norb);
  __syncthreads();
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < P.total; e += gridDim.x * blockDim.x) {
    uint64_t a2, b2;
    double v;
    const int kind = gen_entry(h, P, e, hd, a2, b2, v);
    if (kind == kKeep || (kind == kIfNonzero && v != 0.0)) {
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
cudaError_t launch_column_r(const ColumnLaunch& a, cudaStream_t s) {
  column_kernel<R><<<a.k_grid * a.groups, kNT, 0, s>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Reduced density matrices of the wavefunction in the table (the adjoint of
// the energy with respect to the integrals).  One CTA per determinant D with
// x_D != 0: the diagonal terms over D's occupied pairs, then every single and
// double excitation D' of D (all of them: the RDM is a property of the
// wavefunction, so no integral screening) with x_D' looked up in the table.
// The operator phases are those of the column generation, i.e. of
// <D'|a+_r a_p|D> and <D'|a+_r a+_s a_q a_p|D> in the interleaved order.
// Accumulated unnormalised, in spin blocks (see RdmLaunch).

__global__ void rdm_list_kernel(const Slot* slots, size_t n, unsigned* list, unsigned long long* count,
                                unsigned long long cap) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const Slot sl = slots[i];
    if (slot_vacant(sl.a, sl.b)) continue;
    if (sl.x == 0.0) continue;
    const unsigned long long j = atomicAdd(count, 1ull);
    if (j < cap) list[j] = static_cast<unsigned>(i);
  }
}

// Canonical index of a same-spin pair block element: (p, q) and (r, s) put in
// increasing order; returns the sign of the reordering.
__device__ __forceinline__ double pair_canon(int& p, int& q) {
  if (p < q) return 1.0;
  const int t = p;
  p = q;
  q = t;
  return -1.0;
}

__device__ __forceinline__ size_t idx4(int n, int p, int q, int r, int s) {
  return ((static_cast<size_t>(p) * n + q) * n + r) * n + s;
}

__global__ void __launch_bounds__(kNT) rdm_kernel(RdmLaunch R) {
  __shared__ Prelude P;
  const int n = R.ham.norb;
  const int warp = threadIdx.x >> 5;
  for (long long li = blockIdx.x; li < R.nlist; li += gridDim.x) {
    const Slot* sd = R.tab.slots + R.list[li];
    const Det D{sd->a, sd->b};
    const double xd = sd->x;
    __syncthreads();  // P of the previous determinant is no longer read
    if (warp == 0) build_prelude(P, D, n);
    __syncthreads();
    // Diagonal: gamma_pp, Gamma_pqpq over occupied pairs.
    {
      const double w = xd * xd;
      const int na = P.na, nb = P.nb;
      for (int t = threadIdx.x; t < na + nb; t += blockDim.x) {
        if (t < na)
          atomicAdd(R.g1a + static_cast<size_t>(P.occA[t]) * n + P.occA[t], w);
        else
          atomicAdd(R.g1b + static_cast<size_t>(P.occB[t - na]) * n + P.occB[t - na], w);
      }
      for (int t = threadIdx.x; t < na * na; t += blockDim.x) {
        const int i = t / na, j = t - i * na;
        if (i < j) {
          const int p = P.occA[i], q = P.occA[j];
          atomicAdd(R.g2aa + idx4(n, p, q, p, q), w);
        }
      }
      for (int t = threadIdx.x; t < nb * nb; t += blockDim.x) {
        const int i = t / nb, j = t - i * nb;
        if (i < j) {
          const int p = P.occB[i], q = P.occB[j];
          atomicAdd(R.g2bb + idx4(n, p, q, p, q), w);
        }
      }
      for (int t = threadIdx.x; t < na * nb; t += blockDim.x) {
        const int i = t / nb, j = t - i * nb;
        const int p = P.occA[i], q = P.occB[j];
        atomicAdd(R.g2ab + idx4(n, p, q, p, q), w);
      }
    }
    // Excitations.
    for (int e = 1 + threadIdx.x; e < P.total; e += blockDim.x) {
      const uint64_t a = P.a, b = P.b;
      int kind, p = 0, q = 0, r = 0, s = 0;
      uint64_t a2, b2;
      bool neg;
      if (e < P.off2) {
        const int t = e - 1;
        const int i = t / P.va;
        p = P.occA[i];
        r = P.virA[t - i * P.va];
        kind = 1;
        neg = sign_alpha(a, b, p, r);
        a2 = a ^ (1ull << p) ^ (1ull << r);
        b2 = b;
      } else if (e < P.off3) {
        const int t = e - P.off2;
        const int i = t / P.vb;
        p = P.occB[i];
        r = P.virB[t - i * P.vb];
        kind = 2;
        neg = sign_beta(a, b, p, r);
        a2 = a;
        b2 = b ^ (1ull << p) ^ (1ull << r);
      } else if (e < P.off4) {
        const int t = e - P.off3;
        const int op = t / P.ca_vir, vp = t - op * P.ca_vir;
        int i, j, ri, sj;
        pair_decode(op, i, j);
        pair_decode(vp, ri, sj);
        p = P.occA[i];
        q = P.occA[j];
        r = P.virA[ri];
        s = P.virA[sj];
        kind = 3;
        neg = sign_aa(a, b, p, q, r, s);
        a2 = a ^ (1ull << p) ^ (1ull << q) ^ (1ull << r) ^ (1ull << s);
        b2 = b;
      } else if (e < P.off5) {
        const int t = e - P.off4;
        const int op = t / P.cb_vir, vp = t - op * P.cb_vir;
        int i, j, ri, sj;
        pair_decode(op, i, j);
        pair_decode(vp, ri, sj);
        p = P.occB[i];
        q = P.occB[j];
        r = P.virB[ri];
        s = P.virB[sj];
        kind = 4;
        neg = sign_bb(a, b, p, q, r, s);
        a2 = a;
        b2 = b ^ (1ull << p) ^ (1ull << q) ^ (1ull << r) ^ (1ull << s);
      } else {
        int t = e - P.off5;
        const int sbi = t % P.vb;
        t /= P.vb;
        const int rai = t % P.va;
        t /= P.va;
        const int pbi = t % P.nb;
        const int pai = t / P.nb;
        p = P.occA[pai];  // alpha: p -> r
        r = P.virA[rai];
        q = P.occB[pbi];  // beta: q -> s
        s = P.virB[sbi];
        kind = 5;
        neg = sign_ab(a, b, p, r, q, s);
        a2 = a ^ (1ull << p) ^ (1ull << r);
        b2 = b ^ (1ull << q) ^ (1ull << s);
      }
      const long long slot = table_find(R.tab, a2, b2);
      if (slot < 0) continue;
      const double x2 = R.tab.slots[slot].x;
      if (x2 == 0.0) continue;
      const double w = neg ? -(xd * x2) : xd * x2;
      switch (kind) {
        case 1:  // <a+_r a_p> and the spectators k: <a+_r a+_k a_k a_p>
          atomicAdd(R.g1a + static_cast<size_t>(r) * n + p, w);
          for (int x = 0; x < P.na; ++x) {
            const int k = P.occA[x];
            if (k == p) continue;
            int c1 = r, c2 = k, d1 = p, d2 = k;
            const double sg = pair_canon(c1, c2) * pair_canon(d1, d2);
            atomicAdd(R.g2aa + idx4(n, c1, c2, d1, d2), sg * w);
          }
          for (int x = 0; x < P.nb; ++x) {
            const int k = P.occB[x];
            atomicAdd(R.g2ab + idx4(n, r, k, p, k), w);
          }
          break;
        case 2:
          atomicAdd(R.g1b + static_cast<size_t>(r) * n + p, w);
          for (int x = 0; x < P.nb; ++x) {
            const int k = P.occB[x];
            if (k == p) continue;
            int c1 = r, c2 = k, d1 = p, d2 = k;
            const double sg = pair_canon(c1, c2) * pair_canon(d1, d2);
            atomicAdd(R.g2bb + idx4(n, c1, c2, d1, d2), sg * w);
          }
          for (int x = 0; x < P.na; ++x) {
            const int k = P.occA[x];
            atomicAdd(R.g2ab + idx4(n, k, r, k, p), w);
          }
          break;
        case 3:  // <a+_r a+_s a_q a_p>, p < q, r < s
          atomicAdd(R.g2aa + idx4(n, r, s, p, q), w);
          break;
        case 4:
          atomicAdd(R.g2bb + idx4(n, r, s, p, q), w);
          break;
        default:  // <a+_r(alpha) a+_s(beta) a_q(beta) a_p(alpha)>
          atomicAdd(R.g2ab + idx4(n, r, s, p, q), w);
          break;
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

int column_list_size(int m) { return m <= 32 ? 32 : (m <= 64 ? 64 : 128); }

int column_groups(int entries, int k, int resident) {
  // About three rounds of kNT entries per CTA ...
  int g = (entries + 3 * kNT - 1) / (3 * kNT);
  // ... or, when k columns of such CTAs leave resident CTA slots empty, as
  // many CTAs as fill them, down to one round each.
  if (resident > 0 && k > 0) {
    const int fill = (resident + k - 1) / k;
    const int one_round = (entries + kNT - 1) / kNT;
    g = std::max(g, std::min(fill, one_round));
  }
  // ... and at most 96: the last CTA of a column merges all of its CTAs'
  // lists at the end of the launch, so long columns take longer CTAs (the
  // 271,945-entry columns of 42 orbitals, 24 + 24 electrons, one sweep of
  // 64-column launches: 1074 us per launch with 355 CTAs each, 957 us with
  // the cap's 96, 932 us with 89).
  g = std::min(g, 96);
  return g < 1 ? 1 : g;
}

cudaError_t launch_column(const ColumnLaunch& a, cudaStream_t s) {
  if (a.m <= 32) return launch_column_r<1>(a, s);
  if (a.m <= 64) return launch_column_r<2>(a, s);
  return launch_column_r<4>(a, s);
}

cudaError_t launch_column_batch(const ColumnBatch& b, cudaStream_t s) {
  if (b.n < 1 || b.n > kMaxBatch) return cudaErrorInvalidValue;
  const int ctas = b.cta_begin[b.n];
  const int m = b.L[0].m;
  if (m <= 32)
    column_kernel_batch<1><<<ctas, kNT, 0, s>>>(b);
  else if (m <= 64)
    column_kernel_batch<2><<<ctas, kNT, 0, s>>>(b);
  else
    column_kernel_batch<4><<<ctas, kNT, 0, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_rdm_list(const TableDev& t, size_t capacity, unsigned* list, unsigned long long* count,
                            unsigned long long cap, cudaStream_t s) {
  rdm_list_kernel<<<148 * 8, 256, 0, s>>>(t.slots, capacity, list, count, cap);
  return cudaGetLastError();
}

cudaError_t launch_rdm(const RdmLaunch& r, cudaStream_t s) {
  if (r.nlist <= 0) return cudaSuccess;
  const long long blocks = r.nlist < 148LL * 16 ? r.nlist : 148LL * 16;
  rdm_kernel<<<static_cast<unsigned>(blocks), kNT, 0, s>>>(r);
  return cudaGetLastError();
}

// Scattered-access ceiling of the table, for the column kernel's roofline: a
// stream of pseudo-random slots, each touched the way a column entry touches
// its slot (the 16-byte key, then x and an FP64 atomic add on z that returns
// the old value; the add is of zero, so the table keeps its values).  ILP
// slots are in flight per thread; the grid fills every SM.
// MODE 0: the 16-byte key, x and an FP64 atomic add of zero with its return,
// as a column entry touches its slot; 1: key and x loads only; 2: the atomic
// with return only; 3: key load and an atomic add whose return is unused
// (a reduction, no round trip).
template <int ILP, int MODE>
__global__ void __launch_bounds__(256) scatter_probe_kernel(Slot* slots, uint64_t mask, long long entries,
                                                            uint64_t seed, double* sink) {
  double acc = 0.0;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x * ILP;
  for (long long e0 = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) * ILP; e0 < entries;
       e0 += stride) {
    uint64_t sl[ILP], ka[ILP], kb[ILP];
#pragma unroll
    for (int q = 0; q < ILP; ++q) {
      sl[q] = fmix64(seed ^ static_cast<uint64_t>(e0 + q)) & mask;
      ka[q] = kb[q] = 0;
      if (MODE != 2 && e0 + q < entries) load_key(slots + sl[q], ka[q], kb[q]);
    }
#pragma unroll
    for (int q = 0; q < ILP; ++q) {
      if (e0 + q < entries && ka[q] != ~0ull - 1ull) {  // uses the key, as a probe does
        Slot* sp = slots + sl[q];
        if (MODE == 0) acc += sp->x + atomicAdd(&sp->z, 0.0) + static_cast<double>(kb[q] & 1ull);
        if (MODE == 1) acc += sp->x + static_cast<double>(kb[q] & 1ull);
        if (MODE == 2) acc += atomicAdd(&sp->z, 0.0);
        if (MODE == 3) {
          atomicAdd(&sp->z, 0.0);
          acc += static_cast<double>(kb[q] & 1ull);
        }
      }
    }
  }
  if (acc == 1234.5678) *sink = acc;  // keeps the loads
}

template <int MODE>
void scatter_probe_mode(const TableDev& t, long long entries, int ilp, int ctas, uint64_t seed, double* sink,
                        cudaStream_t s) {
  if (ilp >= 4)
    scatter_probe_kernel<4, MODE><<<ctas, 256, 0, s>>>(t.slots, t.mask, entries, seed, sink);
  else
    scatter_probe_kernel<1, MODE><<<ctas, 256, 0, s>>>(t.slots, t.mask, entries, seed, sink);
}

cudaError_t scatter_probe(const TableDev& t, long long entries, int ilp, int ctas, uint64_t seed, double* sink,
                          cudaStream_t s, int mode) {
  if (ctas < 1 || mode < 0 || mode > 3) return cudaErrorInvalidValue;
  if (mode == 0) scatter_probe_mode<0>(t, entries, ilp, ctas, seed, sink, s);
  if (mode == 1) scatter_probe_mode<1>(t, entries, ilp, ctas, seed, sink, s);
  if (mode == 2) scatter_probe_mode<2>(t, entries, ilp, ctas, seed, sink, s);
  if (mode == 3) scatter_probe_mode<3>(t, entries, ilp, ctas, seed, sink, s);
  return cudaGetLastError();
}

cudaError_t debug_column(const HamDev& h, Det d, double hdiag, uint64_t* a_out, uint64_t* b_out,
                         double* v_out, int cap, int* n_out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(n_out, 0, sizeof(int), s);
  if (e != cudaSuccess) return e;
  debug_column_kernel<<<64, kNT, 0, s>>>(h, d, hdiag, a_out, b_out, v_out, cap, n_out);
  return cudaGetLastError();
}

}  // namespace mcd
