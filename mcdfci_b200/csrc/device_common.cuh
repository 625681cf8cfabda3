// Device building blocks: determinant bit operations, fermionic signs in the
// reference's spin-orbital order, the hash of a determinant, and the
// open-addressing table of (x, z) in HBM.
#pragma once

#include <cstdint>

#include "dd.h"
#include "mcd_types.h"

namespace mcd {

// ---------------------------------------------------------------------------
// Bit masks over one 64-bit occupation string.
__device__ __forceinline__ uint64_t mask_below(int p) {  // bits [0, p)
  return p >= 64 ? ~0ull : ((1ull << p) - 1ull);
}
__device__ __forceinline__ uint64_t mask_open(int lo, int hi) {  // (lo, hi)
  return mask_below(hi) & ~mask_below(lo + 1);
}
__device__ __forceinline__ uint64_t mask_left_closed(int lo, int hi) {  // [lo, hi)
  return mask_below(hi) & ~mask_below(lo);
}
__device__ __forceinline__ uint64_t mask_right_closed(int lo, int hi) {  // (lo, hi]
  return mask_below(hi + 1) & ~mask_below(lo + 1);
}

// The reference's sign of an excitation i -> a is the parity of the occupied
// spin-orbitals strictly between i and a in interleaved order (alpha p = 2p,
// beta p = 2p+1), evaluated on the determinant with i removed
// (Determinant::parity, src/determinant.h:103-111,148-152; used at
// src/hamiltonian.h:349-353 and 395-403).  In alpha/beta strings:
//   alpha p->r: alpha bits in (lo,hi), beta bits in [lo,hi)
//   beta  p->r: beta bits in (lo,hi),  alpha bits in (lo,hi]
// with lo = min(p,r), hi = max(p,r).  The returned value is the count's parity.
__device__ __forceinline__ int sign_alpha(uint64_t a, uint64_t b, int p, int r) {
  const int lo = min(p, r), hi = max(p, r);
  return (__popcll(a & mask_open(lo, hi)) + __popcll(b & mask_left_closed(lo, hi))) & 1;
}
__device__ __forceinline__ int sign_beta(uint64_t a, uint64_t b, int p, int r) {
  const int lo = min(p, r), hi = max(p, r);
  return (__popcll(b & mask_open(lo, hi)) + __popcll(a & mask_right_closed(lo, hi))) & 1;
}

// Sequential sign of a double excitation: first (p->r) on the determinant, then
// (q->s) on the result (src/hamiltonian.h:397-403).  For an alpha-beta double
// the two excitations commute, so alpha-first gives the reference's sign
// whichever of the two comes first in interleaved order.
__device__ __forceinline__ int sign_aa(uint64_t a, uint64_t b, int p, int q, int r, int s) {
  const int s1 = sign_alpha(a, b, p, r);
  const uint64_t a1 = a ^ (1ull << p) ^ (1ull << r);
  return s1 ^ sign_alpha(a1, b, q, s);
}
__device__ __forceinline__ int sign_bb(uint64_t a, uint64_t b, int p, int q, int r, int s) {
  const int s1 = sign_beta(a, b, p, r);
  const uint64_t b1 = b ^ (1ull << p) ^ (1ull << r);
  return s1 ^ sign_beta(a, b1, q, s);
}
__device__ __forceinline__ int sign_ab(uint64_t a, uint64_t b, int pa, int ra, int pb, int sb) {
  const int s1 = sign_alpha(a, b, pa, ra);
  const uint64_t a1 = a ^ (1ull << pa) ^ (1ull << ra);
  return s1 ^ sign_beta(a1, b, pb, sb);
}

// Interleaved spin-orbital words of a determinant (the reference's
// Determinant<N>::repr): word w holds spatial orbitals 32w..32w+31.
__device__ __forceinline__ uint64_t spread32(uint64_t x) {
  x &= 0xFFFFFFFFull;
  x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
  x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
  x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
  x = (x | (x << 2)) & 0x3333333333333333ull;
  x = (x | (x << 1)) & 0x5555555555555555ull;
  return x;
}
__device__ __forceinline__ uint64_t interleaved_word(uint64_t a, uint64_t b, int w) {
  return spread32(a >> (32 * w)) | (spread32(b >> (32 * w)) << 1);
}

// The reference's determinant order used to break ties between equal
// gradients (detComp_global, src/wavefunction.h:30-36): words compared from
// word 0, first differing word decides through the sign of the wrapped
// difference.  Returns >0 if x sorts after y.
__device__ __forceinline__ int det_ref_compare(uint64_t xa, uint64_t xb, uint64_t ya, uint64_t yb, int nwords) {
  int w = 0;
  uint64_t xw = interleaved_word(xa, xb, 0), yw = interleaved_word(ya, yb, 0);
  for (w = 0; w < nwords - 1 && xw == yw; ++w) {
    xw = interleaved_word(xa, xb, w + 1);
    yw = interleaved_word(ya, yb, w + 1);
  }
  const long long diff = static_cast<long long>(xw - yw);
  return (diff > 0) - (diff < 0);
}

// ---------------------------------------------------------------------------
// Hashing: two rounds of the 64-bit murmur3 finaliser.
__device__ __forceinline__ uint64_t fmix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ull;
  k ^= k >> 33;
  return k;
}
__device__ __forceinline__ uint64_t det_hash(uint64_t a, uint64_t b) {
  return fmix64(a ^ fmix64(b + 0x9E3779B97F4A7C15ull));
}

// 16-byte key access.  The key is written once, EMPTY -> key, by a 128-bit
// compare-and-swap; readers use a 128-bit relaxed load, so a key is never
// observed half-written.
__device__ __forceinline__ void load_key(const Slot* s, uint64_t& a, uint64_t& b) {
  asm volatile(
      "{\n\t.reg .b128 d;\n\t"
      "ld.relaxed.gpu.global.b128 d, [%2];\n\t"
      "mov.b128 {%0, %1}, d;\n\t}"
      : "=l"(a), "=l"(b)
      : "l"(s)
      : "memory");
}
__device__ __forceinline__ void cas_key(Slot* s, uint64_t na, uint64_t nb, uint64_t& oa, uint64_t& ob) {
  const uint64_t ea = kEmptyKey, eb = kEmptyKey;
  asm volatile(
      "{\n\t.reg .b128 d, c, n;\n\t"
      "mov.b128 c, {%2, %3};\n\t"
      "mov.b128 n, {%4, %5};\n\t"
      "atom.global.relaxed.gpu.cas.b128 d, [%6], c, n;\n\t"
      "mov.b128 {%0, %1}, d;\n\t}"
      : "=l"(oa), "=l"(ob)
      : "l"(ea), "l"(eb), "l"(na), "l"(nb), "l"(s)
      : "memory");
}
__device__ __forceinline__ double load_relaxed(const double* p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}

// Linear probing, continuing from the home slot i whose key (ka, kb) the
// caller has already loaded (so that the first probe can be in flight while
// the caller does other work).  Returns the slot index of (a,b) or -1 if absent.
__device__ __forceinline__ long long table_find_from(const TableDev& t, uint64_t a, uint64_t b, uint64_t i,
                                                     uint64_t ka, uint64_t kb) {
  for (int p = 0; p < t.max_probe; ++p) {
    if (p > 0) load_key(t.slots + i, ka, kb);
    if (ka == a && kb == b) return static_cast<long long>(i);
    if (ka == kEmptyKey && kb == kEmptyKey) return -1;
    i = (i + 1) & t.mask;
  }
  atomicOr(t.err, kErrProbe);
  return -1;
}

__device__ __forceinline__ long long table_find(const TableDev& t, uint64_t a, uint64_t b) {
  const uint64_t i = det_hash(a, b) & t.mask;
  uint64_t ka, kb;
  load_key(t.slots + i, ka, kb);
  return table_find_from(t, a, b, i, ka, kb);
}

// Find, and insert when `insert` (one loop for both, so that the lanes of a
// warp that insert and those that only update stay on one path), continuing
// from a loaded home slot as table_find_from.
__device__ __forceinline__ long long table_probe_from(const TableDev& t, uint64_t a, uint64_t b, uint64_t i,
                                                      uint64_t ka, uint64_t kb, bool insert, bool& inserted) {
  inserted = false;
  for (int p = 0; p < t.max_probe; ++p) {
    if (p > 0) load_key(t.slots + i, ka, kb);
    if (ka == a && kb == b) return static_cast<long long>(i);
    if (ka == kEmptyKey && kb == kEmptyKey) {
      if (!insert) return -1;
      uint64_t oa, ob;
      cas_key(t.slots + i, a, b, oa, ob);
      if (oa == kEmptyKey && ob == kEmptyKey) {
        inserted = true;
        atomicAdd(t.n_occupied, 1ull);
        return static_cast<long long>(i);
      }
      if (oa == a && ob == b) return static_cast<long long>(i);
    }
    i = (i + 1) & t.mask;
  }
  atomicOr(t.err, kErrProbe);
  return -1;
}

// Find or insert, continuing from a loaded home slot as table_find_from.
// `inserted` is set when this call created the slot (x = z = 0 from the
// table's initialisation).  Returns -1 only when the probe limit is hit,
// after raising kErrProbe.
__device__ __forceinline__ long long table_upsert_from(const TableDev& t, uint64_t a, uint64_t b, uint64_t i,
                                                       uint64_t ka, uint64_t kb, bool& inserted) {
  inserted = false;
  for (int p = 0; p < t.max_probe; ++p) {
    if (p > 0) load_key(t.slots + i, ka, kb);
    if (ka == a && kb == b) return static_cast<long long>(i);
    if (ka == kEmptyKey && kb == kEmptyKey) {
      uint64_t oa, ob;
      cas_key(t.slots + i, a, b, oa, ob);
      if (oa == kEmptyKey && ob == kEmptyKey) {
        inserted = true;
        atomicAdd(t.n_occupied, 1ull);
        return static_cast<long long>(i);
      }
      if (oa == a && ob == b) return static_cast<long long>(i);
    }
    i = (i + 1) & t.mask;
  }
  atomicOr(t.err, kErrProbe);
  return -1;
}

__device__ __forceinline__ long long table_upsert(const TableDev& t, uint64_t a, uint64_t b, bool& inserted) {
  const uint64_t i = det_hash(a, b) & t.mask;
  uint64_t ka, kb;
  load_key(t.slots + i, ka, kb);
  return table_upsert_from(t, a, b, i, ka, kb, inserted);
}

// gcd_grad score of a determinant, |x xx scale^2 + z| (CoordinatePickGcdGrad,
// src/solver.h:118-143), with xss = xx scale^2 in double-double.
__device__ __forceinline__ double score_of(double x, double z, dd xss) {
  if (x == 0.0) return fabs(z);
  const dd t = dd_add_d(dd_mul_d(xss, x), z);
  return fabs(t.hi + t.lo);
}

// ---------------------------------------------------------------------------
// Section clock: thread 0 of a CTA adds the SM cycles since the previous mark
// to acc[i].  Marks are placed right after block-wide barriers, so each entry
// is the duration of one phase of the CTA.  acc may be null (no timing).
struct SectionClock {
  unsigned long long* acc;
  long long t;
  __device__ __forceinline__ void start() {
    if (threadIdx.x == 0) t = clock64();
  }
  __device__ __forceinline__ void mark(int i) {
    if (acc != nullptr && threadIdx.x == 0) {
      const long long now = clock64();
      atomicAdd(acc + i, static_cast<unsigned long long>(now - t));
      t = now;
    }
  }
};

// ---------------------------------------------------------------------------
// Warp helpers.
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ dd warp_sum_dd(dd v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dd w{__shfl_xor_sync(0xffffffffu, v.hi, o), __shfl_xor_sync(0xffffffffu, v.lo, o)};
    v = dd_add(v, w);
  }
  return v;
}

}  // namespace mcd
