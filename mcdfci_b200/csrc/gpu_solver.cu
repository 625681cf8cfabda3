#include "gpu_solver.h"

#include "device_common.cuh"

#include <algorithm>
#include <cstddef>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <future>
#include <iomanip>
#include <iostream>
#include <map>
#include <mutex>
#include <sstream>

namespace mcd {

// ---------------------------------------------------------------------------
// Table kernels.

__global__ void table_fill_kernel(Slot* slots, size_t n) {
  const Slot e{kEmptyKey, kEmptyKey, 0.0, 0.0};
  const Slot r{kEmptyKey, kReservedKeyB, 0.0, 0.0};
  const bool reserve = n == (static_cast<size_t>(1) << 32);  // slot 2^32-1 is the "no slot" marker
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    slots[i] = (reserve && i == n - 1) ? r : e;
}

__global__ void table_sums_kernel(const Slot* slots, size_t n, dd* partial, unsigned long long* count) {
  __shared__ dd sxx[32], sxz[32];
  dd axx{0, 0}, axz{0, 0};
  unsigned long long c = 0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const Slot s = slots[i];
    if (slot_vacant(s.a, s.b)) continue;
    ++c;
    axx = dd_add(axx, dd_two_prod(s.x, s.x));
    axz = dd_add(axz, dd_two_prod(s.x, s.z));
  }
  axx = warp_sum_dd(axx);
  axz = warp_sum_dd(axz);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sxx[warp] = axx;
    sxz[warp] = axz;
  }
  atomicAdd(count, c);
  __syncthreads();
  if (threadIdx.x == 0) {
    dd t1{0, 0}, t2{0, 0};
    for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) {
      t1 = dd_add(t1, sxx[w]);
      t2 = dd_add(t2, sxz[w]);
    }
    partial[2 * blockIdx.x] = t1;
    partial[2 * blockIdx.x + 1] = t2;
  }
}

// Residual of the stored vector: partial[b] = sum over block b's slots of
// (z - e x)^2 and x^2 in double-double.  With z = H x (z_threshold = 0 keeps
// every connected determinant), sqrt(sum (z - e x)^2 / sum x^2) with e =
// x'z / x'x is ||H c - E c|| / ||c|| for the coefficients c = scale x.
__global__ void table_resid_kernel(const Slot* slots, size_t n, dd e, dd* partial) {
  __shared__ dd srr[32], sxx[32];
  dd arr{0, 0}, axx{0, 0};
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const Slot s = slots[i];
    if (slot_vacant(s.a, s.b)) continue;
    const dd r = dd_add_d(dd_neg(dd_mul_d(e, s.x)), s.z);
    arr = dd_add(arr, dd_mul(r, r));
    axx = dd_add(axx, dd_two_prod(s.x, s.x));
  }
  arr = warp_sum_dd(arr);
  axx = warp_sum_dd(axx);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    srr[warp] = arr;
    sxx[warp] = axx;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    dd t1{0, 0}, t2{0, 0};
    for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w) {
      t1 = dd_add(t1, srr[w]);
      t2 = dd_add(t2, sxx[w]);
    }
    partial[2 * blockIdx.x] = t1;
    partial[2 * blockIdx.x + 1] = t2;
  }
}

// ---------------------------------------------------------------------------
// Compaction: the slots that survive (x != 0, or |z| above a limit) are
// copied in slot order into a buffer (per-block counts, then per-block
// in-order writes at prefix-sum offsets, so that the survivor list depends
// only on the table's contents), the table is cleared and they are inserted
// again.  The current candidate lists are saved before and re-found after.

__device__ __forceinline__ bool compact_keeps(const Slot& s, double zlim) {
  if (slot_vacant(s.a, s.b)) return false;
  return s.x != 0.0 || fabs(s.z) > zlim;
}

__global__ void compact_count_kernel(const Slot* slots, size_t n, size_t chunk, double zlim,
                                     unsigned long long* counts) {
  __shared__ unsigned long long ws[32];
  const size_t beg = blockIdx.x * chunk, end = beg + chunk < n ? beg + chunk : n;
  unsigned long long c = 0;
  for (size_t i = beg + threadIdx.x; i < end; i += blockDim.x) c += compact_keeps(slots[i], zlim) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(~0u, c, o);
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += ws[w];
    counts[blockIdx.x] = t;
  }
}

__global__ void compact_write_kernel(const Slot* slots, size_t n, size_t chunk, double zlim,
                                     const unsigned long long* offsets, Slot* out) {
  __shared__ unsigned ws[33];
  const size_t beg = blockIdx.x * chunk, end = beg + chunk < n ? beg + chunk : n;
  unsigned long long pos = offsets[blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (size_t base = beg; base < end; base += blockDim.x) {
    const size_t i = base + threadIdx.x;
    Slot sl{};
    const bool keep = i < end && compact_keeps(sl = slots[i], zlim);
    const unsigned b = __ballot_sync(~0u, keep);
    if (lane == 0) ws[warp] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned run = 0;
      for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
        const unsigned c = ws[w];
        ws[w] = run;
        run += c;
      }
      ws[32] = run;
    }
    __syncthreads();
    if (keep) out[pos + ws[warp] + __popc(b & lanemask_lt())] = sl;
    pos += ws[32];
    __syncthreads();
  }
}

__global__ void compact_reinsert_kernel(TableDev t, const Slot* src, size_t cnt) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cnt;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const Slot s = src[i];
    bool inserted;
    const long long j = table_upsert(t, s.a, s.b, inserted);
    if (j >= 0) {
      t.slots[j].x = s.x;
      t.slots[j].z = s.z;
    }
  }
}

__global__ void rehash_kernel(const Slot* src, size_t n, TableDev t) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const Slot s = src[i];
    if (slot_vacant(s.a, s.b)) continue;
    bool inserted;
    const long long j = table_upsert(t, s.a, s.b, inserted);
    if (j >= 0) {
      t.slots[j].x = s.x;
      t.slots[j].z = s.z;
    }
  }
}

// Doubling rehash with no atomics on global memory for all but a few slots.
// When a table of C slots doubles, an entry whose home is p = hash & (C-1)
// gets the home p or p + C (bit C of its hash).  Take the old slots strictly
// between two empty ones e0 < e1 (a run of whole clusters): every entry sits
// at or after its home with no empty slot between, so its home is in
// (e0, e1), and for each x there the entries with homes in [x, e1) filled old
// slots in [x, e1), so there are at most e1 - x of them.  Linear probing then
// places the run's lower entries within [e0, e1) and its upper entries within
// [e0 + C, e1 + C), in any insertion order.  CTA b owns the run from the
// first empty slot at or after b * kRehashChunk to the first at or after
// (b + 1) * kRehashChunk, or to the table's last empty slot: it places the
// entries in shared memory (a 32-bit compare-and-swap per probe) and writes
// both new ranges whole, empty slots included, so the new table needs no
// separate fill.  These runs tile [W, Z) (W the first empty slot, Z the last).
// The cluster that wraps from slot C-1 to slot 0 belongs to the extra last
// CTA: it empties [Z, C + W) and [Z + C, 2C) + [0, W), which by the same
// count hold all that cluster's entries, and inserts them with the global
// compare-and-swap.  A run longer than kRehashRange takes that global path
// too, within its own ranges.  The entry count does not change.
constexpr int kRehashChunk = 1024;
constexpr int kRehashRange = 2048;
constexpr int kRehashThreads = 256;

__device__ __forceinline__ bool old_slot_empty(const Slot* src, long long i) {
  const ulonglong2 k = __ldg(reinterpret_cast<const ulonglong2*>(src + i));
  return k.x == kEmptyKey && k.y == kEmptyKey;
}

// First empty slot of src in [from, to), else `to`.  Whole warp.
__device__ __forceinline__ long long warp_first_empty(const Slot* src, long long from, long long to) {
  const int lane = threadIdx.x & 31;
  for (long long base = from; base < to; base += 32) {
    const long long i = base + lane;
    const unsigned m = __ballot_sync(~0u, i < to && old_slot_empty(src, i));
    if (m) return base + (__ffs(m) - 1);
  }
  return to;
}

// Last empty slot of src in [from, to), else -1.  Whole warp.
__device__ __forceinline__ long long warp_last_empty(const Slot* src, long long from, long long to) {
  const int lane = threadIdx.x & 31;
  for (long long top = to; top > from; top -= 32) {
    const long long i = top - 1 - lane;
    const unsigned m = __ballot_sync(~0u, i >= from && old_slot_empty(src, i));
    if (m) return top - __ffs(m);
  }
  return -1;
}

// Inserts an entry absent from t, probing at most `limit` slots from its
// home; false when none of them was empty.
__device__ __forceinline__ bool rehash_insert_global(const TableDev& t, const Slot& s, long long limit) {
  uint64_t i = det_hash(s.a, s.b) & t.mask;
  for (long long p = 0; p < limit; ++p) {
    uint64_t ka, kb;
    load_key(t.slots + i, ka, kb);
    if (ka == kEmptyKey && kb == kEmptyKey) {
      uint64_t oa, ob;
      cas_key(t.slots + i, s.a, s.b, oa, ob);
      if (oa == kEmptyKey && ob == kEmptyKey) {
        t.slots[i].x = s.x;
        t.slots[i].z = s.z;
        return true;
      }
    }
    i = (i + 1) & t.mask;
  }
  return false;
}

// src: the old table of C slots (a power of two, no reserved slot); t: the
// new one of 2C slots, written whole.  Grid: C / kRehashChunk + 1 CTAs of
// kRehashThreads.  force_global sends every run down the global path.
__global__ void rehash_double_kernel(const Slot* __restrict__ src, long long C, TableDev t, int force_global) {
  __shared__ int s_lo[kRehashRange], s_hi[kRehashRange];
  __shared__ long long s_e[2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const Slot empty{kEmptyKey, kEmptyKey, 0.0, 0.0};
  Slot* dst = t.slots;
  const long long nchunks = C / kRehashChunk;

  if (blockIdx.x == nchunks) {
    // The cluster through slot C-1 and slot 0.
    if (warp == 0) {
      const long long w = warp_first_empty(src, 0, C);
      if (lane == 0) s_e[0] = w;
    } else if (warp == 1) {
      const long long z = warp_last_empty(src, 0, C);
      if (lane == 0) s_e[1] = z;
    }
    __syncthreads();
    const long long W = s_e[0], Z = s_e[1];
    if (W >= C || Z < 0) {  // no empty slot: never, the occupancy limit is below 1
      if (threadIdx.x == 0) atomicOr(t.err, kErrProbe);
      return;
    }
    const long long n = C - Z + W;  // the length of each of the two regions
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
      dst[Z + i] = empty;
      dst[(Z + C + i) & (2 * C - 1)] = empty;
    }
    __syncthreads();
    for (long long i = 1 + threadIdx.x; i < n; i += blockDim.x) {
      const Slot sl = src[(Z + i) & (C - 1)];
      if (sl.a == kEmptyKey && sl.b == kEmptyKey) continue;
      if (!rehash_insert_global(t, sl, n)) atomicOr(t.err, kErrProbe);
    }
    return;
  }

  const long long s = static_cast<long long>(blockIdx.x) * kRehashChunk;
  if (warp == 0) {
    const long long e0 = warp_first_empty(src, s, C);
    if (lane == 0) s_e[0] = e0;
  } else if (warp == 1) {
    long long e1 = warp_first_empty(src, s + kRehashChunk, C);
    if (e1 == C) e1 = warp_last_empty(src, s, s + kRehashChunk);
    if (lane == 0) s_e[1] = e1;
  }
  __syncthreads();
  const long long e0 = s_e[0], e1 = s_e[1];
  // e0 == C: no empty slot from s on (inside the wrapping cluster);
  // e1 == e0: no run starts in this chunk.
  if (e0 >= C || e1 <= e0) return;
  const long long L = e1 - e0;

  if (L > kRehashRange || force_global) {
    for (long long i = threadIdx.x; i < L; i += blockDim.x) {
      dst[e0 + i] = empty;
      dst[e0 + C + i] = empty;
    }
    __syncthreads();
    for (long long i = 1 + threadIdx.x; i < L; i += blockDim.x) {
      const Slot sl = src[e0 + i];
      if (sl.a == kEmptyKey && sl.b == kEmptyKey) continue;
      if (!rehash_insert_global(t, sl, L)) atomicOr(t.err, kErrProbe);
    }
    return;
  }

  const int n = static_cast<int>(L);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    s_lo[i] = -1;
    s_hi[i] = -1;
  }
  __syncthreads();
  for (int i = 1 + threadIdx.x; i < n; i += blockDim.x) {
    const ulonglong2 k = __ldg(reinterpret_cast<const ulonglong2*>(src + e0 + i));
    if (k.x == kEmptyKey && k.y == kEmptyKey) continue;
    const uint64_t h = det_hash(k.x, k.y);
    int* arr = (h & static_cast<uint64_t>(C)) ? s_hi : s_lo;
    const long long d = static_cast<long long>(h & static_cast<uint64_t>(C - 1)) - e0;
    if (d <= 0 || d > i) {
      atomicOr(t.err, kErrProbe);  // a home outside its run: not a linear-probing table
      continue;
    }
    int p = static_cast<int>(d);
    while (p < n && atomicCAS(arr + p, -1, i) != -1) ++p;
    if (p >= n) atomicOr(t.err, kErrProbe);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int jl = s_lo[i], jh = s_hi[i];
    dst[e0 + i] = jl >= 0 ? src[e0 + jl] : empty;
    dst[e0 + C + i] = jh >= 0 ? src[e0 + jh] : empty;
  }
}

// Candidate lists: (col < k_cur, i < cand_n[col]).  save: the slots'
// contents; restore: find or insert each saved determinant, its new slot.
__global__ void compact_cand_save_kernel(const Slot* slots, const IterState* st, const unsigned* cand_slot, int m,
                                         Slot* saved) {
  const int col = blockIdx.x;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    Slot e{kEmptyKey, kEmptyKey, 0.0, 0.0};
    if (col < st->k_cur && i < st->cand_n[col]) e = slots[cand_slot[col * m + i]];
    saved[col * m + i] = e;
  }
}

__global__ void compact_cand_restore_kernel(TableDev t, const IterState* st, const Slot* saved, unsigned* cand_slot,
                                            int m) {
  const int col = blockIdx.x;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    if (!(col < st->k_cur && i < st->cand_n[col])) continue;
    const Slot s = saved[col * m + i];
    bool inserted;
    const long long j = table_upsert(t, s.a, s.b, inserted);
    if (j < 0) continue;  // table error word already set
    if (inserted) {
      t.slots[j].x = s.x;
      t.slots[j].z = s.z;
    }
    cand_slot[col * m + i] = static_cast<unsigned>(j);
  }
}

cudaError_t launch_rehash(const Slot* src, size_t n, const TableDev& t, cudaStream_t s) {
  rehash_kernel<<<148 * 8, 256, 0, s>>>(src, n, t);
  return cudaGetLastError();
}

cudaError_t launch_rehash_double(const Slot* src, size_t n, const TableDev& t, bool force_global, cudaStream_t s) {
  if (n < static_cast<size_t>(kRehashChunk) || (n & (n - 1)) != 0 || t.mask != 2 * n - 1) return cudaErrorInvalidValue;
  const size_t blocks = n / kRehashChunk + 1;
  rehash_double_kernel<<<static_cast<unsigned>(blocks), kRehashThreads, 0, s>>>(src, static_cast<long long>(n), t,
                                                                                force_global ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_table_fill(Slot* slots, size_t n, cudaStream_t s) {
  table_fill_kernel<<<148 * 8, 256, 0, s>>>(slots, n);
  return cudaGetLastError();
}

cudaError_t launch_table_sums(const Slot* slots, size_t n, dd* partial, unsigned long long* count, int nblocks,
                              cudaStream_t s) {
  table_sums_kernel<<<nblocks, 256, 0, s>>>(slots, n, partial, count);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------

namespace {

template <typename T>
T* device_alloc(size_t count, const char* what) {
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, count * sizeof(T));
  if (e != cudaSuccess)
    throw McdError(MCD_ERR_CUDA, std::string("cudaMalloc(") + what + ", " + std::to_string(count * sizeof(T)) +
                                     " bytes): " + cudaGetErrorString(e));
  return static_cast<T*>(p);
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Pinned host words for the occupancy reads, two per solver, from blocks
// that stay allocated for the life of the process (page-locking a fresh
// block costs more than a solver's other set-up), reused as solvers go.
std::mutex g_pin_mu;
std::vector<unsigned long long*> g_pin_free;

unsigned long long* pinned_words_acquire() {
  std::lock_guard<std::mutex> lock(g_pin_mu);
  if (g_pin_free.empty()) {
    constexpr int kPairs = 256;
    void* p = nullptr;
    const cudaError_t e = cudaMallocHost(&p, kPairs * 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) throw McdError(MCD_ERR_CUDA, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
    auto* b = static_cast<unsigned long long*>(p);
    for (int i = kPairs - 1; i >= 0; --i) g_pin_free.push_back(b + 2 * i);
  }
  unsigned long long* w = g_pin_free.back();
  g_pin_free.pop_back();
  return w;
}

void pinned_words_release(unsigned long long* w) {
  std::lock_guard<std::mutex> lock(g_pin_mu);
  g_pin_free.push_back(w);
}

// Pinned host blocks for the Hamiltonian-table upload, kept for the process
// and reused (a copy from pageable memory runs at a fraction of the DMA
// rate): the smallest free block that holds `bytes`, else a new one of at
// least 8 MB; nullptr when pinned memory cannot be had (the caller then
// uploads from pageable memory).
struct StagingBlock {
  void* p = nullptr;
  size_t bytes = 0;
};
std::vector<StagingBlock> g_stage_free;

StagingBlock staging_acquire(size_t bytes) {
  std::lock_guard<std::mutex> lock(g_pin_mu);
  int best = -1;
  for (int i = 0; i < static_cast<int>(g_stage_free.size()); ++i)
    if (g_stage_free[i].bytes >= bytes && (best < 0 || g_stage_free[i].bytes < g_stage_free[best].bytes)) best = i;
  if (best >= 0) {
    const StagingBlock b = g_stage_free[best];
    g_stage_free.erase(g_stage_free.begin() + best);
    return b;
  }
  StagingBlock b;
  b.bytes = std::max<size_t>(bytes, static_cast<size_t>(8) << 20);
  if (cudaMallocHost(&b.p, b.bytes) != cudaSuccess) {
    (void)cudaGetLastError();
    return StagingBlock{};
  }
  return b;
}

void staging_release(const StagingBlock& b) {
  if (!b.p) return;
  std::lock_guard<std::mutex> lock(g_pin_mu);
  g_stage_free.push_back(b);
}

}  // namespace

void GpuSolver::check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw McdError(MCD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t GpuSolver::full_capacity(const Fcidump& fci, double max_memory) {
  // Table sizing as run_cdfci_wrapper (src/run_wrapper.h:203-213): the
  // largest power of two of determinants whose reference footprint
  // (8*N + 16 bytes, N words per determinant) stays below max_memory.
  const int n_words = 1 + (fci.norb - 1) / 64;
  const double bytes_per_det = static_cast<double>(n_words * 8 + 16);
  size_t pow2 = 8;
  while (static_cast<double>(pow2) * bytes_per_det < max_memory * 1073741824.0) pow2 *= 2;
  return pow2 / 2;
}

GpuSolver::GpuSolver(const Fcidump& fci, const SolverOptions& opt) : opt_(opt) {
  // Option validation (read_input, src/run_wrapper.h:89-119, and this build's limits).
  if (opt_.coordinate_pick != MCD_PICK_GCD_GRAD)
    throw McdError(MCD_ERR_INVALID, "the coordinate pick method is not implemented.");
  if (opt_.coordinate_update == MCD_UPDATE_LS)
    throw McdError(MCD_ERR_UNSUPPORTED,
                   "coordinate_update \"ls\" is not implemented on the GPU; use \"eig\".");
  if (opt_.coordinate_update != MCD_UPDATE_EIG)
    throw McdError(MCD_ERR_INVALID, "the coordinate update method is not implemented.");
  if (!(opt_.max_memory > 0.0))
    throw McdError(MCD_ERR_INVALID,
                   "solver:cdfci:max_memory is invalid. It is the maximum memory (GB) allowed for the "
                   "wavefunction. Please set a positive number.");
  if (opt_.report_interval < 1) throw McdError(MCD_ERR_INVALID, "solver:cdfci:report_interval must be >= 1.");
  if (opt_.num_iterations < 0) throw McdError(MCD_ERR_INVALID, "solver:cdfci:num_iterations must be >= 0.");
  if (opt_.z_threshold_search && opt_.report_interval < 1000)
    throw McdError(MCD_ERR_INVALID, "Please set report_interval >= 1000 when z_threshold_search = true.");
  if (opt_.k < 1 || opt_.k > kMaxK)
    throw McdError(MCD_ERR_UNSUPPORTED, "num_of_coordinate must be in 1.." + std::to_string(kMaxK) + ".");
  if (opt_.m < 1 || opt_.m > kMaxM)
    throw McdError(MCD_ERR_UNSUPPORTED, "estimate must be in 1.." + std::to_string(kMaxM) + ".");
  if (opt_.groups < 0) throw McdError(MCD_ERR_INVALID, "groups must be >= 0.");
  zt_ = opt_.z_threshold;
  uhf_ = fci.uhf;
  if (opt_.z_threshold_search && zt_ < 1e-10) zt_ = 1e-10;

  using clock = std::chrono::steady_clock;
  auto ms_since = [](clock::time_point t) { return std::chrono::duration<double, std::milli>(clock::now() - t).count(); };
  // The host tables are built on a host thread while this one sets up the
  // device and allocates; they are joined before the upload.  Errors keep
  // the order of a serial build: the tables' own checks first, then the
  // reference determinant's.
  double host_ms = 0.0;
  std::future<HamHost> host = std::async(std::launch::async, [&fci, &host_ms, thr = opt_.threshold] {
    const auto t = std::chrono::steady_clock::now();
    HamHost h = build_hamiltonian(fci, thr);
    host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
    return h;
  });
  auto join_host = [&] {
    try {
      ham_ = host.get();
    } catch (const std::invalid_argument& e) {
      throw McdError(MCD_ERR_INVALID, e.what());
    }
    setup_ms_[0] = host_ms;
  };
  {
    std::exception_ptr ref_err;
    try {
      std::string warning;
      if (opt_.ref_det_occ.empty()) {
        ref_ = hartree_fock(fci, &warning);
        if (!warning.empty() && opt_.verbose) std::cout << warning << std::endl << std::endl;
      } else {
        ref_ = ref_det_from_occ(fci, opt_.ref_det_occ);
      }
    } catch (const std::invalid_argument&) {
      ref_err = std::current_exception();
    }
    // Inputs that the tables reject end here, before any device work.
    if (ref_err || fci.norb % 2 || !(opt_.threshold >= 0.0)) {
      join_host();
      try {
        std::rethrow_exception(ref_err);
      } catch (const std::invalid_argument& e) {
        throw McdError(MCD_ERR_INVALID, e.what());
      }
    }
  }
  na_ = __builtin_popcountll(ref_.a);
  nb_ = __builtin_popcountll(ref_.b);
  if (na_ >= 64)  // its only determinant would carry the empty-slot key
    throw McdError(MCD_ERR_UNSUPPORTED, "64 alpha electrons in 64 orbitals (a single determinant) is not supported.");
  entries_ = column_entries(fci.norb / 2, na_, nb_);
  if (entries_ < 0) throw McdError(MCD_ERR_UNSUPPORTED, "a Hamiltonian column has more than 2^31 entries.");
  n_words_ = 1 + (fci.norb - 1) / 64;

  // Table sizing as run_cdfci_wrapper (src/run_wrapper.h:203-213): the
  // largest power of two of determinants whose reference footprint
  // (8*N + 16 bytes) stays below max_memory; max_wavefunction_size is 0.79 of it.
  const size_t pow2 = full_capacity(fci, opt_.max_memory);
  max_capacity_ = pow2;
  max_size_ = static_cast<unsigned long long>(0.79 * static_cast<double>(pow2));
  if (max_capacity_ > (1ull << 32))
    throw McdError(MCD_ERR_UNSUPPORTED, "max_memory asks for more than 2^32 hash slots (128 GB).");

  // Device.
  const auto t_dev = clock::now();
  if (opt_.device >= 0) check(cudaSetDevice(opt_.device), "cudaSetDevice");
  check(cudaGetDevice(&device_), "cudaGetDevice");
  if (opt_.stream) {
    stream_ = opt_.stream;
  } else {
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    own_stream_ = true;
  }
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "cudaDeviceGetAttribute");
  groups_rule_ = column_groups(entries_, opt_.k, opt_.fill_gpu ? 3 * sms : 0);
  groups_ = opt_.groups > 0 ? opt_.groups : groups_rule_;
  if (opt_.autotune && opt_.groups == 0 && groups_ > kMaxGroups) groups_ = kMaxGroups;
  list_ = column_list_size(opt_.m);

  // First table: large enough that two graphs' worth of iterations, each
  // inserting at most k whole columns, keep it below 3/4 full, and at least
  // 2^16 slots; the whole table when growth is off, or when the device could
  // not hold this table and the full one at once (the last growth needs both).
  {
    size_t free_b = 0, total_b = 0;
    check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t margin = static_cast<size_t>(1) << 30;
    budget_slots_ = free_b > margin ? (free_b - margin) / sizeof(Slot) : 0;
    // (or num_iterations, when a solve asks for fewer)
    const double first_iters = static_cast<double>(
        std::min<long long>(2 * graph_iters_, std::max<long long>(1, opt_.num_iterations)));
    const double per_chunk = (first_iters * opt_.k + 1.0) * static_cast<double>(entries_);
    size_t c = static_cast<size_t>(1) << 16;
    while (c < max_capacity_ && 0.75 * static_cast<double>(c) < per_chunk) c <<= 1;
    if (!opt_.table_growth || opt_.table || c >= max_capacity_ || c + max_capacity_ > budget_slots_)
      c = max_capacity_;
    capacity_ = c;
  }
  setup_ms_[7] = ms_since(t_dev);

  auto t_alloc = clock::now();
  auto t_join = t_alloc;
  double alloc_ms = 0.0;
  StagingBlock stage;
  try {
    // Hamiltonian tables in one allocation, sized from the orbital count
    // while the host tables are still being built.
    const size_t no = static_cast<size_t>(fci.norb / 2), nso = static_cast<size_t>(fci.norb);
    const size_t npr = no * (no - 1) / 2;
    const size_t n_hd = nso, n_d2 = nso * nso, n_sh = 2 * no * no, n_st = 2 * no * no * nso, n_sp = 2 * no,
                 n_vss = 2 * npr * npr, n_wab = no * no * no * no;
    size_t off = 0;
    const size_t o_hd = off;
    off = align_up(off + n_hd * 8, 256);
    const size_t o_d2 = off;
    off = align_up(off + n_d2 * 8, 256);
    const size_t o_sh = off;
    off = align_up(off + n_sh * 8, 256);
    const size_t o_st = off;
    off = align_up(off + n_st * 8, 256);
    const size_t o_sp = off;
    off = align_up(off + n_sp * 8, 256);
    const size_t o_vss = off;
    off = align_up(off + std::max<size_t>(n_vss, 1) * 8, 256);
    const size_t o_wab = off;
    off = align_up(off + n_wab * 8, 256);
    // The iteration's small buffers, in the same allocation after the tables.
    // Per-CTA partial lists for the largest CTA count the autotuner tries.
    const size_t parts = static_cast<size_t>(opt_.k) * std::max(groups_, opt_.autotune ? kMaxGroups : 1);
    const size_t mk = static_cast<size_t>(kMaxK) * opt_.m;
    size_t mo = off;
    auto carve = [&](size_t bytes) {
      const size_t o = mo;
      mo = align_up(mo + bytes, 256);
      return o;
    };
    const size_t o_state = carve(sizeof(IterState)), o_cs = carve(mk * sizeof(double)),
                 o_cl = carve(mk * sizeof(unsigned)), o_h = carve((static_cast<size_t>(kMaxK) * kMaxK + 2 * kMaxK + 4) * sizeof(double)),
                 o_err = carve(sizeof(unsigned)), o_occ = carve(sizeof(unsigned long long)),
                 o_sect = carve((kLeaderSections + kColumnSections) * sizeof(unsigned long long)),
                 o_pk = carve(parts * list_ * sizeof(unsigned long long)), o_ps = carve(parts * list_ * sizeof(unsigned)),
                 o_psum = carve(parts * kPartSum * sizeof(double)), o_done = carve(kMaxK * sizeof(unsigned));
    d_tables_ = device_alloc<unsigned char>(mo, "hamiltonian tables and iteration buffers");
    unsigned char* base = static_cast<unsigned char*>(d_tables_);
    auto up = [&](size_t o, const void* src, size_t bytes) {
      if (bytes) check(cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, stream_), "upload tables");
    };
    hd_.norb = static_cast<int>(no);
    hd_.nso = static_cast<int>(nso);
    hd_.npair = static_cast<int>(npr);
    hd_.ecore = fci.core_energy;
    hd_.hdiag = reinterpret_cast<const double*>(base + o_hd);
    hd_.d2 = reinterpret_cast<const double*>(base + o_d2);
    hd_.sh = reinterpret_cast<const double*>(base + o_sh);
    hd_.st = reinterpret_cast<const double*>(base + o_st);
    hd_.spres = reinterpret_cast<const uint64_t*>(base + o_sp);
    hd_.vss = reinterpret_cast<const double*>(base + o_vss);
    hd_.wab = reinterpret_cast<const double*>(base + o_wab);

    if (opt_.table) {
      if (opt_.table_slots != capacity_)
        throw McdError(MCD_ERR_INVALID, "the given table has " + std::to_string(opt_.table_slots) +
                                            " slots; max_memory gives " + std::to_string(capacity_) + ".");
      d_slots_ = opt_.table;
      own_table_ = false;
    } else {
      d_slots_ = device_alloc<Slot>(capacity_, "hash wavefunction");
    }
    unsigned char* mb = static_cast<unsigned char*>(d_tables_);
    d_state_ = reinterpret_cast<IterState*>(mb + o_state);
    d_cand_score_ = reinterpret_cast<double*>(mb + o_cs);
    d_cand_slot_ = reinterpret_cast<unsigned*>(mb + o_cl);
    d_hsub_ = reinterpret_cast<double*>(mb + o_h);
    d_err_ = reinterpret_cast<unsigned*>(mb + o_err);
    d_occ_ = reinterpret_cast<unsigned long long*>(mb + o_occ);
    d_sect_ = reinterpret_cast<unsigned long long*>(mb + o_sect);
    d_part_key_ = reinterpret_cast<unsigned long long*>(mb + o_pk);
    d_part_slot_ = reinterpret_cast<unsigned*>(mb + o_ps);
    d_part_sum_ = reinterpret_cast<double*>(mb + o_psum);
    d_done_ = reinterpret_cast<unsigned*>(mb + o_done);
    check(cudaMemsetAsync(d_sect_, 0, (kLeaderSections + kColumnSections) * sizeof(unsigned long long), stream_),
          "memset");
    check(cudaMemsetAsync(d_done_, 0, kMaxK * sizeof(unsigned), stream_), "memset");
    h_occ_ = pinned_words_acquire();
    for (auto& e : ev_occ_) check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");

    // The host tables, then their upload.
    alloc_ms = ms_since(t_alloc);
    t_join = clock::now();
    join_host();
    ref_diag_ = diagonal_element(ham_, ref_);
    if (ham_.hdiag.size() != n_hd || ham_.d2.size() != n_d2 || ham_.sh.size() != n_sh || ham_.st.size() != n_st ||
        ham_.spres.size() != n_sp || ham_.vss.size() != n_vss || ham_.wab.size() != n_wab)
      throw std::logic_error("host table sizes differ from the device allocation.");
    // Through a pinned staging block, filled on the host task pool in
    // 256 KB pieces, as one copy; from pageable memory when none is had.
    stage = staging_acquire(off);
    if (stage.p) {
      unsigned char* st = static_cast<unsigned char*>(stage.p);
      struct Piece {
        size_t dst;
        const unsigned char* src;
        size_t bytes;
      };
      std::vector<Piece> pieces;
      auto add = [&](size_t o, const void* src, size_t bytes) {
        constexpr size_t kPiece = static_cast<size_t>(256) << 10;
        for (size_t b = 0; b < bytes; b += kPiece)
          pieces.push_back({o + b, static_cast<const unsigned char*>(src) + b, std::min(kPiece, bytes - b)});
      };
      add(o_hd, ham_.hdiag.data(), n_hd * 8);
      add(o_d2, ham_.d2.data(), n_d2 * 8);
      add(o_sh, ham_.sh.data(), n_sh * 8);
      add(o_st, ham_.st.data(), n_st * 8);
      add(o_sp, ham_.spres.data(), n_sp * 8);
      add(o_vss, ham_.vss.data(), n_vss * 8);
      add(o_wab, ham_.wab.data(), n_wab * 8);
      const auto t_copy = clock::now();
      host_parallel(static_cast<int>(pieces.size()),
                    [&](int i) { std::memcpy(st + pieces[i].dst, pieces[i].src, pieces[i].bytes); });
      setup_ms_[8] = ms_since(t_copy);
      check(cudaMemcpyAsync(base, st, off, cudaMemcpyHostToDevice, stream_), "upload tables");
    } else {
      up(o_hd, ham_.hdiag.data(), n_hd * 8);
      up(o_d2, ham_.d2.data(), n_d2 * 8);
      up(o_sh, ham_.sh.data(), n_sh * 8);
      up(o_st, ham_.st.data(), n_st * 8);
      up(o_sp, ham_.spres.data(), n_sp * 8);
      up(o_vss, ham_.vss.data(), n_vss * 8);
      up(o_wab, ham_.wab.data(), n_wab * 8);
    }
  } catch (...) {
    if (stage.p) {
      cudaStreamSynchronize(stream_);
      staging_release(stage);
    }
    release();
    throw;
  }

  td_.slots = d_slots_;
  td_.mask = capacity_ - 1;
  td_.max_probe = static_cast<int>(std::min<size_t>(capacity_, 1u << 14));
  td_.err = d_err_;
  td_.n_occupied = d_occ_;

  cl_.ham = hd_;
  cl_.tab = td_;
  cl_.st = d_state_;
  cl_.cand_score = d_cand_score_;
  cl_.cand_slot = d_cand_slot_;
  cl_.part_key = d_part_key_;
  cl_.part_slot = d_part_slot_;
  cl_.part_sum = d_part_sum_;
  cl_.done = d_done_;
  cl_.m = opt_.m;
  cl_.groups = groups_;
  cl_.k_grid = opt_.k;
  cl_.na = na_;
  cl_.nb = nb_;

  ll_.ham = hd_;
  ll_.tab = td_;
  ll_.st = d_state_;
  ll_.cand_score = d_cand_score_;
  ll_.cand_slot = d_cand_slot_;
  ll_.hsub_out = d_hsub_;
  ll_.sect = d_sect_;
  ll_.m = opt_.m;
  ll_.k_req = opt_.k;
  ll_.eig_method = opt_.eig_method;
  const auto t_sync = clock::now();
  const cudaError_t sync_err = cudaStreamSynchronize(stream_);
  setup_ms_[9] = ms_since(t_sync);
  staging_release(stage);
  check(sync_err, "table upload");
  setup_ms_[1] = alloc_ms;
  setup_ms_[2] = ms_since(t_join);
}

GpuSolver::~GpuSolver() { release(); }

void GpuSolver::release() {
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  if (stream_) cudaStreamSynchronize(stream_);
  cudaFree(d_tables_);
  if (own_table_) cudaFree(d_slots_);
  cudaFree(d_misc_);
  d_misc_ = nullptr;
  d_sect_ = nullptr;
  d_part_key_ = nullptr;
  d_part_slot_ = nullptr;
  d_part_sum_ = nullptr;
  d_done_ = nullptr;
  d_tables_ = nullptr;
  d_slots_ = nullptr;
  d_state_ = nullptr;
  d_cand_score_ = nullptr;
  d_cand_slot_ = nullptr;
  d_hsub_ = nullptr;
  d_err_ = nullptr;
  d_occ_ = nullptr;
  if (h_occ_) pinned_words_release(h_occ_);
  h_occ_ = nullptr;
  for (auto& e : ev_occ_) {
    if (e) cudaEventDestroy(e);
    e = nullptr;
  }
  if (own_stream_ && stream_) cudaStreamDestroy(stream_);
  stream_ = nullptr;
  own_stream_ = false;
}

void GpuSolver::reset() {
  const auto t0 = std::chrono::steady_clock::now();
  check(launch_table_fill(d_slots_, capacity_, stream_), "table fill");
  check(cudaMemsetAsync(d_err_, 0, sizeof(unsigned), stream_), "memset");
  check(cudaMemsetAsync(d_occ_, 0, sizeof(unsigned long long), stream_), "memset");
  check(cudaStreamSynchronize(stream_), "table fill");
  setup_ms_[3] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  std::memset(&h_state_, 0, sizeof(h_state_));
  h_state_.zt = zt_;
  h_state_.n_words = n_words_;
  h_state_.k_req = opt_.k;
  h_state_.m = opt_.m;
  h_state_.occupancy_limit = static_cast<unsigned long long>(0.79 * static_cast<double>(max_size_));
  check(cudaMemcpyAsync(d_state_, &h_state_, sizeof(IterState), cudaMemcpyHostToDevice, stream_), "state upload");
  check(launch_init(ll_, ref_, ref_diag_, stream_), "init");
  check(launch_column(cl_, stream_), "column (init)");
  // The initial column inserts at most one column's entries.
  iters_enqueued_ = 0;
  occ_iters_[0] = occ_iters_[1] = -1;
  occ_exact_ = static_cast<unsigned long long>(entries_);
  occ_exact_iters_ = 0;
}

void GpuSolver::build_graph() {
  const auto t0 = std::chrono::steady_clock::now();
  // Launch attributes are set outside the capture.
  check(prepare_leader(ll_), "leader attributes");
  cudaGraph_t g = nullptr;
  check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
  for (long long i = 0; i < graph_iters_; ++i) {
    launch_leader(ll_, stream_);
    launch_column(cl_, stream_);
  }
  check(cudaStreamEndCapture(stream_, &g), "end capture");
  check(cudaGraphInstantiate(&graph_, g, 0), "graph instantiate");
  cudaGraphDestroy(g);
  setup_ms_[4] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

size_t GpuSolver::next_capacity(size_t c) const {
  size_t n = c * 2;
  // The growth after this one would need this table and the full one at once.
  if (n < max_capacity_ && n + max_capacity_ > budget_slots_) n = max_capacity_;
  return std::min(n, max_capacity_);
}

void GpuSolver::record_occupancy(long long iters) {
  iters_enqueued_ += iters;
  if (capacity_ >= max_capacity_) return;
  const int i = occ_next_;
  check(cudaMemcpyAsync(h_occ_ + i, d_occ_, sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_),
        "occupancy read");
  check(cudaEventRecord(ev_occ_[i], stream_), "cudaEventRecord");
  occ_iters_[i] = iters_enqueued_;
  occ_next_ = 1 - i;
}

void GpuSolver::ensure_room(long long upcoming) {
  if (capacity_ >= max_capacity_) return;
  const double per_iter = static_cast<double>(opt_.k) * static_cast<double>(entries_);
  // The newest occupancy known without waiting for the last chunk: the read
  // after the chunk before it (usually done, since the last chunk is queued
  // behind it), else the last synchronous read.
  unsigned long long known = occ_exact_;
  long long at = occ_exact_iters_;
  const int older = occ_next_;  // a ring of two: the next slot to write holds the older read
  if (occ_iters_[older] > at) {
    check(cudaEventSynchronize(ev_occ_[older]), "occupancy wait");
    known = h_occ_[older];
    at = occ_iters_[older];
  }
  auto fits = [&](unsigned long long occ, long long iters, size_t cap) {
    return static_cast<double>(occ) + static_cast<double>(iters) * per_iter <= 0.75 * static_cast<double>(cap);
  };
  // Linear probing slows as the load rises (a probe walks longer runs): on
  // the 24-orbital 6+6 workload at k = 32 the column kernel takes 63 us at
  // load 0.12, 64 us at 0.24 and 72 us at 0.47, with the same wavefunction.
  // So the table also doubles once the load it has reached passes
  // kGrowLoad, while max_memory allows.
  constexpr double kGrowLoad = 0.25;
  auto light = [&](unsigned long long occ, size_t cap) {
    return static_cast<double>(occ) <= kGrowLoad * static_cast<double>(cap);
  };
  if (fits(known, iters_enqueued_ - at + upcoming, capacity_) && light(known, capacity_)) return;
  // Might not fit, or is past the load: wait for everything enqueued and
  // grow until it fits and is below the load.
  check(cudaStreamSynchronize(stream_), "synchronize");
  unsigned long long occ = 0;
  check(cudaMemcpy(&occ, d_occ_, sizeof(occ), cudaMemcpyDeviceToHost), "occupancy read");
  occ_exact_ = occ;
  occ_exact_iters_ = iters_enqueued_;
  size_t cap = capacity_;
  while (cap < max_capacity_ && (!fits(occ, upcoming, cap) || !light(occ, cap))) cap = next_capacity(cap);
  if (cap != capacity_) grow_to(cap);
}

bool GpuSolver::grow_now(int mode, long long* wrap) {
  if (mode < 0 || mode > 2) throw McdError(MCD_ERR_INVALID, "growth mode must be 0, 1 or 2.");
  if (capacity_ >= max_capacity_) return false;
  read_state();
  if (wrap) {
    const size_t w = std::min<size_t>(capacity_, static_cast<size_t>(1) << 16);
    std::vector<Slot> head(w), tail(w);
    check(cudaMemcpy(head.data(), d_slots_, w * sizeof(Slot), cudaMemcpyDeviceToHost), "table read");
    check(cudaMemcpy(tail.data(), d_slots_ + (capacity_ - w), w * sizeof(Slot), cudaMemcpyDeviceToHost), "table read");
    auto empty = [](const Slot& x) { return x.a == kEmptyKey && x.b == kEmptyKey; };
    long long first = -1, last = -1;
    for (size_t i = 0; i < w && first < 0; ++i)
      if (empty(head[i])) first = static_cast<long long>(i);
    for (size_t i = w; i-- > 0 && last < 0;)
      if (empty(tail[i])) last = static_cast<long long>(i);
    *wrap = (first < 0 || last < 0) ? -1 : first + static_cast<long long>(w) - 1 - last;
  }
  grow_to(next_capacity(capacity_), mode);
  return true;
}

void GpuSolver::grow_to(size_t new_capacity, int mode) {
  const auto t0 = std::chrono::steady_clock::now();
  read_state();  // applies the pending end of the iteration; nothing in flight
  const auto t_alloc = std::chrono::steady_clock::now();
  const int m = opt_.m;
  Slot* fresh = nullptr;
  Slot* saved = nullptr;
  try {
    fresh = device_alloc<Slot>(new_capacity, "hash wavefunction (growth)");
    saved = device_alloc<Slot>(static_cast<size_t>(kMaxK) * m, "candidates");
  } catch (const McdError& e) {
    if (fresh) cudaFree(fresh);
    throw McdError(MCD_ERR_CUDA, std::string("the hash table could not grow to ") + std::to_string(new_capacity) +
                                     " slots (device memory taken since the solver was created?): " + e.what());
  }
  const auto t1 = std::chrono::steady_clock::now();
  TableDev t = td_;
  t.slots = fresh;
  t.mask = new_capacity - 1;
  t.max_probe = static_cast<int>(std::min<size_t>(new_capacity, 1u << 14));
  // A doubling (below 2^32 slots, where no slot is reserved) moves runs of
  // clusters whole and writes every new slot; anything else is a fill and an
  // insert of every entry, which recounts the occupancy.
  const bool doubling = mode != 2 && new_capacity == 2 * capacity_ && new_capacity < (static_cast<size_t>(1) << 32);
  cudaError_t e = cudaSuccess;
  if (!doubling) {
    e = launch_table_fill(fresh, new_capacity, stream_);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_occ_, 0, sizeof(unsigned long long), stream_);
  }
  if (e == cudaSuccess) {
    compact_cand_save_kernel<<<kMaxK, 128, 0, stream_>>>(d_slots_, d_state_, d_cand_slot_, m, saved);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = doubling ? launch_rehash_double(d_slots_, capacity_, t, mode == 1, stream_)
                 : launch_rehash(d_slots_, capacity_, t, stream_);
  if (e == cudaSuccess) {
    compact_cand_restore_kernel<<<kMaxK, 128, 0, stream_>>>(t, d_state_, saved, d_cand_slot_, m);
    e = cudaGetLastError();
  }
  unsigned long long occ = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&occ, d_occ_, sizeof(occ), cudaMemcpyDeviceToHost, stream_);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream_);
  const auto t2 = std::chrono::steady_clock::now();
  cudaFree(saved);
  if (e != cudaSuccess) {
    cudaFree(fresh);
    check(e, "table growth");
  }
  cudaFree(d_slots_);
  const auto t3 = std::chrono::steady_clock::now();
  setup_ms_[10] += std::chrono::duration<double, std::milli>(t1 - t_alloc).count();
  setup_ms_[11] += std::chrono::duration<double, std::milli>(t2 - t1).count();
  setup_ms_[12] += std::chrono::duration<double, std::milli>(t3 - t2).count();
  d_slots_ = fresh;
  capacity_ = new_capacity;
  td_ = t;
  cl_.tab = td_;
  ll_.tab = td_;
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
  ++growths_;
  occ_exact_ = occ;
  occ_exact_iters_ = iters_enqueued_;
  occ_iters_[0] = occ_iters_[1] = -1;
  setup_ms_[5] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  read_state();  // a probe-limit error during the rehash surfaces here
}

void GpuSolver::launch_chunk(long long n) {
  if (n == graph_iters_) {
    if (!graph_) build_graph();
    check(cudaGraphLaunch(graph_, stream_), "graph launch");
    return;
  }
  for (long long i = 0; i < n; ++i) {
    check(launch_leader(ll_, stream_), "leader");
    check(launch_column(cl_, stream_), "column");
  }
}

namespace {
std::mutex g_tune_mu;
std::map<std::vector<int>, int> g_tune_cache;  // (norb, na, nb, k, m, SMs) -> CTAs per column
}  // namespace

void GpuSolver::set_groups(int g) {
  if (g == groups_) return;
  groups_ = g;
  cl_.groups = g;
  if (graph_) cudaGraphExecDestroy(graph_);
  graph_ = nullptr;
}

long long GpuSolver::autotune_groups(long long budget) {
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "cudaDeviceGetAttribute");
  const std::vector<int> key{ham_.norb, na_, nb_, opt_.k, opt_.m, sms};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      set_groups(it->second);
      tuned_ = true;
      return 0;
    }
  }
  // Candidates around the rule, within 1..kMaxGroups.
  std::vector<int> cand;
  for (int g : {groups_rule_, groups_rule_ / 2, groups_rule_ * 2, groups_rule_ * 3 / 4, groups_rule_ * 3 / 2, 8, 16,
                32, 64}) {
    g = std::max(1, std::min(g, kMaxGroups));
    if (std::find(cand.begin(), cand.end(), g) == cand.end()) cand.push_back(g);
  }
  if (budget < kTuneIters * static_cast<long long>(cand.size())) return 0;  // not enough iterations yet
  tuned_ = true;
  long long done = 0;
  int best = groups_;
  double best_us = 1e300;
  tune_trials_.clear();
  for (int g : cand) {
    set_groups(g);
    double lead = 0.0, col = 0.0, tot = 0.0;
    run_iterations_timed(kTuneIters, &lead, &col, &tot);
    done += kTuneIters;
    const double us = 1000.0 * col / kTuneIters;
    tune_trials_.push_back({g, us});
    if (us < best_us) {
      best_us = us;
      best = g;
    }
  }
  set_groups(best);
  // A trial that ended in a device error (a full table, say) timed no work:
  // surface the error instead of keeping its choice.
  read_state();
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune_cache[key] = best;
  return done;
}

void GpuSolver::run_iterations(long long n) {
  if (opt_.autotune && !tuned_ && opt_.groups == 0) n -= autotune_groups(n);
  while (n > 0) {
    const long long c = std::min(n, graph_iters_);
    ensure_room(c);
    launch_chunk(c);
    record_occupancy(c);
    n -= c;
  }
}

void GpuSolver::run_iterations_timed(long long n, double* leader_ms, double* column_ms, double* total_ms) {
  *leader_ms = *column_ms = *total_ms = 0.0;
  if (n <= 0) return;
  // Per iteration: before the leader, between the kernels, after the column
  // kernel; a table growth between two iterations counts in the total only.
  std::vector<cudaEvent_t> ev(static_cast<size_t>(3 * n));
  for (auto& e : ev) check(cudaEventCreate(&e), "cudaEventCreate");
  try {
    for (long long i0 = 0; i0 < n; i0 += graph_iters_) {
      const long long c = std::min(n - i0, graph_iters_);
      ensure_room(c);
      for (long long i = i0; i < i0 + c; ++i) {
        check(cudaEventRecord(ev[3 * i], stream_), "cudaEventRecord");
        check(launch_leader(ll_, stream_), "leader");
        check(cudaEventRecord(ev[3 * i + 1], stream_), "cudaEventRecord");
        check(launch_column(cl_, stream_), "column");
        check(cudaEventRecord(ev[3 * i + 2], stream_), "cudaEventRecord");
      }
      record_occupancy(c);
    }
    check(cudaEventSynchronize(ev[3 * n - 1]), "cudaEventSynchronize");
    for (long long i = 0; i < n; ++i) {
      float a = 0.f, b = 0.f;
      check(cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]), "cudaEventElapsedTime");
      check(cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]), "cudaEventElapsedTime");
      *leader_ms += a;
      *column_ms += b;
    }
    float t = 0.f;
    check(cudaEventElapsedTime(&t, ev[0], ev[3 * n - 1]), "cudaEventElapsedTime");
    *total_ms = t;
  } catch (...) {
    for (auto& e : ev) cudaEventDestroy(e);
    throw;
  }
  for (auto& e : ev) cudaEventDestroy(e);
}

void GpuSolver::read_state() {
  check(launch_finish(ll_, stream_), "finish");
  check(cudaMemcpyAsync(&h_state_, d_state_, sizeof(IterState), cudaMemcpyDeviceToHost, stream_), "state read");
  unsigned err = 0;
  check(cudaMemcpyAsync(&err, d_err_, sizeof(unsigned), cudaMemcpyDeviceToHost, stream_), "error read");
  check(cudaStreamSynchronize(stream_), "synchronize");
  if (err) {
    if (err & (kErrProbe | kErrOverflow))
      throw McdError(MCD_ERR_OVERFLOW, "The hash table is full. Please increase max_memory or z_threshold.");
    if (err & kErrEig)
      throw McdError(MCD_ERR_EIG,
                     "The subspace eigenvalue problem failed (its lowest eigenvalue must be negative: the method "
                     "minimises ||H + x x^T||_F^2, which needs a negative ground-state energy; a positive core "
                     "energy in the FCIDUMP can make it positive).");
    if (err & kErrCandidates) throw McdError(MCD_ERR_NO_CANDIDATES, "The candidate list is empty.");
    throw McdError(MCD_ERR_CUDA, "device error word " + std::to_string(err));
  }
}

mcd_report GpuSolver::report() {
  const auto t0 = std::chrono::steady_clock::now();
  read_state();
  mcd_report r{};
  r.iteration = h_state_.iter;
  const dd xz{dd_to_d(h_state_.xz), 0.0};
  r.energy = dd_to_d(dd_div(xz, h_state_.xx));
  r.dx_max = h_state_.dx_max;
  r.x_size = h_state_.x_size;
  r.z_size = h_state_.z_size;
  r.cols_size = h_state_.emitted;
  r.updates = h_state_.updates;
  r.scale = dd_to_d(h_state_.scale);
  r.max_residual = h_state_.eig_residual_max;
  r.z_threshold = zt_;
  r.emitted_total = h_state_.emitted_total;
  r.updates_total = h_state_.updates_total;
  r.occupied = 0;
  check(cudaMemcpy(&r.occupied, d_occ_, sizeof(unsigned long long), cudaMemcpyDeviceToHost), "occupancy read");
  r.last_k = h_state_.k_cur;
  r.inv_steps_last = h_state_.inv_steps_curr;
  r.inv_updates = h_state_.inv_updates;
  r.inv_steps = h_state_.inv_steps;
  r.eig_fallbacks = h_state_.eig_fallbacks;
  r.max_abs_evec = h_state_.max_abs_evec;
  occ_exact_ = r.occupied;
  occ_exact_iters_ = iters_enqueued_;
  setup_ms_[6] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return r;
}

void GpuSolver::wavefunction(std::vector<Det>& dets, std::vector<double>& x) {
  read_state();
  const unsigned long long cap = h_state_.x_size + 64;
  unsigned* d_list = device_alloc<unsigned>(cap, "x list");
  unsigned long long* d_count = nullptr;
  try {
    d_count = device_alloc<unsigned long long>(1, "x count");
    check(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), stream_), "memset");
    check(launch_rdm_list(td_, capacity_, d_list, d_count, cap, stream_), "x list");
    unsigned long long cnt = 0;
    check(cudaMemcpyAsync(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost, stream_), "count read");
    check(cudaStreamSynchronize(stream_), "synchronize");
    if (cnt > cap) throw McdError(MCD_ERR_CUDA, "more nonzero coefficients than x_size counted");
    std::vector<unsigned> list(cnt);
    if (cnt) check(cudaMemcpy(list.data(), d_list, cnt * sizeof(unsigned), cudaMemcpyDeviceToHost), "list read");
    std::sort(list.begin(), list.end());
    dets.resize(cnt);
    x.resize(cnt);
    for (size_t i = 0; i < cnt; ++i) {
      Slot sl;
      check(cudaMemcpy(&sl, d_slots_ + list[i], sizeof(Slot), cudaMemcpyDeviceToHost), "slot read");
      dets[i] = Det{sl.a, sl.b};
      x[i] = sl.x;
    }
  } catch (...) {
    cudaFree(d_list);
    if (d_count) cudaFree(d_count);
    throw;
  }
  cudaFree(d_list);
  cudaFree(d_count);
}

void GpuSolver::rdm(std::vector<double>& rdm1, std::vector<double>& rdm2) {
  if (uhf_) throw McdError(MCD_ERR_UNSUPPORTED, "RDMs are implemented for RHF FCIDUMPs.");
  read_state();
  const int n = ham_.norb;
  const size_t n2 = static_cast<size_t>(n) * n, n4 = n2 * n2;
  const unsigned long long cap = h_state_.x_size + 64;
  std::vector<void*> owned;
  auto alloc = [&](size_t bytes, const char* what) {
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      for (void* q : owned) cudaFree(q);
      throw McdError(MCD_ERR_CUDA, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
    }
    owned.push_back(p);
    return p;
  };
  try {
    auto* d_list = static_cast<unsigned*>(alloc(cap * sizeof(unsigned), "rdm list"));
    auto* d_count = static_cast<unsigned long long*>(alloc(sizeof(unsigned long long), "rdm count"));
    auto* d_g = static_cast<double*>(alloc((2 * n2 + 3 * n4) * sizeof(double), "rdm"));
    check(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), stream_), "memset");
    check(cudaMemsetAsync(d_g, 0, (2 * n2 + 3 * n4) * sizeof(double), stream_), "memset");
    check(launch_rdm_list(td_, capacity_, d_list, d_count, cap, stream_), "rdm list");
    unsigned long long cnt = 0;
    check(cudaMemcpyAsync(&cnt, d_count, sizeof(cnt), cudaMemcpyDeviceToHost, stream_), "count read");
    check(cudaStreamSynchronize(stream_), "synchronize");
    if (cnt > cap) throw McdError(MCD_ERR_CUDA, "more nonzero coefficients than x_size counted");
    RdmLaunch r{};
    r.ham = hd_;
    r.tab = td_;
    r.list = d_list;
    r.nlist = static_cast<long long>(cnt);
    r.g1a = d_g;
    r.g1b = d_g + n2;
    r.g2aa = d_g + 2 * n2;
    r.g2bb = r.g2aa + n4;
    r.g2ab = r.g2bb + n4;
    check(launch_rdm(r, stream_), "rdm");
    std::vector<double> g(2 * n2 + 3 * n4);
    check(cudaMemcpyAsync(g.data(), d_g, g.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_), "rdm read");
    check(cudaStreamSynchronize(stream_), "synchronize");
    for (void* q : owned) cudaFree(q);
    owned.clear();
    const double norm = 1.0 / dd_to_d(h_state_.xx);
    const double* g1a = g.data();
    const double* g1b = g1a + n2;
    const double* aa = g1b + n2;
    const double* bb = aa + n4;
    const double* ab = bb + n4;
    rdm1.assign(n2, 0.0);
    rdm2.assign(n4, 0.0);
    for (size_t i = 0; i < n2; ++i) rdm1[i] = (g1a[i] + g1b[i]) * norm;
    auto I = [n](int p, int q, int r, int s) { return ((static_cast<size_t>(p) * n + q) * n + r) * n + s; };
    for (int p = 0; p < n; ++p)
      for (int q = 0; q < n; ++q)
        for (int r = 0; r < n; ++r)
          for (int s2 = 0; s2 < n; ++s2) {
            // Same-spin blocks from their canonical p < q, r < s elements.
            double same = 0.0;
            if (p != q && r != s2) {
              const int cp = p < q ? p : q, cq = p < q ? q : p, cr = r < s2 ? r : s2, cs = r < s2 ? s2 : r;
              const double sg = ((p < q) ? 1.0 : -1.0) * ((r < s2) ? 1.0 : -1.0);
              same = sg * (aa[I(cp, cq, cr, cs)] + bb[I(cp, cq, cr, cs)]);
            }
            // Opposite spins: (alpha, beta) + (beta, alpha) = ab[p][q][r][s] + ab[q][p][s][r].
            rdm2[I(p, q, r, s2)] = (same + ab[I(p, q, r, s2)] + ab[I(q, p, s2, r)]) * norm;
          }
  } catch (...) {
    for (void* q : owned) cudaFree(q);
    throw;
  }
}

unsigned long long GpuSolver::compact(double z_threshold) {
  read_state();  // applies the pending end of the iteration; no work in flight
  if (!(z_threshold >= zt_)) throw McdError(MCD_ERR_INVALID, "compaction needs z_threshold >= the current one.");
  const double sc = std::fabs(dd_to_d(h_state_.scale));
  // |dz scale| > zt is the insertion rule; |z scale| <= zt is dropped here.
  const double zlim = z_threshold / std::max(sc, 1e-300);
  const int nb = 148 * 8;
  const size_t chunk = (capacity_ + nb - 1) / nb;
  const int m = opt_.m;
  std::vector<void*> owned;
  auto alloc = [&](size_t bytes, const char* what) {
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess)
      throw McdError(MCD_ERR_CUDA, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
    owned.push_back(p);
    return p;
  };
  unsigned long long occ = 0;
  try {
    auto* d_counts = static_cast<unsigned long long*>(alloc(nb * sizeof(unsigned long long), "compaction counts"));
    compact_count_kernel<<<nb, 256, 0, stream_>>>(d_slots_, capacity_, chunk, zlim, d_counts);
    check(cudaGetLastError(), "compaction count");
    std::vector<unsigned long long> counts(nb), offs(nb);
    check(cudaMemcpyAsync(counts.data(), d_counts, nb * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_),
          "counts read");
    check(cudaStreamSynchronize(stream_), "synchronize");
    unsigned long long total = 0;
    for (int b = 0; b < nb; ++b) {
      offs[b] = total;
      total += counts[b];
    }
    check(cudaMemcpyAsync(d_counts, offs.data(), nb * sizeof(unsigned long long), cudaMemcpyHostToDevice, stream_),
          "offsets");
    auto* d_out = static_cast<Slot*>(alloc(std::max<unsigned long long>(total, 1) * sizeof(Slot), "compaction buffer"));
    auto* d_saved = static_cast<Slot*>(alloc(static_cast<size_t>(kMaxK) * m * sizeof(Slot), "candidates"));
    compact_cand_save_kernel<<<kMaxK, 128, 0, stream_>>>(d_slots_, d_state_, d_cand_slot_, m, d_saved);
    check(cudaGetLastError(), "candidates save");
    compact_write_kernel<<<nb, 256, 0, stream_>>>(d_slots_, capacity_, chunk, zlim, d_counts, d_out);
    check(cudaGetLastError(), "compaction write");
    check(launch_table_fill(d_slots_, capacity_, stream_), "table clear");
    check(cudaMemsetAsync(d_occ_, 0, sizeof(unsigned long long), stream_), "memset");
    compact_reinsert_kernel<<<148 * 8, 256, 0, stream_>>>(td_, d_out, total);
    check(cudaGetLastError(), "reinsert");
    compact_cand_restore_kernel<<<kMaxK, 128, 0, stream_>>>(td_, d_state_, d_saved, d_cand_slot_, m);
    check(cudaGetLastError(), "candidates restore");
    check(cudaMemcpyAsync(&occ, d_occ_, sizeof(occ), cudaMemcpyDeviceToHost, stream_), "occupancy read");
    check(cudaStreamSynchronize(stream_), "synchronize");
    for (void* q : owned) cudaFree(q);
    owned.clear();
  } catch (...) {
    for (void* q : owned) cudaFree(q);
    throw;
  }
  zt_ = z_threshold;
  h_state_.zt = zt_;
  h_state_.z_size = occ;
  check(cudaMemcpyAsync(reinterpret_cast<char*>(d_state_) + offsetof(IterState, zt), &h_state_.zt, sizeof(double),
                        cudaMemcpyHostToDevice, stream_), "zt upload");
  check(cudaMemcpyAsync(reinterpret_cast<char*>(d_state_) + offsetof(IterState, z_size), &h_state_.z_size,
                        sizeof(unsigned long long), cudaMemcpyHostToDevice, stream_), "z_size upload");
  check(cudaStreamSynchronize(stream_), "synchronize");
  read_state();
  return occ;
}

// ---------------------------------------------------------------------------
// Checkpoint: header, iteration state, the occupied slots in slot order and
// the candidate lists by determinant; loading rebuilds the table by insertion.

namespace {
constexpr char kCkptMagic[8] = {'M', 'C', 'D', 'F', 'C', 'I', 'K', '2'};
struct CkptHeader {
  char magic[8];
  int32_t nso, na, nb, k, m, pad;
  double ecore;
  uint64_t ham_hash;  // FNV-1a over the bytes of the Hamiltonian tables
  uint64_t state_bytes, nslots, ncand;
};

uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
  const unsigned char* c = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= c[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

// Identifies the integrals a checkpoint was made with: the same FCIDUMP and
// hamiltonian threshold give the same tables, bit for bit.
uint64_t ham_fingerprint(const HamHost& h) {
  uint64_t f = 0xcbf29ce484222325ull;
  f = fnv1a(f, h.hdiag.data(), h.hdiag.size() * sizeof(double));
  f = fnv1a(f, h.d2.data(), h.d2.size() * sizeof(double));
  f = fnv1a(f, h.sh.data(), h.sh.size() * sizeof(double));
  f = fnv1a(f, h.st.data(), h.st.size() * sizeof(double));
  f = fnv1a(f, h.spres.data(), h.spres.size() * sizeof(uint64_t));
  f = fnv1a(f, h.vss.data(), h.vss.size() * sizeof(double));
  f = fnv1a(f, h.wab.data(), h.wab.size() * sizeof(double));
  return fnv1a(f, &h.ecore, sizeof(double));
}
}  // namespace

void GpuSolver::gather_slots(double zlim, std::vector<Slot>& out) {
  const int nb = 148 * 8;
  const size_t chunk = (capacity_ + nb - 1) / nb;
  unsigned long long* d_counts = device_alloc<unsigned long long>(nb, "gather counts");
  Slot* d_out = nullptr;
  try {
    compact_count_kernel<<<nb, 256, 0, stream_>>>(d_slots_, capacity_, chunk, zlim, d_counts);
    check(cudaGetLastError(), "gather count");
    std::vector<unsigned long long> counts(nb), offs(nb);
    check(cudaMemcpyAsync(counts.data(), d_counts, nb * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream_),
          "counts read");
    check(cudaStreamSynchronize(stream_), "synchronize");
    unsigned long long total = 0;
    for (int b = 0; b < nb; ++b) {
      offs[b] = total;
      total += counts[b];
    }
    check(cudaMemcpyAsync(d_counts, offs.data(), nb * sizeof(unsigned long long), cudaMemcpyHostToDevice, stream_),
          "offsets");
    d_out = device_alloc<Slot>(std::max<unsigned long long>(total, 1), "gather buffer");
    compact_write_kernel<<<nb, 256, 0, stream_>>>(d_slots_, capacity_, chunk, zlim, d_counts, d_out);
    check(cudaGetLastError(), "gather write");
    out.resize(total);
    if (total)
      check(cudaMemcpyAsync(out.data(), d_out, total * sizeof(Slot), cudaMemcpyDeviceToHost, stream_), "slots read");
    check(cudaStreamSynchronize(stream_), "synchronize");
  } catch (...) {
    cudaFree(d_counts);
    if (d_out) cudaFree(d_out);
    throw;
  }
  cudaFree(d_counts);
  cudaFree(d_out);
}

void GpuSolver::slots(std::vector<Slot>& out) {
  read_state();
  gather_slots(-1.0, out);
}

void GpuSolver::checkpoint_save(const std::string& path) {
  read_state();
  std::vector<Slot> slots;
  gather_slots(-1.0, slots);
  const int m = opt_.m;
  std::vector<Slot> cand(static_cast<size_t>(kMaxK) * m);
  Slot* d_saved = device_alloc<Slot>(cand.size(), "candidates");
  try {
    compact_cand_save_kernel<<<kMaxK, 128, 0, stream_>>>(d_slots_, d_state_, d_cand_slot_, m, d_saved);
    check(cudaGetLastError(), "candidates save");
    check(cudaMemcpyAsync(cand.data(), d_saved, cand.size() * sizeof(Slot), cudaMemcpyDeviceToHost, stream_),
          "candidates read");
    check(cudaStreamSynchronize(stream_), "synchronize");
  } catch (...) {
    cudaFree(d_saved);
    throw;
  }
  cudaFree(d_saved);
  CkptHeader h{};
  std::memcpy(h.magic, kCkptMagic, 8);
  h.nso = ham_.nso;
  h.na = na_;
  h.nb = nb_;
  h.k = opt_.k;
  h.m = m;
  h.ecore = ham_.ecore;
  h.ham_hash = ham_fingerprint(ham_);
  h.state_bytes = sizeof(IterState);
  h.nslots = slots.size();
  h.ncand = cand.size();
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw McdError(MCD_ERR_INVALID, "cannot write the checkpoint file " + path);
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(&h_state_, sizeof(IterState), 1, f) == 1 &&
            (slots.empty() || std::fwrite(slots.data(), sizeof(Slot), slots.size(), f) == slots.size()) &&
            std::fwrite(cand.data(), sizeof(Slot), cand.size(), f) == cand.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) throw McdError(MCD_ERR_INVALID, "writing the checkpoint file " + path + " failed");
}

void GpuSolver::checkpoint_load(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw McdError(MCD_ERR_INVALID, "cannot read the checkpoint file " + path);
  CkptHeader h{};
  IterState st{};
  std::vector<Slot> slots, cand;
  bool ok = std::fread(&h, sizeof(h), 1, f) == 1;
  if (ok && std::memcmp(h.magic, kCkptMagic, 8) != 0) ok = false;
  if (ok && (h.nso != ham_.nso || h.na != na_ || h.nb != nb_ || h.k != opt_.k || h.m != opt_.m ||
             h.ecore != ham_.ecore || h.ham_hash != ham_fingerprint(ham_) ||
             h.state_bytes != sizeof(IterState) || h.ncand != static_cast<uint64_t>(kMaxK) * opt_.m)) {
    std::fclose(f);
    throw McdError(MCD_ERR_INVALID, "the checkpoint " + path + " belongs to another problem or other options");
  }
  if (ok) ok = std::fread(&st, sizeof(st), 1, f) == 1;
  if (ok) {
    slots.resize(h.nslots);
    cand.resize(h.ncand);
    ok = (slots.empty() || std::fread(slots.data(), sizeof(Slot), slots.size(), f) == slots.size()) &&
         std::fread(cand.data(), sizeof(Slot), cand.size(), f) == cand.size();
  }
  std::fclose(f);
  if (!ok) throw McdError(MCD_ERR_INVALID, "the checkpoint file " + path + " is not readable");
  const unsigned long long limit = static_cast<unsigned long long>(0.79 * static_cast<double>(max_size_));
  if (slots.size() > limit)
    throw McdError(MCD_ERR_OVERFLOW, "The hash table is full. Please increase max_memory or z_threshold.");
  check(cudaStreamSynchronize(stream_), "synchronize");
  // A table that grows on demand is enlarged first to hold the saved entries
  // below 3/4 full (its contents are replaced anyway).
  {
    size_t cap = capacity_;
    while (cap < max_capacity_ && static_cast<double>(slots.size()) > 0.75 * static_cast<double>(cap))
      cap = next_capacity(cap);
    if (cap != capacity_) {
      Slot* fresh = device_alloc<Slot>(cap, "hash wavefunction (checkpoint)");
      cudaFree(d_slots_);
      d_slots_ = fresh;
      capacity_ = cap;
      td_.slots = fresh;
      td_.mask = cap - 1;
      td_.max_probe = static_cast<int>(std::min<size_t>(cap, 1u << 14));
      cl_.tab = td_;
      ll_.tab = td_;
      if (graph_) cudaGraphExecDestroy(graph_);
      graph_ = nullptr;
      ++growths_;
    }
  }
  Slot* d_in = device_alloc<Slot>(std::max<size_t>(slots.size(), 1), "checkpoint slots");
  Slot* d_saved = nullptr;
  try {
    d_saved = device_alloc<Slot>(cand.size(), "checkpoint candidates");
    if (!slots.empty())
      check(cudaMemcpyAsync(d_in, slots.data(), slots.size() * sizeof(Slot), cudaMemcpyHostToDevice, stream_),
            "slots upload");
    check(cudaMemcpyAsync(d_saved, cand.data(), cand.size() * sizeof(Slot), cudaMemcpyHostToDevice, stream_),
          "candidates upload");
    st.occupancy_limit = limit;  // this table's, not the saved one's
    st.pending = 0;
    check(cudaMemcpyAsync(d_state_, &st, sizeof(IterState), cudaMemcpyHostToDevice, stream_), "state upload");
    check(cudaMemsetAsync(d_err_, 0, sizeof(unsigned), stream_), "memset");
    check(launch_table_fill(d_slots_, capacity_, stream_), "table clear");
    check(cudaMemsetAsync(d_occ_, 0, sizeof(unsigned long long), stream_), "memset");
    compact_reinsert_kernel<<<148 * 8, 256, 0, stream_>>>(td_, d_in, slots.size());
    check(cudaGetLastError(), "reinsert");
    compact_cand_restore_kernel<<<kMaxK, 128, 0, stream_>>>(td_, d_state_, d_saved, d_cand_slot_, opt_.m);
    check(cudaGetLastError(), "candidates restore");
    check(cudaStreamSynchronize(stream_), "synchronize");
  } catch (...) {
    cudaFree(d_in);
    if (d_saved) cudaFree(d_saved);
    throw;
  }
  cudaFree(d_in);
  cudaFree(d_saved);
  zt_ = st.zt;
  iters_enqueued_ = 0;
  occ_iters_[0] = occ_iters_[1] = -1;
  occ_exact_ = slots.size();
  occ_exact_iters_ = 0;
  read_state();
}

void GpuSolver::scalars(dd* xx, dd* scale, dd* xz, long long* iter) {
  read_state();
  *xx = h_state_.xx;
  *scale = h_state_.scale;
  *xz = h_state_.xz;
  *iter = h_state_.iter;
}

int GpuSolver::solve(mcd_report_cb cb, void* user) {
  const bool v = opt_.verbose;
  if (v) {
    std::cout << "CDFCI calculation" << std::endl << "-----------------" << std::endl;
    std::cout << "Hartree Fock determinant occupied spin-orbitals:" << std::endl;
    for (int so : det_spin_orbitals(ref_, ham_.norb)) std::cout << so << "  ";
    std::cout << std::endl;
    std::cout << "Hartree Fock energy: " << std::fixed << std::setprecision(10) << ref_diag_ << std::endl
              << std::endl;
  }
  while (true) {
    reset();
    const auto t0 = std::chrono::steady_clock::now();
    if (v) {
      std::cout << std::setw(13) << std::left << "Iteration";
      std::cout << std::setw(18) << std::right << "Energy";
      std::cout << std::setw(18) << "|dx|_max";
      std::cout << std::setw(12) << "|x|_0";
      std::cout << std::setw(12) << "|z|_0";
      std::cout << std::setw(10) << "|H[I]|_0";
      std::cout << std::setw(10) << "upds";
      std::cout << std::setw(10) << "Time";
      std::cout << std::setw(10) << "scale";
      std::cout << std::endl;
    }
    unsigned long long last_z = 0;
    bool restart = false;
    double energy = 0.0;
    const long long chunks = opt_.num_iterations / opt_.report_interval;
    for (long long c = 0; c < chunks; ++c) {
      run_iterations(opt_.report_interval);
      mcd_report r = report();
      r.time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      energy = r.energy;
      if (v) {
        std::cout << std::setw(13) << std::left << (c + 1) * opt_.report_interval;
        std::cout << std::setw(18) << std::right << std::fixed << std::setprecision(10) << r.energy;
        std::cout << std::setw(18) << std::scientific << std::setprecision(4) << r.dx_max;
        std::cout << std::setw(12) << r.x_size;
        std::cout << std::setw(12) << r.z_size;
        std::cout << std::setw(10) << r.cols_size;
        std::cout << std::setw(10) << r.updates;
        std::cout << std::setw(10) << std::fixed << std::setprecision(2) << r.time_s;
        std::cout << std::setw(10) << std::fixed << std::setprecision(6) << r.scale;
        std::cout << std::endl;
        // The reference's fields (src/solver.h:787-798) with this solver's
        // quantities: iterations solved by shifted inverse iteration, their
        // steps, and the change made by the last refinement step; the
        // updates that fell back to the full reduction are counted after.
        const IterState& S = h_state_;
        const double nit = S.inv_updates > 0 ? static_cast<double>(S.inv_updates) : 1.0;
        std::printf(
            "[LOG] max residual: %e, max eigenvector entry: %e, number of iterations provoking inv iters: %llu, "
            "avg number of inv iters: %.1f, curr number of inv iters: %d, avg diff inv iter makes: %e, curr diff "
            "inv iter makes: %e, max diff inv iter makes: %e, full reductions after a failed shift: %llu.\n",
            r.max_residual, S.max_abs_evec, static_cast<unsigned long long>(S.inv_updates),
            static_cast<double>(S.inv_steps) / nit, S.inv_steps_curr, S.inv_diff_sum / nit, S.inv_diff_curr,
            S.inv_diff_max, static_cast<unsigned long long>(S.eig_fallbacks));
        std::fflush(stdout);
      }
      if (cb && cb(&r, user) != 0) {
        result_energy_ = energy;
        return MCD_STOPPED;
      }
      // z_threshold search (src/solver.h:802-810).
      if (opt_.z_threshold_search) {
        int ncand = 0;
        for (int i = 0; i < h_state_.k_cur; ++i) ncand += h_state_.cand_n[i];
        const double inc = 1000.0 * static_cast<double>(r.z_size - last_z) / std::max(ncand, 1) /
                           static_cast<double>(opt_.report_interval);
        if (inc >= 1.0 && static_cast<double>(r.z_size) > 0.7 * static_cast<double>(max_size_)) {
          restart = true;
          break;
        }
      }
      // Compaction under max_memory: before the table fills, double
      // z_threshold and drop the entries with x = 0 and |z scale| below it.
      if (opt_.compaction && static_cast<double>(r.occupied) > 0.6 * static_cast<double>(h_state_.occupancy_limit)) {
        unsigned long long occ = r.occupied;
        for (int round = 0; round < 30 && static_cast<double>(occ) > 0.4 * static_cast<double>(h_state_.occupancy_limit);
             ++round)
          occ = compact(std::max(2.0 * zt_, 1e-10));
        if (v)
          std::cout << "compaction: z_threshold " << std::scientific << std::setprecision(2) << zt_ << ", |z|_0 "
                    << occ << std::endl;
        r.z_size = occ;
      }
      last_z = r.z_size;
      if (static_cast<double>(r.z_size) > 0.79 * static_cast<double>(max_size_))
        throw McdError(MCD_ERR_OVERFLOW, "The hash table is full. Please increase max_memory or z_threshold.");
    }
    if (restart) {
      zt_ *= 2.0;
      if (v)
        std::cout << "z_threshold_search: z_threshold is too small. Increase z_threhold to " << std::scientific
                  << std::setprecision(2) << zt_ << " and restart." << std::endl;
      continue;
    }
    result_energy_ = energy;
    return MCD_OK;
  }
}

std::vector<std::pair<Det, double>> GpuSolver::column(Det d) {
  const int cap = entries_;
  uint64_t* da = device_alloc<uint64_t>(cap, "debug");
  uint64_t* db = device_alloc<uint64_t>(cap, "debug");
  double* dv = device_alloc<double>(cap, "debug");
  int* dn = device_alloc<int>(1, "debug");
  std::vector<std::pair<Det, double>> out;
  try {
    check(debug_column(hd_, d, diagonal_element(ham_, d), da, db, dv, cap, dn, stream_), "debug column");
    int n = 0;
    check(cudaMemcpyAsync(&n, dn, sizeof(int), cudaMemcpyDeviceToHost, stream_), "copy");
    check(cudaStreamSynchronize(stream_), "sync");
    n = std::min(n, cap);
    std::vector<uint64_t> ha(n), hb(n);
    std::vector<double> hv(n);
    if (n) {
      check(cudaMemcpy(ha.data(), da, n * 8, cudaMemcpyDeviceToHost), "copy");
      check(cudaMemcpy(hb.data(), db, n * 8, cudaMemcpyDeviceToHost), "copy");
      check(cudaMemcpy(hv.data(), dv, n * 8, cudaMemcpyDeviceToHost), "copy");
    }
    for (int i = 0; i < n; ++i) out.push_back({Det{ha[i], hb[i]}, hv[i]});
  } catch (...) {
    cudaFree(da);
    cudaFree(db);
    cudaFree(dv);
    cudaFree(dn);
    throw;
  }
  cudaFree(da);
  cudaFree(db);
  cudaFree(dv);
  cudaFree(dn);
  return out;
}

std::vector<double> GpuSolver::hsub(const std::vector<Det>& dets) {
  const int k = static_cast<int>(dets.size());
  Det* dd_ = device_alloc<Det>(std::max(k, 1), "debug");
  double* dh = device_alloc<double>(std::max(k * k, 1), "debug");
  std::vector<double> out(static_cast<size_t>(k) * k);
  check(cudaMemcpyAsync(dd_, dets.data(), k * sizeof(Det), cudaMemcpyHostToDevice, stream_), "copy");
  check(debug_hsub(hd_, dd_, k, dh, stream_), "debug hsub");
  check(cudaMemcpyAsync(out.data(), dh, out.size() * 8, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "sync");
  cudaFree(dd_);
  cudaFree(dh);
  return out;
}

void GpuSolver::table_sums(dd* xx, dd* xz, unsigned long long* occupied) {
  read_state();
  const int nb = 148 * 4;
  dd* dp = device_alloc<dd>(2 * nb, "debug");
  unsigned long long* dc = device_alloc<unsigned long long>(1, "debug");
  std::vector<dd> hp(2 * nb);
  unsigned long long c = 0;
  check(cudaMemsetAsync(dc, 0, 8, stream_), "memset");
  check(launch_table_sums(d_slots_, capacity_, dp, dc, nb, stream_), "table sums");
  check(cudaMemcpyAsync(hp.data(), dp, hp.size() * sizeof(dd), cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaMemcpyAsync(&c, dc, 8, cudaMemcpyDeviceToHost, stream_), "copy");
  check(cudaStreamSynchronize(stream_), "sync");
  cudaFree(dp);
  cudaFree(dc);
  dd a{0, 0}, b{0, 0};
  for (int i = 0; i < nb; ++i) {
    a = dd_add(a, hp[2 * i]);
    b = dd_add(b, hp[2 * i + 1]);
  }
  *xx = a;
  *xz = b;
  *occupied = c;
}

double GpuSolver::residual() {
  read_state();
  const int nb = 148 * 4;
  dd* dp = device_alloc<dd>(2 * nb, "residual");
  std::vector<dd> hp(2 * nb);
  const dd e = dd_div(h_state_.xz, h_state_.xx);
  table_resid_kernel<<<nb, 256, 0, stream_>>>(d_slots_, capacity_, e, dp);
  cudaError_t err = cudaGetLastError();
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(hp.data(), dp, hp.size() * sizeof(dd), cudaMemcpyDeviceToHost, stream_);
  if (err == cudaSuccess) err = cudaStreamSynchronize(stream_);
  cudaFree(dp);
  check(err, "residual");
  dd rr{0, 0}, xx{0, 0};
  for (int i = 0; i < nb; ++i) {
    rr = dd_add(rr, hp[2 * i]);
    xx = dd_add(xx, hp[2 * i + 1]);
  }
  return std::sqrt(dd_to_d(rr) / dd_to_d(xx));
}

std::vector<unsigned long long> GpuSolver::column_sections(bool enable) {
  std::vector<unsigned long long> v(kColumnSections);
  check(cudaStreamSynchronize(stream_), "sync");
  check(cudaMemcpy(v.data(), d_sect_ + kLeaderSections, v.size() * 8, cudaMemcpyDeviceToHost), "copy");
  check(cudaMemset(d_sect_ + kLeaderSections, 0, v.size() * 8), "memset");
  unsigned long long* want = enable ? d_sect_ + kLeaderSections : nullptr;
  if (cl_.sect != want) {  // the descriptor is recorded in the graph: rebuild it
    cl_.sect = want;
    if (graph_) cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  return v;
}

double GpuSolver::scatter_rate(long long entries, int reps, int ilp, int ctas_per_sm, int mode) {
  if (entries <= 0 || reps <= 0) throw McdError(MCD_ERR_INVALID, "entries and reps must be positive.");
  if (ctas_per_sm < 0 || ctas_per_sm > 8) throw McdError(MCD_ERR_INVALID, "ctas_per_sm must be in 0..8.");
  int sms = 0;
  check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_), "cudaDeviceGetAttribute");
  const int ctas = sms * (ctas_per_sm == 0 ? 8 : ctas_per_sm);
  double* sink = device_alloc<double>(1, "probe");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float ms = 0.0f;
  try {
    check(cudaEventCreate(&e0), "cudaEventCreate");
    check(cudaEventCreate(&e1), "cudaEventCreate");
    check(scatter_probe(td_, entries, ilp, ctas, 0x5eedull, sink, stream_, mode), "scatter probe");
    check(cudaEventRecord(e0, stream_), "cudaEventRecord");
    for (int r = 0; r < reps; ++r)
      check(scatter_probe(td_, entries, ilp, ctas, 0x5eedull + 7919ull * (r + 1), sink, stream_, mode),
            "scatter probe");
    check(cudaEventRecord(e1, stream_), "cudaEventRecord");
    check(cudaEventSynchronize(e1), "cudaEventSynchronize");
    check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
  } catch (...) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  return static_cast<double>(entries) * reps / (static_cast<double>(ms) * 1e-3);
}

std::vector<unsigned long long> GpuSolver::leader_sections() {
  std::vector<unsigned long long> v(kLeaderSections);
  check(cudaStreamSynchronize(stream_), "sync");
  check(cudaMemcpy(v.data(), d_sect_, v.size() * 8, cudaMemcpyDeviceToHost), "copy");
  check(cudaMemset(d_sect_, 0, v.size() * 8), "memset");
  return v;
}

int GpuSolver::last_eig_inputs(double* hsub, double* x, double* z, double xx[2], double xz[2], int cap) {
  read_state();
  const int k = h_state_.k_cur;
  std::vector<double> buf(static_cast<size_t>(kMaxK) * kMaxK + 2 * kMaxK + 4);
  check(cudaMemcpy(buf.data(), d_hsub_, buf.size() * sizeof(double), cudaMemcpyDeviceToHost), "read eig inputs");
  if (k > cap) return k;
  const double* in = buf.data() + static_cast<size_t>(kMaxK) * kMaxK;
  for (int i = 0; i < k * k; ++i) if (hsub) hsub[i] = buf[i];
  for (int i = 0; i < k; ++i) {
    if (x) x[i] = in[i];
    if (z) z[i] = in[kMaxK + i];
  }
  if (xx) { xx[0] = in[2 * kMaxK]; xx[1] = in[2 * kMaxK + 1]; }
  if (xz) { xz[0] = in[2 * kMaxK + 2]; xz[1] = in[2 * kMaxK + 3]; }
  return k;
}

std::vector<std::pair<Det, double>> GpuSolver::picked() {
  read_state();
  std::vector<std::pair<Det, double>> out;
  for (int i = 0; i < h_state_.k_cur; ++i) out.push_back({h_state_.det[i], h_state_.dx[i]});
  return out;
}

}  // namespace mcd
