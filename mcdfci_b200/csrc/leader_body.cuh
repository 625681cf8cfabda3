// Device code of the leader: the serial part of one mCDFCI iteration, run by
// one CTA of 512 threads (leader_body), with its helpers; included by the
// leader kernels (leader_kernel.cu).
//
//   finish iteration t-1   z[D_c] = new_z_c for the picked D_c (the exact
//                          recompute that overwrites the accumulated z,
//                          src/wavefunction.h:557-565); xz += sum_c dot_c
//                          (src/wavefunction.h:583); occupancy check
//                          (src/wavefunction.h:594-599)
//   refetch                (x, z) of every column's candidates from the table
//                          (src/wavefunction.h:567-575)
//   pick                   the k distinct determinants with the largest
//                          |x*xx*scale^2 + z|, ties to the larger determinant
//                          in the reference order (CoordinatePickGcdGrad,
//                          src/solver.h:118-143,196-224)
//   H_sub                  k x k sub-matrix (CDFCI::get_hamiltonian_submatrix,
//                          src/solver.h:637-670): upper triangle from
//                          get_off_diagonal(det_i, det_j) for i < j, diagonal
//                          from get_diagonal (src/hamiltonian.h:252-328)
//   eig update             dx, scale and xx (CoordinateUpdateEig,
//                          src/solver.h:333-609)
//   update_x               x[D_c] += dx_c, xz += z[D_c] * dx_c
//                          (WaveFunctionCuckoo::update_x, src/wavefunction.h:425-451)
//   publish                the k picked determinants, dx, H_cc, xx*scale^2
//                          and scale for the column kernel.
#pragma once

#include "eig.cuh"
#include "device_common.cuh"
#include "kernels.h"

namespace mcd {
namespace {


constexpr int kLT = kEigThreads;  // 512
constexpr int kLW = kLT / 32;     // warps

// ---------------------------------------------------------------------------
// Matrix elements between two determinants.

// Single p->r of spin s summed over the occupied spin-orbitals of (a, b) in
// interleaved order.
__device__ double single_value_det(const HamDev& h, int s, int p, int r, uint64_t a, uint64_t b) {
  const int n = h.norb;
  const size_t base = (static_cast<size_t>(s) * n + p) * n + r;
  const double* st = h.st + base * h.nso;
  double v = h.sh[base];
  uint64_t u = a | b;
  while (u) {
    const int q = __ffsll(static_cast<long long>(u)) - 1;
    u &= u - 1;
    if ((a >> q) & 1ull) v += st[2 * q];
    if ((b >> q) & 1ull) v += st[2 * q + 1];
  }
  return v;
}

__device__ __forceinline__ int lowest_bit(uint64_t x) { return __ffsll(static_cast<long long>(x)) - 1; }

// <d2|H|d1> computed from d1's side, as HamiltonianMolecule::get_off_diagonal(d1, d2).
__device__ double off_diagonal(const HamDev& h, Det d1, Det d2) {
  const uint64_t da = d1.a ^ d2.a, db = d1.b ^ d2.b;
  const int na = __popcll(da), nb = __popcll(db);
  const int n = h.norb;
  if (na + nb == 2) {
    if (na == 2) {
      const int p = lowest_bit(da & d1.a), r = lowest_bit(da & d2.a);
      if (!((h.spres[p] >> r) & 1ull)) return 0.0;
      double v = single_value_det(h, 0, p, r, d1.a, d1.b);
      return sign_alpha(d1.a, d1.b, p, r) ? -v : v;
    }
    if (nb == 2) {
      const int p = lowest_bit(db & d1.b), r = lowest_bit(db & d2.b);
      if (!((h.spres[n + p] >> r) & 1ull)) return 0.0;
      double v = single_value_det(h, 1, p, r, d1.a, d1.b);
      return sign_beta(d1.a, d1.b, p, r) ? -v : v;
    }
    return 0.0;
  }
  if (na + nb == 4) {
    const size_t np = static_cast<size_t>(h.npair);
    if (na == 4) {
      uint64_t o = da & d1.a, v = da & d2.a;
      const int p = lowest_bit(o);
      o &= o - 1;
      const int q = lowest_bit(o);
      const int r = lowest_bit(v);
      v &= v - 1;
      const int s = lowest_bit(v);
      const double val = h.vss[static_cast<size_t>(pair_index(p, q)) * np + pair_index(r, s)];
      return sign_aa(d1.a, d1.b, p, q, r, s) ? -val : val;
    }
    if (nb == 4) {
      uint64_t o = db & d1.b, v = db & d2.b;
      const int p = lowest_bit(o);
      o &= o - 1;
      const int q = lowest_bit(o);
      const int r = lowest_bit(v);
      v &= v - 1;
      const int s = lowest_bit(v);
      const double val = h.vss[(np + pair_index(p, q)) * np + pair_index(r, s)];
      return sign_bb(d1.a, d1.b, p, q, r, s) ? -val : val;
    }
    if (na == 2 && nb == 2) {
      const int pa = lowest_bit(da & d1.a), ra = lowest_bit(da & d2.a);
      const int pb = lowest_bit(db & d1.b), sb = lowest_bit(db & d2.b);
      const double val = h.wab[((static_cast<size_t>(pa) * n + pb) * n + ra) * n + sb];
      return sign_ab(d1.a, d1.b, pa, ra, pb, sb) ? -val : val;
    }
  }
  return 0.0;
}

// Diagonal element by one warp (lane-partial sums, fixed reduction order).
// occ: 128-byte per-warp scratch.
__device__ double diagonal_warp(const HamDev& h, Det d, unsigned char* occ) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = lanemask_lt();
  int nocc = 0;
  for (int j = 0; j < 4; ++j) {
    const int s = lane + 32 * j;
    const int p = s >> 1;
    const bool o = p < h.norb && ((((s & 1) ? d.b : d.a) >> p) & 1ull);
    const unsigned m = __ballot_sync(~0u, o);
    if (o) occ[nocc + __popc(m & lt)] = static_cast<unsigned char>(s);
    nocc += __popc(m);
  }
  __syncwarp();
  // <i|h|i> over the occupied i and <ij||ij> over the occupied pairs i < j,
  // the (i, j) terms spread over the lanes (independent loads).
  double v = 0.0;
  for (int x = lane; x < nocc; x += 32) v += h.hdiag[occ[x]];
  const int nn = nocc * nocc;
#pragma unroll 4
  for (int t = lane; t < nn; t += 32) {
    const int x = t / nocc, y = t - x * nocc;
    if (y > x) v += h.d2[static_cast<size_t>(occ[x]) * h.nso + occ[y]];
  }
  v = warp_sum(v);
  __syncwarp();
  return __shfl_sync(~0u, v, 0) + h.ecore;
}

// ---------------------------------------------------------------------------
// Eig update.  Inputs x[k], z[k] in shared memory; H (row-major k x k,
// symmetric: dsyevr with UPLO='L' on the row-major array reads its upper
// triangle, and callers fill the lower one from it) in shared or global
// memory; `work` is shared scratch of eig_work_doubles(k) doubles.  Outputs
// dx[k] (shared), new xx and scale.

struct EigResult {
  dd xx, scale;
  int branch;
  bool ok;
  double resid;
  double lambda;     // the eigenvalue (Rayleigh quotient of the vector)
  double max_evec;   // max |v_i| over i >= 1 (branch 1) or i >= 0 (branch 2)
  int shift_steps;   // steps of the shifted solver, 0 when the reduction ran
  double shift_diff; // change made by its last refinement step
  bool fallback;     // the shifted solver was tried and the reduction ran instead
};

constexpr int kEigVecs = 18;

// Shared scratch of eig_update: B (lda), 18 vectors, and for k + 1 <=
// kShiftMaxN the explicit inverse of the shifted solver's Cholesky factor
// and the inverse of B - sigma I formed from it.
__host__ __device__ constexpr size_t eig_work_doubles(int k) {
  return static_cast<size_t>(k + 1) * eig_lda(k + 1) + kEigVecs * static_cast<size_t>(k + 1) +
         (k + 1 <= kShiftMaxN ? 2 * static_cast<size_t>(k + 1) * eig_lda(k + 1) : 0) + 64;
}

// drop: the last update's energy drop E - lambda (0 = unknown).  When it is
// known and B has at most kShiftMaxN rows, the shifted solver runs first with
// sigma = E - max(16 drop, 1e-9 (1 + |E|)) below the current energy E = xz/xx
// (an upper bound of lambda_1: the current vector lies in the subspace, and
// its Rayleigh quotient there is xz/xx) and the current vector as the start;
// the reduction runs when that fails or its residual is not below 1e-11
// (1 + |lambda|).  method 2: the bordered fixed point (eig_lowest_bordered)
// runs first for k <= kBorderMaxK, the reduction when it does not certify its
// result or the residual check fails.  The first iteration's problem (branch
// 2, no bordering row) always takes the reduction.
__device__ EigResult eig_update(const double* H, int k, const double* x, const double* z, dd xx, dd xz,
                                double* dx, double* work, SectionClock& clk, double drop, int method) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ double s_b00, s_y1, s_res;
  __shared__ dd s_sum3[3];
  __shared__ double s_sgn;
  __shared__ int s_branch;
  __shared__ dd s_rq;
  EigResult res;
  res.shift_steps = 0;
  res.shift_diff = 0.0;
  res.fallback = false;

  // B = [[b00, b'], [b, H]] in A (leading dimension lda); H's block at (1, 1)
  // also serves the first-iteration k x k problem.
  const int lda = eig_lda(k + 1);
  double* A = work;
  double* vec = work + static_cast<size_t>(k + 1) * lda;
  const int vs = k + 1;
  EigVecs V;
  V.d = vec;
  V.e = vec + vs;
  V.e2 = vec + 2 * vs;
  V.u0 = vec + 3 * vs;
  V.tau = vec + 4 * vs;
  V.num = vec + 5 * vs;
  V.den = vec + 6 * vs;
  V.ru = vec + 7 * vs;
  V.l = vec + 8 * vs;
  V.y = vec + 9 * vs;
  V.c = vec + 10 * vs;
  V.g = vec + 11 * vs;
  double* Hx = vec + 12 * vs;    // [k]
  double* bvec = vec + 13 * vs;  // [k+1] first row of B (branch 1)
  double* Bv = vec + 14 * vs;
  double* vhi = vec + 15 * vs;   // normalised eigenvector, hi part
  double* vlo = vec + 16 * vs;   // lo part

  double* Li = vec + kEigVecs * vs;   // [(k+1) x lda] when k + 1 <= kShiftMaxN
  double* Ci = Li + vs * lda;          // [(k+1) x lda] likewise
  auto fill_h = [&]() {
    for (int idx = tid; idx < k * k; idx += blockDim.x) {
      const int i = idx / k, j = idx - i * k;
      if (i <= j) {
        const double v = H[idx];
        A[(i + 1) * lda + (j + 1)] = v;
        A[(j + 1) * lda + (i + 1)] = v;
      }
    }
  };
  fill_h();
  __syncthreads();
  clk.mark(21);
  // H x in double (dsymv, src/solver.h:355); x'x, x'z, x'Hx in double-double,
  // rounded where the reference works in double.
  for (int r = warp; r < k; r += kLW) {
    const double* row = A + (r + 1) * lda + 1;
    double s = 0.0;
    for (int c = lane; c < k; c += 32) s = fma(row[c], x[c], s);
    s = warp_sum(s);
    if (lane == 0) Hx[r] = s;
  }
  __syncthreads();
  clk.mark(22);
  if (warp == 0) {
    dd sxx{0, 0}, sxz{0, 0}, sxhx{0, 0};
    for (int i = lane; i < k; i += 32) {
      sxx = dd_add(sxx, dd_two_prod(x[i], x[i]));
      sxz = dd_add(sxz, dd_two_prod(x[i], z[i]));
      sxhx = dd_add(sxhx, dd_two_prod(x[i], Hx[i]));
    }
    sxx = warp_sum_dd(sxx);
    sxz = warp_sum_dd(sxz);
    sxhx = warp_sum_dd(sxhx);
    if (lane == 0) {
      const double xTx = dd_to_d(sxx), xTz = dd_to_d(sxz), xTHx = dd_to_d(sxhx);
      const double yy = dd_to_d(dd_add_d(xx, -xTx));
      s_branch = fabs(yy) > 1e-14 ? 1 : 2;
      if (s_branch == 1) {
        const double y1 = sqrt(yy);
        dd num = dd_add_d(dd_add_d(xz, -2.0 * xTz), xTHx);
        s_b00 = dd_to_d(dd_div_d(num, yy));
        s_y1 = y1;
      }
    }
  }
  __syncthreads();
  clk.mark(23);
  const int branch = s_branch;
  const int n = branch == 1 ? k + 1 : k;
  const double y1 = s_y1;
  if (branch == 1) {
    // b = (z - Hx) / y1 (src/solver.h:378-383).
    for (int i = tid; i <= k; i += blockDim.x) {
      const double v = i == 0 ? s_b00 : (z[i - 1] - Hx[i - 1]) / y1;
      A[i] = v;
      A[i * lda] = v;
      bvec[i] = v;
    }
  }
  __syncthreads();
  clk.mark(9);

  double* Ae = branch == 1 ? A : A + lda + 1;
  bool shifted = false;
  if (branch == 1 && n <= kShiftMaxN && drop > 0.0) {
    const double e_cur = dd_to_d(dd_div(xz, xx));
    const double delta = fmax(16.0 * drop, 1e-9 * (1.0 + fabs(e_cur)));
    for (int i = tid; i < n; i += blockDim.x) V.y[i] = i == 0 ? y1 : x[i - 1];
    __syncthreads();
    int steps = 0;
    double diff = 0.0;
    shifted = eig_lowest_shifted_warp(A, lda, n, V, e_cur - delta, Li, Ci, &steps, &diff, clk);
    res.shift_steps = shifted ? steps : 0;
    res.shift_diff = shifted ? diff : 0.0;
    if (!shifted) {
      res.fallback = true;
      fill_h();
      for (int i = tid; i <= k; i += blockDim.x) {
        A[i] = bvec[i];
        A[i * lda] = bvec[i];
      }
      __syncthreads();
    }
  }
  bool bordered = false;
  if (!shifted && method == 2 && branch == 1 && k <= kBorderMaxK) {
    int iters = 0;
    double rn = 0.0;
    bordered = eig_lowest_bordered(A, lda, n, V, Li, &iters, &rn, clk);  // Li and Ci as its scratch
    res.shift_steps = bordered ? iters : 0;
    res.shift_diff = rn;
    res.fallback = !bordered;
  }
  clk.mark(16);
  if (!shifted && !bordered) eig_lowest(Ae, lda, n, V, clk);
  clk.mark(13);
  shifted = shifted || bordered;  // a fast solve, checked below

  for (int attempt = 0; attempt < 2; ++attempt) {
  // B v in double, one row per warp (H is symmetric, so its rows are read).
  const double* y = V.y;
  for (int r = warp; r < n; r += kLW) {
    double s = 0.0;
    if (branch == 1) {
      const double* hr = H + (r - 1) * k - 1;  // hr[c] = H[r-1][c-1]
      for (int c = lane; c < n; c += 32) {
        const double brc = (r == 0) ? bvec[c] : (c == 0 ? bvec[r] : hr[c]);
        s = fma(brc, y[c], s);
      }
    } else {
      const double* hr = H + r * k;
      for (int c = lane; c < n; c += 32) s = fma(hr[c], y[c], s);
    }
    s = warp_sum(s);
    if (lane == 0) Bv[r] = s;
  }
  __syncthreads();
  clk.mark(24);
  // Rayleigh quotient y'By / y'y, normalisation in double-double, sign fix,
  // residual ||B v - lambda v||: y'y on warp 0, y'Bv on warp 1 and, for the
  // first iteration's sign, y'x on warp 2; then warp 0 normalises while warp 1
  // forms the quotient and the residual.
  if (warp < 3) {
    dd acc{0, 0};
    double sgn = 0.0;
    for (int i = lane; i < n; i += 32) {
      if (warp == 2)
        sgn = branch == 2 ? fma(y[i], x[i], sgn) : 0.0;
      else
        acc = dd_add(acc, dd_two_prod(y[i], warp == 0 ? y[i] : Bv[i]));
    }
    if (warp == 2) {
      sgn = warp_sum(sgn);
      if (lane == 0) s_sgn = sgn;
    } else {
      acc = warp_sum_dd(acc);
      if (lane == 0) s_sum3[warp] = acc;
    }
  }
  __syncthreads();
  if (warp == 0) {
    const dd nrm = s_sum3[0];
    const double flip = (branch == 1) ? (y[0] < 0.0 ? -1.0 : 1.0) : (s_sgn < 0.0 ? -1.0 : 1.0);
    const dd inv = dd_div(dd{flip, 0.0}, dd_sqrt(nrm));
    for (int i = lane; i < n; i += 32) {
      const dd vi = dd_mul_d(inv, y[i]);
      vhi[i] = vi.hi;
      vlo[i] = vi.lo;
    }
  } else if (warp == 1) {
    const dd nrm = s_sum3[0];
    const dd rq = dd_div(s_sum3[1], nrm);
    const double lam = dd_to_d(rq);
    double acc = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double t = fma(-lam, y[i], Bv[i]);
      acc = fma(t, t, acc);
    }
    acc = warp_sum(acc);
    if (lane == 0) {
      s_rq = rq;
      s_res = sqrt(acc / dd_to_d(nrm));
    }
  }
  __syncthreads();
  // A shifted solve whose residual is not small runs the reduction instead.
  if (!shifted || s_res <= 1e-11 * (1.0 + fabs(dd_to_d(s_rq)))) break;
  shifted = false;
  res.shift_steps = 0;
  res.shift_diff = 0.0;
  res.fallback = true;
  fill_h();
  for (int i = tid; i <= k; i += blockDim.x) {
    A[i] = bvec[i];
    A[i * lda] = bvec[i];
  }
  __syncthreads();
  eig_lowest(Ae, lda, n, V, clk);
  }
  clk.mark(14);
  const dd rq = s_rq;
  const double lam = dd_to_d(rq);
  res.resid = s_res;
  res.branch = branch;
  res.ok = true;
  res.lambda = lam;
  {
    double mv = 0.0;
    if (warp == 0)
      for (int i = lane + (branch == 1 ? 1 : 0); i < n; i += 32) mv = fmax(mv, fabs(vhi[i]));
    for (int o = 16; o > 0; o >>= 1) mv = fmax(mv, __shfl_xor_sync(~0u, mv, o));
    res.max_evec = mv;  // warp 0's value; thread 0 publishes it
  }

  if (branch == 1) {
    // lambda_q = -rq, gamma = v0 / y1, scale = gamma sqrt(lambda_q),
    // xx = lambda_q / scale^2, dx_i = v_{i+1} / gamma - x_i (src/solver.h:516-538).
    const dd lq = dd_neg(rq);
    const dd v0{vhi[0], vlo[0]};
    const dd gamma = dd_div_d(v0, y1);
    res.ok = lq.hi > 0.0 && gamma.hi != 0.0 && isfinite(lq.hi) && isfinite(gamma.hi);
    const dd sc = dd_mul(gamma, dd_sqrt(lq));
    res.scale = sc;
    res.xx = dd_div(lq, dd_mul(sc, sc));
    for (int i = tid; i < k; i += blockDim.x) {
      const dd q = dd_div(dd{vhi[i + 1], vlo[i + 1]}, gamma);
      dx[i] = dd_to_d(dd_add_d(q, -x[i]));
    }
  } else {
    // First iteration: xx = -lambda, scale = 1, dx = v sqrt(-lambda) - x (src/solver.h:552-598).
    res.ok = lam < 0.0 && isfinite(lam);
    const double sq = sqrt(-lam);
    res.xx = dd{-lam, 0.0};
    res.scale = dd{1.0, 0.0};
    for (int i = tid; i < k; i += blockDim.x) dx[i] = (vhi[i] + vlo[i]) * sq - x[i];
  }
  __syncthreads();
  for (int i = tid; i < k; i += blockDim.x)
    if (!isfinite(dx[i])) res.ok = false;
  res.ok = __syncthreads_and(res.ok ? 1 : 0) != 0;
  return res;
}

// ---------------------------------------------------------------------------
// End of iteration t (src/wavefunction.h:557-565,583): z[D_c] = new_z_c for
// the picked determinants, then xz += sum_c dot_c.  Block-wide, on a state
// copy `S` (shared or global); table stores go to global memory.
__device__ void finish_iteration(IterState* S, const TableDev& T) {
  if (!S->pending) return;
  const int k = S->k_cur;
  if (static_cast<int>(threadIdx.x) < k) {
    Slot* sp = T.slots + S->slot[threadIdx.x];
    sp->z = S->newz[threadIdx.x];
  }
  __syncthreads();  // orders the stores for this CTA; the next launch sees them anyway
  if (threadIdx.x < 32) {
    dd acc{0.0, 0.0};
    for (int c = threadIdx.x; c < k; c += 32) acc = dd_add_d(acc, S->dot[c]);
    acc = warp_sum_dd(acc);
    if (threadIdx.x == 0) {
      S->xz = dd_add(S->xz, acc);
      S->pending = 0;
    }
  }
  __syncthreads();
}

__global__ void finish_kernel(LeaderLaunch L) { finish_iteration(L.st, L.tab); }

__device__ __forceinline__ unsigned hash32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Block-wide exclusive position of a kept element within one chunk of
// blockDim.x elements; returns the chunk's kept count through *chunk_total.
__device__ __forceinline__ int block_rank(bool keep, int* wsum, int* chunk_total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned b = __ballot_sync(~0u, keep);
  if (lane == 0) wsum[warp] = __popc(b);
  __syncthreads();
  if (warp == 0) {
    const int v = lane < static_cast<int>(blockDim.x >> 5) ? wsum[lane] : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(~0u, incl, o);
      if (lane >= o) incl += t;
    }
    wsum[lane] = incl - v;  // exclusive
    if (lane == 31) wsum[32] = incl;
  }
  __syncthreads();
  const int pos = wsum[warp] + __popc(b & lanemask_lt());
  *chunk_total = wsum[32];
  __syncthreads();
  return pos;
}

constexpr unsigned kNoSlot = 0xFFFFFFFFu;

// The k best (score, slot) pairs among n candidates (us, sc in shared
// memory) by radix selection on the 64-bit keys bits(score) + 1: scores are
// +0 or positive, so their bit patterns order like their values.  Eight-bit
// digits from the top, one 256-bin shared histogram per pass (warp-aggregated
// counts: the leading digits of nearby scores coincide), until the bin that
// holds the k-th largest key holds exactly the keys still to choose.  The
// chosen keys are then ranked among themselves, in decreasing score and equal
// scores in the reference's determinant order (detComp_global,
// src/wavefunction.h:30-36), and their slots written to out[0..k) in that
// order.  Returns false, writing nothing, when the k-th and (k+1)-th keys are
// equal, so that the caller can choose the set by determinant order.
__device__ bool topk_radix(const unsigned* us, const double* sc, int n, int k, const Slot* slots, int nwords,
                           unsigned* out) {
  __shared__ unsigned s_hist[256];
  __shared__ unsigned long long s_sel_key[kMaxK];
  __shared__ unsigned s_sel_slot[kMaxK];
  __shared__ unsigned long long s_prefix;
  __shared__ unsigned s_need;
  __shared__ int s_state, s_count;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid < 256) s_hist[tid] = 0u;
  if (tid == 0) {
    s_need = static_cast<unsigned>(k);
    s_count = 0;
    s_state = 0;
    s_prefix = 0ull;
  }
  __syncthreads();
  unsigned long long prefix = 0ull;  // the digits chosen so far, lower bits 0
  int state = 0;                     // 0 more digits, 1 set found, 2 tie at the k-th key
  for (int pass = 0; pass < 8 && state == 0; ++pass) {
    const int shift = 56 - 8 * pass;
    const unsigned long long himask = pass == 0 ? 0ull : (~0ull << (shift + 8));
    for (int base = warp * 32; base < n; base += blockDim.x) {
      const int u = base + lane;
      const unsigned long long key =
          u < n ? static_cast<unsigned long long>(__double_as_longlong(sc[u])) + 1ull : 0ull;
      const bool match = u < n && ((key ^ prefix) & himask) == 0ull;
      const unsigned act = __ballot_sync(~0u, match);
      if (match) {
        const unsigned d = static_cast<unsigned>(key >> shift) & 255u;
        const unsigned peers = __match_any_sync(act, d);
        if (lane == __ffs(peers) - 1) atomicAdd(&s_hist[d], static_cast<unsigned>(__popc(peers)));
      }
    }
    __syncthreads();
    if (warp == 0) {
      // Lane l holds bins 255-8l .. 248-8l, in decreasing order.
      const unsigned need = s_need;
      unsigned c[8], t = 0u;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        c[j] = s_hist[255 - 8 * lane - j];
        s_hist[255 - 8 * lane - j] = 0u;
        t += c[j];
      }
      unsigned incl = t;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned v = __shfl_up_sync(~0u, incl, o);
        if (lane >= o) incl += v;
      }
      unsigned run = incl - t;  // keys in higher bins
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        if (run < need && run + c[j] >= need) {
          const unsigned long long d = static_cast<unsigned long long>(255 - 8 * lane - j);
          s_prefix = prefix | (d << shift);
          s_need = need - run;
          s_state = (c[j] == need - run) ? 1 : (pass == 7 ? 2 : 0);
        }
        run += c[j];
      }
    }
    __syncthreads();
    prefix = s_prefix;
    state = s_state;
  }
  if (state != 1) return false;
  // The chosen keys are those >= prefix: exactly k of them.
  for (int base = warp * 32; base < n; base += blockDim.x) {
    const int u = base + lane;
    const unsigned long long key =
        u < n ? static_cast<unsigned long long>(__double_as_longlong(sc[u])) + 1ull : 0ull;
    const bool keep = u < n && key >= prefix;
    const unsigned b = __ballot_sync(~0u, keep);
    if (b == 0u) continue;
    int pos = 0;
    if (lane == 0) pos = atomicAdd(&s_count, __popc(b));
    pos = __shfl_sync(~0u, pos, 0) + __popc(b & lanemask_lt());
    if (keep) {
      s_sel_key[pos] = key;
      s_sel_slot[pos] = us[u];
    }
  }
  __syncthreads();
  if (tid < k) {
    const unsigned long long mine = s_sel_key[tid];
    const unsigned slot = s_sel_slot[tid];
    int rank = 0;
    bool equal = false;
    for (int j = 0; j < k; ++j) {
      const unsigned long long o = s_sel_key[j];
      rank += o > mine;
      equal |= (o == mine) && j != tid;
    }
    if (equal) {  // equal scores: the reference's determinant order
      uint64_t ia, ib;
      load_key(slots + slot, ia, ib);
      for (int j = 0; j < k; ++j) {
        if (j == tid || s_sel_key[j] != mine) continue;
        uint64_t ja, jb;
        load_key(slots + s_sel_slot[j], ja, jb);
        rank += det_ref_compare(ja, jb, ia, ib, nwords) > 0;
      }
    }
    out[rank] = slot;
  }
  __syncthreads();
  return true;
}


__device__ __forceinline__ void leader_body(const LeaderLaunch& L) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ __align__(16) IterState sS;
  __shared__ int s_off[kMaxK + 1];
  __shared__ int s_wsum[33];
  __shared__ int s_R, s_U;
  __shared__ unsigned s_err;
  __shared__ unsigned s_slot[kMaxK];
  __shared__ Det s_det[kMaxK];
  __shared__ double s_x[kMaxK], s_z[kMaxK], s_dx[kMaxK];
  __shared__ unsigned char s_occ[kLW][128];
  __shared__ unsigned long long s_newx;

  IterState* G = L.st;
  const TableDev& T = L.tab;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int m = L.m;
  SectionClock clk{L.sect, 0};
  clk.start();

  // 0. Iteration state into shared memory.
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(G);
    unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sS);
    for (int i = tid; i < static_cast<int>(sizeof(IterState) / 8); i += kLT) dst[i] = src[i];
  }
  if (tid == 0) {
    s_err = *reinterpret_cast<volatile unsigned*>(T.err);
    if (*T.n_occupied > L.st->occupancy_limit) {
      atomicOr(T.err, kErrOverflow);
      s_err |= kErrOverflow;
    }
    s_newx = 0;
  }
  __syncthreads();
  clk.mark(0);

  // 1. Finish the previous iteration (unless finish_kernel already did).
  const int kprev = sS.k_cur;
  finish_iteration(&sS, T);
  if (warp == 0) {
    int run = 0;
    for (int base = 0; base < kMaxK; base += 32) {
      const int cc = (base + lane < kprev) ? sS.cand_n[base + lane] : 0;
      int incl = cc;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(~0u, incl, o);
        if (lane >= o) incl += t;
      }
      s_off[base + lane] = run + incl - cc;
      run += __shfl_sync(~0u, incl, 31);
    }
    if (lane == 0) {
      s_off[kMaxK] = run;
      s_R = run;
    }
  }
  __syncthreads();
  clk.mark(1);
  if (s_err != 0u || s_R == 0) {
    if (tid == 0) {
      if (s_R == 0 && s_err == 0u) atomicOr(T.err, kErrCandidates);
      G->xz = sS.xz;
      G->pending = 0;
      G->k_cur = 0;
    }
    return;
  }

  // 2-3. Candidate slots, with duplicates (one determinant in several
  //      columns) removed through a shared-memory hash set, and their scores
  //      |x*xx*scale^2 + z| refetched from the table.
  const int R = s_R;
  int PR = 2;  // >= 2 keeps the score array (which reuses the hash set) 8-byte aligned
  while (PR < R) PR <<= 1;
  unsigned* us = reinterpret_cast<unsigned*>(smem);  // [PR] slots, compacted in place
  unsigned* hs = us + PR;                             // [2*PR] hash set; then scores (double[PR])
  double* sc = reinterpret_cast<double*>(hs);
  const int H = 2 * PR;
  const dd xss = sS.xss;
  auto slot_of = [&](int r) {  // candidate r: s_off[lo] <= r < s_off[lo+1]
    int lo = 0, hi = kprev;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (s_off[mid] <= r) lo = mid; else hi = mid;
    }
    return L.cand_slot[lo * m + (r - s_off[lo])];
  };
  auto score_at = [&](unsigned slot) {
    const Slot* sp = T.slots + slot;
    const double x = load_relaxed(&sp->x), z = load_relaxed(&sp->z);
    const double g = score_of(x, z, xss);
    return (g >= 0.0) ? g : 0.0;  // a non-finite gradient must not reorder the padding
  };
  auto hash_keep = [&](unsigned s) {  // true for the first copy of slot s
    unsigned h = hash32(s) & static_cast<unsigned>(H - 1);
    for (int probe = 0; probe < H; ++probe) {
      const unsigned old = atomicCAS(&hs[h], kNoSlot, s);
      if (old == kNoSlot) return true;
      if (old == s) return false;
      h = (h + 1) & static_cast<unsigned>(H - 1);
    }
    return false;
  };
  // With at most two candidates per thread (the usual case), each thread
  // fetches its candidates' slots and scores in one go, before the duplicate
  // removal, and the scores are written once the hash set is done with.
  auto gather = [&]() {
    for (int i = tid; i < H; i += kLT) hs[i] = kNoSlot;
    int total = 0;
    if (R <= 2 * kLT) {
      const int r0 = tid, r1 = kLT + tid;
      const unsigned s0 = r0 < R ? slot_of(r0) : kNoSlot;
      const unsigned s1 = r1 < R ? slot_of(r1) : kNoSlot;
      // The candidates' (x, z) loads are issued here and consumed after the
      // duplicate removal, which needs only the slots, so that their latency
      // overlaps it.
      double x0 = 0.0, z0 = 0.0, x1 = 0.0, z1 = 0.0;
      if (r0 < R) {
        x0 = load_relaxed(&T.slots[s0].x);
        z0 = load_relaxed(&T.slots[s0].z);
      }
      if (r1 < R) {
        x1 = load_relaxed(&T.slots[s1].x);
        z1 = load_relaxed(&T.slots[s1].z);
      }
      __syncthreads();
      int p0 = -1, p1 = -1, chunk = 0;
      bool keep = r0 < R && hash_keep(s0);
      int pos = block_rank(keep, s_wsum, &chunk);
      if (keep) {
        us[pos] = s0;
        p0 = pos;
      }
      total = chunk;
      __syncthreads();
      if (R > kLT) {
        keep = r1 < R && hash_keep(s1);
        pos = block_rank(keep, s_wsum, &chunk);
        if (keep) {
          us[total + pos] = s1;
          p1 = total + pos;
        }
        total += chunk;
        __syncthreads();
      }
      // The hash set (which sc overlays) is no longer read.
      auto score_xz = [&](double x, double z) {
        const double g = score_of(x, z, xss);
        return (g >= 0.0) ? g : 0.0;  // as score_at
      };
      if (p0 >= 0) sc[p0] = score_xz(x0, z0);
      if (p1 >= 0) sc[p1] = score_xz(x1, z1);
    } else {
      for (int r = tid; r < R; r += kLT) us[r] = slot_of(r);
      __syncthreads();
      for (int base = 0; base < R; base += kLT) {
        const int r = base + tid;
        const unsigned s = r < R ? us[r] : kNoSlot;
        const bool keep = r < R && hash_keep(s);
        int chunk = 0;
        const int pos = block_rank(keep, s_wsum, &chunk);
        if (keep) us[total + pos] = s;
        total += chunk;
        __syncthreads();
      }
      for (int u = tid; u < total; u += kLT) sc[u] = score_at(us[u]);
    }
    if (tid == 0) s_U = total;
    int Pl = 1;
    while (Pl < total) Pl <<= 1;
    for (int u = total + tid; u < Pl; u += kLT) {
      sc[u] = -1.0;
      us[u] = kNoSlot;
    }
    __syncthreads();
  };
  gather();
  clk.mark(2);
  const int U = s_U;
  const int k = U < L.k_req ? U : L.k_req;

  // 4. The k largest scores, by radix selection over the candidates.  Equal
  //    scores are ordered by the reference's determinant order
  //    (detComp_global, src/wavefunction.h:30-36); when the k-th and (k+1)-th
  //    scores are equal that order decides the set, and the whole candidate
  //    list is sorted instead (rare).
  const bool fast = topk_radix(us, sc, U, k, T.slots, sS.n_words, s_slot);
  clk.mark(3);
  if (!fast) {
    gather();
    int P = 1;
    while (P < U) P <<= 1;
    const int nwords = sS.n_words;
    for (int size = 2; size <= P; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int t = tid; t < (P >> 1); t += kLT) {
          const int i = 2 * stride * (t / stride) + (t % stride);
          const int j = i + stride;
          const double si = sc[i], sj = sc[j];
          bool jfirst;
          if (si != sj) {
            jfirst = sj > si;
          } else {
            const unsigned a = us[i], b = us[j];
            if (a == kNoSlot || b == kNoSlot || a == b) {
              jfirst = false;
            } else {
              uint64_t ia, ib, ja, jb;
              load_key(T.slots + a, ia, ib);
              load_key(T.slots + b, ja, jb);
              jfirst = det_ref_compare(ja, jb, ia, ib, nwords) > 0;
            }
          }
          const bool up = (i & size) == 0;
          if (jfirst == up) {
            sc[i] = sj;
            sc[j] = si;
            const unsigned tmp = us[i];
            us[i] = us[j];
            us[j] = tmp;
          }
        }
        __syncthreads();
      }
    }
    if (tid < k) s_slot[tid] = us[tid];
    __syncthreads();
  }
  clk.mark(4);
  if (tid < k) {
    const Slot* sp = T.slots + s_slot[tid];
    uint64_t a, b;
    load_key(sp, a, b);
    s_det[tid] = Det{a, b};
    s_x[tid] = load_relaxed(&sp->x);
    s_z[tid] = load_relaxed(&sp->z);
  }
  __syncthreads();
  clk.mark(5);

  // 5. H_sub: in shared memory when it fits beside the eig scratch, else in
  //    the global copy (which is written either way for inspection).
  const bool h_in_smem = k <= 64;
  double* Hs = h_in_smem ? reinterpret_cast<double*>(smem) : L.hsub_out;
  double* work = h_in_smem ? Hs + k * k : reinterpret_cast<double*>(smem);
  // One thread per pair i < j (pair t = j(j-1)/2 + i).
  for (int t = tid; t < k * (k - 1) / 2; t += kLT) {
    int j = static_cast<int>((1.0f + sqrtf(1.0f + 8.0f * static_cast<float>(t))) * 0.5f);
    while (j * (j - 1) / 2 > t) --j;
    while (j * (j + 1) / 2 <= t) ++j;
    const int i = t - j * (j - 1) / 2;
    const double v = off_diagonal(L.ham, s_det[i], s_det[j]);
    Hs[i * k + j] = v;
    Hs[j * k + i] = v;
  }
  for (int i = warp; i < k; i += kLW) {
    const double v = diagonal_warp(L.ham, s_det[i], s_occ[warp]);
    if (lane == 0) Hs[i * k + i] = v;
  }
  __threadfence_block();
  __syncthreads();
  clk.mark(6);
  if (h_in_smem)
    for (int t = tid; t < k * k; t += kLT) L.hsub_out[t] = Hs[t];
  {
    double* in = L.hsub_out + kMaxK * kMaxK;
    if (tid < k) {
      in[tid] = s_x[tid];
      in[kMaxK + tid] = s_z[tid];
    }
    if (tid == 0) {
      in[2 * kMaxK] = sS.xx.hi;
      in[2 * kMaxK + 1] = sS.xx.lo;
      in[2 * kMaxK + 2] = sS.xz.hi;
      in[2 * kMaxK + 3] = sS.xz.lo;
    }
  }

  // 6. Eig update.
  const EigResult er =
      eig_update(Hs, k, s_x, s_z, sS.xx, sS.xz, s_dx, work, clk, L.eig_method == 1 ? sS.eig_drop : 0.0, L.eig_method);
  clk.mark(15);
  if (!er.ok) {
    if (tid == 0) {
      atomicOr(T.err, kErrEig);
      G->xz = sS.xz;
      G->pending = 0;
      G->k_cur = 0;
    }
    return;
  }

  // 7. update_x: x[D_i] += dx_i; xz += z_i dx_i; x_size counts dets whose x was 0.
  if (tid < k) {
    Slot* sp = T.slots + s_slot[tid];
    const double x0 = s_x[tid];
    sp->x = x0 + s_dx[tid];
    if (x0 == 0.0) atomicAdd(&s_newx, 1ull);
  }
  __syncthreads();
  clk.mark(7);

  // 8. Publish the next iteration.
  dd zdx{0.0, 0.0};
  double mx = 0.0;
  if (warp == 0) {
    for (int i = lane; i < k; i += 32) {
      zdx = dd_add_d(zdx, s_z[i] * s_dx[i]);
      mx = fmax(mx, fabs(s_dx[i]));
    }
    zdx = warp_sum_dd(zdx);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(~0u, mx, o));
  }
  if (tid == 0) {
    G->xz = dd_add(sS.xz, zdx);
    G->xx = er.xx;
    G->scale = er.scale;
    G->xss = dd_mul(er.xx, dd_mul(er.scale, er.scale));
    G->x_size = sS.x_size + s_newx;
    G->dx_max = mx;
    G->eig_residual_max = fmax(sS.eig_residual_max, er.resid);
    G->last_branch = er.branch;
    // Energy drop of this update, for the next one's shift: the current
    // energy xz/xx minus the eigenvalue (the energy after the update).
    // (only the shifted solver, eig_method 1, uses it)
    const double drop = L.eig_method == 1 ? dd_to_d(dd_div(sS.xz, sS.xx)) - er.lambda : 0.0;
    G->eig_drop = er.branch == 1 && L.eig_method == 1 ? fmax(drop, 1e-300) : 0.0;
    G->max_abs_evec = er.max_evec;
    G->inv_steps_curr = er.shift_steps;
    G->inv_diff_curr = er.shift_diff;
    if (er.shift_steps > 0) {
      G->inv_updates = sS.inv_updates + 1;
      G->inv_steps = sS.inv_steps + er.shift_steps;
      G->inv_diff_sum = sS.inv_diff_sum + er.shift_diff;
      G->inv_diff_max = fmax(sS.inv_diff_max, er.shift_diff);
    }
    if (er.fallback) G->eig_fallbacks = sS.eig_fallbacks + 1;
    G->emitted = 0;
    G->updates = 0;
    G->iter = sS.iter + 1;
    G->k_cur = k;
    G->pending = 1;
  }
  if (tid < k) {
    G->det[tid] = s_det[tid];
    G->slot[tid] = s_slot[tid];
    G->dx[tid] = s_dx[tid];
    G->hdiag[tid] = Hs[tid * k + tid];
  }
  __syncthreads();
  clk.mark(8);
}

}  // namespace
}  // namespace mcd
