// Lowest eigenpair of a small dense symmetric FP64 matrix (n <= kMaxK+1),
// computed in shared memory by one CTA of kEigThreads threads.
//
// The reference calls LAPACK dsyevr (IL=IU=1) and refines the vector with one
// step of __float128 inverse iteration through dgetrf (src/solver.h:400-503).
// Here the work is arranged around the serial dependencies of one CTA:
//   1. Householder reduction to tridiagonal T = Q^T A Q (Golub & Van Loan,
//      Algorithm 8.3.1).  Up to 33 rows (k <= 32) four warps hold the
//      matrix in registers, a row per four lanes, two barriers per step;
//      larger matrices take four warps per 32 rows in shared memory, one
//      pass over the trailing rows per step: the next pivot row is updated first, one column per thread,
//      every thread derives the next reflector from its norm, and then the
//      trailing rows, each split over four lanes, are updated with reflector
//      j while p = tau A u for reflector j+1 is formed.  Reflector j is
//      H_j = I - tau_j u_j u_j^T with u_j = (0..0, A[j][j+1..n)), where
//      A[j][j+1] holds u0_j; row j is not written after step j.
//   2. The lowest eigenvalue of T is bracketed by 128-way multisection on four
//      warps (one per SM sub-partition): T - sigma I is positive definite
//      exactly when every leading principal minor is positive (Sylvester), and
//      the minors follow p_{i+1} = (d_i - sigma) p_i - e_{i-1}^2 p_{i-1}.
//      Meanwhile the other warps form M[i][j] = tau_i u_j^T u_i (j < i) in
//      the lower triangle of A, which the reduction no longer reads.
//   3. Two steps of inverse iteration on T - sigma I with sigma at the lower
//      end of the bracket (positive definite, so LU without pivoting is
//      stable); the bracket is 2.8e-11 of the Gershgorin interval wide, so each
//      step shrinks the other eigenvectors' share by that over the gap.  The LU
//      pivots are the ratios p_{i+1}/p_i of the same minors: one FMA
//      recurrence, then independent divisions.
//   4. Back-transformation v = H_0 H_1 ... H_{n-3} y without a chain of
//      reductions: with c_j = u_j^T y, the coefficients s_j of
//      v = y - sum_j tau_j s_j u_j solve s_j = c_j - sum_{i>j} M[i][j] s_i,
//      a triangular solve of one shuffle and one FMA per step.
// The caller forms the Rayleigh quotient from the original matrix, the
// quantity that the reference's refined step approximates
// (rq = v'Bv + 2 dv'Bv, src/solver.h:516-521).
// Two faster solvers that fall back to the reduction follow: 5, shifted
// inverse iteration from a certified shift, and 6, the bordered fixed point
// (the default), a one-warp iteration on the structure of the subspace matrix
// whose result is certified as the lowest eigenpair by interlacing.
#pragma once

#include "device_common.cuh"

namespace mcd {

constexpr int kEigThreads = 512;
constexpr int kEigBracketWarps = 4;
constexpr int kEigInverseSteps = 2;  // inverse-iteration steps from the bracket's lower end
constexpr int kEigBracketRounds = 5;  // 129^5 = 3.6e10 : 1 reduction of the Gershgorin interval

// Leading dimension of an n x n work matrix: odd, so that the lanes of a warp
// reading one column of consecutive rows hit distinct shared-memory banks.
__host__ __device__ constexpr int eig_lda(int n) { return n | 1; }

__device__ __forceinline__ void bar_named(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Per-index vectors of the solver, n doubles each.
struct EigVecs {
  double *d, *e, *e2;  // diagonal, sub-diagonal and its squares of T
  double *u0, *tau;    // reflectors
  double *num, *den;   // p and w vectors of the reduction; then the minors p_{i+1}, p_i at sigma
  double *ru, *l;      // LU of T - sigma I: 1 / pivot, multipliers
  double *y;           // eigenvector of T, then of A
  double *c, *g;       // back-transformation: u_j^T y and tau_j s_j
};

// Householder scalars for x = (x0, rest) with |rest|^2 = s: u = x + sign(x0)
// mu e_1 maps x to e e_1 with e = -sign(x0) mu; u'u = 2 mu |u0|, tau = 2/u'u.
// Both roots come from the reciprocal square root (about 1 ulp each), with no
// division on the chain: mu = q rsqrt(q), tau = rsqrt(mu |u0|)^2, which keeps
// H_j orthogonal to a few ulp.
__device__ __forceinline__ void eig_reflector(double x0, double s, double& u0, double& tau, double& e) {
  if (s == 0.0) {  // nothing to annihilate: H = I
    u0 = 0.0;
    tau = 0.0;
    e = x0;
    return;
  }
  const double q = fma(x0, x0, s);
  const double mu = q * rsqrt(q);
  const double sg = x0 < 0.0 ? -1.0 : 1.0;
  u0 = fma(sg, mu, x0);
  const double r = rsqrt(mu * fabs(u0));
  tau = r * r;
  e = -sg * mu;
}

// Warps taking part in the reduction of an n x n matrix: four per 32
// trailing rows, so that each row is split over four lanes.
__host__ __device__ constexpr int eig_tridiag_warps(int n) { return 4 * ((n - 1 + 31) / 32); }

// 1. Tridiagonalisation; threads [0, 32*eig_tridiag_warps(n)) only, n >= 2.
// Step j, with reflector j, p = tau_j A u_j and K = tau_j/2 p'u_j known:
//   (a) row j+1 after the update, one column per thread (w = p - K u_j on
//       the fly): its diagonal is d_{j+1}, the rest defines reflector j+1,
//       whose scalars every thread derives from its squared norm and first
//       element;
//   (b) rows j+2.. after the update, each row split over four lanes
//       (interleaved columns), in the same pass as p = tau_{j+1} A u_{j+1}.
// A[j][j+1] is replaced by u0_j, so u_j is row j from column j+1 on.  Each
// lane of a single warp issues only about one shared-memory access per ten
// cycles, so the row pass is spread over four warps per 32 rows, one per SM
// sub-partition, and w and the row scalars go through shared memory rather
// than shuffles.
__device__ __forceinline__ void eig_tridiag(double* A, int lda, int n, const EigVecs& V) {
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int nwc = (n - 1 + 31) / 32;  // warps holding the column owners
  const int T = 32 * 4 * nwc;
  const int rs = wid * 8 + (lane & 7);  // row slot of this thread
  const int seg = lane >> 3;            // its quarter of the row
  double* const P = V.num;
  double* const W = V.den;
  __shared__ double s_part[2][4];
  __shared__ double s_x0[2];
  __shared__ double s_kp[2][16];
  if (n == 2) {
    if (t == 0) {
      V.d[0] = A[0];
      V.e[0] = A[1];
      V.d[1] = A[lda + 1];
    }
    return;
  }
  // Sum over the four lanes of a row, then over the rows of the warp, of a
  // value held by segment 0; partial per warp into s_kp[buf][wid].
  auto kp_partial = [&](double v, int buf) {
    v = warp_sum(v);
    if (lane == 0) s_kp[buf][wid] = v;
  };
  auto part_total = [&](int buf) {
    double v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = q < nwc ? s_part[buf][q] : 0.0;
    return (v[0] + v[1]) + (v[2] + v[3]);
  };
  // The per-warp partials, loaded together and summed in a fixed order.
  auto kp_total = [&](int buf) {  // 4 nwc partials, four at a time
    double k = 0.0;
    for (int g = 0; g < nwc; ++g) {
      const double v0 = s_kp[buf][4 * g], v1 = s_kp[buf][4 * g + 1];
      const double v2 = s_kp[buf][4 * g + 2], v3 = s_kp[buf][4 * g + 3];
      k += (v0 + v1) + (v2 + v3);
    }
    return k;
  };

  // Reflector 0 from row 0.
  double tau, K;
  {
    const int c = 1 + t;
    double sq = 0.0;
    if (c < n) {
      const double a = A[c];
      if (c >= 2) sq = a * a;
      if (c == 1) s_x0[0] = a;
    }
    if (wid < nwc) {
      sq = warp_sum(sq);
      if (lane == 0) s_part[0][wid] = sq;
    }
    bar_named(1, T);
    sq = part_total(0);
    double u0, e0;
    eig_reflector(s_x0[0], sq, u0, tau, e0);
    if (t == 0) {
      V.d[0] = A[0];
      V.e[0] = e0;
      V.u0[0] = u0;
      V.tau[0] = tau;
      A[1] = u0;
    }
    bar_named(1, T);
    // p for reflector 0.
    const int r = 1 + rs;
    double p = 0.0;
    if (r < n) {
      const double* Rr = A + r * lda;
      double p0 = 0.0, p1 = 0.0;
      int cc = 1 + seg;
      for (; cc + 4 < n; cc += 8) {
        p0 = fma(Rr[cc], A[cc], p0);
        p1 = fma(Rr[cc + 4], A[cc + 4], p1);
      }
      if (cc < n) p0 = fma(Rr[cc], A[cc], p0);
      p = p0 + p1;
    }
    p += __shfl_xor_sync(~0u, p, 8);
    p += __shfl_xor_sync(~0u, p, 16);
    p *= tau;
    double kp = 0.0;
    if (r < n && seg == 0) {
      P[r] = p;
      kp = p * A[r];
    }
    kp_partial(kp, 0);
    bar_named(1, T);
    K = 0.5 * tau * kp_total(0);
  }

  for (int j = 0; j + 2 < n; ++j) {
    const int buf = j & 1;
    const double* Uj = A + j * lda;  // u_j from column j+1
    double* R1 = A + (j + 1) * lda;  // the next pivot row
    const bool more = j + 3 < n;     // reflector j+1 exists
    // (a)
    const int c = j + 1 + t;
    double a = 0.0, sq = 0.0;
    if (c < n) {
      const double uc = Uj[c];
      const double wc = fma(-K, uc, P[c]);
      W[c] = wc;
      const double u1 = Uj[j + 1];
      const double w1 = fma(-K, u1, P[j + 1]);
      a = fma(-u1, wc, fma(-w1, uc, R1[c]));
      if (c >= j + 3) sq = a * a;
      if (c == j + 2) s_x0[buf] = a;
      if (c == j + 1) V.d[j + 1] = a;
    }
    if (wid < nwc) {
      sq = warp_sum(sq);
      if (lane == 0) s_part[buf][wid] = sq;
    }
    bar_named(1, T);
    sq = part_total(buf);
    const double x0 = s_x0[buf];
    double u0n = 0.0, taun = 0.0, en = x0;
    if (more) eig_reflector(x0, sq, u0n, taun, en);
    if (t == 0) {
      V.e[j + 1] = en;
      if (more) {
        V.u0[j + 1] = u0n;
        V.tau[j + 1] = taun;
      }
    }
    if (c >= j + 2 && c < n) R1[c] = (c == j + 2 && more) ? u0n : a;
    bar_named(1, T);
    // (b)
    const int r = j + 2 + rs;
    double p = 0.0;
    if (r < n) {
      double* Rr = A + r * lda;
      const double ur = Uj[r], wr = W[r];
      double p0 = 0.0, p1 = 0.0;
      int cc = j + 2 + seg;
      for (; cc + 4 < n; cc += 8) {
        const double x0v = Rr[cc], x1v = Rr[cc + 4];
        const double u0v = Uj[cc], u1v = Uj[cc + 4];
        const double w0v = W[cc], w1v = W[cc + 4];
        const double n0v = R1[cc], n1v = R1[cc + 4];
        const double y0 = fma(-ur, w0v, fma(-wr, u0v, x0v));
        const double y1 = fma(-ur, w1v, fma(-wr, u1v, x1v));
        Rr[cc] = y0;
        Rr[cc + 4] = y1;
        p0 = fma(y0, n0v, p0);
        p1 = fma(y1, n1v, p1);
      }
      if (cc < n) {
        const double y0 = fma(-ur, W[cc], fma(-wr, Uj[cc], Rr[cc]));
        Rr[cc] = y0;
        p0 = fma(y0, R1[cc], p0);
        if (!more) V.d[n - 1] = y0;  // j = n-3: the single element of row n-1
      }
      p = p0 + p1;
    }
    if (more) {
      p += __shfl_xor_sync(~0u, p, 8);
      p += __shfl_xor_sync(~0u, p, 16);
      p *= taun;
      double kp = 0.0;
      if (r < n && seg == 0) {
        P[r] = p;
        kp = p * R1[r];
      }
      kp_partial(kp, buf);
    }
    bar_named(1, T);
    if (more) K = 0.5 * taun * kp_total(buf);
    tau = taun;
  }
}

// Rows of the largest matrix that the register reduction takes.
constexpr int kEigRegRows = 33;

// eig_reflector without branches (s == 0 selects H = I), so that its two
// square roots can be scheduled together with independent work.
__device__ __forceinline__ void eig_reflector_nb(double x0, double s, double& u0, double& tau, double& e) {
  const bool none = s == 0.0;
  const double q = none ? 1.0 : fma(x0, x0, s);
  const double mu = q * rsqrt(q);
  const double sg = x0 < 0.0 ? -1.0 : 1.0;
  const double uu = fma(sg, mu, x0);
  const double r = rsqrt(mu * fabs(uu));
  u0 = none ? 0.0 : uu;
  tau = none ? 0.0 : r * r;
  e = none ? x0 : -sg * mu;
}

// a[i] for a register array of nine and a run-time i in [0, 9): a tree of
// selects on the bits of i, so that a stays in registers.
__device__ __forceinline__ double reg_pick9(const double (&a)[9], int i) {
  const bool b0 = (i & 1) != 0, b1 = (i & 2) != 0, b2 = (i & 4) != 0;
  const double t0 = b0 ? a[1] : a[0], t1 = b0 ? a[3] : a[2];
  const double t2 = b0 ? a[5] : a[4], t3 = b0 ? a[7] : a[6];
  const double s0 = b1 ? t1 : t0, s1 = b1 ? t3 : t2;
  return i >= 8 ? a[8] : (b2 ? s1 : s0);
}

// Shared-memory index of column c in the per-quarter vectors: quarter q
// (columns 9q .. 9q+8) starts at 10q, 16-byte aligned.
__device__ __forceinline__ int qpos(int c) { return c + c / 9; }

// 1 (registers).  Tridiagonalisation of an n x n matrix, 3 <= n <= 33, by
// four warps (one per SM sub-partition) holding the matrix in registers:
// row r = 1..32 belongs to the four lanes 4(r-1)..4(r-1)+3, lane quarter q
// keeping columns 9q..9q+8 (row 0 is only read: A[0][0] is d_0 and every
// reflector acts on indices 1..n-1).  Step j, two barriers:
//   (a) column j (a register picked by j, shuffled within the row) is
//       published, zero in the finished rows, together with row j+1 and each
//       warp's partial of the column's squared norm;
//   (b) every thread forms its row's A x over the published column while
//       reflector j is derived from the four partials (summed in one order:
//       the same scalars everywhere); the column stands for u except at its
//       first element, u0 instead of x0, which the row's element A[r][j+1]
//       (= A[j+1][r], read from the published row) corrects in
//       p = tau A u; then p, u and a partial of u'p are published;
//   (c) K = tau/2 u'p, w_c = p_c - K u_c and the rank-2 update
//       A -= u w' + w u' of the thread's nine elements.
// The published vectors are zero outside the active rows, so no element
// needs a mask, and the finished part of the register matrix no longer
// changes.  Same outputs as eig_tridiag.
__device__ __forceinline__ void eig_tridiag_reg(double* A, int lda, int n, const EigVecs& V) {
  __shared__ __align__(16) double s_x[40];
  __shared__ __align__(16) double s_row[40];
  __shared__ __align__(16) double s_u[40];
  __shared__ __align__(16) double s_p[40];
  __shared__ __align__(16) double s_part[4];
  __shared__ __align__(16) double s_kp[4];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int q = t & 3, r = (t >> 2) + 1, rowl = lane & ~3;
  const bool live = r < n;
  const int pr = qpos(r);
  double a[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const int c = 9 * q + i;
    a[i] = (live && c < n) ? A[r * lda + c] : 0.0;
  }
  if (t < 8) {  // entries that no row writes: column 0, quarter padding, columns 33..35
    const int z = t == 0 ? 0 : (t < 4 ? 10 * t - 1 : 32 + t);
    s_x[z] = s_row[z] = s_u[z] = s_p[z] = 0.0;
  }
  if (t == 0) V.d[0] = A[0];
  const double2* x2 = reinterpret_cast<const double2*>(s_x + 10 * q);
  const double2* u2 = reinterpret_cast<const double2*>(s_u + 10 * q);
  const double2* p2 = reinterpret_cast<const double2*>(s_p + 10 * q);
  double2* row2 = reinterpret_cast<double2*>(s_row + 10 * q);
  int jq = 0, jr = 0;  // j = 9 jq + jr
  int pj1 = 1;         // qpos(j + 1)
  for (int j = 0; j + 2 < n; ++j) {
    // (a)
    const double x = __shfl_sync(~0u, reg_pick9(a, jr), rowl | jq);  // A[r][j]
    const bool act = r >= j + 1;
    const double xp = act ? x : 0.0;
    if (q == 0) {
      if (r == j) V.d[j] = x;  // row j is final after step j-1
      s_x[pr] = xp;
    }
    if (r == j + 1) {
#pragma unroll
      for (int i = 0; i < 4; ++i) row2[i] = make_double2(a[2 * i], a[2 * i + 1]);
      s_row[10 * q + 8] = a[8];
    }
    double sq = (q == 0 && r >= j + 2) ? x * x : 0.0;
    sq += __shfl_xor_sync(~0u, sq, 4);
    sq += __shfl_xor_sync(~0u, sq, 8);
    sq += __shfl_xor_sync(~0u, sq, 16);
    if (lane == 0) s_part[wid] = sq;
    bar_named(1, 128);
    // (b)
    const double x0 = s_x[pj1];
    double pp0 = 0.0, pp1 = 0.0;  // A x over the published column, before the reflector is known
#pragma unroll
    for (int i2 = 0; i2 < 5; ++i2) {
      const double2 v = x2[i2];
      pp0 = fma(a[2 * i2], v.x, pp0);
      if (i2 < 4) pp1 = fma(a[2 * i2 + 1], v.y, pp1);
    }
    double pp = pp0 + pp1;
    pp += __shfl_xor_sync(~0u, pp, 1);
    pp += __shfl_xor_sync(~0u, pp, 2);
    double u0, tau, e;
    eig_reflector_nb(x0, (s_part[0] + s_part[1]) + (s_part[2] + s_part[3]), u0, tau, e);
    const double aj1 = s_row[pr];  // A[j+1][r]
    const double ur = (r == j + 1) ? u0 : xp;
    const double p = act ? tau * fma(aj1, u0 - x0, pp) : 0.0;
    double kp = q == 0 ? ur * p : 0.0;
    kp += __shfl_xor_sync(~0u, kp, 4);
    kp += __shfl_xor_sync(~0u, kp, 8);
    kp += __shfl_xor_sync(~0u, kp, 16);
    if (lane == 0) s_kp[wid] = kp;
    if (q == 0) {
      s_p[pr] = p;
      s_u[pr] = ur;
      if (act && live) A[j * lda + r] = ur;
    }
    if (t == 0) {
      V.e[j] = e;
      V.u0[j] = u0;
      V.tau[j] = tau;
    }
    bar_named(1, 128);
    // (c)
    const double K = 0.5 * tau * ((s_kp[0] + s_kp[1]) + (s_kp[2] + s_kp[3]));
    const double wr = fma(-K, ur, p);
#pragma unroll
    for (int i2 = 0; i2 < 5; ++i2) {
      const double2 u = u2[i2], pv = p2[i2];
      {
        const double wc = fma(-K, u.x, pv.x);
        a[2 * i2] = fma(-ur, wc, fma(-wr, u.x, a[2 * i2]));
      }
      if (i2 < 4) {
        const double wc = fma(-K, u.y, pv.y);
        a[2 * i2 + 1] = fma(-ur, wc, fma(-wr, u.y, a[2 * i2 + 1]));
      }
    }
    if (++jr == 9) {
      jr = 0;
      ++jq;
    }
    pj1 = qpos(j + 2);
  }
  // d_{n-2} = A[n-2][n-2], e_{n-2} = A[n-1][n-2], d_{n-1} = A[n-1][n-1].
  const double y = reg_pick9(a, (n - 2) % 9);
  const double z = reg_pick9(a, (n - 1) % 9);
  if (q == (n - 2) / 9) {
    if (r == n - 2) V.d[n - 2] = y;
    if (r == n - 1) V.e[n - 2] = y;
  }
  if (q == (n - 1) / 9 && r == n - 1) V.d[n - 1] = z;
}

// Rescales a pair of consecutive minors by a power of two when the newer one
// leaves [1e-150, 1e150]; signs and the ratio are unchanged.  Called every
// four recurrence steps, which grow the magnitudes by far less than 1e150.
__device__ __forceinline__ void pair_rescale(double& pc, double& pm) {
  const double a = fabs(pc);
  const double f = a > 1e150 ? 0x1p-500 : (a < 1e-150 && a > 0.0 ? 0x1p+500 : 1.0);
  pc *= f;
  pm *= f;
}

// 2a. Bracket [lo, hi] of the lowest eigenvalue of T, T - lo I positive
// definite; warps [0, kEigBracketWarps).  Returns lo and hi in every thread.
__device__ __forceinline__ void eig_bracket(int n, const EigVecs& V, double& lo_out, double& hi_out) {
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  constexpr int T = 32 * kEigBracketWarps;
  __shared__ int s_first[2][kEigBracketWarps];
  __shared__ double s_lohi[2];
  const double* const d = V.d;
  double* const e2 = V.e2;
  if (warp == 0) {
    double lo = 1e300, hi = -1e300;
    for (int i = lane; i < n; i += 32) {
      const double em = (i > 0) ? fabs(V.e[i - 1]) : 0.0;
      const double ep = (i < n - 1) ? fabs(V.e[i]) : 0.0;
      lo = fmin(lo, d[i] - em - ep);
      hi = fmax(hi, d[i] + em + ep);
      if (i < n - 1) e2[i] = V.e[i] * V.e[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(~0u, lo, o));
      hi = fmax(hi, __shfl_xor_sync(~0u, hi, o));
    }
    if (lane == 0) {
      const double widen = 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300;
      s_lohi[0] = lo - widen;
      s_lohi[1] = hi + widen;
    }
  }
  bar_named(2, T);
  double lo = s_lohi[0], hi = s_lohi[1];
  const double inv = 1.0 / static_cast<double>(T + 1);
  for (int round = 0; round < kEigBracketRounds; ++round) {
    const double w = hi - lo;
    const double sig = fma(w, static_cast<double>(t + 1) * inv, lo);
    // Not positive definite at sig <=> some leading minor <= 0.  No early
    // exit: the loop stays free of data-dependent branches.
    double pm = 1.0, pc = d[0] - sig;
    bool neg = !(pc > 0.0);
    int i = 1;
    for (; i + 3 < n; i += 4) {
      double di[4], ei[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        di[q] = d[i + q];
        ei[q] = e2[i + q - 1];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double pn = fma(di[q] - sig, pc, -ei[q] * pm);
        pm = pc;
        pc = pn;
        neg |= !(pc > 0.0);
      }
      pair_rescale(pc, pm);
    }
    for (; i < n; ++i) {
      const double pn = fma(d[i] - sig, pc, -e2[i - 1] * pm);
      pm = pc;
      pc = pn;
      neg |= !(pc > 0.0);
    }
    const unsigned b = __ballot_sync(~0u, neg);
    if (lane == 0) s_first[round & 1][warp] = b ? warp * 32 + __ffs(b) - 1 : T;
    bar_named(2, T);
    int f = T;
    for (int q = 0; q < kEigBracketWarps; ++q) f = min(f, s_first[round & 1][q]);
    if (f < T) {
      const double nlo = f > 0 ? fma(w, static_cast<double>(f) * inv, lo) : lo;
      hi = fma(w, static_cast<double>(f + 1) * inv, lo);
      lo = nlo;
    } else {
      lo = fma(w, static_cast<double>(T) * inv, lo);
    }
  }
  lo_out = lo;
  hi_out = hi;
}

// 2b. M[i][j] = tau_i u_j^T u_i for 0 <= j < i <= n-3 into A[i][j]; threads
// [t0, t0 + nthreads).
__device__ __forceinline__ void eig_gram(double* A, int lda, int n, const EigVecs& V, int t0, int nthreads) {
  const int nr = n - 2;
  const int P = nr > 1 ? nr * (nr - 1) / 2 : 0;
  for (int idx = static_cast<int>(threadIdx.x) - t0; idx < P; idx += nthreads) {
    int i = static_cast<int>((1.0f + sqrtf(1.0f + 8.0f * static_cast<float>(idx))) * 0.5f);
    while (i * (i - 1) / 2 > idx) --i;
    while (i * (i + 1) / 2 <= idx) ++i;
    const int j = idx - i * (i - 1) / 2;
    const double* ri = A + i * lda;
    const double* rj = A + j * lda;
    double s0 = rj[i + 1] * V.u0[i], s1 = 0.0;
    int c = i + 2;
    for (; c + 1 < n; c += 2) {
      s0 = fma(rj[c], ri[c], s0);
      s1 = fma(rj[c + 1], ri[c + 1], s1);
    }
    if (c < n) s0 = fma(rj[c], ri[c], s0);
    A[i * lda + j] = V.tau[i] * (s0 + s1);
  }
}

// 3. kEigInverseSteps steps of inverse iteration on T - sigma I from a fixed start
// vector; warp 0.  Writes V.y (scaled down whenever its largest element
// passes 1e100).
__device__ __forceinline__ void eig_inverse_iteration(int n, const EigVecs& V, double sigma) {
  const int lane = threadIdx.x & 31;
  const double* const d = V.d;
  const double* const e = V.e;
  const double* const e2 = V.e2;
  double* const num = V.num;
  double* const den = V.den;
  double* const ru = V.ru;
  double* const l = V.l;
  double* const y = V.y;
  for (int i = lane; i < n; i += 32) y[i] = 1.0 + 0.0625 * static_cast<double>((7 * i + 3) % 11);
  if (lane == 0) {
    double pm = 1.0, pc = d[0] - sigma;
    num[0] = pc;
    den[0] = 1.0;
    int i = 1;
    for (; i + 3 < n; i += 4) {
      double di[4], ei[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        di[q] = d[i + q];
        ei[q] = e2[i + q - 1];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double pn = fma(di[q] - sigma, pc, -ei[q] * pm);
        num[i + q] = pn;
        den[i + q] = pc;
        pm = pc;
        pc = pn;
      }
      pair_rescale(pc, pm);
    }
    for (; i < n; ++i) {
      const double pn = fma(d[i] - sigma, pc, -e2[i - 1] * pm);
      num[i] = pn;
      den[i] = pc;
      pm = pc;
      pc = pn;
    }
  }
  __syncwarp();
  for (int i = lane; i < n; i += 32) {
    double u = num[i] / den[i];
    if (!(fabs(u) >= 1e-290)) u = 1e-290;  // also catches a NaN pivot
    ru[i] = 1.0 / u;
  }
  __syncwarp();
  for (int i = lane; i < n; i += 32) l[i] = i > 0 ? e[i - 1] * ru[i - 1] : 0.0;
  __syncwarp();
  if (lane == 0) {
    for (int it = 0; it < kEigInverseSteps; ++it) {
      // L z = y: z_i = y_i - l_i z_{i-1}, in chunks of four (loads first).
      double prev = y[0];
      int i = 1;
      for (; i + 3 < n; i += 4) {
        double li[4], yi[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          li[q] = l[i + q];
          yi[q] = y[i + q];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          prev = fma(-li[q], prev, yi[q]);
          y[i + q] = prev;
        }
      }
      for (; i < n; ++i) {
        prev = fma(-l[i], prev, y[i]);
        y[i] = prev;
      }
      // U y = z: y_i = (z_i - e_i y_{i+1}) / u_i.
      double next = y[n - 1] * ru[n - 1];
      y[n - 1] = next;
      double mx = fabs(next);
      i = n - 2;
      for (; i >= 3; i -= 4) {
        double ei[4], zi[4], ri[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          ei[q] = e[i - q];
          zi[q] = y[i - q];
          ri[q] = ru[i - q];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          next = fma(-ei[q], next, zi[q]) * ri[q];
          y[i - q] = next;
          mx = fmax(mx, fabs(next));
        }
      }
      for (; i >= 0; --i) {
        next = fma(-e[i], next, y[i]) * ru[i];
        y[i] = next;
        mx = fmax(mx, fabs(next));
      }
      if (mx > 1e100)
        for (int q = 0; q < n; ++q) y[q] *= 1e-100;
    }
  }
  __syncwarp();
}

// Block-wide.  On return V.y[0..n) holds an (unnormalised) eigenvector of the
// lowest eigenvalue of the matrix originally in A (n x n, leading dimension
// lda, both triangles); A is overwritten.  clk marks sections 10..12.
__device__ __forceinline__ void eig_lowest(double* A, int lda, int n, const EigVecs& V, SectionClock& clk) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (n == 1) {
    if (tid == 0) V.y[0] = 1.0;
    __syncthreads();
    return;
  }
  if (n >= 3 && n <= kEigRegRows) {
    if (warp < 4) eig_tridiag_reg(A, lda, n, V);
  } else if (warp < eig_tridiag_warps(n)) {
    eig_tridiag(A, lda, n, V);
  }
  __syncthreads();
  clk.mark(10);

  if (warp < kEigBracketWarps) {
    double lo, hi;
    eig_bracket(n, V, lo, hi);
    clk.mark(11);
    if (warp == 0) eig_inverse_iteration(n, V, lo);
    clk.mark(12);
  } else {
    eig_gram(A, lda, n, V, 32 * kEigBracketWarps, static_cast<int>(blockDim.x) - 32 * kEigBracketWarps);
  }
  __syncthreads();

  // 4. Back-transformation.
  double* y = V.y;
  for (int j = warp; j < n - 2; j += kEigThreads / 32) {
    const double* rj = A + j * lda;
    double s = 0.0;
    for (int c = j + 2 + lane; c < n; c += 32) s = fma(rj[c], y[c], s);
    s = warp_sum(s);
    if (lane == 0) V.c[j] = fma(V.u0[j], y[j + 1], s);
  }
  __syncthreads();
  if (warp == 0) {
    constexpr int Q = (kMaxK + 1 + 31) / 32;
    double tq[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int j = lane + 32 * q;
      tq[q] = j < n - 2 ? V.c[j] : 0.0;
    }
    double mrow[Q];  // M[i][lane + 32q], loaded one step ahead
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int j = lane + 32 * q;
      mrow[q] = (n >= 3 && j < n - 3) ? A[(n - 3) * lda + j] : 0.0;
    }
    for (int i = n - 3; i >= 0; --i) {
      double mnext[Q];
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int j = lane + 32 * q;
        mnext[q] = (i >= 1 && j < i - 1) ? A[(i - 1) * lda + j] : 0.0;
      }
      const int qi = i >> 5;
      double own = tq[0];
#pragma unroll
      for (int q = 1; q < Q; ++q) own = (qi == q) ? tq[q] : own;
      const double si = __shfl_sync(~0u, own, i & 31);
      if (lane == (i & 31)) V.g[i] = V.tau[i] * si;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int j = lane + 32 * q;
        if (j < i) tq[q] = fma(-mrow[q], si, tq[q]);
        mrow[q] = mnext[q];
      }
    }
  }
  __syncthreads();
  for (int r = warp; r < n; r += kEigThreads / 32) {
    const int jmax = min(r - 1, n - 3);
    double s = 0.0;
    for (int j = lane; j <= jmax; j += 32) {
      const double ujr = (j == r - 1) ? V.u0[j] : A[j * lda + r];
      s = fma(V.g[j], ujr, s);
    }
    s = warp_sum(s);
    if (lane == 0) y[r] -= s;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// 5. The lowest eigenpair from a certified shift, for matrices of up to
//    kShiftMaxN rows, when a shift sigma just below the lowest eigenvalue and
//    a start vector close to its eigenvector are known (in the solver, the
//    current vector lies in the subspace, its energy bounds the eigenvalue
//    from above, and the last iteration's energy drop says how far below it
//    the eigenvalue is likely to lie).
//    (a) Cholesky factorisation A - sigma I = L L^T in Crout order by one
//        warp (a row per lane), in A's lower triangle, 1/L_jj in V.ru.  It
//        succeeds exactly when A - sigma I is positive definite (Sylvester),
//        which certifies sigma < lambda_1: inverse iteration can then only
//        converge to the lowest eigenvector.  A non-positive pivot returns
//        false.
//    (b) L^-1 explicitly, one thread per column, into Li (lower triangle,
//        zeros above).
//    (c) Power steps v <- C v / |C v| with C = (A - sigma I)^-1 = L^-T L^-1
//        formed once, one matrix-vector product per step (no serial chain),
//        until successive vectors agree to 1e-12 or stop improving; each step
//        divides the other eigenvectors' share by at least
//        (lambda_2 - sigma)/(lambda_1 - sigma).
//    (d) Refinement: C applied to the residual instead of the vector.  With
//        rho = v'Av and r = A v - rho v, exactly (A - sigma I)^-1 v =
//        (v - (A - sigma I)^-1 r) / (rho - sigma).  The explicit inverse is
//        accurate to about n eps cond(L) relative, but r is small, so the
//        step w = v - C r carries that error only on a small correction: an
//        inverse-iteration step at the accuracy of the residual.  A is read
//        from its upper triangle and the diagonal saved in V.d.
//    Returns false (uniform over the block) when (a) fails or (c)/(d) do not
//    converge within their limits; A's lower triangle is then overwritten and
//    the caller rebuilds it.  On success V.y holds the unit eigenvector.
//    *steps receives the power and refinement steps, *diff the change made
//    by the last refinement.  All threads of the block call it; V.y holds
//    the start vector on entry.
constexpr int kShiftMaxN = 65;
constexpr int kShiftPowerSteps = 40;
constexpr int kShiftRefineSteps = 6;

// Per-row values of three rows per lane at most (n <= 96).
constexpr int kShiftQ = 3;

// (a) and (b) with the matrix in registers, for n <= kShiftRegRows: 160
// threads, row r = t/4 held by four lanes, lane quarter q keeping columns
// 9q..9q+8.  Cholesky, right-looking: at step j the owners of column j
// publish it (rows >= j) to a shared vector, and after one barrier every
// thread scales it by 1/sqrt(pivot) and updates its part of the trailing
// matrix; L goes to A's lower triangle, 1/L_jj to V.ru.  Then X = L^-1 by
// forward substitution on the identity, row j published (divided by L_jj)
// and subtracted from the rows below, one barrier per step; X goes to Li.
// Two vectors alternate as the published column or row, so that a step's
// writes never meet the previous step's reads.  Called by the whole block;
// returns false (uniform) on a non-positive pivot.
constexpr int kShiftRegRows = 36;
constexpr int kShiftRegThreads = 160;

__device__ bool shift_factor_reg(double* A, int lda, int n, double sigma, const EigVecs& V, double* Li) {
  const int t = threadIdx.x;
  const bool part = t < kShiftRegThreads;
  const int r = t >> 2, q = t & 3;
  const bool row_ok = part && r < n;
  __shared__ int s_fail;
  double a[9];
#pragma unroll
  for (int e = 0; e < 9; ++e) {
    const int c = 9 * q + e;
    a[e] = (row_ok && c < n) ? A[r * lda + c] - (r == c ? sigma : 0.0) : 0.0;
  }
  if (t == 0) s_fail = 0;
  __syncthreads();
  if (part) {
    for (int j = 0; j < n; ++j) {
      double* col = (j & 1) ? V.g : V.c;
      if (row_ok && r >= j && q == j / 9) col[r] = reg_pick9(a, j - 9 * q);
      bar_named(2, kShiftRegThreads);
      const double d = col[j];
      if (!(d > 0.0)) {
        if (t == 0) s_fail = 1;
        break;
      }
      const double rinv = rsqrt(d);
      if (row_ok && r > j) {
        const double li = col[r] * rinv;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          const int c = 9 * q + e;
          if (c > j && c < n) a[e] = fma(-li, col[c] * rinv, a[e]);
        }
        if (q == 0) A[r * lda + j] = li;
      }
      if (r == j && q == 0) {
        A[j * lda + j] = d * rinv;
        V.ru[j] = rinv;
      }
    }
  }
  __syncthreads();
  if (s_fail) return false;
  if (part) {
    double x[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) x[e] = (row_ok && r == 9 * q + e) ? 1.0 : 0.0;
    for (int j = 0; j < n; ++j) {
      double* row = (j & 1) ? V.den : V.num;
      if (r == j) {
        const double rinv = V.ru[j];
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          const int c = 9 * q + e;
          x[e] *= rinv;
          if (c < n) row[c] = x[e];
        }
      }
      bar_named(2, kShiftRegThreads);
      if (row_ok && r > j) {
        const double lij = A[r * lda + j];
#pragma unroll
        for (int e = 0; e < 9; ++e) {
          const int c = 9 * q + e;
          if (c <= j) x[e] = fma(-lij, row[c], x[e]);
        }
      }
    }
    if (row_ok) {
#pragma unroll
      for (int e = 0; e < 9; ++e) {
        const int c = 9 * q + e;
        if (c < n) Li[r * lda + c] = x[e];
      }
    }
  }
  __syncthreads();
  return true;
}

// The shifted solver: (a) and (b) in registers up to kShiftRegRows rows
// (shift_factor_reg), else by one warp in shared memory (a Crout Cholesky,
// then L^-1 one column per thread); C formed by the whole block into Ci
// (n x lda shared doubles); (c) and (d) by one warp, up to kShiftQ rows per
// lane, shuffle reductions and no block barrier, each refinement step
// adding the residual's product with A (upper triangle and V.d).
__device__ bool eig_lowest_shifted_warp(double* A, int lda, int n, const EigVecs& V, double sigma, double* Li,
                                        double* Ci, int* steps, double* diff, SectionClock& clk) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ bool s_ok;
  __shared__ int s_steps;
  __shared__ double s_diff;
  if (tid == 0) {
    s_ok = true;
    s_steps = 0;
    s_diff = 0.0;
  }
  for (int i = tid; i < n; i += blockDim.x) V.d[i] = A[i * lda + i];
  __syncthreads();

  if (n <= kShiftRegRows) {
    const bool ok = shift_factor_reg(A, lda, n, sigma, V, Li);
    clk.mark(17);
    if (!ok) {
      *steps = 0;
      *diff = 0.0;
      return false;
    }
  } else {
  // (a) Cholesky by warp 0.
  if (warp == 0) {
    bool ok = true;
    for (int j = 0; j < n; ++j) {
      const double* Lj = A + j * lda;
      double sv[kShiftQ];
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) {
        const int i = j + lane + 32 * q;
        sv[q] = 0.0;
        if (i < n) {
          const double* Lr = A + i * lda;
          double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
          int c = 0;
          for (; c + 4 <= j; c += 4) {
            a0 = fma(Lr[c], Lj[c], a0);
            a1 = fma(Lr[c + 1], Lj[c + 1], a1);
            a2 = fma(Lr[c + 2], Lj[c + 2], a2);
            a3 = fma(Lr[c + 3], Lj[c + 3], a3);
          }
          for (; c < j; ++c) a0 = fma(Lr[c], Lj[c], a0);
          const double aij = (i == j) ? Lr[j] - sigma : Lr[j];
          sv[q] = aij - ((a0 + a1) + (a2 + a3));
        }
      }
      const double d = __shfl_sync(~0u, sv[0], 0);
      if (!(d > 0.0)) {
        ok = false;
        break;
      }
      const double r = rsqrt(d);
      if (lane == 0) {
        A[j * lda + j] = d * r;
        V.ru[j] = r;
      }
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) {
        const int i = j + lane + 32 * q;
        if (i > j && i < n) A[i * lda + j] = sv[q] * r;
      }
      __syncwarp();
    }
    if (lane == 0 && !ok) s_ok = false;
  }
  __syncthreads();
  clk.mark(17);
  if (!s_ok) {
    *steps = 0;
    *diff = 0.0;
    return false;
  }

  // (b) L^-1, column j by thread j.
  if (tid < n) {
    const int j = tid;
    for (int i = 0; i < n; ++i) {
      const double* Lr = A + i * lda;
      double a0 = (i == j) ? 1.0 : 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
      int c = 0;
      for (; c + 4 <= i; c += 4) {
        a0 = fma(-Lr[c], Li[c * lda + j], a0);
        a1 = fma(-Lr[c + 1], Li[(c + 1) * lda + j], a1);
        a2 = fma(-Lr[c + 2], Li[(c + 2) * lda + j], a2);
        a3 = fma(-Lr[c + 3], Li[(c + 3) * lda + j], a3);
      }
      for (; c < i; ++c) a0 = fma(-Lr[c], Li[c * lda + j], a0);
      Li[i * lda + j] = ((a0 + a1) + (a2 + a3)) * V.ru[i];
    }
  }
  __syncthreads();
  }
  // C = L^-T L^-1: C[i][j] = sum over c >= max(i, j) of Li[c][i] Li[c][j], one
  // element of the upper triangle per thread, mirrored.
  for (int t = tid; t < n * (n + 1) / 2; t += blockDim.x) {
    int j = static_cast<int>((sqrtf(8.0f * static_cast<float>(t) + 1.0f) - 1.0f) * 0.5f);
    while (j * (j + 1) / 2 > t) --j;
    while ((j + 1) * (j + 2) / 2 <= t) ++j;
    const int i = t - j * (j + 1) / 2;  // i <= j
    double a0 = 0.0, a1 = 0.0;
    int c = j;
    for (; c + 2 <= n; c += 2) {
      a0 = fma(Li[c * lda + i], Li[c * lda + j], a0);
      a1 = fma(Li[(c + 1) * lda + i], Li[(c + 1) * lda + j], a1);
    }
    if (c < n) a0 = fma(Li[c * lda + i], Li[c * lda + j], a0);
    const double v = a0 + a1;
    Ci[i * lda + j] = v;
    Ci[j * lda + i] = v;
  }
  __syncthreads();
  clk.mark(18);

  // (c), (d) by warp 0; rows lane + 32 q.
  if (warp == 0) {
    double v[kShiftQ];
    double nrm = 0.0;
#pragma unroll
    for (int q = 0; q < kShiftQ; ++q) {
      const int i = lane + 32 * q;
      v[q] = i < n ? V.y[i] : 0.0;
      nrm = fma(v[q], v[q], nrm);
    }
    nrm = warp_sum(nrm);
    const double inv0 = rsqrt(nrm);
#pragma unroll
    for (int q = 0; q < kShiftQ; ++q) {
      v[q] *= inv0;
      const int i = lane + 32 * q;
      if (i < n) V.y[i] = v[q];
    }
    __syncwarp();
    // w = M u for the rows of this lane, u in shared memory.
    auto matvec = [&](const double* M, const double* u, double (&w)[kShiftQ]) {
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) {
        const int i = lane + 32 * q;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
        if (i < n) {
          const double* row = M + i * lda;
          int c = 0;
          for (; c + 4 <= n; c += 4) {
            a0 = fma(row[c], u[c], a0);
            a1 = fma(row[c + 1], u[c + 1], a1);
            a2 = fma(row[c + 2], u[c + 2], a2);
            a3 = fma(row[c + 3], u[c + 3], a3);
          }
          for (; c < n; ++c) a0 = fma(row[c], u[c], a0);
        }
        w[q] = (a0 + a1) + (a2 + a3);
      }
    };
    // v <- w / |w|; returns |v_new - v_old|.
    auto normalise_into = [&](double (&w)[kShiftQ]) {
      double ww = 0.0;
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) ww = fma(w[q], w[q], ww);
      ww = warp_sum(ww);
      const double inv = rsqrt(ww);
      double d2 = 0.0;
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) {
        const double vn = w[q] * inv;
        d2 = fma(vn - v[q], vn - v[q], d2);
        v[q] = vn;
      }
      d2 = warp_sum(d2);
      __syncwarp();
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) {
        const int i = lane + 32 * q;
        if (i < n) V.y[i] = v[q];
      }
      __syncwarp();
      return sqrt(d2);
    };
    int nsteps = 0;
    double prev = 1e300;
    for (int it = 0; it < kShiftPowerSteps; ++it) {
      double w[kShiftQ];
      matvec(Ci, V.y, w);
      const double dv = normalise_into(w);
      ++nsteps;
      if (dv < 1e-12 || (dv < 1e-8 && dv > 0.5 * prev)) break;
      prev = dv;
    }
    clk.mark(19);
    bool done = false;
    double last = 0.0;
    for (int it = 0; it < kShiftRefineSteps && !done; ++it) {
      // A v from the upper triangle and the saved diagonal.
      double av[kShiftQ];
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) {
        const int i = lane + 32 * q;
        double a0 = 0.0, a1 = 0.0;
        if (i < n) {
          for (int c = 0; c < n; c += 2) {
            const double e0 = (c == i) ? V.d[i] : (c > i ? A[i * lda + c] : A[c * lda + i]);
            a0 = fma(e0, V.y[c], a0);
            if (c + 1 < n) {
              const int c1 = c + 1;
              const double e1 = (c1 == i) ? V.d[i] : (c1 > i ? A[i * lda + c1] : A[c1 * lda + i]);
              a1 = fma(e1, V.y[c1], a1);
            }
          }
        }
        av[q] = a0 + a1;
      }
      double rho = 0.0;
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) rho = fma(v[q], av[q], rho);
      rho = warp_sum(rho);
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) {
        const int i = lane + 32 * q;
        if (i < n) V.g[i] = av[q] - rho * v[q];
      }
      __syncwarp();
      double t[kShiftQ];
      matvec(Ci, V.g, t);
#pragma unroll
      for (int q = 0; q < kShiftQ; ++q) t[q] = v[q] - t[q];
      last = normalise_into(t);
      ++nsteps;
      done = last < 2e-15 * sqrt(static_cast<double>(n));
    }
    if (lane == 0) {
      s_ok = done;
      s_steps = nsteps;
      s_diff = last;
    }
  }
  __syncthreads();
  clk.mark(20);
  *steps = s_steps;
  *diff = s_diff;
  return s_ok;
}

// ---------------------------------------------------------------------------
// 6. The lowest eigenpair of the bordered matrix B = [[a, b'], [b, C]] (n = k + 1
//    rows, k <= kBorderMaxK) when it lies below the Gershgorin bound of C,
//    g = min_i (C_ii - sum_{j != i} |C_ij|).  By Cauchy interlacing B has exactly
//    one eigenvalue below lambda_1(C) >= g, so an approximate eigenpair (lambda,
//    v) with lambda + ||B v - lambda v|| / ||v|| < g belongs to the lowest
//    eigenvalue (some eigenvalue lies within the residual norm of lambda).  With
//    v = (1, y), D the diagonal of C and E the rest, the last k rows of
//    (B - lambda I) v = 0 read (D - lambda I) y = -(b + E y), and the first row
//    lambda = a + b'y.  One warp iterates
//        y <- -(b + E y) / (d - lambda),   lambda <- a + b'y,
//    which contracts by about max_i sum_j |E_ij| / (d_i - lambda) per step, less
//    than 1 whenever lambda < g (C is strongly diagonal in a subspace of picked
//    determinants, most of which are not connected by a single or double
//    excitation).  The product E y of a step also gives the residual of the
//    current iterate, r_i = (b + E y)_i + (d_i - lambda) y_i (row 0's residual
//    is zero by the choice of lambda), so a step costs one matrix-vector
//    product, a reciprocal per row and one warp reduction of three values, with
//    no block barrier.  The reciprocal of d_i - lambda is one Newton-Raphson
//    step, r <- r + r e with e = 1 - (d_i - lambda) r, from the last step's r,
//    while |e| < 1e-3 (lambda moves less every step, so the error falls
//    quadratically), and a division otherwise (the first steps); an inexact r
//    changes only the step, not the fixed point.  E is sparse (most picked determinants are not
//    connected), so each lane first packs its rows' nonzero entries of E into
//    `pack`, 2 (k + 1) lda doubles of scratch (values of row i from i lda on;
//    after the k rows of values, their columns as 4-byte ints, row i from
//    i (2 lda + 1) on), and a step's product runs over those only.  The
//    iteration stops when ||r|| / ||v|| reaches
//    1e-15 max_i sum_j |B_ij| (or stalls within 16 times that), and gives up
//    when it stops contracting or lambda is not below g; A is only read.
//    Returns true (uniform over the block) with V.y = (1, y) when the pair is
//    certified; *iters receives the steps taken and *resid the final residual
//    norm.  All threads call it.
constexpr int kBorderMaxK = 64;
constexpr int kBorderIters = 64;

__device__ bool eig_lowest_bordered(const double* A, int lda, int n, const EigVecs& V, double* pack, int* iters,
                                    double* resid, SectionClock& clk) {
  __shared__ int s_ok, s_it;
  __shared__ double s_rn;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int k = n - 1;
  if (warp == 0) {
    double* ys = V.y + 1;  // y_j at ys[j]
    const double a = A[0];
    double d[2], b[2], y[2];
    bool own[2];
    int cnt[2];
    double gl = 1e300, nb = 0.0, babs = 0.0;
    // Row i's nonzero off-diagonal entries of C: values at pv + i lda, their
    // columns at pc + i (2 lda + 1) (an odd stride in 4-byte words).
    double* const pv = pack;
    int* const pc = reinterpret_cast<int*>(pack + static_cast<size_t>(k) * lda);
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int i = lane + 32 * q;
      own[q] = i < k;
      const double* row = A + (i + 1) * lda + 1;
      d[q] = own[q] ? row[i] : 0.0;
      b[q] = own[q] ? A[i + 1] : 0.0;
      double off = 0.0;
      int c = 0;
      if (own[q])
        for (int j0 = 0; j0 < k; j0 += 8) {
          double v8[8];  // eight loads in flight before the dependent stores
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) v8[jj] = j0 + jj < k ? row[j0 + jj] : 0.0;
#pragma unroll
          for (int jj = 0; jj < 8; ++jj) {
            const int j = j0 + jj;
            if (j != i && v8[jj] != 0.0) {
              off += fabs(v8[jj]);
              pv[i * lda + c] = v8[jj];
              pc[i * (2 * lda + 1) + c] = j;
              ++c;
            }
          }
        }
      cnt[q] = c;
      y[q] = 0.0;
      if (own[q]) {
        gl = fmin(gl, d[q] - off);
        nb = fmax(nb, fabs(d[q]) + off + fabs(b[q]));
        babs += fabs(b[q]);
        ys[i] = 0.0;
      }
    }
    int cmax = max(cnt[0], cnt[1]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      gl = fmin(gl, __shfl_xor_sync(~0u, gl, o));
      nb = fmax(nb, __shfl_xor_sync(~0u, nb, o));
      babs += __shfl_xor_sync(~0u, babs, o);
      cmax = max(cmax, __shfl_xor_sync(~0u, cmax, o));
    }
    nb = fmax(nb, fabs(a) + babs);
    if (lane == 0) V.y[0] = 1.0;
    __syncwarp();
    clk.mark(17);
    const double tol = 1e-15 * nb;
    const double tol2 = tol * tol;
    double lam = fmin(a, gl) - 1e-3 * (1.0 + fabs(a));
    double rcp[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) rcp[q] = own[q] ? 1.0 / (d[q] - lam) : 0.0;
    // The tests compare squared residual norms |r|^2 / |v|^2 cross-multiplied,
    // so that no division or square root sits on a step's chain.
    double rrp = 1e300, vvp = 1.0;  // |r|^2 and |v|^2 of the previous step
    bool ok = false;
    int t = 0;
    for (; t < kBorderIters; ++t) {
      // s = b + E y_t for this lane's rows, over their packed nonzeros.
      double s[2], yn[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int i = lane + 32 * q;
        const double* rv = pv + i * lda;
        const int* rc = pc + i * (2 * lda + 1);
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (q == 0 || k > 32) {
          const int c = cnt[q];
          int e = 0;
          for (; e + 3 < cmax; e += 4) {
            if (e < c) s0 = fma(rv[e], ys[rc[e]], s0);
            if (e + 1 < c) s1 = fma(rv[e + 1], ys[rc[e + 1]], s1);
            if (e + 2 < c) s2 = fma(rv[e + 2], ys[rc[e + 2]], s2);
            if (e + 3 < c) s3 = fma(rv[e + 3], ys[rc[e + 3]], s3);
          }
          for (; e < cmax; ++e)
            if (e < c) s0 = fma(rv[e], ys[rc[e]], s0);
          s[q] = b[q] + ((s0 + s1) + (s2 + s3));
          if (t > 0) {
            const double x = d[q] - lam;
            const double e = fma(-x, rcp[q], 1.0);  // relative error of rcp as 1 / x
            if (fabs(e) < 1e-3)
              rcp[q] = fma(rcp[q], e, rcp[q]);
            else
              rcp[q] = 1.0 / x;
          }
          yn[q] = own[q] ? -s[q] * rcp[q] : 0.0;
        } else {
          s[q] = 0.0;
          yn[q] = 0.0;
        }
      }
      clk.mark(18);
      // Residual of (lambda_t, v_t), |y_t|^2 and b'y_{t+1}, in one reduction.
      double rr = 0.0, yy = 0.0, by = 0.0;
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        if (!own[q]) continue;
        const double ri = fma(d[q] - lam, y[q], s[q]);
        rr = fma(ri, ri, rr);
        yy = fma(y[q], y[q], yy);
        by = fma(b[q], yn[q], by);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        rr += __shfl_xor_sync(~0u, rr, o);
        yy += __shfl_xor_sync(~0u, yy, o);
        by += __shfl_xor_sync(~0u, by, o);
      }
      const double vv = 1.0 + yy;
      if (!isfinite(rr) || !isfinite(vv)) break;
      // rn <= tol, or rn > rn_prev / 2 and rn <= 16 tol (stalled at rounding)
      const bool small =
          rr <= tol2 * vv || (t >= 2 && rr * vvp > 0.25 * rrp * vv && rr <= 256.0 * tol2 * vv);
      if (t > 0 && small) {
        const double rn = sqrt(rr / vv);
        ok = lam + rn < gl;
        if (lane == 0) s_rn = rn;
        break;
      }
      // not contracting (rn > 0.9 rn_prev), or lambda not below g
      if ((t >= 8 && rr * vvp > 0.81 * rrp * vv) || (t >= 4 && !(lam < gl))) break;
      clk.mark(19);
      rrp = rr;
      vvp = vv;
      __syncwarp();  // every lane has read y_t
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        y[q] = yn[q];
        if (own[q]) ys[lane + 32 * q] = yn[q];
      }
      lam = a + by;
      __syncwarp();
      clk.mark(20);
    }
    if (lane == 0) {
      s_ok = ok;
      s_it = t + 1;
    }
  }
  __syncthreads();
  *iters = s_it;
  if (resid) *resid = s_ok ? s_rn : 0.0;
  return s_ok != 0;
}

}  // namespace mcd
