// Smallest eigenpair of a small dense symmetric FP64 matrix, computed by one
// CTA of 1024 threads in shared memory.
//
// The reference calls LAPACK dsyevr (IL=IU=1) and refines the vector with one
// step of __float128 inverse iteration through dgetrf (src/solver.h:400-503).
// Here, for n <= kMaxK+1:
//   1. Householder reduction to tridiagonal T = Q^T A Q (Golub & Van Loan,
//      Algorithm 8.3.1).  Each step takes two CTA barriers: every warp derives
//      the reflector scalars from the current column itself (identical
//      arithmetic in every warp, so no broadcast barrier), forms p = beta A v
//      for its rows, then, after a barrier, K = beta/2 p'v and the rank-2
//      update of its rows.  Reflector j is kept in row j right of the diagonal,
//      which the reduction never reads again.
//   2. The lowest eigenvalue of T is isolated by 1024-way multisection: each
//      thread counts the eigenvalues below its shift from the signs of the
//      characteristic polynomials of the leading sub-matrices (Sturm's
//      theorem), computed by the three-term recurrence with power-of-two
//      rescaling, four rounds.
//   3. Inverse iteration on T - sigma I with sigma at the lower end of the
//      isolating interval (positive definite, so no pivoting), three solves.
//   4. Back-transformation v = Q y by warp 0 with y in registers.
// The caller forms the Rayleigh quotient in double-double from the original
// matrix, which is the quantity the reference's refined step approximates
// (rq = v'Bv + 2 dv'Bv, src/solver.h:516-521).
#pragma once

#include "device_common.cuh"

namespace mcd {

constexpr int kEigThreads = 1024;

struct EigScratch {
  double* A;     // n x n, row-major, leading dimension lda
  int lda;
  double* d;     // [n] diagonal of T
  double* e;     // [n] sub-diagonal of T
  double* e2;    // [n] e^2
  double* beta;  // [n] reflector coefficients
  double* hv;    // [n] scratch
  double* p;     // [n] scratch
  double* y;     // [n] eigenvector (output)
  double* part;  // [32] per-warp partials
  double* scal;  // [8] scalars
  int* ibest;    // [1]
};

// Reflector scalars of column j (rows j+1..n-1), computed identically by
// every lane of every warp: beta, 1/v0 and the new sub-diagonal mu.
__device__ __forceinline__ void house_scalars(const double* A, int lda, int j, int m, double& bet, double& inv_v0,
                                              double& mu) {
  const int lane = threadIdx.x & 31;
  double s = 0.0;
  for (int i = 1 + lane; i < m; i += 32) {
    const double v = A[(j + 1 + i) * lda + j];
    s = fma(v, v, s);
  }
  s = __shfl_sync(~0u, warp_sum(s), 0);
  const double x0 = A[(j + 1) * lda + j];
  bet = 0.0;
  inv_v0 = 0.0;
  mu = x0;
  if (s != 0.0) {
    mu = sqrt(x0 * x0 + s);
    const double v0 = (x0 <= 0.0) ? x0 - mu : -s / (x0 + mu);
    bet = 2.0 * v0 * v0 / (s + v0 * v0);
    inv_v0 = 1.0 / v0;
  }
}

// Block-wide.  On return ws.y[0..n) holds an (unnormalised) eigenvector of the
// lowest eigenvalue of the matrix originally in ws.A; ws.A is overwritten.
__device__ void smallest_eigvec(EigScratch& ws, int n, SectionClock& clk) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NT = blockDim.x;
  const int NW = NT >> 5;
  double* A = ws.A;
  const int lda = ws.lda;

  if (n == 1) {
    if (tid == 0) ws.y[0] = 1.0;
    __syncthreads();
    return;
  }

  // 1. Tridiagonalisation.
  for (int j = 0; j + 2 < n; ++j) {
    const int m = n - j - 1;
    double bet, inv_v0, mu;
    house_scalars(A, lda, j, m, bet, inv_v0, mu);
    if (tid == 0) {
      ws.beta[j] = bet;
      ws.e[j] = mu;
      ws.d[j] = A[j * lda + j];
    }
    if (bet == 0.0) continue;  // column already reduced; T keeps e[j] = x0
    const double* colj = A + (j + 1) * lda + j;  // element i at colj[i * lda]
    // p = beta * A22 * v for this warp's rows.
    for (int r = warp; r < m; r += NW) {
      const double* row = A + (j + 1 + r) * lda + (j + 1);
      double acc = 0.0;
      for (int c = lane; c < m; c += 32) {
        const double hc = (c == 0) ? 1.0 : colj[c * lda] * inv_v0;
        acc = fma(row[c], hc, acc);
      }
      acc = warp_sum(acc);
      if (lane == 0) ws.p[r] = bet * acc;
    }
    __syncthreads();
    // K = beta/2 * p'v (identical in every warp), then A22 -= v w' + w v'.
    double kp = 0.0;
    for (int r = lane; r < m; r += 32) {
      const double hr = (r == 0) ? 1.0 : colj[r * lda] * inv_v0;
      kp = fma(ws.p[r], hr, kp);
    }
    const double K = 0.5 * bet * __shfl_sync(~0u, warp_sum(kp), 0);
    for (int r = warp; r < m; r += NW) {
      const double hr = (r == 0) ? 1.0 : colj[r * lda] * inv_v0;
      const double wr = ws.p[r] - K * hr;
      double* row = A + (j + 1 + r) * lda + (j + 1);
      for (int c = lane; c < m; c += 32) {
        const double hc = (c == 0) ? 1.0 : colj[c * lda] * inv_v0;
        const double wc = ws.p[c] - K * hc;
        row[c] -= hr * wc + wr * hc;
      }
    }
    if (warp == NW - 1)
      for (int c = lane; c < m; c += 32) A[j * lda + (j + 1 + c)] = (c == 0) ? 1.0 : colj[c * lda] * inv_v0;
    __syncthreads();
  }
  if (tid == 0) {
    ws.d[n - 2] = A[(n - 2) * lda + (n - 2)];
    ws.e[n - 2] = A[(n - 1) * lda + (n - 2)];
    ws.d[n - 1] = A[(n - 1) * lda + (n - 1)];
  }
  __syncthreads();
  clk.mark(10);

  // 2. Multisection for the lowest eigenvalue of T.
  if (warp == 0) {
    double lo = 1e300, hi = -1e300;
    for (int i = lane; i < n; i += 32) {
      const double em = (i > 0) ? fabs(ws.e[i - 1]) : 0.0;
      const double ep = (i < n - 1) ? fabs(ws.e[i]) : 0.0;
      lo = fmin(lo, ws.d[i] - em - ep);
      hi = fmax(hi, ws.d[i] + em + ep);
      if (i < n - 1) ws.e2[i] = ws.e[i] * ws.e[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(~0u, lo, o));
      hi = fmax(hi, __shfl_xor_sync(~0u, hi, o));
    }
    if (lane == 0) {
      const double widen = 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300;
      ws.scal[2] = lo - widen;
      ws.scal[3] = hi + widen;
    }
  }
  __syncthreads();
  for (int round = 0; round < 4; ++round) {
    const double lo = ws.scal[2], hi = ws.scal[3];
    if (tid == 0) *ws.ibest = NT;
    __syncthreads();
    const double sig = lo + (hi - lo) * (static_cast<double>(tid + 1) / static_cast<double>(NT + 1));
    // Sign changes in p_0 = 1, p_1 = d_0 - sig, p_i = (d_{i-1} - sig) p_{i-1} - e_{i-2}^2 p_{i-2};
    // a zero takes the sign opposite to its predecessor.
    double pm = 1.0, pc = ws.d[0] - sig;
    int sprev = 1, cnt = 0;
    int sc = (pc > 0.0) ? 1 : (pc < 0.0 ? -1 : -sprev);
    cnt += (sc != sprev);
    sprev = sc;
    for (int i = 1; i < n; ++i) {
      const double pn = (ws.d[i] - sig) * pc - ws.e2[i - 1] * pm;
      pm = pc;
      pc = pn;
      const double big = fabs(pc) + fabs(pm);
      if (big > 1e150 || (big < 1e-150 && big > 0.0)) {
        const double f = big > 1e150 ? 0x1p-500 : 0x1p+500;
        pc *= f;
        pm *= f;
      }
      sc = (pc > 0.0) ? 1 : (pc < 0.0 ? -1 : -sprev);
      cnt += (sc != sprev);
      sprev = sc;
    }
    if (cnt >= 1) atomicMin(ws.ibest, tid);
    __syncthreads();
    if (tid == 0) {
      const int t = *ws.ibest;
      if (t < NT) {
        ws.scal[3] = lo + (hi - lo) * (static_cast<double>(t + 1) / static_cast<double>(NT + 1));
        if (t > 0) ws.scal[2] = lo + (hi - lo) * (static_cast<double>(t) / static_cast<double>(NT + 1));
      } else {
        ws.scal[2] = lo + (hi - lo) * (static_cast<double>(NT) / static_cast<double>(NT + 1));
      }
    }
    __syncthreads();
  }
  clk.mark(11);

  // 3. Inverse iteration on T - sigma I (thread 0; 1/u and l reuse hv and p).
  if (tid == 0) {
    const double sigma = ws.scal[2];
    const double tiny = 1e-290;
    double* ru = ws.hv;
    double* l = ws.p;
    double u = ws.d[0] - sigma;
    if (fabs(u) < tiny) u = tiny;
    ru[0] = 1.0 / u;
    for (int i = 1; i < n; ++i) {
      const double li = ws.e[i - 1] * ru[i - 1];
      l[i] = li;
      u = (ws.d[i] - sigma) - li * ws.e[i - 1];
      if (fabs(u) < tiny) u = tiny;
      ru[i] = 1.0 / u;
    }
    double* y = ws.y;
    for (int i = 0; i < n; ++i) y[i] = 1.0 + 0.0625 * static_cast<double>((7 * i + 3) % 11);
    for (int it = 0; it < 3; ++it) {
      double prev = y[0];
      for (int i = 1; i < n; ++i) {
        prev = y[i] - l[i] * prev;
        y[i] = prev;
      }
      double next = y[n - 1] * ru[n - 1];
      y[n - 1] = next;
      double mx = fabs(next);
      for (int i = n - 2; i >= 0; --i) {
        next = (y[i] - ws.e[i] * next) * ru[i];
        y[i] = next;
        mx = fmax(mx, fabs(next));
      }
      const double inv = mx > 0.0 ? 1.0 / mx : 1.0;
      for (int i = 0; i < n; ++i) y[i] *= inv;
    }
  }
  __syncthreads();
  clk.mark(12);

  // 4. Back-transformation y <- H_0 ... H_{n-3} y (warp 0, y in registers:
  //    lane holds y[lane + 32q]).
  if (warp == 0) {
    constexpr int QY = (kMaxK + 1 + 31) / 32;
    double yr[QY];
#pragma unroll
    for (int q = 0; q < QY; ++q) {
      const int t = lane + 32 * q;
      yr[q] = t < n ? ws.y[t] : 0.0;
    }
    for (int j = n - 3; j >= 0; --j) {
      const double bet = ws.beta[j];
      if (bet == 0.0) continue;
      const double* hvj = A + j * lda;  // v_j[i] at hvj[j + 1 + i]
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < QY; ++q) {
        const int t = lane + 32 * q;
        if (t > j && t < n) s = fma(hvj[t], yr[q], s);
      }
      s = __shfl_sync(~0u, warp_sum(s), 0) * bet;
#pragma unroll
      for (int q = 0; q < QY; ++q) {
        const int t = lane + 32 * q;
        if (t > j && t < n) yr[q] -= s * hvj[t];
      }
    }
#pragma unroll
    for (int q = 0; q < QY; ++q) {
      const int t = lane + 32 * q;
      if (t < n) ws.y[t] = yr[q];
    }
  }
  __syncthreads();
}

}  // namespace mcd
