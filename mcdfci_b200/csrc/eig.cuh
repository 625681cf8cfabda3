// Smallest eigenpair of a small dense symmetric FP64 matrix, computed by one
// CTA of 1024 threads in shared memory.
//
// The reference calls LAPACK dsyevr (IL=IU=1) and refines the vector with one
// step of __float128 inverse iteration through dgetrf (src/solver.h:400-503).
// Here, for n <= kMaxK+1:
//   1. Householder reduction to tridiagonal T = Q^T A Q (Golub & Van Loan,
//      Algorithm 8.3.1), one reflector per step with the rank-2 update spread
//      over the CTA;
//   2. the lowest eigenvalue of T isolated by 1024-way multisection with Sturm
//      counts (each thread evaluates one shift), three rounds;
//   3. inverse iteration on T - sigma I (sigma at the lower end of the isolating
//      interval, so the matrix is positive definite and needs no pivoting);
//   4. back-transformation v = Q y with the stored reflectors.
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
  double* hv;    // [n] current reflector
  double* p;     // [n]
  double* y;     // [n] eigenvector (output)
  double* part;  // [32] per-warp partials
  double* scal;  // [8] scalars
  int* ibest;    // [1]
};

// Block-wide.  On return ws.y[0..n) holds an (unnormalised) eigenvector of the
// lowest eigenvalue of the matrix originally in ws.A; ws.A is overwritten.
__device__ void smallest_eigvec(EigScratch& ws, int n, SectionClock& clk) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int NT = blockDim.x;
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
    if (warp == 0) {
      double s = 0.0;
      for (int i = 1 + lane; i < m; i += 32) {
        const double v = A[(j + 1 + i) * lda + j];
        s += v * v;
      }
      s = warp_sum(s);
      if (lane == 0) {
        const double x0 = A[(j + 1) * lda + j];
        double bet = 0.0, v0 = 1.0, mu = x0;
        if (s != 0.0) {
          mu = sqrt(x0 * x0 + s);
          v0 = (x0 <= 0.0) ? x0 - mu : -s / (x0 + mu);
          bet = 2.0 * v0 * v0 / (s + v0 * v0);
        }
        ws.scal[0] = bet;
        ws.scal[1] = v0;
        ws.beta[j] = bet;
        ws.e[j] = mu;
        ws.d[j] = A[j * lda + j];
      }
    }
    __syncthreads();
    const double bet = ws.scal[0], v0 = ws.scal[1];
    if (bet == 0.0) continue;  // column already reduced; T keeps e[j] = x0
    const double inv_v0 = 1.0 / v0;
    for (int i = tid; i < m; i += NT) {
      const double h = (i == 0) ? 1.0 : A[(j + 1 + i) * lda + j] * inv_v0;
      ws.hv[i] = h;
    }
    __syncthreads();
    double wp = 0.0;
    for (int r = warp; r < m; r += 32) {
      const double* row = A + (j + 1 + r) * lda + (j + 1);
      double s = 0.0;
      for (int c = lane; c < m; c += 32) s += row[c] * ws.hv[c];
      s = warp_sum(s);
      const double pr = bet * s;
      if (lane == 0) ws.p[r] = pr;
      wp += pr * ws.hv[r];
    }
    if (lane == 0) ws.part[warp] = wp;
    __syncthreads();
    double ptv = 0.0;
    for (int w = 0; w < 32; ++w) ptv += ws.part[w];
    const double K = 0.5 * bet * ptv;
    for (int idx = tid; idx < m * m; idx += NT) {
      const int r = idx / m, c = idx - r * m;
      const double hr = ws.hv[r], hc = ws.hv[c];
      const double wr = ws.p[r] - K * hr, wc = ws.p[c] - K * hc;
      A[(j + 1 + r) * lda + (j + 1 + c)] -= hr * wc + wr * hc;
    }
    for (int i = tid; i < m; i += NT) A[(j + 1 + i) * lda + j] = ws.hv[i];
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
    double lo = 1e300, hi = -1e300, emax = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double em = (i > 0) ? fabs(ws.e[i - 1]) : 0.0;
      const double ep = (i < n - 1) ? fabs(ws.e[i]) : 0.0;
      lo = fmin(lo, ws.d[i] - em - ep);
      hi = fmax(hi, ws.d[i] + em + ep);
      if (i < n - 1) {
        ws.e2[i] = ws.e[i] * ws.e[i];
        emax = fmax(emax, ws.e2[i]);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(~0u, lo, o));
      hi = fmax(hi, __shfl_xor_sync(~0u, hi, o));
      emax = fmax(emax, __shfl_xor_sync(~0u, emax, o));
    }
    if (lane == 0) {
      const double widen = 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300;
      ws.scal[2] = lo - widen;
      ws.scal[3] = hi + widen;
      ws.scal[4] = 2.2250738585072014e-308 * fmax(1.0, emax);  // pivmin
    }
  }
  __syncthreads();
  const double pivmin = ws.scal[4];
  for (int round = 0; round < 3; ++round) {
    const double lo = ws.scal[2], hi = ws.scal[3];
    if (tid == 0) *ws.ibest = NT;
    __syncthreads();
    const double sig = lo + (hi - lo) * (static_cast<double>(tid + 1) / static_cast<double>(NT + 1));
    double q = ws.d[0] - sig;
    if (fabs(q) < pivmin) q = -pivmin;
    int cnt = q < 0.0;
    for (int i = 1; i < n; ++i) {
      q = (ws.d[i] - sig) - ws.e2[i - 1] / q;
      if (fabs(q) < pivmin) q = -pivmin;
      cnt += q < 0.0;
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

  // 3. Inverse iteration on T - sigma I (thread 0; u and l reuse hv and p).
  if (tid == 0) {
    const double sigma = ws.scal[2];
    const double tiny = 1e-290;
    double* ru = ws.hv;  // 1 / u_i
    double* l = ws.p;
    double u = ws.d[0] - sigma;
    if (fabs(u) < tiny) u = tiny;
    ru[0] = 1.0 / u;
    for (int i = 1; i < n; ++i) {
      l[i] = ws.e[i - 1] * ru[i - 1];
      u = (ws.d[i] - sigma) - l[i] * ws.e[i - 1];
      if (fabs(u) < tiny) u = tiny;
      ru[i] = 1.0 / u;
    }
    double* y = ws.y;
    for (int i = 0; i < n; ++i) y[i] = 1.0 + 0.0625 * static_cast<double>((7 * i + 3) % 11);
    for (int it = 0; it < 3; ++it) {
      for (int i = 1; i < n; ++i) y[i] -= l[i] * y[i - 1];
      y[n - 1] *= ru[n - 1];
      for (int i = n - 2; i >= 0; --i) y[i] = (y[i] - ws.e[i] * y[i + 1]) * ru[i];
      double mx = 0.0;
      for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(y[i]));
      const double inv = mx > 0.0 ? 1.0 / mx : 1.0;
      for (int i = 0; i < n; ++i) y[i] *= inv;
    }
  }
  __syncthreads();

  clk.mark(12);

  // 4. Back-transformation y <- H_0 ... H_{n-3} y (warp 0).
  if (warp == 0) {
    for (int j = n - 3; j >= 0; --j) {
      const double bet = ws.beta[j];
      if (bet == 0.0) continue;
      const int m = n - j - 1;
      double s = 0.0;
      for (int i = lane; i < m; i += 32) s += A[(j + 1 + i) * lda + j] * ws.y[j + 1 + i];
      s = warp_sum(s) * bet;
      for (int i = lane; i < m; i += 32) ws.y[j + 1 + i] -= s * A[(j + 1 + i) * lda + j];
      __syncwarp();
    }
  }
  __syncthreads();
}

}  // namespace mcd
