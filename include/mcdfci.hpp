/*
 * C++ facades with the reference's interface names, over the C ABI of
 * mcdfci.h (header-only; link with -lmcdfci).  A host written against the
 * reference's classes keeps its names and call shapes:
 *
 *   Determinant        Determinant<N> (src/determinant.h:24-123) as an
 *                      (alpha, beta) pair, with the reference's interleaved
 *                      spin-orbital numbering for occupied_orbitals()
 *   Fcidump            Fcidump (src/input.h:57-152)
 *   Hamiltonian        Hamiltonian<N> (src/hamiltonian.h:25-54): get_diagonal,
 *                      get_off_diagonal, get_column, on the GPU tables
 *   WaveFunction       WaveFunction<N> (src/wavefunction.h:163-221): xx,
 *                      scale, xz, x_size, size of the GPU hash wavefunction
 *   CoordinatePickGcdGrad, CoordinateUpdateEig
 *                      CoordinatePick<N> / CoordinateUpdate<N>
 *                      (src/solver.h:94-101,230-250); the update's
 *                      operator() runs one subspace eigenproblem
 *   Solver, CDFCI      Solver (src/solver.h:613-619) and CDFCI<N>::solve
 *                      (src/solver.h:831-893)
 *
 * The reference templates these on N, the 64-bit words of a determinant;
 * here one type covers every N this library supports (up to 64 spatial
 * orbitals per spin).  Errors are thrown as mcdfci::Error (a
 * std::runtime_error carrying the MCD_* code), std::invalid_argument for bad
 * input and std::overflow_error for a full table, as the reference throws.
 */
#ifndef MCDFCI_HPP
#define MCDFCI_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mcdfci.h"

namespace mcdfci {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& what) : std::runtime_error(what), code(code) {}
  int code;
};

inline void check(int rc) {
  if (rc == MCD_OK || rc == MCD_STOPPED) return;
  const std::string msg = mcd_last_error();
  if (rc == MCD_ERR_INVALID) throw std::invalid_argument(msg);
  if (rc == MCD_ERR_OVERFLOW) throw std::overflow_error(msg);
  throw Error(rc, msg);
}

struct Determinant {
  uint64_t alpha = 0, beta = 0;  // bit p: spatial orbital p of that spin

  Determinant() = default;
  Determinant(uint64_t a, uint64_t b) : alpha(a), beta(b) {}
  // From spin-orbital indices in the reference's order (2p alpha, 2p+1 beta).
  static Determinant from_occupied(const std::vector<int>& occ) {
    Determinant d;
    for (int so : occ) (so & 1 ? d.beta : d.alpha) |= uint64_t{1} << (so >> 1);
    return d;
  }
  // DeterminantDecoded::occupied_orbitals (src/determinant.h:155-179).
  std::vector<int> occupied_orbitals() const {
    std::vector<int> out;
    for (int p = 0; p < 64; ++p) {
      if ((alpha >> p) & 1) out.push_back(2 * p);
      if ((beta >> p) & 1) out.push_back(2 * p + 1);
    }
    return out;
  }
  bool operator==(const Determinant& o) const { return alpha == o.alpha && beta == o.beta; }
};

class Fcidump {
 public:
  explicit Fcidump(const std::string& path) { check(mcd_fcidump_read(path.c_str(), &f_)); }
  ~Fcidump() { mcd_fcidump_free(f_); }
  Fcidump(const Fcidump&) = delete;
  Fcidump& operator=(const Fcidump&) = delete;
  mcd_problem problem() const {
    mcd_problem p;
    check(mcd_fcidump_problem(f_, &p));
    return p;
  }
  int norb() const { return problem().norb; }    // spin-orbitals, as the reference's Fcidump::norb
  int nelec() const { return problem().nelec; }
  const mcd_fcidump* handle() const { return f_; }

 private:
  mcd_fcidump* f_ = nullptr;
};

class Hamiltonian {
 public:
  explicit Hamiltonian(mcd_solver* s) : s_(s) {}
  double get_diagonal(const Determinant& d) const {
    double h = 0.0;
    check(mcd_debug_hsub(s_, &d.alpha, &d.beta, 1, &h));
    return h;
  }
  // <d2|H|d1>, computed from d1's side as the reference's get_off_diagonal(d1, d2).
  double get_off_diagonal(const Determinant& d1, const Determinant& d2) const {
    const uint64_t a[2] = {d1.alpha, d2.alpha}, b[2] = {d1.beta, d2.beta};
    double h[4];
    check(mcd_debug_hsub(s_, a, b, 2, h));
    return h[1];
  }
  // get_column (src/hamiltonian.h:412-424): the diagonal and every stored
  // single and double excitation with its matrix element.
  std::vector<std::pair<Determinant, double>> get_column(const Determinant& d) const {
    int64_t n = 0;
    check(mcd_debug_column(s_, d.alpha, d.beta, nullptr, nullptr, nullptr, 0, &n));
    std::vector<uint64_t> a(static_cast<size_t>(n)), b(static_cast<size_t>(n));
    std::vector<double> v(static_cast<size_t>(n));
    check(mcd_debug_column(s_, d.alpha, d.beta, a.data(), b.data(), v.data(), n, &n));
    std::vector<std::pair<Determinant, double>> out;
    out.reserve(a.size());
    for (size_t i = 0; i < a.size(); ++i) out.push_back({Determinant(a[i], b[i]), v[i]});
    return out;
  }

 private:
  mcd_solver* s_;
};

class WaveFunction {
 public:
  explicit WaveFunction(mcd_solver* s) : s_(s) {}
  // The scalars in double-double, returned as long double (the reference
  // keeps them in __float128).
  long double xx() const { return scalar(0); }
  long double scale() const { return scalar(1); }
  long double xz() const { return scalar(2); }
  size_t x_size() const { return report().x_size; }
  size_t size() const { return report().occupied; }
  // The determinants with nonzero x and their x (coefficients are scale * x).
  std::vector<std::pair<Determinant, double>> x() const {
    int64_t n = 0;
    check(mcd_debug_wavefunction(s_, nullptr, nullptr, nullptr, 0, &n));
    std::vector<uint64_t> a(static_cast<size_t>(n)), b(static_cast<size_t>(n));
    std::vector<double> v(static_cast<size_t>(n));
    check(mcd_debug_wavefunction(s_, a.data(), b.data(), v.data(), n, &n));
    std::vector<std::pair<Determinant, double>> out;
    for (size_t i = 0; i < a.size(); ++i) out.push_back({Determinant(a[i], b[i]), v[i]});
    return out;
  }

 private:
  long double scalar(int i) const {
    double v[3][2];
    int64_t it = 0;
    check(mcd_scalars(s_, v[0], v[1], v[2], &it));
    return static_cast<long double>(v[i][0]) + static_cast<long double>(v[i][1]);
  }
  mcd_report report() const {
    mcd_report r;
    check(mcd_get_report(s_, &r));
    return r;
  }
  mcd_solver* s_;
};

struct CoordinatePickGcdGrad {
  int method() const { return MCD_PICK_GCD_GRAD; }
};

struct CoordinateUpdateEig {
  int method() const { return MCD_UPDATE_EIG; }
  // CoordinateUpdateEig::operator() (src/solver.h:333-609) on one subproblem:
  // H_sub (k x k, row-major, its upper triangle read), the picked x and z,
  // the wavefunction's xx and xz; returns dx, and the new xx and scale.
  std::vector<double> operator()(const std::vector<double>& h_sub, const std::vector<double>& x,
                                 const std::vector<double>& z, long double xx, long double xz,
                                 long double* new_xx = nullptr, long double* new_scale = nullptr) const {
    const int32_t k = static_cast<int32_t>(x.size());
    if (z.size() != x.size() || h_sub.size() != x.size() * x.size())
      throw std::invalid_argument("H_sub must be k x k and z must have k elements.");
    const double xxp[2] = {static_cast<double>(xx), static_cast<double>(xx - static_cast<double>(xx))};
    const double xzp[2] = {static_cast<double>(xz), static_cast<double>(xz - static_cast<double>(xz))};
    std::vector<double> dx(x.size());
    double nxx[2], nsc[2];
    int32_t branch = 0;
    check(mcd_debug_eig(k, h_sub.data(), x.data(), z.data(), xxp, xzp, dx.data(), nxx, nsc, &branch));
    if (new_xx) *new_xx = static_cast<long double>(nxx[0]) + nxx[1];
    if (new_scale) *new_scale = static_cast<long double>(nsc[0]) + nsc[1];
    return dx;
  }
};

class Solver {
 public:
  virtual ~Solver() = default;
  double result_energy = 0.0;
};

// CDFCI<N> over one GPU solver: created from the FCIDUMP and the solver
// options (mcd_options, with the reference's defaults from
// mcd_options_default), it owns the Hamiltonian tables and the wavefunction.
class CDFCI : public Solver {
 public:
  CDFCI(const Fcidump& fci, const mcd_options& option) : option_(option) {
    check(mcd_create_from_fcidump(fci.handle(), &option_, &s_));
  }
  ~CDFCI() override { mcd_destroy(s_); }
  CDFCI(const CDFCI&) = delete;
  CDFCI& operator=(const CDFCI&) = delete;

  Hamiltonian hamiltonian() const { return Hamiltonian(s_); }
  WaveFunction wavefunction() const { return WaveFunction(s_); }

  // CDFCI<N>::solve(h, pick, update, k, m) (src/solver.h:831-893): k and m
  // are those the solver was created with (num_of_coordinate, estimate).
  int solve(const Hamiltonian&, const CoordinatePickGcdGrad&, const CoordinateUpdateEig&, int k, int m) {
    if (k != option_.num_of_coordinate || m != option_.estimate)
      throw std::invalid_argument("k and m must be the solver's num_of_coordinate and estimate.");
    const int rc = mcd_solve(s_, nullptr, nullptr);
    check(rc);
    check(mcd_result(s_, &result_energy));
    return rc == MCD_OK ? 0 : rc;
  }
  mcd_solver* handle() const { return s_; }

 private:
  mcd_options option_;
  mcd_solver* s_ = nullptr;
};

}  // namespace mcdfci

#endif  // MCDFCI_HPP
