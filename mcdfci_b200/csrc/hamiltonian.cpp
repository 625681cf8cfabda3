// Table construction.  Every value is formed from the spin-orbital integrals
// G(i,j,a,b) = <ij|ab> (0 when absent, and only for i <= j, as the reference's
// map) with the same floating-point expression the reference uses, so table
// entries are bit-identical to the reference's excitation lists:
//
//   same-spin double  <ij||ab> = G(i,j,a,b) - G(i,j,b,a), i<j, a<b
//                     (construct_double_excitation, src/hamiltonian.h:142-162;
//                      an entry present only as (b,a) is stored as -G(i,j,b,a),
//                      which equals 0 - G(i,j,b,a))
//   opposite-spin     G(i,j,a,b) for the interleaved-ordered pair i<j, with a of
//                     i's spin and b of j's spin (src/hamiltonian.h:135-141)
//   single            <i|h|a> and <ik||ak> = G(i,k,a,k) - G(i,k,k,a) (i <= k) or
//                     G(k,i,k,a) - G(k,i,a,k) (i > k)  (src/hamiltonian.h:176-210)
//   diagonal          <i|h|i>, <ij||ij> = G(i,j,i,j) - G(i,j,j,i)  (:226-245)
//
// Layout for the kernels (spatial indices p,q,r,s; spin s = 0 alpha, 1 beta):
//   vss[s][P(p,q)][P(r,s)]  same-spin double p,q -> r,s (p<q, r<s), P(p,q) = q(q-1)/2+p
//   wab[pa][pb][ra][sb]     alpha pa->ra together with beta pb->sb
//   sh[s][p][r], st[s][p][r][k]  single p->r of spin s; k runs over spin-orbitals
#include "hamiltonian.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <unistd.h>
#include <cmath>
#include <stdexcept>
#include <thread>
#include <vector>

namespace mcd {

namespace {

// A pool of up to 15 worker threads, started on first use and kept for the
// process: run(n, f) calls f(i) for every i in [0, n) on the workers and the
// calling thread, each taking the next unclaimed i from a shared counter (the
// tasks differ in cost), and returns when all are done.  Every i writes its
// own part of the tables, so no two threads share one.  Calls from several
// threads take turns.  A process forked from one that started the pool has
// none of its threads, so it starts a pool of its own.
class TaskPool {
 public:
  static TaskPool& get() {
    static std::mutex mu;
    static TaskPool* pool = nullptr;  // kept to the end of the process, like its threads
    static pid_t owner = 0;
    std::lock_guard<std::mutex> lk(mu);
    if (!pool || owner != getpid()) {
      pool = new TaskPool();
      owner = getpid();
    }
    return *pool;
  }
  void run(int n, const std::function<void(int)>& f) {
    std::lock_guard<std::mutex> turn(run_mu_);
    if (workers_ == 0 || n <= 1) {
      for (int i = 0; i < n; ++i) f(i);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      job_ = &f;
      n_ = n;
      next_.store(0);
      busy_ = workers_;
      ++gen_;
    }
    cv_.notify_all();
    work(f, n);
    std::unique_lock<std::mutex> lk(mu_);
    done_cv_.wait(lk, [&] { return busy_ == 0; });
    job_ = nullptr;
  }

 private:
  TaskPool() {
    const int hw = static_cast<int>(std::thread::hardware_concurrency());
    workers_ = std::max(0, std::min(hw > 0 ? hw : 1, 16) - 1);
    for (int t = 0; t < workers_; ++t) std::thread([this] { loop(); }).detach();
  }
  void work(const std::function<void(int)>& f, int n) {
    for (int i = next_.fetch_add(1); i < n; i = next_.fetch_add(1)) f(i);
  }
  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      const std::function<void(int)>* f;
      int n;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen; });
        seen = gen_;
        f = job_;
        n = n_;
      }
      work(*f, n);
      std::lock_guard<std::mutex> lk(mu_);
      if (--busy_ == 0) done_cv_.notify_one();
    }
  }
  std::mutex run_mu_, mu_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(int)>* job_ = nullptr;
  int n_ = 0, busy_ = 0, workers_ = 0;
  unsigned long long gen_ = 0;
  std::atomic<int> next_{0};
};

}  // namespace

HamHost build_hamiltonian(const Fcidump& fci, double thr) {
  if (!(thr >= 0.0)) throw std::invalid_argument("hamiltonian:threshold must be >= 0.");
  if (fci.norb % 2) throw std::invalid_argument("an odd number of spin-orbitals is not supported.");
  HamHost h;
  const int nso = fci.norb;
  const int n = nso / 2;
  h.norb = n;
  h.nso = nso;
  h.npair = n * (n - 1) / 2;
  h.ecore = fci.core_energy;

  auto spin = [](int so) { return so & 1; };
  auto sp = [](int so) { return so >> 1; };

  // Reject couplings between alpha and beta spin-orbitals (an RHF file's
  // expansion has none; UHF files and arrays from the C ABI are checked).
  for (int i = 0; i < nso && !fci.spin_conserving; ++i)
    for (int a = 0; a < nso; ++a)
      if (spin(i) != spin(a) && std::fabs(fci.h(i, a)) > thr)
        throw std::invalid_argument("one-electron integrals couple alpha and beta spin-orbitals.");
  for (int i = 0; i < nso && !fci.spin_conserving; ++i)
    for (int j = i; j < nso; ++j)
      for (int a = 0; a < nso; ++a)
        for (int b = 0; b < nso; ++b) {
          const double v = fci.g(i, j, a, b);
          if (v != 0.0 && (spin(i) != spin(a) || spin(j) != spin(b)) && std::fabs(v) > thr)
            throw std::invalid_argument("two-electron integrals couple alpha and beta spin-orbitals.");
        }

  h.hdiag.resize(nso);
  for (int i = 0; i < nso; ++i) h.hdiag[i] = fci.h(i, i);
  h.d2.assign(static_cast<size_t>(nso) * nso, 0.0);
  for (int i = 0; i < nso; ++i)
    for (int j = i + 1; j < nso; ++j) h.d2[i * nso + j] = fci.g(i, j, i, j) - fci.g(i, j, j, i);

  // Singles, same-spin and opposite-spin doubles: one pool of tasks, the
  // most expensive (opposite-spin rows) first.  Every task writes each entry
  // of its rows (0 where the value is not above the threshold), so the
  // tables need no clearing first.
  const size_t np = static_cast<size_t>(h.npair);
  h.sh.resize(2 * static_cast<size_t>(n) * n);
  h.st.resize(2 * static_cast<size_t>(n) * n * nso);
  h.spres.assign(2 * static_cast<size_t>(n), 0);
  h.vss.resize(2 * np * np);
  h.wab.resize(static_cast<size_t>(n) * n * n * n);
  // Single excitations p -> r of spin s, every r.
  auto singles = [&](int s, int p) {
    uint64_t pres = 0;
    for (int r = 0; r < n; ++r) {
      const int i = 2 * p + s, a = 2 * r + s;
      const double one = fci.h(i, a);
      double maxv = std::fabs(one);
      double* t = &h.st[((static_cast<size_t>(s) * n + p) * n + r) * nso];
      for (int k = 0; k < nso; ++k) {
        double v;
        if (i <= k)
          v = fci.g(i, k, a, k) - fci.g(i, k, k, a);
        else
          v = fci.g(k, i, k, a) - fci.g(k, i, a, k);
        t[k] = v;
        maxv = std::max(maxv, std::fabs(v));
      }
      h.sh[(static_cast<size_t>(s) * n + p) * n + r] = one;
      if (maxv > thr) pres |= 1ull << r;
    }
    h.spres[s * n + p] = pres;
  };
  // Same-spin doubles out of the pairs (p, q), p < q, of spin s: rows P(p, q).
  auto same_spin = [&](int s, int q) {
    for (int p = 0; p < q; ++p) {
      const int i = 2 * p + s, j = 2 * q + s;
      double* row = &h.vss[(s * np + pair_index(p, q)) * np];
      for (int ss = 1; ss < n; ++ss)
        for (int r = 0; r < ss; ++r) {
          const int a = 2 * r + s, b = 2 * ss + s;
          const double v = fci.g(i, j, a, b) - fci.g(i, j, b, a);
          row[pair_index(r, ss)] = std::fabs(v) > thr ? v : 0.0;
        }
    }
  };
  // Opposite-spin doubles out of alpha pa and beta pb: n x n entries.
  auto opposite_spin = [&](int pa, int pb) {
    double* blk = &h.wab[(static_cast<size_t>(pa) * n + pb) * n * n];
    for (int ra = 0; ra < n; ++ra)
      for (int sb = 0; sb < n; ++sb) {
        double v;
        if (pa <= pb)  // alpha pa (2pa) precedes beta pb (2pb+1)
          v = fci.g(2 * pa, 2 * pb + 1, 2 * ra, 2 * sb + 1);
        else
          v = fci.g(2 * pb + 1, 2 * pa, 2 * sb + 1, 2 * ra);
        blk[ra * n + sb] = std::fabs(v) > thr ? v : 0.0;
      }
  };
  const int n_ab = n * n, n_ss = 2 * n, n_s = 2 * n;
  TaskPool::get().run(n_ab + n_ss + n_s, [&](int t) {
    if (t < n_ab) {
      opposite_spin(t / n, t % n);
    } else if (t < n_ab + n_ss) {
      const int u = t - n_ab;
      same_spin(u / n, n - 1 - u % n);  // larger q (more pairs) first
    } else {
      const int u = t - n_ab - n_ss;
      singles(u / n, u % n);
    }
  });
  (void)sp;
  return h;
}

void host_parallel(int n, const std::function<void(int)>& f) { TaskPool::get().run(n, f); }

Det det_from_spin_orbitals(const std::vector<int>& occ) {
  Det d{0, 0};
  for (int so : occ) {
    if (so & 1)
      d.b |= 1ull << (so >> 1);
    else
      d.a |= 1ull << (so >> 1);
  }
  return d;
}

std::vector<int> det_spin_orbitals(const Det& d, int norb) {
  std::vector<int> occ;
  for (int p = 0; p < norb; ++p) {
    if ((d.a >> p) & 1) occ.push_back(2 * p);
    if ((d.b >> p) & 1) occ.push_back(2 * p + 1);
  }
  return occ;
}

Det hartree_fock(const Fcidump& fci, std::string* warning) {
  std::vector<std::pair<int, double>> sorted;
  if (fci.orbital_energy.empty()) {
    for (int i = 0; i < fci.norb; ++i) sorted.push_back({i, static_cast<double>(i)});
    if (warning) *warning = "Warning: no orbital energy found. Assume orbitals are sorted.";
  } else {
    for (const auto& e : fci.orbital_energy) sorted.push_back(e);
  }
  std::stable_sort(sorted.begin(), sorted.end(),
                   [](const auto& x, const auto& y) { return x.second < y.second; });
  const int n_alpha = (fci.nelec + fci.ms2) / 2;
  const int n_beta = (fci.nelec - fci.ms2) / 2;
  if (fci.nelec > static_cast<int>(sorted.size()))
    throw std::invalid_argument("NELEC exceeds the number of spin-orbitals with an orbital energy.");
  std::vector<int> occ;
  for (int i = 0, ia = 0, ib = 0; i < fci.nelec; ++i) {
    const int orb = sorted[i].first;
    if (orb % 2 == 0 && ia < n_alpha) {
      occ.push_back(orb);
      ++ia;
    } else if (orb % 2 == 1 && ib < n_beta) {
      occ.push_back(orb);
      ++ib;
    }
  }
  return det_from_spin_orbitals(occ);
}

Det ref_det_from_occ(const Fcidump& fci, const std::vector<int>& occ) {
  std::vector<int> valid;
  for (int o : occ)
    if (o >= 0 && o < fci.norb && std::find(valid.begin(), valid.end(), o) == valid.end()) valid.push_back(o);
  if (static_cast<int>(valid.size()) != fci.nelec)
    throw std::invalid_argument(
        "Reference determinant is invalid. The number of valid orbitals does not match the number of "
        "electrons. Please provide " +
        std::to_string(fci.nelec) + " orbitals from 0 to " + std::to_string(fci.norb - 1) +
        " or remove the argument.");
  return det_from_spin_orbitals(valid);
}

double diagonal_element(const HamHost& h, const Det& d) {
  const std::vector<int> occ = det_spin_orbitals(d, h.norb);
  double v = 0.0;
  for (size_t x = 0; x < occ.size(); ++x) {
    v += h.hdiag[occ[x]];
    for (size_t y = x + 1; y < occ.size(); ++y) v += h.d2[occ[x] * h.nso + occ[y]];
  }
  return v + h.ecore;
}

}  // namespace mcd
