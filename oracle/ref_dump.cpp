// Golden-vector dump driver for the mCDFCI oracle.
//
// TEST INFRASTRUCTURE ONLY.  This file is compiled by oracle/Makefile against
// the reference's own headers (src/run_wrapper.h and what it includes); it is
// never linked into the product.  It calls the reference classes directly and
// prints what they compute, so the fixtures under tests/golden/ come from the
// reference itself rather than from a restatement:
//
//   columns  HamiltonianMolecule<N>::get_column / get_diagonal
//            (src/hamiltonian.h:252-272, 336-424) for a random walk of
//            determinants starting at get_hartree_fock (src/hamiltonian.h:469-492)
//   hsub     CDFCI<N>::get_hamiltonian_submatrix (src/solver.h:637-670)
//   eig      CoordinateUpdateEig<N>::operator() (src/solver.h:333-609), captured
//            inside a real CDFCI<N>::solve run (src/solver.h:672-893)
//
// Determinants are printed as the reference stores them: N 64-bit words of the
// interleaved spin-orbital string (bit 2p = alpha p, bit 2p+1 = beta p,
// src/input.h:242-243).  Doubles are printed with 17 significant digits, which
// round-trips exactly.  __float128 scalars are printed as an unevaluated pair
// (hi, lo) of doubles.
#include "run_wrapper.h"

#include <cstdio>
#include <random>
#include <set>
#include <string>
#include <vector>

namespace {

template <int N>
void put_det(FILE* f, const Determinant<N>& d) {
  fputc('[', f);
  for (int t = 0; t < N; ++t)
    fprintf(f, "%s%llu", t ? ", " : "", (unsigned long long)d.repr[t]);
  fputc(']', f);
}

void put_q(FILE* f, QUAD_PRECISION q) {
  double hi = (double)q;
  double lo = (double)(q - (QUAD_PRECISION)hi);
  fprintf(f, "[%.17g, %.17g]", hi, lo);
}

template <int N>
std::vector<Determinant<N>> random_walk(HamiltonianMolecule<N>& h,
                                        unsigned seed, int ndets) {
  std::mt19937_64 rng(seed);
  std::vector<Determinant<N>> dets;
  std::set<std::array<size_t, N>> seen;
  Determinant<N> cur = h.get_hartree_fock();
  dets.push_back(cur);
  seen.insert(cur.repr);
  int guard = 0;
  while ((int)dets.size() < ndets && guard++ < 100000) {
    DeterminantDecoded<N> dec(cur);
    auto col = h.get_column(dec);
    if (col.size() < 2) break;
    size_t j = 1 + rng() % (col.size() - 1);
    cur = col[j].first;
    if (seen.insert(cur.repr).second) dets.push_back(cur);
  }
  return dets;
}

template <int N>
int dump_columns(Fcidump& fci, double thr, unsigned seed, int ndets,
                 FILE* f) {
  HamiltonianMolecule<N> h(fci, thr);
  Determinant<N>::constuct_masks();
  auto dets = random_walk<N>(h, seed, ndets);
  fprintf(f, "{\"norb\": %d, \"nelec\": %d, \"ms2\": %d, \"n_words\": %d,\n",
          fci.norb, fci.nelec, fci.ms2, N);
  fprintf(f, "\"hf\": ");
  put_det<N>(f, h.get_hartree_fock());
  fprintf(f, ",\n\"dets\": [\n");
  for (size_t d = 0; d < dets.size(); ++d) {
    DeterminantDecoded<N> dec(dets[d]);
    auto col = h.get_column(dec);
    fprintf(f, "{\"det\": ");
    put_det<N>(f, dets[d]);
    fprintf(f, ", \"diag\": %.17g, \"col\": [", h.get_diagonal(dec));
    for (size_t e = 0; e < col.size(); ++e) {
      fprintf(f, "%s[", e ? ", " : "");
      put_det<N>(f, col[e].first);
      fprintf(f, ", %.17g]", col[e].second);
    }
    fprintf(f, "]}%s\n", d + 1 < dets.size() ? "," : "");
  }
  fprintf(f, "]}\n");
  return 0;
}

template <int N>
int dump_hsub(Fcidump& fci, double thr, unsigned seed, int k, int nsets,
              FILE* f) {
  HamiltonianMolecule<N> h(fci, thr);
  Determinant<N>::constuct_masks();
  // A long walk gives a pool of mutually close determinants, so most pairs
  // in a set are singles or doubles of each other.
  auto pool = random_walk<N>(h, seed, 4 * k);
  std::mt19937_64 rng(seed + 17);
  Option opt = Option::object();
  CDFCI<N> solver(opt);
  fprintf(f, "{\"norb\": %d, \"n_words\": %d, \"sets\": [\n", fci.norb, N);
  for (int s = 0; s < nsets; ++s) {
    std::vector<size_t> idx(pool.size());
    for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
    std::shuffle(idx.begin(), idx.end(), rng);
    int kk = std::min<int>(k, (int)pool.size());
    WaveFunctionVector<N> picked;
    for (int i = 0; i < kk; ++i)
      picked.data.push_back({pool[idx[i]], {0.0, 0.0}});
    std::vector<double> H(kk * kk);
    solver.get_hamiltonian_submatrix(h, picked, H.data());
    fprintf(f, "{\"dets\": [");
    for (int i = 0; i < kk; ++i) {
      if (i) fprintf(f, ", ");
      put_det<N>(f, picked.data[i].first);
    }
    fprintf(f, "], \"hsub\": [");
    for (int i = 0; i < kk * kk; ++i)
      fprintf(f, "%s%.17g", i ? ", " : "", H[i]);
    fprintf(f, "]}%s\n", s + 1 < nsets ? "," : "");
  }
  fprintf(f, "]}\n");
  return 0;
}

// Records the inputs and outputs of selected calls of the reference's eig
// update while a real solve runs.
template <int N>
class DumpingEig : public CoordinateUpdateEig<N> {
 public:
  FILE* f = nullptr;
  std::set<long> which;
  long calls = 0;
  int written = 0;

  std::vector<double> operator()(double* H_sub, WaveFunction<N>& xz,
                                 WaveFunctionVector<N>& sub) override {
    const bool dump = which.count(calls) > 0;
    const int k = (int)sub.data.size();
    std::vector<double> H(H_sub, H_sub + k * k);
    QUAD_PRECISION xx0 = xz.xx(), xz0 = xz.xz(), sc0 = xz.scale();
    std::vector<double> x(k), z(k);
    for (int i = 0; i < k; ++i) {
      x[i] = sub.data[i].second[0];
      z[i] = sub.data[i].second[1];
    }
    auto res = CoordinateUpdateEig<N>::operator()(H_sub, xz, sub);
    if (dump) {
      fprintf(f, "%s{\"call\": %ld, \"k\": %d, \"hsub\": [", written ? ",\n" : "",
              calls, k);
      for (int i = 0; i < k * k; ++i) fprintf(f, "%s%.17g", i ? ", " : "", H[i]);
      fprintf(f, "], \"x\": [");
      for (int i = 0; i < k; ++i) fprintf(f, "%s%.17g", i ? ", " : "", x[i]);
      fprintf(f, "], \"z\": [");
      for (int i = 0; i < k; ++i) fprintf(f, "%s%.17g", i ? ", " : "", z[i]);
      fprintf(f, "], \"xx\": ");
      put_q(f, xx0);
      fprintf(f, ", \"xz\": ");
      put_q(f, xz0);
      fprintf(f, ", \"scale\": ");
      put_q(f, sc0);
      fprintf(f, ", \"dx\": [");
      for (int i = 0; i < k; ++i) fprintf(f, "%s%.17g", i ? ", " : "", res[i]);
      fprintf(f, "], \"new_xx\": ");
      put_q(f, xz.xx());
      fprintf(f, ", \"new_scale\": ");
      put_q(f, xz.scale());
      fprintf(f, "}");
      ++written;
    }
    ++calls;
    return res;
  }
};

// Mirrors the sizing in run_cdfci_wrapper (src/run_wrapper.h:203-213) and the
// wiring in run_cdfci<N> (src/run_wrapper.h:124-173), with the eig functor
// swapped for the recording subclass above.
template <int N>
int dump_eig(Option& option, Fcidump& fci, const std::vector<long>& which,
             FILE* f) {
  int n = N;
  int bytes_per_det = n * 8 + 16;
  size_t cap = 8;
  double max_memory = option["solver"]["cdfci"]["max_memory"];
  while (cap * bytes_per_det < max_memory * 1073741824) cap *= 2;
  cap /= 2;
  option["solver"]["cdfci"]["max_wavefunction_size"] =
      static_cast<size_t>(0.79 * cap);
  HamiltonianMolecule<N> h(fci, option["hamiltonian"]["threshold"]);
  Option cdfci_option = option["solver"]["cdfci"];
  CDFCI<N> solver(cdfci_option);
  CoordinatePickGcdGrad<N> pick;
  DumpingEig<N> upd;
  upd.f = f;
  upd.which.insert(which.begin(), which.end());
  Determinant<N>::constuct_masks();
  int k = option["solver"]["cdfci"]["num_of_coordinate"];
  int m = option["solver"]["cdfci"]["estimate"];
  fprintf(f, "{\"calls\": [\n");
  solver.solve(h, pick, upd, k, m);
  fprintf(f, "],\n\"energy\": %.17g}\n", solver.result_energy);
  return 0;
}

int usage() {
  fprintf(stderr,
          "usage: ref_dump columns FCIDUMP THRESHOLD SEED NDETS OUT\n"
          "       ref_dump hsub FCIDUMP THRESHOLD SEED K NSETS OUT\n"
          "       ref_dump eig INPUT.json OUT CALL [CALL ...]\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) return usage();
  std::string mode = argv[1];
  try {
    if (mode == "columns" && argc == 7) {
      Fcidump fci(argv[2]);
      FILE* f = fopen(argv[6], "w");
      int nw = 1 + (fci.norb - 1) / 64;
      int rc = nw == 1 ? dump_columns<1>(fci, atof(argv[3]), atoi(argv[4]), atoi(argv[5]), f)
                       : dump_columns<2>(fci, atof(argv[3]), atoi(argv[4]), atoi(argv[5]), f);
      fclose(f);
      return rc;
    }
    if (mode == "hsub" && argc == 8) {
      Fcidump fci(argv[2]);
      FILE* f = fopen(argv[7], "w");
      int nw = 1 + (fci.norb - 1) / 64;
      int rc = nw == 1 ? dump_hsub<1>(fci, atof(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]), f)
                       : dump_hsub<2>(fci, atof(argv[3]), atoi(argv[4]), atoi(argv[5]), atoi(argv[6]), f);
      fclose(f);
      return rc;
    }
    if (mode == "eig" && argc >= 5) {
      Option option = read_input(argv[2]);
      Fcidump fci(option["hamiltonian"]["fcidump_path"]);
      std::vector<long> which;
      for (int i = 4; i < argc; ++i) which.push_back(atol(argv[i]));
      FILE* f = fopen(argv[3], "w");
      int nw = 1 + (fci.norb - 1) / 64;
      int rc = nw == 1 ? dump_eig<1>(option, fci, which, f)
                       : dump_eig<2>(option, fci, which, f);
      fclose(f);
      return rc;
    }
  } catch (const std::exception& e) {
    fprintf(stderr, "ERROR: %s\n", e.what());
    return 1;
  }
  return usage();
}
