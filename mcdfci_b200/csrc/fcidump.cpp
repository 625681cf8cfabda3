// FCIDUMP reader.  Behaviour follows the reference reader (src/input.h:88-338):
//  * header = the lines before the first line containing "&END" or "/";
//    NORB, NELEC, MS2 are required, UHF optional (default .FALSE. with a warning);
//  * the body is read as whitespace-separated records "value i a j b" until the
//    first record that does not parse;
//  * i,a,j,b all non-zero: two-electron <ij|ab> = (ia|jb), inserted for the
//    four index permutations <ij|ab>, <ib|aj>, <aj|ib>, <ab|ij>, each stored
//    under the ordered key (min, max) with the pair swapped when i > j; for RHF
//    every permutation is expanded to the alpha-alpha, beta-beta, alpha-beta and
//    beta-alpha spin-orbital blocks.  The first value stored for a key wins;
//  * a non-zero (and not all four non-zero): one-electron <i|h|a>, written
//    symmetrically (later lines overwrite);
//  * only i non-zero: orbital energy of i (first value wins);
//  * all zero: core energy (later lines overwrite).
#include "fcidump.h"

#include <fstream>
#include <iostream>
#include <regex>
#include <sstream>

namespace mcd {
namespace {

struct Builder {
  Fcidump& d;
  explicit Builder(Fcidump& dd) : d(dd) {}

  void alloc() {
    const size_t n = static_cast<size_t>(d.norb);
    d.h1.assign(n * n, 0.0);
    d.g2.assign(n * n * n * n, 0.0);
    d.g2_set.assign(n * n * n * n, 0);
  }

  void put(int i, int j, int a, int b, double v) {
    const size_t n = static_cast<size_t>(d.norb);
    const size_t idx = ((static_cast<size_t>(i) * n + j) * n + a) * n + b;
    if (!d.g2_set[idx]) {
      d.g2[idx] = v;
      d.g2_set[idx] = 1;
    }
  }

  // Keeps i <= j; when i == j both orders are stored.
  void insert(int i, int j, int a, int b, double v) {
    if (i <= j) put(i, j, a, b, v);
    if (i >= j) put(j, i, b, a, v);
  }

  static int alpha(int i) { return 2 * i - 2; }
  static int beta(int i) { return 2 * i - 1; }

  void rhf_insert(int i, int j, int a, int b, double v) {
    insert(alpha(i), alpha(j), alpha(a), alpha(b), v);
    insert(beta(i), beta(j), beta(a), beta(b), v);
    insert(alpha(i), beta(j), alpha(a), beta(b), v);
    insert(beta(i), alpha(j), beta(a), alpha(b), v);
  }
};

int read_int_param(const std::string& header, const std::string& name) {
  std::regex r(name + R"([ ]*=[ ]*(\d+))");
  std::smatch m;
  if (!std::regex_search(header, m, r)) throw std::invalid_argument(name + " is not found.");
  return std::stoi(m[1].str());
}

bool read_uhf_param(const std::string& header) {
  std::regex r(R"(UHF[ ]*=[ .]*(FALSE|TRUE))");
  std::smatch m;
  if (!std::regex_search(header, m, r)) {
    std::cerr << "Warning: FCIDUMP optional parameter UHF is not found. Use default value 0."
              << std::endl
              << std::endl;
    return false;
  }
  return m[1].str() == "TRUE";
}

}  // namespace

Fcidump read_fcidump(const std::string& path) {
  Fcidump d;
  try {
    std::ifstream f(path);
    if (f.fail()) throw std::invalid_argument("Failed to open the FCIDUMP file " + path);
    std::string header, line;
    while (std::getline(f, line) && line.find("&END") == std::string::npos &&
           line.find("/") == std::string::npos) {
      header += " ";
      header += line;
    }
    header += " &END";
    if (f.eof()) throw std::invalid_argument("FCIDUMP has the wrong header.");

    d.norb = read_int_param(header, "NORB");
    d.nelec = read_int_param(header, "NELEC");
    d.ms2 = read_int_param(header, "MS2");
    d.uhf = read_uhf_param(header);
    d.spin_conserving = !d.uhf;  // rhf_insert writes alpha-alpha and beta-beta pairs only
    const int nfile = d.norb;  // largest index allowed in the body
    if (!d.uhf) d.norb *= 2;
    if (d.norb <= 0 || d.norb > 2 * kMaxOrb)
      throw std::invalid_argument("NORB outside the supported range 1.." +
                                  std::to_string(d.uhf ? 2 * kMaxOrb : kMaxOrb) + ".");
    Builder b(d);
    b.alloc();

    double v;
    int i, a, j, bb;
    while (f >> v >> i >> a >> j >> bb) {
      if (i < 0 || a < 0 || j < 0 || bb < 0 || i > nfile || a > nfile || j > nfile || bb > nfile)
        throw std::invalid_argument("integral index outside 0.." + std::to_string(nfile) + ".");
      if (i && a && j && bb) {
        if (d.uhf) {
          b.insert(i - 1, j - 1, a - 1, bb - 1, v);
          b.insert(i - 1, bb - 1, a - 1, j - 1, v);
          b.insert(a - 1, j - 1, i - 1, bb - 1, v);
          b.insert(a - 1, bb - 1, i - 1, j - 1, v);
        } else {
          b.rhf_insert(i, j, a, bb, v);
          b.rhf_insert(i, bb, a, j, v);
          b.rhf_insert(a, j, i, bb, v);
          b.rhf_insert(a, bb, i, j, v);
        }
      } else if (a) {
        const size_t n = static_cast<size_t>(d.norb);
        if (d.uhf) {
          d.h1[(i - 1) * n + (a - 1)] = v;
          d.h1[(a - 1) * n + (i - 1)] = v;
        } else {
          const int ai = Builder::alpha(i), bi = Builder::beta(i);
          const int aa = Builder::alpha(a), ba = Builder::beta(a);
          d.h1[ai * n + aa] = v;
          d.h1[bi * n + ba] = v;
          d.h1[aa * n + ai] = v;
          d.h1[ba * n + bi] = v;
        }
      } else if (i) {
        if (d.uhf) {
          d.orbital_energy.insert({i - 1, v});
        } else {
          d.orbital_energy.insert({Builder::alpha(i), v});
          d.orbital_energy.insert({Builder::beta(i), v});
        }
      } else {
        d.core_energy = v;
      }
    }
  } catch (const std::exception& e) {
    throw std::invalid_argument("Can not read the FCIDUMP file " + path + ". " + e.what());
  }
  return d;
}

Fcidump fcidump_from_arrays(int norb_spin, int nelec, int ms2, bool uhf, double ecore,
                            const double* h1, const double* g2, const double* orbital_energy) {
  if (norb_spin <= 0 || norb_spin > 2 * kMaxOrb || (norb_spin & 1))
    throw std::invalid_argument("norb (spin-orbitals) must be even and in 2.." +
                                std::to_string(2 * kMaxOrb) + ".");
  if (!h1 || !g2) throw std::invalid_argument("h1 and g2 must not be NULL.");
  Fcidump d;
  d.norb = norb_spin;
  d.nelec = nelec;
  d.ms2 = ms2;
  d.uhf = uhf;
  d.core_energy = ecore;
  const size_t n = static_cast<size_t>(norb_spin);
  d.h1.assign(h1, h1 + n * n);
  d.g2.assign(g2, g2 + n * n * n * n);
  d.g2_set.assign(n * n * n * n, 1);
  // Keys (i, j) with i > j are not part of the reference's map.
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < i; ++j)
      for (size_t ab = 0; ab < n * n; ++ab) {
        d.g2[(i * n + j) * n * n + ab] = 0.0;
        d.g2_set[(i * n + j) * n * n + ab] = 0;
      }
  if (orbital_energy)
    for (int i = 0; i < norb_spin; ++i) d.orbital_energy.insert({i, orbital_energy[i]});
  return d;
}

}  // namespace mcd
