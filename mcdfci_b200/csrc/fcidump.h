// FCIDUMP reader with the reference's semantics (src/input.h:57-338).
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "mcd_types.h"

namespace mcd {

// Integrals of one FCIDUMP in spin-orbital form.  Spin-orbital 2p is alpha p
// and 2p+1 is beta p for RHF input; UHF input is already spin-orbital
// (src/input.h:203-243).
struct Fcidump {
  int norb = 0;   // spin-orbitals (NORB*2 for RHF), as the reference's Fcidump::norb
  int nelec = 0;
  int ms2 = 0;
  bool uhf = false;
  // True when every integral conserves spin by construction (the RHF
  // expansion of a file), so that the tables need not check it.
  bool spin_conserving = false;
  double core_energy = 0.0;
  std::vector<double> h1;       // [norb*norb] <i|h|a>
  // <ij|ab> stored densely at ((i*norb+j)*norb+a)*norb+b for i <= j, the only
  // keys the reference's map holds (insert_two_body_, src/input.h:304-316).
  // An absent entry reads as 0, as get_two_body_integral does (src/input.h:319-330).
  std::vector<double> g2;
  std::vector<uint8_t> g2_set;  // first insertion wins, as std::unordered_map::insert
  std::map<int, double> orbital_energy;  // first insertion wins

  double g(int i, int j, int a, int b) const {
    if (i > j) return 0.0;
    return g2[((static_cast<size_t>(i) * norb + j) * norb + a) * norb + b];
  }
  double h(int i, int a) const { return h1[static_cast<size_t>(i) * norb + a]; }
};

// Reads `path`.  Throws std::invalid_argument with the reference's messages
// ("Can not read the FCIDUMP file <path>. <reason>").  Where the reference has
// undefined behaviour (an index outside 0..NORB, a missing core-energy line)
// this reader throws, respectively defaults the core energy to 0.
Fcidump read_fcidump(const std::string& path);

// Builds the same structure from dense spin-orbital arrays (the C-ABI path).
Fcidump fcidump_from_arrays(int norb_spin, int nelec, int ms2, bool uhf, double ecore,
                            const double* h1, const double* g2, const double* orbital_energy);

}  // namespace mcd
