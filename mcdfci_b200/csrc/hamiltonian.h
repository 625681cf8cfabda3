// Host-side Hamiltonian: the tables the kernels read, built from an Fcidump
// with the reference's definitions (HamiltonianMolecule<N>, src/hamiltonian.h:56-493).
#pragma once

#include <string>
#include <functional>
#include <memory>
#include <utility>
#include <vector>

#include "fcidump.h"
#include "mcd_types.h"

namespace mcd {

// std::allocator whose value construction leaves doubles uninitialised, for
// tables that their builder writes in full.
template <typename T>
struct DefaultInitAllocator : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = DefaultInitAllocator<U>;
  };
  DefaultInitAllocator() = default;
  template <typename U>
  DefaultInitAllocator(const DefaultInitAllocator<U>&) noexcept {}
  template <typename U>
  void construct(U* p) noexcept {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... A>
  void construct(U* p, A&&... a) {
    ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
  }
};
using TableVec = std::vector<double, DefaultInitAllocator<double>>;

struct HamHost {
  int norb = 0;   // spatial orbitals
  int nso = 0;    // spin-orbitals
  int npair = 0;  // norb*(norb-1)/2
  double ecore = 0.0;
  std::vector<double> hdiag;    // [nso]
  std::vector<double> d2;       // [nso*nso]
  TableVec sh;                  // [2][norb][norb]
  TableVec st;                  // [2][norb][norb][nso]
  std::vector<uint64_t> spres;  // [2][norb]
  TableVec vss;                 // [2][npair][npair]
  TableVec wab;                 // [norb^4]
};

// Builds the tables.  `threshold` is hamiltonian:threshold: a double
// excitation is stored if |value| > threshold (src/hamiltonian.h:137-162); a
// single p->r is stored if max(|<p|h|r>|, max_k |<pk||rk>|) > threshold
// (src/hamiltonian.h:176-210).  Throws std::invalid_argument for a negative
// threshold, an odd spin-orbital count, or integrals that couple alpha and
// beta spin-orbitals (spin-changing excitations), none of which the
// alpha/beta determinant layout represents.
HamHost build_hamiltonian(const Fcidump& fci, double threshold);

// f(i) for every i in [0, n) on the host task pool that builds the tables
// (up to 16 threads, the caller included); returns when all are done.
void host_parallel(int n, const std::function<void(int)>& f);

// Determinant helpers (host).
Det det_from_spin_orbitals(const std::vector<int>& occ);
std::vector<int> det_spin_orbitals(const Det& d, int norb);

// The reference's Hartree-Fock guess (HamiltonianMolecule::get_hartree_fock,
// src/hamiltonian.h:447-492): spin-orbitals sorted by orbital energy (by index
// with a warning when the FCIDUMP has none), then the first NELEC of them are
// offered in order, alpha ones kept while fewer than (NELEC+MS2)/2 are set and
// beta ones while fewer than (NELEC-MS2)/2.  Equal energies keep index order.
Det hartree_fock(const Fcidump& fci, std::string* warning);

// Reference determinant from `ref_det_occ` (CDFCI::get_ref_det,
// src/solver.h:895-919): spin-orbitals outside 0..norb-1 are ignored and the
// count must equal NELEC.
Det ref_det_from_occ(const Fcidump& fci, const std::vector<int>& occ);

// Diagonal element, summed in the reference's order (src/hamiltonian.h:257-272).
double diagonal_element(const HamHost& h, const Det& d);

}  // namespace mcd
