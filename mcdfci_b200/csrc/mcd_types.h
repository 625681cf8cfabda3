// Types shared by the host code and the sm_100a kernels.
#pragma once

#include <cstdint>

#include "dd.h"

#if defined(__CUDACC__)
#define MCD_HD __host__ __device__ __forceinline__
#define MCD_ALIGN(n) __align__(n)
#else
#define MCD_HD inline
#define MCD_ALIGN(n) alignas(n)
#endif

namespace mcd {

// Spatial orbitals per spin string: one uint64 per spin.
constexpr int kMaxOrb = 64;
// Coordinates picked per iteration (num_of_coordinate) and candidates kept
// per column (estimate).
constexpr int kMaxK = 128;
constexpr int kMaxM = 128;
// Key of an empty hash slot.  A determinant can only equal it if all 64
// alpha and all 64 beta orbitals are occupied.
constexpr uint64_t kEmptyKey = ~0ull;
// A table of exactly 2^32 slots keeps its last slot, whose index equals the
// 32-bit "no slot" marker of the candidate lists, out of use: it holds the
// key (kEmptyKey, kReservedKeyB), which no determinant of fewer than 64
// alpha electrons matches, so every probe passes over it.
constexpr uint64_t kReservedKeyB = ~0ull - 1ull;

// A slot that holds no determinant: empty, or the reserved last slot.
MCD_HD bool slot_vacant(uint64_t a, uint64_t b) { return a == kEmptyKey && (b == kEmptyKey || b == kReservedKeyB); }

// A Slater determinant as a pair of occupation strings: bit p of `a` is the
// alpha spin-orbital of spatial orbital p, bit p of `b` the beta one.  The
// reference stores the same information interleaved (bit 2p alpha, bit 2p+1
// beta; src/input.h:242-243, src/determinant.h:24-123).
struct Det {
  uint64_t a, b;
};

// One open-addressing hash slot in HBM: key (alpha, beta), coefficient x and
// gradient z.  32 bytes, so a slot is exactly one DRAM sector.
struct MCD_ALIGN(32) Slot {
  uint64_t a, b;
  double x, z;
};

// Device-resident Hamiltonian tables derived from the FCIDUMP (see
// hamiltonian.cpp for how each is formed from the reference's definitions).
struct HamDev {
  int norb;    // spatial orbitals
  int nso;     // spin-orbitals = 2*norb
  int npair;   // norb*(norb-1)/2
  double ecore;
  const double* hdiag;    // [nso]           <i|h|i>
  const double* d2;       // [nso*nso]       <ij||ij> for i<j (interleaved index)
  const double* sh;       // [2][norb][norb] <p|h|r> for spin s
  const double* st;       // [2][norb][norb][nso] <pk||rk> for spin s, k any spin-orbital
  const uint64_t* spres;  // [2][norb] bit r set if the single p->r is stored
  const double* vss;      // [2][npair][npair] <pq||rs>, p<q, r<s, same spin, 0 if dropped
  const double* wab;      // [norb][norb][norb][norb] alpha p->r with beta q->s, 0 if dropped
};

MCD_HD int pair_index(int p, int q) { return q * (q - 1) / 2 + p; }  // p < q

// Error bits written to the device error word; the host turns them into
// MCD_ERR_* status codes.
enum : unsigned {
  kErrProbe = 1u,      // probe limit hit: the table is (nearly) full
  kErrOverflow = 2u,   // occupancy above the reference's 0.79 * max_wavefunction_size
  kErrEig = 4u,        // subspace eigenproblem produced a non-finite or invalid update
  kErrCandidates = 8u, // no candidate determinant to pick
};

// The open-addressing (x, z) table in HBM.
struct TableDev {
  Slot* slots;
  uint64_t mask;           // capacity - 1 (capacity is a power of two)
  int max_probe;           // bounded probe sequence
  unsigned* err;           // error word
  unsigned long long* n_occupied;
};

}  // namespace mcd
