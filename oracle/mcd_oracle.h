/*
 * CPU restatement of the reference's Hamiltonian path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ (and nothing in the product) to
 * check the GPU kernels.  It follows the reference's own data layout and
 * loops rather than the GPU design:
 *   determinants  interleaved spin-orbital bit strings, nw 64-bit words
 *                 (Determinant<N>, src/determinant.h:24-123)
 *   parity        bits in [min(i,a), max(i,a)) (src/determinant.h:103-111)
 *   tables        per spin-orbital pair a list of (a, b, value) built from
 *                 the FCIDUMP entries present in the reference's map, sorted
 *                 by |value| (src/hamiltonian.h:113-219)
 *   column        diagonal, singles, doubles in that order
 *                 (src/hamiltonian.h:252-424)
 * Pinned against fixtures printed by the reference itself (tests/golden).
 */
#ifndef MCD_ORACLE_H
#define MCD_ORACLE_H

#include <stdint.h>

typedef struct oracle oracle;

/* Parses an FCIDUMP as src/input.h:88-338 does and builds the tables with
 * hamiltonian:threshold `thr`.  Returns NULL on failure (message in err). */
oracle* oracle_load(const char* path, double thr, char* err, int errlen);
void oracle_free(oracle* o);

/* Header values: spin-orbitals, electrons, ms2, words per determinant. */
void oracle_info(const oracle* o, int32_t* nso, int32_t* nelec, int32_t* ms2, int32_t* nw, double* ecore);

/* Dense copies of the parsed integrals: h1[nso*nso], g2[nso^4] (keys i <= j). */
void oracle_integrals(const oracle* o, double* h1, double* g2);

/* Hartree-Fock determinant (src/hamiltonian.h:447-492), nw words. */
void oracle_hartree_fock(const oracle* o, uint64_t* det);

/* get_column: writes up to cap entries (nw words each + value); returns the count. */
int64_t oracle_column(const oracle* o, const uint64_t* det, uint64_t* dets_out, double* vals_out, int64_t cap);

/* get_diagonal and get_off_diagonal(d1, d2). */
double oracle_diagonal(const oracle* o, const uint64_t* det);
double oracle_off_diagonal(const oracle* o, const uint64_t* d1, const uint64_t* d2);

/* get_hamiltonian_submatrix (src/solver.h:637-670) for k determinants. */
void oracle_hsub(const oracle* o, const uint64_t* dets, int32_t k, double* h);

#endif
