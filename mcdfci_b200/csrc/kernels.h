// Host-visible interface of the sm_100a kernels.
//
// One mCDFCI iteration (CDFCI<N>::solve inner loop, src/solver.h:701-759) is
// two launches on the solver's stream:
//
//   leader_kernel   (1 CTA)  finishes the previous iteration's z-update
//                            (reinsert the exact z of the picked determinants,
//                            accumulate xz), refetches the candidates, picks the
//                            next k coordinates, builds H_sub, solves the
//                            (k+1)x(k+1) eigenproblem and applies x += dx;
//   column_kernel   (k x G CTAs, G per column) generates the k Hamiltonian columns
//                            and applies z += H_col * dx to the hash table,
//                            keeping each column's top-m candidates.
//
// All scalar solver state lives in IterState in device memory, so iterations
// run back-to-back without host round trips and can be captured in a graph.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "mcd_types.h"

namespace mcd {

struct IterState {
  // Solver scalars, carried in double-double (the reference uses __float128).
  dd xx;       // |x|^2 of the stored (scaled) vector
  dd scale;    // true coefficients = scale * x
  dd xz;       // x^T z = x^T H x
  dd xss;      // xx * scale^2, used for gradients |x*xss + z|
  double zt;   // z_threshold
  int n_words; // interleaved words per determinant in the reference layout (tie-break order)
  int k_req;   // num_of_coordinate
  int m;       // estimate
  int pad0;
  long long iter;  // completed iterations (0 after initialisation)

  // Current iteration (written by the leader, read by the column kernel).
  int k_cur;
  int pad1;
  Det det[kMaxK];
  long long slot[kMaxK];
  double dx[kMaxK];
  double hdiag[kMaxK];

  // Column kernel outputs for the current iteration.
  double newz[kMaxK];  // exact (H x)_c recomputed over the column
  double dot[kMaxK];   // sum over the column of dz * x
  int cand_n[kMaxK];

  // Counters.
  unsigned long long x_size;        // reference x_size (src/wavefunction.h:425-451)
  unsigned long long z_size;        // reference z_size: dets inserted by the z-update
  unsigned long long emitted;       // column entries of the last iteration (|H[I]|_0)
  unsigned long long updates;       // z updates of the last iteration (upds)
  unsigned long long occupancy_limit;  // 0.79 * max_wavefunction_size
  double dx_max;                    // max |dx| of the last iteration
  double eig_residual_max;          // max ||B v - lambda v|| seen so far
  int last_branch;                  // 1: (k+1)x(k+1) problem, 2: k x k (first iteration)
  int pending;                      // 1: the column kernel ran and its z reinsert / xz update is not applied yet
  unsigned long long emitted_total; // column entries over all iterations
  unsigned long long updates_total; // z updates over all iterations

  // Subspace eigenproblem statistics (the [LOG] line).
  double eig_drop;                  // last update's energy drop xz/xx - lambda (0: unknown)
  double max_abs_evec;              // max |v_i|, i >= 1, of the last eigenvector
  unsigned long long inv_updates;   // updates solved by shifted inverse iteration
  unsigned long long inv_steps;     // their inverse-iteration steps, summed
  unsigned long long eig_fallbacks; // shifted solves that fell back to the reduction
  double inv_diff_sum;              // sum of the changes made by their last step
  double inv_diff_max;
  double inv_diff_curr;
  int inv_steps_curr;               // steps of the last update (0: the reduction ran)
  int pad2;
};

struct ColumnLaunch {
  HamDev ham;
  TableDev tab;
  IterState* st;
  double* cand_score;     // [kMaxK][m] score of each column's candidates
  unsigned* cand_slot;    // [kMaxK][m] their hash slots (tables have at most 2^32 slots)
  unsigned long long* part_key;  // [kMaxK][groups][list] per-CTA candidate lists
  unsigned* part_slot;           // [kMaxK][groups][list]
  double* part_sum;              // [kMaxK][groups][kPartSum] per-CTA new_z, dot and entry counters
  unsigned* done;                // [kMaxK] CTAs finished per column (reset by the last one)
  unsigned long long* sect;  // [kColumnSections] SM cycles per phase of thread 0's rounds, or null
  int m;
  int groups;             // CTAs per column
  int k_grid;             // columns launched (>= k_cur)
  int na, nb;             // electrons per spin (fixed by the starting determinant)
};

struct LeaderLaunch {
  HamDev ham;
  TableDev tab;
  IterState* st;
  const double* cand_score;
  const unsigned* cand_slot;
  double* hsub_out;       // [kMaxK*kMaxK] last H_sub (row-major, k_cur x k_cur), then the last eig
                          // update's other inputs: x[kMaxK], z[kMaxK], xx (hi, lo), xz (hi, lo)
  unsigned long long* sect;  // [kLeaderSections] SM cycles per phase of the leader kernel, or null
  int m;
  int k_req;
  int eig_method;          // 1: shifted inverse iteration first when the last energy drop is known
};

// Several independent instances advanced by the same two launches per
// iteration: one leader CTA per instance, and the column CTAs of all
// instances in one grid (instance i owns CTAs [cta_begin[i], cta_begin[i+1])).
// Passed by value as kernel parameters (well under the 32 KB limit), so that
// every CTA reads its instance's descriptor from the constant bank.  All
// instances of a batch share k and m.
constexpr int kMaxBatch = 64;

// Per-CTA partial values of the column kernel: new_z, dot, and the emitted,
// updated and inserted entry counts (exact in a double).
constexpr int kPartSum = 5;
struct LeaderBatch {
  int n;
  LeaderLaunch L[kMaxBatch];
};
struct ColumnBatch {
  int n;
  int cta_begin[kMaxBatch + 1];
  ColumnLaunch L[kMaxBatch];
};
static_assert(sizeof(LeaderBatch) <= 32000 && sizeof(ColumnBatch) <= 32000, "kernel parameters above 32 KB");

// Reduced density matrices of the wavefunction in the table, unnormalised
// (divide by sum x^2), in spin blocks over spatial orbitals (n = ham.norb):
//   g1a[r*n+p]          = sum <a+_{r alpha} a_{p alpha}>           (g1b: beta)
//   g2aa[((p*n+q)*n+r)*n+s], p < q, r < s only
//                       = sum <a+_p a+_q a_s a_r> (all alpha)      (g2bb: beta)
//   g2ab[((p*n+q)*n+r)*n+s] = sum <a+_{p alpha} a+_{q beta} a_{s beta} a_{r alpha}>
struct RdmLaunch {
  HamDev ham;
  TableDev tab;
  const unsigned* list;  // slots of the determinants with x != 0
  long long nlist;
  double *g1a, *g1b, *g2aa, *g2bb, *g2ab;
};

// Phases of the leader kernel timed into LeaderLaunch::sect: 0 state load,
// 1 finish + prefix, 2 candidate gather (slots, dedupe, scores), 3 top-k,
// 4 full sort when the k-th score is tied, 5 picked determinants, 6 H_sub,
// 7 update_x, 8 publish, 9 eig setup, 10 tridiagonalisation, 11 multisection,
// 12 inverse iteration, 13 back-transformation, 14 Rayleigh quotient,
// 15 eig finish,
// 16 the fast solver of eig_method 1 or 2 (when it runs, in place of 10-13:
// its set-up and, when it fails, the restore), the rest of it in 17-20:
// method 1: 17 Cholesky factorisation, 18 explicit inverse, 19 power steps,
// 20 refinement steps; method 2: 17 set-up (packing of H_sub's nonzeros, the
// bounds), 18 products and reciprocals of its steps, 19 their reductions and
// tests, 20 their stores.  The eig set-up (9) is split further: 21 H_sub into
// B, 22 H x, 23 the double-double sums of x'x, x'z, x'Hx (9 is then the first
// row of B), and the Rayleigh quotient (14): 24 the product B v (14 is then
// the double-double quotient, normalisation and residual).
constexpr int kLeaderSections = 25;

// Phases of the column kernel timed into ColumnLaunch::sect (thread 0 of each
// CTA, summed): 0 entry decode and integral value, 1 slot probe, 2 x load,
// z atomic and score, 3 candidate offer, 4 rounds counted, 5 prelude (CTA
// start to the first round), 6 CTA list merge, store and ticket, 7 the
// column's final merge (last CTA), 8 CTAs counted, 9 final merges counted.
constexpr int kColumnSections = 10;

// Launchers (column_kernel.cu / leader_kernel.cu).
int column_entries(int norb, int na, int nb);
// Length of the per-CTA candidate lists for `estimate` m (32, 64 or 128).
int column_list_size(int m);
// CTAs per column for a column of `entries` entries.
// CTAs per column: about three rounds of 256 entries each, or more when k
// such columns would leave some of `resident` CTA slots of the GPU empty
// (resident = 0: never more); at most 96.
int column_groups(int entries, int k, int resident);
// The most CTAs per column the autotuner tries, and its iterations per trial.
constexpr int kMaxGroups = 96;
constexpr int kTuneIters = 16;
cudaError_t launch_column(const ColumnLaunch& a, cudaStream_t s);
cudaError_t launch_leader(const LeaderLaunch& a, cudaStream_t s);
// Sets, on the current device, the launch attribute launch_leader needs for
// a (its dynamic shared-memory limit); for use before a stream capture.
cudaError_t prepare_leader(const LeaderLaunch& a);
cudaError_t launch_leader_batch(const LeaderBatch& b, cudaStream_t s);
cudaError_t launch_column_batch(const ColumnBatch& b, cudaStream_t s);
cudaError_t launch_init(const LeaderLaunch& a, Det hf, double hf_diag, cudaStream_t s);
// Applies the pending end of the last iteration (z reinsert of the picked
// determinants, xz += dot), so that reported energies and table contents are
// those after a complete iteration.  Idempotent.
cudaError_t launch_finish(const LeaderLaunch& a, cudaStream_t s);
// Every occupied slot of `src` (n slots) inserted into table t with its x and z.
cudaError_t launch_rehash(const Slot* src, size_t n, const TableDev& t, cudaStream_t s);
// The same for a table t of exactly 2n slots (n a power of two >= 1024, below
// 2^32 in t), which it writes whole (no fill first) and whose occupancy
// count it leaves as it is; force_global inserts every entry with the global
// compare-and-swap instead of placing runs of clusters in shared memory.
cudaError_t launch_rehash_double(const Slot* src, size_t n, const TableDev& t, bool force_global, cudaStream_t s);
// Table initialisation (all slots empty) and whole-table sums.
cudaError_t launch_table_fill(Slot* slots, size_t n, cudaStream_t s);
cudaError_t launch_table_sums(const Slot* slots, size_t n, dd* partial, unsigned long long* count, int nblocks,
                              cudaStream_t s);

// Slots with x != 0 into list (up to cap; *count receives the total).
cudaError_t launch_rdm_list(const TableDev& t, size_t capacity, unsigned* list, unsigned long long* count,
                            unsigned long long cap, cudaStream_t s);
cudaError_t launch_rdm(const RdmLaunch& r, cudaStream_t s);

// Debug / parity entry points (synchronous).
// Column of one determinant: writes up to `cap` (a, b, value) entries.
// Scattered-access probe of the table: `entries` pseudo-random slots, each
// read (key, x) and given an atomic add of zero on z; ilp 1 or 4 slots in
// flight per thread; `ctas` CTAs of 256 threads.  `sink`: one device double,
// written only to keep loads.
// mode 0: key, x and atomic with return; 1: key and x only; 2: atomic with
// return only; 3: key and an atomic add without return.
cudaError_t scatter_probe(const TableDev& t, long long entries, int ilp, int ctas, uint64_t seed, double* sink,
                          cudaStream_t s, int mode = 0);
cudaError_t debug_column(const HamDev& h, Det d, double hdiag, uint64_t* a_out, uint64_t* b_out,
                         double* v_out, int cap, int* n_out, cudaStream_t s);
cudaError_t debug_hsub(const HamDev& h, const Det* dets, int k, double* hsub, cudaStream_t s);
// One eig update on given inputs (device pointers); writes dx[k], xx_scale[0] =
// new xx, xx_scale[1] = new scale, the branch taken and an error word.  The
// lower triangle of hsub is overwritten with its upper triangle.
// drop > 0: the last update's energy drop, which lets the shifted solver run
// first (as the leader does); *steps (device int) receives its steps, 0 when
// the reduction ran.
cudaError_t debug_eig(int k, double* hsub, const double* x, const double* z, dd xx, dd xz, double* dx,
                      dd* xx_scale, int* branch, unsigned* err, cudaStream_t s, double drop = 0.0,
                      int* steps = nullptr, int method = 1);
size_t leader_smem_bytes(int k, int m);

// debug_eig on HOST buffers with its device buffers in a file-scope device
// array (leader_kernel.cu) instead of cudaMalloc: no allocation.  k <= 128;
// returns cudaErrorInvalidValue above.  Runs on stream s and synchronises it.
// Calls that overlap on one device share the array and race.
constexpr int kStaticEigMaxK = 128;
cudaError_t eig_update_static(int k, const double* hsub, const double* x, const double* z, dd xx, dd xz,
                              double* dx, dd* new_xx_scale, int* branch, unsigned* err, cudaStream_t s);

}  // namespace mcd
