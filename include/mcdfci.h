/*
 * mcdfci_b200 C ABI: multi-coordinate-descent FCI (mCDFCI) on one B200.
 *
 * Drop-in for the solver path of ninotreve/mcdfci's cdfci_omp.  The reference
 * has no FFI; its boundary is run_cdfci<N>(Option&, Fcidump&) -> double
 * (src/run_wrapper.h:124-173) over the C++ interfaces Hamiltonian<N>
 * (src/hamiltonian.h:25-54), WaveFunction<N> (src/wavefunction.h:163-221),
 * CoordinatePick<N> / CoordinateUpdate<N> (src/solver.h:94-101,230-250) and
 * Solver / CDFCI<N> (src/solver.h:613-893).  The entry points below replace
 * that boundary with plain pointers and sizes; no C++ exception and no CUDA
 * or torch type crosses it.  Every function returns an MCD_* status; the text
 * of the last error is available from mcd_last_error().
 *
 * Determinants cross the ABI as (alpha, beta) pairs of uint64 occupation
 * strings: bit p of alpha is spatial orbital p with spin alpha.  The
 * reference's layout interleaves them (bit 2p alpha, bit 2p+1 beta,
 * src/input.h:242-243).
 *
 * All arithmetic is FP64; the solver scalars xx, scale and xz (__float128 in
 * the reference) are double-double and cross the ABI as (hi, lo) pairs.
 */
#ifndef MCDFCI_H
#define MCDFCI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MCD_OK 0
/* z_threshold_search asks for a restart with a doubled z_threshold; the
 * reference's CDFCI<N>::solve returns -1 (src/solver.h:803-808). */
#define MCD_RESTART (-1)
#define MCD_ERR_INVALID 1      /* bad input or option (std::invalid_argument in the reference) */
#define MCD_ERR_OVERFLOW 2     /* "The hash table is full..." (std::overflow_error, src/solver.h:813-817) */
#define MCD_ERR_EIG 3          /* subspace eigenproblem failed (the reference exits, src/solver.h:447-450) */
#define MCD_ERR_CUDA 4         /* CUDA runtime error, or no usable GPU */
#define MCD_ERR_UNSUPPORTED 5  /* outside this build's limits (norb > 64, k or estimate > 128, ...) */
#define MCD_ERR_NO_CANDIDATES 6 /* the candidate list became empty */
#define MCD_STOPPED 7          /* the report callback asked to stop */

/* coordinate_pick / coordinate_update values (src/run_wrapper.h:136-156). */
#define MCD_PICK_GCD_GRAD 0
#define MCD_UPDATE_EIG 1
#define MCD_UPDATE_LS 2 /* accepted by the reference but not implemented here: MCD_ERR_UNSUPPORTED */

typedef struct mcd_solver mcd_solver;   /* opaque: one solver bound to one GPU */
typedef struct mcd_batch mcd_batch;     /* opaque: several solver instances advanced together on one GPU */
typedef struct mcd_fcidump mcd_fcidump; /* opaque: a parsed FCIDUMP (host memory) */

/* Integrals in spin-orbital form, as the reference's Fcidump holds them
 * (src/input.h:57-86). */
typedef struct mcd_problem {
  int32_t norb;   /* spin-orbitals: 2 x NORB for RHF, NORB for UHF; even, <= 128 */
  int32_t nelec;
  int32_t ms2;
  int32_t uhf;
  double core_energy;
  const double* h1;             /* [norb*norb] <i|h|a> */
  const double* g2;             /* [norb^4] <ij|ab> at ((i*norb+j)*norb+a)*norb+b; used for i <= j, 0 = absent */
  const double* orbital_energy; /* [norb] or NULL (then the Hartree-Fock guess assumes index order) */
} mcd_problem;

/* The solver:cdfci and hamiltonian options of the input deck, with the
 * reference's defaults (src/run_wrapper.h:64-80) set by mcd_options_default. */
typedef struct mcd_options {
  int64_t num_iterations;      /* 10 */
  int64_t report_interval;     /* 1 */
  int32_t num_of_coordinate;   /* k, 1 */
  int32_t estimate;            /* m, 100 */
  double z_threshold;          /* 0 */
  int32_t z_threshold_search;  /* 0 */
  double max_memory;           /* GB for the wavefunction; required > 0 */
  double threshold;            /* hamiltonian:threshold, 1e-13 */
  const int32_t* ref_det_occ;  /* NULL, or spin-orbital indices of the reference determinant */
  int32_t n_ref_det_occ;
  int32_t coordinate_pick;     /* MCD_PICK_GCD_GRAD */
  int32_t coordinate_update;   /* MCD_UPDATE_EIG (the reference's default, "ls", is unsupported) */
  int32_t groups;              /* CTAs per Hamiltonian column; 0 = chosen from the column length */
  int32_t verbose;             /* 1: print the reference's report table to stdout */
  void* stream;                /* cudaStream_t to run on; NULL = a stream owned by the solver */
  int32_t device;              /* CUDA device ordinal; -1 = the current device */
  /* 1: compaction under max_memory (no counterpart in the reference): when the
   * table passes 60% of its occupancy limit at a report, z_threshold doubles
   * and the entries with x = 0 and |z scale| <= z_threshold are removed, until
   * it is below 40%, instead of failing with MCD_ERR_OVERFLOW.  0 by default. */
  int32_t compaction;
  /* 1 (default): the hash table starts at the size two 64-iteration chunks
   * (or num_iterations, when fewer) of worst-case inserts need (k whole
   * columns per iteration, kept below 3/4 full) and doubles, rehashing into
   * a new allocation between chunks, when those could pass 3/4 or when its
   * load passes 1/4 (shorter probes), up to the table max_memory gives;
   * occupancy limits and results are those of the full table.  0: the full table is allocated at creation, as the reference
   * reserves its table.  A growth that finds the device memory taken by
   * others fails with MCD_ERR_CUDA.  No counterpart in the reference. */
  int32_t table_growth;
  /* The subspace eigenproblem's method.  0: the full reduction for every
   * update (Householder, multisection, inverse iteration).  1: first by
   * shifted inverse iteration (a Cholesky factorisation of B - sigma I, sigma
   * below the current energy by 16 times the last energy drop, certifies
   * sigma < lambda_1; the current vector starts it), its steps run by one warp
   * on the explicit inverse, with the full reduction when that fails.  2
   * (default): first by the bordered fixed point: with B = [[a, b'], [b,
   * H_sub]] and v = (1, y), one warp iterates y <- -(b + E y) / (d - lambda),
   * lambda <- a + b'y (d the diagonal of H_sub, E the rest, kept as its
   * nonzeros), and the result is taken when lambda plus the residual norm
   * lies below the Gershgorin bound of H_sub, which makes it the lowest
   * eigenvalue (Cauchy interlacing); the full reduction otherwise, and for
   * k > 64.  On 24 orbitals, k = 32, method 2 certifies every update after the
   * first few in 12-17 steps, method 1 costs as much as the reduction late in a
   * solve and more early on.  No counterpart in the reference (LAPACK dsyevr,
   * src/solver.h:400-411). */
  int32_t eig_method;
  /* 1: with groups = 0, the CTAs per Hamiltonian column are chosen from
   * timed trials the first time at least 16 iterations per candidate are run
   * (the trials are iterations of the solve), among values around the fixed
   * rule's, the fastest column kernel kept and remembered for the process
   * per (orbitals, electrons, k, m, SM count).  0 (default): the fixed rule.
   * No counterpart in the reference. */
  int32_t autotune;
} mcd_options;

/* One line of the reference's report table (src/solver.h:761-798). */
typedef struct mcd_report {
  int64_t iteration;
  double energy;        /* xz / xx */
  double dx_max;        /* |dx|_max of the last iteration */
  uint64_t x_size;      /* |x|_0 */
  uint64_t z_size;      /* |z|_0 */
  uint64_t cols_size;   /* |H[I]|_0: column entries of the last iteration */
  uint64_t updates;     /* upds: z updates of the last iteration */
  double time_s;        /* wall time since the start of the solve */
  double scale;
  double max_residual;  /* max ||B v - lambda v|| of the subspace eigenproblems */
  double z_threshold;
  uint64_t emitted_total; /* column entries processed since the last reset */
  uint64_t updates_total; /* z updates since the last reset */
  uint64_t occupied;      /* occupied hash slots */
  int32_t last_k;         /* determinants picked in the last iteration */
  int32_t inv_steps_last; /* inverse-iteration steps of the last eigenproblem (0: full reduction) */
  uint64_t inv_updates;   /* eigenproblems solved by shifted inverse iteration since the reset */
  uint64_t inv_steps;     /* their steps, summed */
  uint64_t eig_fallbacks; /* shifted solves that fell back to the full reduction */
  double max_abs_evec;    /* max |v_i|, i >= 1, of the last subspace eigenvector */
} mcd_report;

/* Called after every report_interval iterations; return nonzero to stop. */
typedef int (*mcd_report_cb)(const mcd_report* report, void* user);

/* Called for each instance of a batch after every report_interval
 * iterations; return MCD_CB_RETIRE to stop advancing that instance (it keeps
 * its state, and the batch's later launches leave it out, so the others run
 * on a smaller grid), any other nonzero value to stop the batch. */
#define MCD_CB_RETIRE 2
typedef int (*mcd_batch_report_cb)(int32_t instance, const mcd_report* report, void* user);

/* ---- Input ------------------------------------------------------------- */

/* Fcidump::Fcidump(path) (src/input.h:88-152). */
int mcd_fcidump_read(const char* path, mcd_fcidump** out);
/* A view of the parsed integrals; valid until mcd_fcidump_free.
 * orbital_energy is NULL unless the FCIDUMP lists an energy for every orbital. */
int mcd_fcidump_problem(const mcd_fcidump* f, mcd_problem* view);
void mcd_fcidump_free(mcd_fcidump* f);

/* Defaults of read_input (src/run_wrapper.h:61-80). */
void mcd_options_default(mcd_options* o);

/* ---- Solver ------------------------------------------------------------ */

/* HamiltonianMolecule<N>(fci, threshold) + CDFCI<N>(option) + the table
 * sizing of run_cdfci_wrapper (src/run_wrapper.h:203-213): builds the
 * Hamiltonian tables on the GPU and allocates the hash wavefunction. */
int mcd_create(const mcd_problem* problem, const mcd_options* options, mcd_solver** out);
/* The same, from a parsed FCIDUMP, keeping its orbital energies as read
 * (a partial list included), as run_cdfci_wrapper does (src/run_wrapper.h:175-241). */
int mcd_create_from_fcidump(const mcd_fcidump* f, const mcd_options* options, mcd_solver** out);
void mcd_destroy(mcd_solver* s);

/* CDFCI<N>::solve(h, pick, update, k, m) (src/solver.h:831-893): initial
 * state, num_iterations iterations with a report every report_interval,
 * restarts with a doubled z_threshold under z_threshold_search.  Returns
 * MCD_OK or an error status. */
int mcd_solve(mcd_solver* s, mcd_report_cb cb, void* user);

/* Lower-level control (bench and tests).  mcd_reset puts the wavefunction in
 * the initial state (x = e_ref, z = H[:, ref], src/solver.h:862-873);
 * mcd_run_iterations enqueues n iterations on the solver's stream without
 * waiting; mcd_get_report waits and reads the state. */
int mcd_reset(mcd_solver* s);
int mcd_run_iterations(mcd_solver* s, int64_t n);
/* n iterations with a CUDA event recorded on the solver's stream between
 * every two kernels; waits and returns the summed device time of the leader
 * kernels, of the column kernels, and the total, in milliseconds. */
int mcd_run_iterations_timed(mcd_solver* s, int64_t n, double* leader_ms, double* column_ms, double* total_ms);
int mcd_get_report(mcd_solver* s, mcd_report* r);
/* Solver::result_energy (src/solver.h:613-619) of the last solve. */
int mcd_result(const mcd_solver* s, double* energy);
/* The cudaStream_t the solver runs on. */
int mcd_stream(const mcd_solver* s, void** stream);
/* Solver-side scalars: xx, scale, xz as (hi, lo) pairs; iteration count. */
int mcd_scalars(mcd_solver* s, double xx[2], double scale[2], double xz[2], int64_t* iteration);

/* ---- Batches ------------------------------------------------------------
 *
 * No counterpart in the reference, which solves several systems (the points
 * of a binding curve) one after another with separate runs
 * (experiments/4.4-binding-curve/dissociation.sh:2-9).  A batch holds up to 64
 * instances, each an FCIDUMP of its own size with its own hash wavefunction
 * of options->max_memory GB (the tables carved from one device allocation,
 * committed at creation), all with the same options (k, m, z_threshold,
 * num_iterations, report_interval; z_threshold_search is not supported).  One
 * iteration advances every instance with two launches: one leader CTA per
 * instance and the column CTAs of all instances in one grid; each instance
 * computes exactly what it would alone. */
int mcd_batch_create(const mcd_fcidump* const* fcidumps, int32_t n, const mcd_options* options, mcd_batch** out);
void mcd_batch_destroy(mcd_batch* b);
int mcd_batch_size(const mcd_batch* b, int32_t* n);
/* Initial state of every instance, then num_iterations iterations with a
 * report of each active instance every report_interval (callback may be
 * NULL), until every instance is retired or num_iterations is reached. */
int mcd_batch_solve(mcd_batch* b, mcd_batch_report_cb cb, void* user);
int mcd_batch_reset(mcd_batch* b);
int mcd_batch_run_iterations(mcd_batch* b, int64_t n);
int mcd_batch_run_iterations_timed(mcd_batch* b, int64_t n, double* leader_ms, double* column_ms, double* total_ms);
int mcd_batch_get_report(mcd_batch* b, int32_t instance, mcd_report* r);
/* mcd_debug_table_sums of one instance: sum x^2 and sum x z over its table
 * (double-double) and its occupied slots. */
int mcd_batch_table_sums(mcd_batch* b, int32_t instance, double xx[2], double xz[2], uint64_t* occupied);
/* mcd_residual of one instance: ||H c - E c|| / ||c|| of its current vector. */
int mcd_batch_residual(mcd_batch* b, int32_t instance, double* residual);
/* Energies of the last batch solve, one per instance. */
int mcd_batch_result(const mcd_batch* b, double* energies);

/* ---- Energy gradient ------------------------------------------------------
 *
 * No counterpart in the reference.  The energy is variational, so its
 * derivative with respect to the integrals is the reduced density matrices of
 * the wavefunction: dE/dh_PQ = rdm1[P][Q] and dE/d(PR|QS) = rdm2[P][Q][R][S]/2
 * for independent entries of the dense spatial integral arrays.  mcd_rdm
 * computes them from the current wavefunction on the GPU (one pass over the
 * determinants with nonzero coefficients, recomputing their single and double
 * excitations): rdm1[P*n+Q] = sum_s <a+_{Ps} a_{Qs}>, rdm2[((P*n+Q)*n+R)*n+S] =
 * sum_{s,t} <a+_{Ps} a+_{Qt} a_{St} a_{Rs}>, normalised, n spatial orbitals,
 * so that E = sum h_PQ rdm1[P][Q] + 1/2 sum (PR|QS) rdm2[P][Q][R][S] + E_core.
 * RHF FCIDUMPs only (MCD_ERR_UNSUPPORTED for UHF). */
int mcd_rdm(mcd_solver* s, double* rdm1, double* rdm2);

/* ||H c - E c|| / ||c|| of the current vector c = scale x, E = x'z / x'x,
 * summed over the table's x and z (exact with z_threshold = 0, where z = H x
 * on every connected determinant; with z_threshold > 0 the truncated z gives
 * an estimate).  No counterpart in the reference, which reports only the
 * residual of each subspace eigenproblem (src/solver.h:419-424). */
int mcd_residual(mcd_solver* s, double* residual);

/* ---- Checkpoint / restart -------------------------------------------------
 *
 * No counterpart in the reference.  mcd_checkpoint_save writes the
 * wavefunction (every occupied slot: determinant, x, z) and the iteration
 * state (scalars in double-double, counters, candidate lists) to a binary
 * file; mcd_checkpoint_load, on a solver created for the same FCIDUMP with the
 * same num_of_coordinate and estimate, replaces its state with the file's, so
 * that mcd_run_iterations continues the saved solve.  The table may differ in
 * size (max_memory) if it holds the saved entries (else MCD_ERR_OVERFLOW). */
int mcd_checkpoint_save(mcd_solver* s, const char* path);
int mcd_checkpoint_load(mcd_solver* s, const char* path);

/* Text of the last error on this thread. */
const char* mcd_last_error(void);

/* The whole cdfci_omp main (src/main.cpp:19-36): read the JSON input deck,
 * the FCIDUMP it names, print the header and the report table, solve.
 * Returns 0 on success and 1 on error, as main does. */
int mcd_run_json(const char* input_json_path);

/* ---- Parity / debug ---------------------------------------------------- */

/* HamiltonianMolecule::get_column (src/hamiltonian.h:412-424) of one
 * determinant: up to `cap` (alpha, beta, value) entries, in this build's
 * enumeration order.  *n_out receives the total count. */
int mcd_debug_column(mcd_solver* s, uint64_t alpha, uint64_t beta, uint64_t* alpha_out, uint64_t* beta_out,
                     double* value_out, int64_t cap, int64_t* n_out);
/* CDFCI::get_hamiltonian_submatrix (src/solver.h:637-670): H[i*k+j] =
 * get_off_diagonal(det_i, det_j) for i != j, get_diagonal on the diagonal. */
int mcd_debug_hsub(mcd_solver* s, const uint64_t* alpha, const uint64_t* beta, int32_t k, double* hsub);
/* CoordinateUpdateEig::operator() (src/solver.h:333-609) on given inputs, on
 * the current CUDA device: returns dx[k], the new xx and scale as (hi, lo),
 * and the branch (1: (k+1)x(k+1) problem, 2: k x k first-iteration problem). */
int mcd_debug_eig(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                  const double xz[2], double* dx, double new_xx[2], double new_scale[2], int32_t* branch);
/* mcd_debug_eig with the leader's first method: `drop` > 0 stands for the
 * previous update's energy drop, so that shifted inverse iteration from a
 * Cholesky factorisation of B - sigma I, sigma = xz/xx - max(16 drop, 1e-9
 * (1 + |xz/xx|)), runs before the full reduction, as in a solve; *steps
 * receives its steps, 0 when it fell back to the reduction.  Same outputs. */
int mcd_debug_eig_shifted(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                          const double xz[2], double drop, double* dx, double new_xx[2], double new_scale[2],
                          int32_t* branch, int32_t* steps);
/* mcd_debug_eig with a given method, as mcd_options.eig_method selects it:
 * 0 the full reduction, 1 shifted inverse iteration first (`drop` > 0 as in
 * mcd_debug_eig_shifted), 2 the bordered fixed point first (`drop` unused).
 * *steps receives the fast method's steps, 0 when the reduction ran. */
int mcd_debug_eig_method(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                         const double xz[2], int32_t method, double drop, double* dx, double new_xx[2],
                         double new_scale[2], int32_t* branch, int32_t* steps);
/* mcd_debug_eig without any allocation: no counterpart in the reference.
 * The same kernel and results, but its device buffers are a file-scope
 * static device array of 134 KB (k <= 128; a larger k returns
 * MCD_ERR_UNSUPPORTED) instead of cudaMalloc/cudaFree per call, for callers
 * that cannot allocate: a host whose device memory is committed to the hash
 * wavefunction, or one that cannot take the device-wide synchronisation of
 * cudaFree while a solver runs on another stream.  Inputs and outputs are
 * host buffers; the call runs on `stream` (NULL = the legacy default stream)
 * on the current device and synchronises that stream before it returns.
 * The first call on each device finds the array's address and sets the
 * kernel's shared-memory limit: make it before any stream capture on that
 * device.  The kernel writes every output word on each call, so nothing has
 * to start at zero.  Calls that overlap on one device (two host threads)
 * share the array and race: serialise them. */
int mcd_eig_update_static(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                          const double xz[2], double* dx, double new_xx[2], double new_scale[2], int32_t* branch,
                          void* stream);
/* One compaction now (see mcd_options.compaction) with the given z_threshold
 * (>= the current one); *occupied receives the slots in use after it. */
int mcd_debug_compact(mcd_solver* s, double z_threshold, uint64_t* occupied);
/* One table growth now, as the solver makes when the table fills: the next
 * size (double, or the full one), rehashed by mode 0 (the solver's: a
 * doubling moves runs of whole clusters through shared memory and writes
 * every new slot), 1 (the doubling with every entry inserted by global
 * compare-and-swap) or 2 (fill, then an atomic insert of every entry).
 * *wrap_slots receives the length of the old table's cluster through its
 * last and first slots (0 when either is empty, -1 when longer than 2^16).
 * MCD_ERR_INVALID at the full size.  No counterpart in the reference (its
 * table has a fixed size). */
int mcd_debug_grow(mcd_solver* s, int32_t mode, int64_t* wrap_slots);
/* WaveFunctionCuckoo::debug_calculate_xx_xz (src/wavefunction.h:640-651):
 * sum over the table of x^2 and x*z (double-double), and the slot count. */
int mcd_debug_table_sums(mcd_solver* s, double xx[2], double xz[2], uint64_t* occupied);
/* The hash table: slots now, slots at full size (max_memory), growths so far. */
int mcd_debug_table_info(const mcd_solver* s, uint64_t* capacity, uint64_t* max_capacity, int32_t* growths);
/* Host wall time of the solver's set-up stages in milliseconds, up to n
 * (<= 13) of them: 0 Hamiltonian tables (host, on a host thread during 7 and
 * 1), 1 device allocations at creation, 2 the wait for the host tables and
 * their upload, 3 table fill of the last reset (synchronised), 4 CUDA graph
 * builds, 5 table growths, 6 report read-backs, 7 device and stream set-up,
 * 8 and 9 parts of 2 (the copy into pinned staging, the final stream
 * synchronisation), 10, 11 and 12 parts of 5 (the new table's allocation,
 * its fill and the rehash into it, the release of the old table), summed
 * since creation.  No counterpart in the reference. */
int mcd_debug_setup_times(const mcd_solver* s, double* ms, int32_t n);
/* The autotuner's record: the fixed rule's CTAs per column, the chosen
 * ones, and up to cap trials (CTAs per column, column-kernel microseconds
 * per iteration); *n receives the number of trials (0 before tuning, or
 * when the choice came from the process's cache). */
int mcd_debug_autotune_info(const mcd_solver* s, int32_t* rule, int32_t* chosen, int32_t* trial_groups,
                            double* trial_us, int32_t cap, int32_t* n);
/* Launch shape of the column kernel: CTAs per column, length of the per-CTA
 * candidate lists, and entries per Hamiltonian column.  No counterpart in the
 * reference (it has no GPU launch). */
int mcd_debug_launch_info(mcd_solver* s, int32_t* groups, int32_t* list_size, int32_t* entries_per_column);
/* Scattered-access ceiling of this solver's table, for the column kernel's
 * roofline: slots per second over reps launches of `entries` pseudo-random
 * slots, each touched as a column entry touches its slot (16-byte key, x, an
 * FP64 atomic add of zero on z, so the values stay), ilp = 1 or 4 slots in
 * flight per thread, ctas_per_sm CTAs of 256 threads per SM (1..8; 0 = 8).
 * No counterpart in the reference. */
int mcd_debug_scatter_rate(mcd_solver* s, int64_t entries, int32_t reps, int32_t ilp, int32_t ctas_per_sm,
                           double* slots_per_s);
/* mcd_debug_scatter_rate with the slot touched in one of four ways, to split
 * the ceiling between its parts: mode 0 as a column entry (key, x, atomic
 * add with return), 1 key and x loads only, 2 the atomic with return only,
 * 3 the key load and an atomic add whose return is unused.  No counterpart
 * in the reference. */
int mcd_debug_scatter_rate_mode(mcd_solver* s, int64_t entries, int32_t reps, int32_t ilp, int32_t ctas_per_sm,
                                int32_t mode, double* slots_per_s);
/* SM cycles spent in each phase of the leader kernel (21 phases: state load,
 * finish, candidate gather, top-k, tie sort, picked, H_sub, update_x, publish,
 * eig setup, tridiagonalisation, multisection, inverse iteration,
 * back-transformation, Rayleigh quotient, eig finish, shifted inverse
 * iteration set-up, its Cholesky factorisation, explicit inverse, power steps
 * and refinement steps), summed over launches since the previous call, which
 * resets them.  No counterpart in the reference. */
int mcd_debug_leader_sections(mcd_solver* s, uint64_t* cycles, int32_t n);
/* The determinants with nonzero x and their x (the coefficients are scale * x),
 * sorted by slot; up to cap of them, *n_out receives the count. */
int mcd_debug_wavefunction(mcd_solver* s, uint64_t* alpha, uint64_t* beta, double* x, int64_t cap, int64_t* n_out);
/* SM cycles of thread 0 of every column-kernel CTA in each phase (10
 * values: per round entry decode and integral value, slot probe, x load, z
 * atomic and score, candidate offer; the number of rounds; per CTA the
 * prelude before the first round, the CTA list merge, store and ticket, the
 * column's final merge by its last CTA; the number of CTAs and of final
 * merges), summed since the previous call, which resets them; enable = 1
 * turns the timers on for later launches, 0 off (the default).  No
 * counterpart in the reference. */
int mcd_debug_column_sections(mcd_solver* s, uint64_t* cycles, int32_t n, int32_t enable);
/* Every occupied slot of the hash wavefunction (determinant, x, z), in slot
 * order, after the end of the last iteration is applied; up to cap of them,
 * *n_out receives the count.  No counterpart in the reference. */
int mcd_debug_slots(mcd_solver* s, uint64_t* alpha, uint64_t* beta, double* x, double* z, int64_t cap,
                    int64_t* n_out);
/* The inputs of the last iteration's subspace eigenproblem, the arguments of
 * CoordinateUpdateEig::operator() (src/solver.h:333-345): H_sub (k x k,
 * row-major), the picked coordinates' x and z before the update, and the
 * double-double xx and xz.  *k_out = k; nothing is written when k > cap. */
int mcd_debug_last_eig(mcd_solver* s, double* hsub, double* x, double* z, double xx[2], double xz[2], int32_t cap,
                       int32_t* k_out);
/* The determinants picked in the last iteration (alpha, beta, dx); *k_out <= cap. */
int mcd_debug_picked(mcd_solver* s, uint64_t* alpha, uint64_t* beta, double* dx, int32_t cap, int32_t* k_out);

#ifdef __cplusplus
}
#endif

#endif /* MCDFCI_H */
