// GPU solver: owns the device tables, the hash wavefunction and the iteration
// state, and runs the reference's solve loop (CDFCI<N>::solve,
// src/solver.h:672-893) as launches on one CUDA stream.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/mcdfci.h"
#include "fcidump.h"
#include "hamiltonian.h"
#include "kernels.h"

namespace mcd {

struct SolverOptions {
  long long num_iterations = 10;
  long long report_interval = 1;
  int k = 1;
  int m = 100;
  double z_threshold = 0.0;
  bool z_threshold_search = false;
  double max_memory = 0.0;
  double threshold = 1e-13;
  std::vector<int> ref_det_occ;
  int coordinate_pick = MCD_PICK_GCD_GRAD;
  int coordinate_update = MCD_UPDATE_EIG;
  int groups = 0;
  bool fill_gpu = true;  // with groups = 0: spread few columns over more CTAs (a batch fills the GPU itself)
  bool compaction = false;
  // The hash table starts small and doubles (rehashing into a new
  // allocation) as it fills, up to the size max_memory gives; false: the
  // whole table is allocated at creation, as the reference reserves it.
  bool table_growth = true;
  // Subspace eigenproblem: 0 the full reduction every time; 1 shifted
  // inverse iteration first, with the reduction when it fails.
  int eig_method = 2;
  // Choose the CTAs per Hamiltonian column from timed trials (real
  // iterations of the solve) the first time enough iterations are run, and
  // remember the choice per (orbitals, electrons, k, m, SM count).
  bool autotune = false;
  // A table the caller owns, of exactly the slots max_memory gives
  // (full_capacity): the solver uses it, never grows or frees it.
  Slot* table = nullptr;
  size_t table_slots = 0;
  bool verbose = false;
  cudaStream_t stream = nullptr;
  int device = -1;
};

// Status with a message; thrown inside the library, turned into a return code
// at the C ABI.
struct McdError : std::runtime_error {
  int code;
  McdError(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

class GpuSolver {
 public:
  GpuSolver(const Fcidump& fci, const SolverOptions& opt);
  // Slots of the full table for this FCIDUMP and max_memory (GB).
  static size_t full_capacity(const Fcidump& fci, double max_memory);
  ~GpuSolver();
  GpuSolver(const GpuSolver&) = delete;
  GpuSolver& operator=(const GpuSolver&) = delete;

  // Full solve with reports and z_threshold_search restarts.
  int solve(mcd_report_cb cb, void* user);
  // Initial state with the current z_threshold.
  void reset();
  // Enqueue n iterations (asynchronous).
  void run_iterations(long long n);
  // Run n iterations with direct launches and a CUDA event between every
  // two kernels on the solver's stream; waits, and returns the summed
  // leader-kernel and column-kernel device times and the total (ms).
  void run_iterations_timed(long long n, double* leader_ms, double* column_ms, double* total_ms);
  // Apply the pending end-of-iteration step, wait, and read the state.
  mcd_report report();

  double result_energy() const { return result_energy_; }
  cudaStream_t stream() const { return stream_; }
  void scalars(dd* xx, dd* scale, dd* xz, long long* iter);

  // Parity / debug.
  std::vector<std::pair<Det, double>> column(Det d);
  std::vector<double> hsub(const std::vector<Det>& dets);
  void table_sums(dd* xx, dd* xz, unsigned long long* occupied);
  // ||H c - E c|| / ||c|| of the current vector, from the table's x and z
  // (exact when z_threshold = 0, so that z = H x on every connected determinant).
  double residual();
  // Every occupied slot (determinant, x, z) in slot order, after the pending
  // end of the last iteration.
  void slots(std::vector<Slot>& out);
  std::vector<std::pair<Det, double>> picked();
  // The last eig update's inputs: k, H_sub (k x k), x, z (k each), xx, xz.
  int last_eig_inputs(double* hsub, double* x, double* z, double xx[2], double xz[2], int cap);
  // Spin-summed spatial 1- and 2-RDM of the current wavefunction, normalised
  // (rdm1[P*n+Q] = sum_s <a+_{Ps} a_{Qs}>, rdm2[((P*n+Q)*n+R)*n+S] =
  // sum_{s,t} <a+_{Ps} a+_{Qt} a_{St} a_{Rs}>, n spatial orbitals), so that
  // E = sum h_PQ rdm1 + 1/2 sum (PR|QS) rdm2 + E_core.
  void rdm(std::vector<double>& rdm1, std::vector<double>& rdm2);
  // Raise z_threshold to `z_threshold` and remove the entries with x = 0 and
  // |z scale| <= z_threshold, rebuilding the table; returns the occupied slots.
  unsigned long long compact(double z_threshold);
  // Doubles the table now (grow_to's modes); *wrap receives the slots of
  // the old table's cluster through its last and first slots (0 when either
  // is empty; -1 when longer than 2^16).  False at the full size.
  bool grow_now(int mode, long long* wrap);
  // Checkpoint of the wavefunction and the iteration state (binary file);
  // loading needs a solver for the same problem, k and m, and a table large
  // enough for the saved entries, and continues where the saved solve stopped.
  void checkpoint_save(const std::string& path);
  void checkpoint_load(const std::string& path);
  // The determinants with x != 0 and their x (scaled: coefficients are scale * x).
  void wavefunction(std::vector<Det>& dets, std::vector<double>& x);
  // Leader-kernel phase timers (SM cycles summed over launches since the last call).
  std::vector<unsigned long long> leader_sections();
  // Column-kernel phase timers (kColumnSections values since the last call,
  // which resets them); `enable` turns them on or off for later launches.
  std::vector<unsigned long long> column_sections(bool enable);
  // Slots per second of the scattered-access probe on this solver's table
  // (reps timed launches of `entries` slots after one untimed launch), with
  // ctas_per_sm CTAs of 256 threads per SM (0: 8, every thread slot).
  double scatter_rate(long long entries, int reps, int ilp, int ctas_per_sm, int mode = 0);

  const HamHost& ham() const { return ham_; }
  Det reference_det() const { return ref_; }
  long long table_capacity() const { return static_cast<long long>(capacity_); }
  long long table_max_capacity() const { return static_cast<long long>(max_capacity_); }
  int table_growths() const { return growths_; }
  // Host wall time of the set-up stages, in milliseconds (kSetupStages values):
  // 0 Hamiltonian tables on the host (built on a host thread during 7 and 1),
  // 1 device allocations of the constructor, 2 the wait for the host tables
  // after 1 and their upload, 3 table fill of the last
  // reset (synchronised), 4 CUDA graph builds, 5 table growths, 6 report
  // read-backs (finish, state copy, synchronisation), 7 device and stream
  // set-up (device, stream, attributes, free memory), summed since creation;
  // 8 and 9 are parts of 2: the copy of the tables into pinned staging and
  // the constructor's final synchronisation with the stream; 10, 11 and 12
  // are parts of 5: the new table's allocation, its fill and the rehash into
  // it (synchronised), and the release of the old table.
  static constexpr int kSetupStages = 13;
  const double* setup_ms() const { return setup_ms_; }
  unsigned long long max_wavefunction_size() const { return max_size_; }
  int groups() const { return groups_; }
  int groups_rule() const { return groups_rule_; }
  const std::vector<std::pair<int, double>>& tune_trials() const { return tune_trials_; }
  // Launch descriptors and the column CTA count, for running this instance
  // inside a batch (GpuBatch) on the same stream.
  const LeaderLaunch& leader_launch() const { return ll_; }
  const ColumnLaunch& column_launch() const { return cl_; }
  int column_ctas() const { return cl_.k_grid * cl_.groups; }
  int device() const { return device_; }
  int list_size() const { return list_; }
  int entries_per_column() const { return entries_; }

 private:
  void check(cudaError_t e, const char* what);
  void release();
  void read_state();
  void raise_device_error();
  void build_graph();
  void gather_slots(double zlim, std::vector<Slot>& out);  // occupied slots kept by zlim, in slot order
  // Table growth: before `upcoming` iterations are enqueued, make sure that
  // the table keeps its load below 3/4 even if every one of them inserts a
  // whole column per coordinate, and that the load reached is at most 1/4
  // (shorter probes), from the occupancy read (lagged by one chunk) after
  // earlier chunks; grows, synchronously, when either might not hold.
  void ensure_room(long long upcoming);
  // Rehash into a table of new_capacity slots.  mode 0: a doubling moves runs
  // of clusters (launch_rehash_double), other sizes fill and insert; 1: the
  // doubling with every entry inserted by global compare-and-swap; 2: fill
  // and insert whatever the size.
  void grow_to(size_t new_capacity, int mode = 0);
  size_t next_capacity(size_t c) const;     // the capacity after c
  void record_occupancy(long long iters);   // async occupancy read after a chunk of iters
  void launch_chunk(long long n);           // n <= graph_iters_ iterations, graph or direct
  // The autotuner: trials of kTuneIters iterations per candidate CTA count,
  // the fastest column kernel kept; returns the iterations it ran.
  long long autotune_groups(long long budget);
  void set_groups(int g);

  SolverOptions opt_;
  HamHost ham_;
  Det ref_{0, 0};
  double ref_diag_ = 0.0;
  int na_ = 0, nb_ = 0, entries_ = 0, groups_ = 1, list_ = 32, n_words_ = 1;
  bool uhf_ = false;
  size_t capacity_ = 0;             // hash slots now (power of two)
  size_t max_capacity_ = 0;         // hash slots max_memory gives (the reference's table)
  size_t budget_slots_ = 0;         // device memory for two tables at once, in slots
  int growths_ = 0;
  bool own_table_ = true;
  int groups_rule_ = 1;      // the CTAs per column the fixed rule gives
  bool tuned_ = false;
  std::vector<std::pair<int, double>> tune_trials_;  // (CTAs per column, column kernel us per iteration)
  double setup_ms_[kSetupStages] = {};
  // Occupancy reads after the last two chunks: pinned host words, events, and
  // the iterations enqueued since the reset when each was recorded.
  unsigned long long* h_occ_ = nullptr;
  cudaEvent_t ev_occ_[2] = {nullptr, nullptr};
  long long occ_iters_[2] = {-1, -1};
  int occ_next_ = 0;
  long long iters_enqueued_ = 0;      // since the last reset
  unsigned long long occ_exact_ = 0;  // occupancy read synchronously ...
  long long occ_exact_iters_ = 0;     // ... after this many enqueued iterations
  unsigned long long max_size_ = 0; // reference max_wavefunction_size
  double zt_ = 0.0;
  double result_energy_ = 0.0;

  cudaStream_t stream_ = nullptr;
  bool own_stream_ = false;
  int device_ = 0;
  void* d_tables_ = nullptr;
  void* d_misc_ = nullptr;  // unused: the buffers from d_state_ to d_done_ follow the tables in d_tables_
  Slot* d_slots_ = nullptr;
  IterState* d_state_ = nullptr;
  double* d_cand_score_ = nullptr;
  unsigned* d_cand_slot_ = nullptr;
  double* d_hsub_ = nullptr;
  unsigned* d_err_ = nullptr;
  unsigned long long* d_occ_ = nullptr;
  unsigned long long* d_sect_ = nullptr;
  unsigned long long* d_part_key_ = nullptr;
  unsigned* d_part_slot_ = nullptr;
  double* d_part_sum_ = nullptr;
  unsigned* d_done_ = nullptr;
  HamDev hd_{};
  TableDev td_{};
  ColumnLaunch cl_{};
  LeaderLaunch ll_{};
  IterState h_state_{};

  cudaGraphExec_t graph_ = nullptr;
  static constexpr long long graph_iters_ = 64;
};

}  // namespace mcd
