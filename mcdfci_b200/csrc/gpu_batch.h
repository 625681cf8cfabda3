// Several independent mCDFCI instances (for example the points of a
// dissociation curve, each its own FCIDUMP) advanced together on one GPU.
// The instances are split into a few groups, each on its own stream: one
// leader CTA per instance of the group and the column CTAs of the whole group
// in one grid, two launches per iteration per group, recorded 64 iterations
// at a time in a CUDA graph.  The groups run concurrently, so that one group's
// single-SM leader CTAs overlap another group's column grid.  Each instance keeps its own Hamiltonian tables, hash
// table and iteration state (a GpuSolver on the batch's stream), and its CTA
// layout is that of its own single-instance launch.  No counterpart in the
// reference, which solves a curve one point after another
// (experiments/4.4-binding-curve/dissociation.sh:2-9).
#pragma once

#include <memory>
#include <vector>

#include "gpu_solver.h"

namespace mcd {

class GpuBatch {
 public:
  // opt applies to every instance (k, m, z_threshold, max_memory per
  // instance, num_iterations, report_interval); z_threshold_search is not
  // supported in a batch.
  GpuBatch(const std::vector<const Fcidump*>& fcis, const SolverOptions& opt);
  ~GpuBatch();
  GpuBatch(const GpuBatch&) = delete;
  GpuBatch& operator=(const GpuBatch&) = delete;

  int size() const { return static_cast<int>(inst_.size()); }
  void reset();
  void run_iterations(long long n);
  void run_iterations_timed(long long n, double* leader_ms, double* column_ms, double* total_ms);
  mcd_report report(int i);
  // num_iterations iterations of every instance, a report of each every
  // report_interval; cb(instance, report) returning MCD_CB_RETIRE stops that
  // instance (it keeps its state and energy, and later launches leave it
  // out), any other nonzero value stops the batch.  Ends when every
  // instance is retired or num_iterations is reached.
  int solve(int (*cb)(int, const mcd_report*, void*), void* user);
  // Instances still advanced by run_iterations (all of them after a reset).
  int active() const;
  double result_energy(int i) const { return energies_.at(static_cast<size_t>(i)); }
  GpuSolver& instance(int i) { return *inst_.at(static_cast<size_t>(i)); }
  cudaStream_t stream() const { return stream_; }

 private:
  void check(cudaError_t e, const char* what);

  struct Group {
    std::unique_ptr<LeaderBatch> lb;
    std::unique_ptr<ColumnBatch> cb;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
  };
  void join_streams();
  void launch_iteration(Group& g);
  void build_graphs();
  // The groups' launch descriptors over the active instances (instance i in
  // group i % groups); drops the graphs.
  void set_groups();

  SolverOptions opt_;
  std::vector<std::unique_ptr<GpuSolver>> inst_;
  std::vector<Group> groups_;
  std::vector<cudaEvent_t> join_;  // one per group: the end of its last enqueued work
  cudaStream_t stream_ = nullptr;  // group 0's stream; the others wait on it and it waits on them
  bool own_stream_ = false;
  long long graph_iters_ = 0;
  std::vector<double> energies_;
  std::vector<char> active_;
  Slot* pool_ = nullptr;  // every instance's hash table, one allocation
};

}  // namespace mcd
