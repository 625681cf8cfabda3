#include "gpu_batch.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <exception>
#include <thread>
#include <vector>
#include <cstdio>
#include <iomanip>
#include <iostream>

namespace mcd {

// Concurrent groups of a batch: two let one group's leader CTAs (one SM each)
// run under the other group's column grid.
#ifndef MCD_BATCH_GROUPS
#define MCD_BATCH_GROUPS 2
#endif
namespace {
constexpr int kBatchGroups = MCD_BATCH_GROUPS;
}  // namespace

void GpuBatch::check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw McdError(MCD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

GpuBatch::GpuBatch(const std::vector<const Fcidump*>& fcis, const SolverOptions& opt) : opt_(opt) {
  if (fcis.empty() || static_cast<int>(fcis.size()) > kMaxBatch)
    throw McdError(MCD_ERR_UNSUPPORTED, "a batch holds 1.." + std::to_string(kMaxBatch) + " instances.");
  if (opt_.z_threshold_search)
    throw McdError(MCD_ERR_UNSUPPORTED, "z_threshold_search is not supported in a batch.");
  if (opt_.device >= 0) check(cudaSetDevice(opt_.device), "cudaSetDevice");
  const int ng = std::min(kBatchGroups, static_cast<int>(fcis.size()));
  try {
    if (opt_.stream) {
      stream_ = opt_.stream;
    } else {
      check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
      own_stream_ = true;
    }
    groups_.resize(static_cast<size_t>(ng));
    join_.assign(static_cast<size_t>(ng), nullptr);
    for (int g = 0; g < ng; ++g) {
      if (g == 0)
        groups_[0].stream = stream_;
      else
        check(cudaStreamCreateWithFlags(&groups_[g].stream, cudaStreamNonBlocking), "cudaStreamCreate");
      check(cudaEventCreateWithFlags(&join_[g], cudaEventDisableTiming), "cudaEventCreate");
      groups_[g].lb = std::make_unique<LeaderBatch>();
      groups_[g].cb = std::make_unique<ColumnBatch>();
      groups_[g].lb->n = groups_[g].cb->n = 0;
      groups_[g].cb->cta_begin[0] = 0;
    }
    // The instances' tables carved from one allocation, each a power of two
    // of 32-byte slots (so every table starts aligned).
    std::vector<size_t> caps(fcis.size());
    size_t total = 0;
    for (size_t i = 0; i < fcis.size(); ++i) total += caps[i] = GpuSolver::full_capacity(*fcis[i], opt_.max_memory);
    void* pool = nullptr;
    cudaError_t ae = cudaMalloc(&pool, total * sizeof(Slot));
    if (ae != cudaSuccess)
      throw McdError(MCD_ERR_CUDA, "cudaMalloc(batch tables, " + std::to_string(total * sizeof(Slot)) +
                                       " bytes): " + cudaGetErrorString(ae));
    pool_ = static_cast<Slot*>(pool);
    // Instance i goes to group i % ng, on that group's stream.  The
    // instances are independent, so they are constructed on up to eight host
    // threads (host tables, uploads); the device is named explicitly because
    // each thread has its own current device.  The first failure in instance
    // order is the one reported.
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    const size_t n = fcis.size();
    std::vector<SolverOptions> each(n, opt_);
    size_t off = 0;
    for (size_t i = 0; i < n; ++i) {
      each[i].device = dev;
      each[i].stream = groups_[i % static_cast<size_t>(ng)].stream;
      each[i].verbose = false;
      each[i].fill_gpu = false;      // the batch's columns fill the GPU together
      each[i].table_growth = false;  // the batch launches its instances' kernels itself
      each[i].table = pool_ + off;
      each[i].table_slots = caps[i];
      off += caps[i];
    }
    inst_.resize(n);
    std::vector<std::exception_ptr> errs(n);
    std::atomic<size_t> next{0};
    auto build = [&] {
      for (size_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) {
        try {
          inst_[i] = std::make_unique<GpuSolver>(*fcis[i], each[i]);
        } catch (...) {
          errs[i] = std::current_exception();
        }
      }
    };
    const size_t nt = std::min<size_t>(n, 8);
    std::vector<std::thread> th;
    for (size_t t = 1; t < nt; ++t) th.emplace_back(build);
    build();
    for (auto& x : th) x.join();
    for (const auto& e : errs)
      if (e) std::rethrow_exception(e);
    energies_.assign(fcis.size(), 0.0);
    active_.assign(fcis.size(), 1);
    set_groups();
  } catch (...) {
    inst_.clear();
    if (pool_) cudaFree(pool_);
    pool_ = nullptr;
    for (size_t g = 0; g < groups_.size(); ++g)
      if (g > 0 && groups_[g].stream) cudaStreamDestroy(groups_[g].stream);
    for (auto e : join_)
      if (e) cudaEventDestroy(e);
    if (own_stream_ && stream_) cudaStreamDestroy(stream_);
    throw;
  }
}

GpuBatch::~GpuBatch() {
  for (size_t g = 0; g < groups_.size(); ++g) {
    if (groups_[g].graph) cudaGraphExecDestroy(groups_[g].graph);
  }
  inst_.clear();
  if (pool_) cudaFree(pool_);
  for (size_t g = 1; g < groups_.size(); ++g)
    if (groups_[g].stream) cudaStreamDestroy(groups_[g].stream);
  for (auto e : join_)
    if (e) cudaEventDestroy(e);
  if (own_stream_ && stream_) cudaStreamDestroy(stream_);
}

// Make every group's stream wait for the others' enqueued work, so that a
// later operation on any of them (a report, a reset) sees all of it.
void GpuBatch::join_streams() {
  for (size_t g = 0; g < groups_.size(); ++g) check(cudaEventRecord(join_[g], groups_[g].stream), "cudaEventRecord");
  for (size_t g = 0; g < groups_.size(); ++g)
    for (size_t h = 0; h < groups_.size(); ++h)
      if (g != h) check(cudaStreamWaitEvent(groups_[g].stream, join_[h], 0), "cudaStreamWaitEvent");
}

void GpuBatch::set_groups() {
  const size_t ng = groups_.size();
  for (Group& G : groups_) {
    if (G.graph) cudaGraphExecDestroy(G.graph);
    G.graph = nullptr;
    G.lb->n = G.cb->n = 0;
    G.cb->cta_begin[0] = 0;
  }
  for (size_t i = 0; i < inst_.size(); ++i) {
    if (!active_[i]) continue;
    Group& G = groups_[i % ng];
    const int j = G.lb->n;
    G.lb->L[j] = inst_[i]->leader_launch();
    G.cb->L[j] = inst_[i]->column_launch();
    G.cb->cta_begin[j + 1] = G.cb->cta_begin[j] + inst_[i]->column_ctas();
    G.lb->n = G.cb->n = j + 1;
  }
}

int GpuBatch::active() const {
  int n = 0;
  for (char a : active_) n += a ? 1 : 0;
  return n;
}

void GpuBatch::reset() {
  for (auto& s : inst_) s->reset();
  if (active() != size()) {
    active_.assign(inst_.size(), 1);
    set_groups();
  }
  join_streams();
}

void GpuBatch::launch_iteration(Group& g) {
  if (g.lb->n == 0) return;
  check(launch_leader_batch(*g.lb, g.stream), "batched leader");
  check(launch_column_batch(*g.cb, g.stream), "batched column");
}

void GpuBatch::build_graphs() {
  graph_iters_ = 64;
  for (Group& G : groups_) {
    if (G.lb->n == 0) continue;
    launch_iteration(G);  // sets launch attributes outside capture
    cudaGraph_t g = nullptr;
    check(cudaStreamBeginCapture(G.stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    for (long long i = 0; i < graph_iters_; ++i) {
      launch_leader_batch(*G.lb, G.stream);
      launch_column_batch(*G.cb, G.stream);
    }
    check(cudaStreamEndCapture(G.stream, &g), "end capture");
    check(cudaGraphInstantiate(&G.graph, g, 0), "graph instantiate");
    cudaGraphDestroy(g);
  }
}

void GpuBatch::run_iterations(long long n) {
  if (n <= 0 || active() == 0) return;
  bool built = false;
  for (const Group& G : groups_) built = built || G.graph != nullptr;
  if (!built) {
    build_graphs();
    --n;
  }
  while (n >= graph_iters_) {
    for (Group& G : groups_)
      if (G.graph) check(cudaGraphLaunch(G.graph, G.stream), "graph launch");
    n -= graph_iters_;
  }
  for (; n > 0; --n)
    for (Group& G : groups_) launch_iteration(G);
  join_streams();
}

// Device time of n iterations of the whole batch (CUDA events on group 0's
// stream around work that every group joins).  With the groups overlapping,
// the time is not split by kernel: leader_ms and column_ms stay 0.
void GpuBatch::run_iterations_timed(long long n, double* leader_ms, double* column_ms, double* total_ms) {
  *leader_ms = *column_ms = *total_ms = 0.0;
  if (n <= 0 || active() == 0) return;
  cudaEvent_t a = nullptr, b = nullptr;
  check(cudaEventCreate(&a), "cudaEventCreate");
  check(cudaEventCreate(&b), "cudaEventCreate");
  try {
    join_streams();
    check(cudaEventRecord(a, stream_), "cudaEventRecord");
    join_streams();
    for (long long i = 0; i < n; ++i)
      for (Group& G : groups_) launch_iteration(G);
    join_streams();
    check(cudaEventRecord(b, stream_), "cudaEventRecord");
    check(cudaEventSynchronize(b), "cudaEventSynchronize");
    float t = 0.f;
    check(cudaEventElapsedTime(&t, a, b), "cudaEventElapsedTime");
    *total_ms = t;
  } catch (...) {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    throw;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
}

mcd_report GpuBatch::report(int i) { return inst_.at(static_cast<size_t>(i))->report(); }

int GpuBatch::solve(int (*cb)(int, const mcd_report*, void*), void* user) {
  reset();
  const auto t0 = std::chrono::steady_clock::now();
  const long long chunks = opt_.num_iterations / opt_.report_interval;
  for (long long c = 0; c < chunks && active() > 0; ++c) {
    run_iterations(opt_.report_interval);
    bool stop = false, retired = false;
    for (int i = 0; i < size(); ++i) {
      if (!active_[static_cast<size_t>(i)]) continue;
      mcd_report r = report(i);
      r.time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      energies_[static_cast<size_t>(i)] = r.energy;
      if (opt_.verbose) {
        std::cout << "instance " << std::setw(3) << i << "  iteration " << std::setw(10) << r.iteration
                  << "  energy " << std::fixed << std::setprecision(10) << r.energy << "  |x|_0 " << r.x_size
                  << "  |z|_0 " << r.z_size << "  time " << std::setprecision(2) << r.time_s << std::endl;
      }
      const int rc = cb ? cb(i, &r, user) : 0;
      if (rc == MCD_CB_RETIRE) {
        active_[static_cast<size_t>(i)] = 0;
        retired = true;
      } else if (rc != 0) {
        stop = true;
      }
    }
    if (stop) return MCD_STOPPED;
    if (retired) set_groups();
  }
  for (int i = 0; i < size(); ++i)
    if (active_[static_cast<size_t>(i)]) energies_[static_cast<size_t>(i)] = report(i).energy;
  return MCD_OK;
}

}  // namespace mcd
