#include "gpu_batch.h"

#include <chrono>
#include <cstdio>
#include <iomanip>
#include <iostream>

namespace mcd {

void GpuBatch::check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw McdError(MCD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

GpuBatch::GpuBatch(const std::vector<const Fcidump*>& fcis, const SolverOptions& opt) : opt_(opt) {
  if (fcis.empty() || static_cast<int>(fcis.size()) > kMaxBatch)
    throw McdError(MCD_ERR_UNSUPPORTED, "a batch holds 1.." + std::to_string(kMaxBatch) + " instances.");
  if (opt_.z_threshold_search)
    throw McdError(MCD_ERR_UNSUPPORTED, "z_threshold_search is not supported in a batch.");
  if (opt_.device >= 0) check(cudaSetDevice(opt_.device), "cudaSetDevice");
  if (opt_.stream) {
    stream_ = opt_.stream;
  } else {
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    own_stream_ = true;
  }
  try {
    SolverOptions each = opt_;
    each.stream = stream_;
    each.verbose = false;
    for (const Fcidump* f : fcis) inst_.push_back(std::make_unique<GpuSolver>(*f, each));
    lb_ = std::make_unique<LeaderBatch>();
    cb_ = std::make_unique<ColumnBatch>();
    lb_->n = cb_->n = size();
    cb_->cta_begin[0] = 0;
    for (int i = 0; i < size(); ++i) {
      lb_->L[i] = inst_[i]->leader_launch();
      cb_->L[i] = inst_[i]->column_launch();
      cb_->cta_begin[i + 1] = cb_->cta_begin[i] + inst_[i]->column_ctas();
    }
    energies_.assign(fcis.size(), 0.0);
  } catch (...) {
    inst_.clear();
    if (own_stream_) cudaStreamDestroy(stream_);
    throw;
  }
}

GpuBatch::~GpuBatch() {
  if (graph_) cudaGraphExecDestroy(graph_);
  inst_.clear();
  if (own_stream_ && stream_) cudaStreamDestroy(stream_);
}

void GpuBatch::reset() {
  for (auto& s : inst_) s->reset();
}

void GpuBatch::launch_iteration() {
  check(launch_leader_batch(*lb_, stream_), "batched leader");
  check(launch_column_batch(*cb_, stream_), "batched column");
}

void GpuBatch::build_graph() {
  launch_iteration();  // sets launch attributes outside capture
  graph_iters_ = 64;
  cudaGraph_t g = nullptr;
  check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
  for (long long i = 0; i < graph_iters_; ++i) {
    launch_leader_batch(*lb_, stream_);
    launch_column_batch(*cb_, stream_);
  }
  check(cudaStreamEndCapture(stream_, &g), "end capture");
  check(cudaGraphInstantiate(&graph_, g, 0), "graph instantiate");
  cudaGraphDestroy(g);
}

void GpuBatch::run_iterations(long long n) {
  if (n <= 0) return;
  if (!graph_) {
    build_graph();
    --n;
  }
  while (n >= graph_iters_) {
    check(cudaGraphLaunch(graph_, stream_), "graph launch");
    n -= graph_iters_;
  }
  for (; n > 0; --n) launch_iteration();
}

void GpuBatch::run_iterations_timed(long long n, double* leader_ms, double* column_ms, double* total_ms) {
  *leader_ms = *column_ms = *total_ms = 0.0;
  if (n <= 0) return;
  std::vector<cudaEvent_t> ev(static_cast<size_t>(2 * n + 1));
  for (auto& e : ev) check(cudaEventCreate(&e), "cudaEventCreate");
  try {
    check(cudaEventRecord(ev[0], stream_), "cudaEventRecord");
    for (long long i = 0; i < n; ++i) {
      check(launch_leader_batch(*lb_, stream_), "batched leader");
      check(cudaEventRecord(ev[2 * i + 1], stream_), "cudaEventRecord");
      check(launch_column_batch(*cb_, stream_), "batched column");
      check(cudaEventRecord(ev[2 * i + 2], stream_), "cudaEventRecord");
    }
    check(cudaEventSynchronize(ev[2 * n]), "cudaEventSynchronize");
    for (long long i = 0; i < n; ++i) {
      float a = 0.f, b = 0.f;
      check(cudaEventElapsedTime(&a, ev[2 * i], ev[2 * i + 1]), "cudaEventElapsedTime");
      check(cudaEventElapsedTime(&b, ev[2 * i + 1], ev[2 * i + 2]), "cudaEventElapsedTime");
      *leader_ms += a;
      *column_ms += b;
    }
    float t = 0.f;
    check(cudaEventElapsedTime(&t, ev[0], ev[2 * n]), "cudaEventElapsedTime");
    *total_ms = t;
  } catch (...) {
    for (auto& e : ev) cudaEventDestroy(e);
    throw;
  }
  for (auto& e : ev) cudaEventDestroy(e);
}

mcd_report GpuBatch::report(int i) { return inst_.at(static_cast<size_t>(i))->report(); }

int GpuBatch::solve(int (*cb)(int, const mcd_report*, void*), void* user) {
  reset();
  const auto t0 = std::chrono::steady_clock::now();
  const long long chunks = opt_.num_iterations / opt_.report_interval;
  for (long long c = 0; c < chunks; ++c) {
    run_iterations(opt_.report_interval);
    bool stop = false;
    for (int i = 0; i < size(); ++i) {
      mcd_report r = report(i);
      r.time_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      energies_[static_cast<size_t>(i)] = r.energy;
      if (opt_.verbose) {
        std::cout << "instance " << std::setw(3) << i << "  iteration " << std::setw(10) << r.iteration
                  << "  energy " << std::fixed << std::setprecision(10) << r.energy << "  |x|_0 " << r.x_size
                  << "  |z|_0 " << r.z_size << "  time " << std::setprecision(2) << r.time_s << std::endl;
      }
      if (cb && cb(i, &r, user) != 0) stop = true;
    }
    if (stop) return MCD_STOPPED;
  }
  for (int i = 0; i < size(); ++i) energies_[static_cast<size_t>(i)] = report(i).energy;
  return MCD_OK;
}

}  // namespace mcd
