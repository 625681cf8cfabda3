// extern "C" layer: the only boundary of the library (include/mcdfci.h).
// Exceptions stop here and become MCD_* status codes with a message kept per
// thread for mcd_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <memory>
#include <string>
#include <vector>

#include "../../include/mcdfci.h"
#include "fcidump.h"
#include "gpu_batch.h"
#include "gpu_solver.h"
#include "json.h"

struct mcd_solver {
  std::unique_ptr<mcd::GpuSolver> impl;
};

struct mcd_batch {
  std::unique_ptr<mcd::GpuBatch> impl;
};

struct mcd_fcidump {
  mcd::Fcidump f;
  std::vector<double> orbital_energy;  // dense copy when every spin-orbital has one
};

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

template <typename F>
int guarded(F&& f) {
  try {
    g_last_error.clear();
    return f();
  } catch (const mcd::McdError& e) {
    return fail(e.code, e.what());
  } catch (const std::invalid_argument& e) {
    return fail(MCD_ERR_INVALID, e.what());
  } catch (const std::bad_alloc&) {
    return fail(MCD_ERR_INVALID, "host memory allocation failed");
  } catch (const std::exception& e) {
    return fail(MCD_ERR_INVALID, e.what());
  }
}

mcd::SolverOptions to_options(const mcd_options* o) {
  mcd::SolverOptions s;
  s.num_iterations = o->num_iterations;
  s.report_interval = o->report_interval;
  s.k = o->num_of_coordinate;
  s.m = o->estimate;
  s.z_threshold = o->z_threshold;
  s.z_threshold_search = o->z_threshold_search != 0;
  s.max_memory = o->max_memory;
  s.threshold = o->threshold;
  if (o->ref_det_occ && o->n_ref_det_occ > 0) s.ref_det_occ.assign(o->ref_det_occ, o->ref_det_occ + o->n_ref_det_occ);
  s.coordinate_pick = o->coordinate_pick;
  s.coordinate_update = o->coordinate_update;
  s.groups = o->groups;
  s.compaction = o->compaction != 0;
  s.table_growth = o->table_growth != 0;
  if (o->eig_method < 0 || o->eig_method > 2) throw mcd::McdError(MCD_ERR_INVALID, "eig_method must be 0, 1 or 2.");
  s.eig_method = o->eig_method;
  s.autotune = o->autotune != 0;
  s.verbose = o->verbose != 0;
  s.stream = static_cast<cudaStream_t>(o->stream);
  s.device = o->device;
  return s;
}

mcd::Fcidump problem_to_fcidump(const mcd_problem* p) {
  if (!p) throw mcd::McdError(MCD_ERR_INVALID, "problem is NULL.");
  return mcd::fcidump_from_arrays(p->norb, p->nelec, p->ms2, p->uhf != 0, p->core_energy, p->h1, p->g2,
                                  p->orbital_energy);
}

void print_header() {
  std::cout << "mcdfci-b200: multi-coordinate-descent FCI on one GPU" << std::endl << std::endl;
  int dev = 0;
  cudaDeviceProp prop{};
  if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
    std::cout << "GPU: " << prop.name << " (" << prop.multiProcessorCount << " SMs, "
              << prop.totalGlobalMem / (1024.0 * 1024 * 1024) << " GiB)" << std::endl;
  std::cout << "=======================================================" << std::endl << std::endl;
}

// read_input (src/run_wrapper.h:61-122): defaults, merge-patch, validation.
mcd::Json read_input(const std::string& path) {
  mcd::Json cd = mcd::Json::object();
  cd["num_iterations"] = mcd::Json::number(10);
  cd["report_interval"] = mcd::Json::number(1);
  cd["coordinate_pick"] = mcd::Json::string("gcd_grad");
  cd["coordinate_update"] = mcd::Json::string("ls");
  cd["ref_det_occ"] = mcd::Json::array();
  cd["z_threshold"] = mcd::Json::number(0.0);
  cd["z_threshold_search"] = mcd::Json::boolean(false);
  cd["max_wavefunction_size"] = mcd::Json::number(1);
  cd["max_memory"] = mcd::Json::number(0.0);
  cd["num_of_coordinate"] = mcd::Json::number(1);
  cd["estimate"] = mcd::Json::number(100);
  mcd::Json hm = mcd::Json::object();
  hm["type"] = mcd::Json::string("molecule");
  hm["threshold"] = mcd::Json::number(1e-13);

  mcd::Json option = mcd::Json::parse_file(path);
  cd.merge_patch(option.at("solver").at("cdfci"));
  option["solver"]["cdfci"] = cd;
  hm.merge_patch(option.at("hamiltonian"));
  option["hamiltonian"] = hm;

  if (option.at("hamiltonian").at("type").as_string("hamiltonian:type") != "molecule")
    throw std::invalid_argument(
        "hamiltonian:type is invalid. Currently the only supported Hamiltonian is \"molecule\".");
  const double max_memory = cd.at("max_memory").as_number("max_memory");
  if (max_memory <= 0.0)
    throw std::invalid_argument(
        "solver:cdfci:max_memory is invalid. It is the maximum memory (GB) allowed for the wavefunction. "
        "Please set a positive number.");
  const bool search = cd.at("z_threshold_search").as_bool("z_threshold_search");
  const double zt = cd.at("z_threshold").as_number("z_threshold");
  if (search) {
    std::cout << "Warning: z cut-off threshold auto search (z_threshold_search) is enabled. This feature is "
                 "experimental and may not always work."
              << std::endl
              << std::endl;
    if (zt < 1e-10)
      std::cout << "Warning: The initial z_threshold may be too small. Set z_threshold = 1.00e-10" << std::endl
                << std::endl;
  }
  if (search && cd.at("report_interval").as_number("report_interval") < 1000)
    throw std::invalid_argument("Please set report_interval >= 1000 when z_threshold_search = true.");
  return option;
}

void options_from_json(const mcd::Json& option, mcd_options* o, std::vector<int32_t>* occ) {
  const mcd::Json& cd = option.at("solver").at("cdfci");
  mcd_options_default(o);
  o->num_iterations = static_cast<int64_t>(cd.at("num_iterations").as_number("num_iterations"));
  o->report_interval = static_cast<int64_t>(cd.at("report_interval").as_number("report_interval"));
  o->num_of_coordinate = static_cast<int32_t>(cd.at("num_of_coordinate").as_number("num_of_coordinate"));
  o->estimate = static_cast<int32_t>(cd.at("estimate").as_number("estimate"));
  o->z_threshold = cd.at("z_threshold").as_number("z_threshold");
  o->z_threshold_search = cd.at("z_threshold_search").as_bool("z_threshold_search") ? 1 : 0;
  o->max_memory = cd.at("max_memory").as_number("max_memory");
  o->threshold = option.at("hamiltonian").at("threshold").as_number("hamiltonian:threshold");
  if (cd.has("groups")) o->groups = static_cast<int32_t>(cd.at("groups").as_number("groups"));
  if (cd.has("compaction")) o->compaction = cd.at("compaction").as_bool("compaction") ? 1 : 0;
  if (cd.has("table_growth")) o->table_growth = cd.at("table_growth").as_bool("table_growth") ? 1 : 0;
  if (cd.has("eig_method")) o->eig_method = static_cast<int32_t>(cd.at("eig_method").as_number("eig_method"));
  if (cd.has("autotune")) o->autotune = cd.at("autotune").as_bool("autotune") ? 1 : 0;
  const std::string pick = cd.at("coordinate_pick").as_string("coordinate_pick");
  const std::string upd = cd.at("coordinate_update").as_string("coordinate_update");
  if (pick != "gcd_grad") throw mcd::McdError(MCD_ERR_INVALID, "the coordinate pick method \"" + pick + "\" is not implemented.");
  if (upd == "eig")
    o->coordinate_update = MCD_UPDATE_EIG;
  else if (upd == "ls")
    o->coordinate_update = MCD_UPDATE_LS;
  else
    throw mcd::McdError(MCD_ERR_INVALID, "the coordinate update method \"" + upd + "\" is not implemented.");
  for (const auto& v : cd.at("ref_det_occ").items()) occ->push_back(static_cast<int32_t>(v.as_number("ref_det_occ")));
  o->ref_det_occ = occ->empty() ? nullptr : occ->data();
  o->n_ref_det_occ = static_cast<int32_t>(occ->size());
}

}  // namespace

extern "C" {

const char* mcd_last_error(void) { return g_last_error.c_str(); }

void mcd_options_default(mcd_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->num_iterations = 10;
  o->report_interval = 1;
  o->num_of_coordinate = 1;
  o->estimate = 100;
  o->z_threshold = 0.0;
  o->z_threshold_search = 0;
  o->max_memory = 0.0;
  o->threshold = 1e-13;
  o->coordinate_pick = MCD_PICK_GCD_GRAD;
  o->coordinate_update = MCD_UPDATE_EIG;
  o->groups = 0;
  o->compaction = 0;
  o->table_growth = 1;
  o->eig_method = 2;
  o->autotune = 0;
  o->verbose = 0;
  o->stream = nullptr;
  o->device = -1;
}

int mcd_fcidump_read(const char* path, mcd_fcidump** out) {
  return guarded([&] {
    if (!path || !out) return fail(MCD_ERR_INVALID, "path and out must not be NULL.");
    *out = nullptr;
    auto f = std::make_unique<mcd_fcidump>();
    f->f = mcd::read_fcidump(path);
    if (static_cast<int>(f->f.orbital_energy.size()) == f->f.norb) {
      f->orbital_energy.resize(f->f.norb);
      for (const auto& kv : f->f.orbital_energy) f->orbital_energy[kv.first] = kv.second;
    }
    *out = f.release();
    return MCD_OK;
  });
}

int mcd_fcidump_problem(const mcd_fcidump* f, mcd_problem* v) {
  if (!f || !v) return fail(MCD_ERR_INVALID, "NULL argument.");
  v->norb = f->f.norb;
  v->nelec = f->f.nelec;
  v->ms2 = f->f.ms2;
  v->uhf = f->f.uhf ? 1 : 0;
  v->core_energy = f->f.core_energy;
  v->h1 = f->f.h1.data();
  v->g2 = f->f.g2.data();
  v->orbital_energy = f->orbital_energy.empty() ? nullptr : f->orbital_energy.data();
  return MCD_OK;
}

void mcd_fcidump_free(mcd_fcidump* f) { delete f; }

int mcd_create(const mcd_problem* problem, const mcd_options* options, mcd_solver** out) {
  return guarded([&] {
    if (!out || !options) return fail(MCD_ERR_INVALID, "options and out must not be NULL.");
    *out = nullptr;
    mcd::Fcidump fci = problem_to_fcidump(problem);
    auto s = std::make_unique<mcd_solver>();
    s->impl = std::make_unique<mcd::GpuSolver>(fci, to_options(options));
    *out = s.release();
    return MCD_OK;
  });
}

// Internal: create from an already parsed FCIDUMP, keeping its orbital energies.
static int create_from_fcidump(const mcd::Fcidump& fci, const mcd_options* options, mcd_solver** out) {
  return guarded([&] {
    *out = nullptr;
    auto s = std::make_unique<mcd_solver>();
    s->impl = std::make_unique<mcd::GpuSolver>(fci, to_options(options));
    *out = s.release();
    return MCD_OK;
  });
}

int mcd_create_from_fcidump(const mcd_fcidump* f, const mcd_options* options, mcd_solver** out) {
  if (!f || !options || !out) return fail(MCD_ERR_INVALID, "NULL argument.");
  return create_from_fcidump(f->f, options, out);
}

void mcd_destroy(mcd_solver* s) { delete s; }

// ---- Batches ----------------------------------------------------------------

int mcd_batch_create(const mcd_fcidump* const* fcidumps, int32_t n, const mcd_options* options, mcd_batch** out) {
  return guarded([&] {
    if (!fcidumps || !options || !out) return fail(MCD_ERR_INVALID, "NULL argument.");
    *out = nullptr;
    if (n < 1) return fail(MCD_ERR_INVALID, "a batch needs at least one FCIDUMP.");
    std::vector<const mcd::Fcidump*> f;
    for (int32_t i = 0; i < n; ++i) {
      if (!fcidumps[i]) return fail(MCD_ERR_INVALID, "NULL FCIDUMP in the batch.");
      f.push_back(&fcidumps[i]->f);
    }
    auto b = std::make_unique<mcd_batch>();
    b->impl = std::make_unique<mcd::GpuBatch>(f, to_options(options));
    *out = b.release();
    return MCD_OK;
  });
}

void mcd_batch_destroy(mcd_batch* b) { delete b; }

int mcd_batch_size(const mcd_batch* b, int32_t* n) {
  if (!b || !n) return fail(MCD_ERR_INVALID, "NULL argument.");
  *n = b->impl->size();
  return MCD_OK;
}

int mcd_batch_solve(mcd_batch* b, mcd_batch_report_cb cb, void* user) {
  return guarded([&] {
    if (!b) return fail(MCD_ERR_INVALID, "batch is NULL.");
    return b->impl->solve(cb, user);
  });
}

int mcd_batch_reset(mcd_batch* b) {
  return guarded([&] {
    if (!b) return fail(MCD_ERR_INVALID, "batch is NULL.");
    b->impl->reset();
    return MCD_OK;
  });
}

int mcd_batch_run_iterations(mcd_batch* b, int64_t n) {
  return guarded([&] {
    if (!b) return fail(MCD_ERR_INVALID, "batch is NULL.");
    b->impl->run_iterations(n);
    return MCD_OK;
  });
}

int mcd_batch_run_iterations_timed(mcd_batch* b, int64_t n, double* leader_ms, double* column_ms, double* total_ms) {
  return guarded([&] {
    if (!b || !leader_ms || !column_ms || !total_ms) return fail(MCD_ERR_INVALID, "NULL argument.");
    b->impl->run_iterations_timed(n, leader_ms, column_ms, total_ms);
    return MCD_OK;
  });
}

int mcd_batch_table_sums(mcd_batch* b, int32_t instance, double xx[2], double xz[2], uint64_t* occupied) {
  return guarded([&] {
    if (!b) return fail(MCD_ERR_INVALID, "batch is NULL.");
    if (instance < 0 || instance >= b->impl->size()) return fail(MCD_ERR_INVALID, "instance out of range.");
    mcd::dd a, c;
    unsigned long long n = 0;
    b->impl->instance(instance).table_sums(&a, &c, &n);
    if (xx) { xx[0] = a.hi; xx[1] = a.lo; }
    if (xz) { xz[0] = c.hi; xz[1] = c.lo; }
    if (occupied) *occupied = n;
    return MCD_OK;
  });
}

int mcd_batch_residual(mcd_batch* b, int32_t instance, double* residual) {
  return guarded([&] {
    if (!b || !residual) return fail(MCD_ERR_INVALID, "NULL argument.");
    if (instance < 0 || instance >= b->impl->size()) return fail(MCD_ERR_INVALID, "instance out of range.");
    *residual = b->impl->instance(instance).residual();
    return MCD_OK;
  });
}

int mcd_batch_get_report(mcd_batch* b, int32_t instance, mcd_report* r) {
  return guarded([&] {
    if (!b || !r) return fail(MCD_ERR_INVALID, "NULL argument.");
    if (instance < 0 || instance >= b->impl->size()) return fail(MCD_ERR_INVALID, "instance out of range.");
    *r = b->impl->report(instance);
    return MCD_OK;
  });
}

int mcd_batch_result(const mcd_batch* b, double* energies) {
  if (!b || !energies) return fail(MCD_ERR_INVALID, "NULL argument.");
  for (int i = 0; i < b->impl->size(); ++i) energies[i] = b->impl->result_energy(i);
  return MCD_OK;
}

int mcd_solve(mcd_solver* s, mcd_report_cb cb, void* user) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    return s->impl->solve(cb, user);
  });
}

int mcd_reset(mcd_solver* s) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    s->impl->reset();
    return MCD_OK;
  });
}

int mcd_run_iterations(mcd_solver* s, int64_t n) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    s->impl->run_iterations(n);
    return MCD_OK;
  });
}

int mcd_run_iterations_timed(mcd_solver* s, int64_t n, double* leader_ms, double* column_ms, double* total_ms) {
  return guarded([&] {
    if (!s || !leader_ms || !column_ms || !total_ms) return fail(MCD_ERR_INVALID, "NULL argument.");
    s->impl->run_iterations_timed(n, leader_ms, column_ms, total_ms);
    return MCD_OK;
  });
}

int mcd_get_report(mcd_solver* s, mcd_report* r) {
  return guarded([&] {
    if (!s || !r) return fail(MCD_ERR_INVALID, "NULL argument.");
    *r = s->impl->report();
    return MCD_OK;
  });
}

int mcd_result(const mcd_solver* s, double* energy) {
  if (!s || !energy) return fail(MCD_ERR_INVALID, "NULL argument.");
  *energy = s->impl->result_energy();
  return MCD_OK;
}

int mcd_stream(const mcd_solver* s, void** stream) {
  if (!s || !stream) return fail(MCD_ERR_INVALID, "NULL argument.");
  *stream = s->impl->stream();
  return MCD_OK;
}

int mcd_scalars(mcd_solver* s, double xx[2], double scale[2], double xz[2], int64_t* iteration) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    mcd::dd a, b, c;
    long long it = 0;
    s->impl->scalars(&a, &b, &c, &it);
    if (xx) { xx[0] = a.hi; xx[1] = a.lo; }
    if (scale) { scale[0] = b.hi; scale[1] = b.lo; }
    if (xz) { xz[0] = c.hi; xz[1] = c.lo; }
    if (iteration) *iteration = it;
    return MCD_OK;
  });
}

int mcd_run_json(const char* input_json_path) {
  try {
    print_header();
    if (!input_json_path)
      throw std::invalid_argument("No input file specified. Please use the path of the input file as the first argument.");
    mcd::Json option = read_input(input_json_path);
    const std::string path = option.at("hamiltonian").at("fcidump_path").as_string("hamiltonian:fcidump_path");
    mcd::Fcidump fci = mcd::read_fcidump(path);
    const int n = 1 + (fci.norb - 1) / 64;
    std::cout << "FCIDUMP information" << std::endl << "-------------------" << std::endl;
    std::cout << "Number of elections: " << fci.nelec << std::endl;
    std::cout << "Number of spin-orbitals: " << fci.norb << std::endl;
    std::cout << "Ms2: " << fci.ms2 << std::endl;
    std::cout << "Hartree Fock: " << (fci.uhf ? "unrestricted" : "restricted") << std::endl << std::endl;
    std::cout << "Number of 64-bit words per determinant in the reference layout: " << n << std::endl;
    std::cout << "Determinant storage: alpha/beta uint64 strings, 32-byte hash slots" << std::endl << std::endl;
    mcd_options o;
    std::vector<int32_t> occ;
    options_from_json(option, &o, &occ);
    o.verbose = 1;
    std::cout << "Input option" << std::endl << "------------" << std::endl << option.dump(4) << std::endl;
    mcd_solver* s = nullptr;
    int rc = create_from_fcidump(fci, &o, &s);
    if (rc != MCD_OK) throw std::runtime_error(g_last_error);
    std::cout << "Note:" << std::endl;
    std::cout << "The hash wavefunction has " << s->impl->table_capacity() << " slots of 32 bytes ("
              << std::fixed << std::setprecision(3) << s->impl->table_capacity() * 32.0 / 1073741824.0
              << " GB) and can store " << s->impl->max_wavefunction_size() << " determinants at most." << std::endl;
    std::cout << "Each Hamiltonian column has " << s->impl->entries_per_column() << " candidate entries, "
              << s->impl->groups() << " CTA(s) per column." << std::endl
              << std::endl;
    rc = mcd_solve(s, nullptr, nullptr);
    const std::string err = g_last_error;
    mcd_destroy(s);
    if (rc != MCD_OK) throw std::runtime_error(err);
    return 0;
  } catch (const std::exception& e) {
    std::cerr << std::endl << "ERROR: " << e.what() << std::endl;
    g_last_error = e.what();
    return 1;
  }
}

int mcd_debug_column(mcd_solver* s, uint64_t alpha, uint64_t beta, uint64_t* alpha_out, uint64_t* beta_out,
                     double* value_out, int64_t cap, int64_t* n_out) {
  return guarded([&] {
    if (!s || !n_out) return fail(MCD_ERR_INVALID, "NULL argument.");
    auto col = s->impl->column(mcd::Det{alpha, beta});
    *n_out = static_cast<int64_t>(col.size());
    for (int64_t i = 0; i < cap && i < static_cast<int64_t>(col.size()); ++i) {
      alpha_out[i] = col[i].first.a;
      beta_out[i] = col[i].first.b;
      value_out[i] = col[i].second;
    }
    return MCD_OK;
  });
}

int mcd_debug_hsub(mcd_solver* s, const uint64_t* alpha, const uint64_t* beta, int32_t k, double* hsub) {
  return guarded([&] {
    if (!s || !alpha || !beta || !hsub || k < 1) return fail(MCD_ERR_INVALID, "bad argument.");
    std::vector<mcd::Det> dets(k);
    for (int i = 0; i < k; ++i) dets[i] = mcd::Det{alpha[i], beta[i]};
    auto h = s->impl->hsub(dets);
    std::memcpy(hsub, h.data(), h.size() * sizeof(double));
    return MCD_OK;
  });
}

}  // extern "C"

namespace {

// mcd_debug_eig / mcd_debug_eig_shifted: one eig update on the current device
// from host buffers; the device buffers are released on every path.
int debug_eig_host(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                   const double xz[2], double drop, int method, double* dx, double new_xx[2],
                   double new_scale[2], int32_t* branch, int32_t* steps) {
  if (k < 1 || k > mcd::kMaxK) return fail(MCD_ERR_UNSUPPORTED, "k must be in 1..128.");
  if (!hsub || !x || !z || !xx || !xz || !dx || !new_xx || !new_scale) return fail(MCD_ERR_INVALID, "NULL argument.");
  struct Buffers {
    double *h = nullptr, *x = nullptr, *z = nullptr, *dx = nullptr;
    mcd::dd* out = nullptr;
    int *br = nullptr, *steps = nullptr;
    unsigned* err = nullptr;
    ~Buffers() {
      cudaFree(h);
      cudaFree(x);
      cudaFree(z);
      cudaFree(dx);
      cudaFree(out);
      cudaFree(br);
      cudaFree(steps);
      cudaFree(err);
    }
  } b;
  auto ck = [](cudaError_t e) {
    if (e != cudaSuccess) throw mcd::McdError(MCD_ERR_CUDA, cudaGetErrorString(e));
  };
  ck(cudaMalloc(&b.h, sizeof(double) * k * k));
  ck(cudaMalloc(&b.x, sizeof(double) * k));
  ck(cudaMalloc(&b.z, sizeof(double) * k));
  ck(cudaMalloc(&b.dx, sizeof(double) * k));
  ck(cudaMalloc(&b.out, sizeof(mcd::dd) * 2));
  ck(cudaMalloc(&b.br, sizeof(int)));
  ck(cudaMalloc(&b.steps, sizeof(int)));
  ck(cudaMalloc(&b.err, sizeof(unsigned)));
  ck(cudaMemcpy(b.h, hsub, sizeof(double) * k * k, cudaMemcpyHostToDevice));
  ck(cudaMemcpy(b.x, x, sizeof(double) * k, cudaMemcpyHostToDevice));
  ck(cudaMemcpy(b.z, z, sizeof(double) * k, cudaMemcpyHostToDevice));
  ck(cudaMemset(b.steps, 0, sizeof(int)));
  ck(mcd::debug_eig(k, b.h, b.x, b.z, mcd::dd{xx[0], xx[1]}, mcd::dd{xz[0], xz[1]}, b.dx, b.out, b.br, b.err, 0,
                    drop, b.steps, method));
  mcd::dd out[2];
  int br = 0, st = 0;
  unsigned err = 0;
  ck(cudaMemcpy(dx, b.dx, sizeof(double) * k, cudaMemcpyDeviceToHost));
  ck(cudaMemcpy(out, b.out, sizeof(out), cudaMemcpyDeviceToHost));
  ck(cudaMemcpy(&br, b.br, sizeof(int), cudaMemcpyDeviceToHost));
  ck(cudaMemcpy(&st, b.steps, sizeof(int), cudaMemcpyDeviceToHost));
  ck(cudaMemcpy(&err, b.err, sizeof(unsigned), cudaMemcpyDeviceToHost));
  new_xx[0] = out[0].hi;
  new_xx[1] = out[0].lo;
  new_scale[0] = out[1].hi;
  new_scale[1] = out[1].lo;
  if (branch) *branch = br;
  if (steps) *steps = st;
  if (err) return fail(MCD_ERR_EIG, "The subspace eigenvalue problem failed.");
  return MCD_OK;
}

}  // namespace

extern "C" {

int mcd_debug_eig(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                  const double xz[2], double* dx, double new_xx[2], double new_scale[2], int32_t* branch) {
  return guarded([&] { return debug_eig_host(k, hsub, x, z, xx, xz, 0.0, 0, dx, new_xx, new_scale, branch, nullptr); });
}

int mcd_debug_eig_shifted(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                          const double xz[2], double drop, double* dx, double new_xx[2], double new_scale[2],
                          int32_t* branch, int32_t* steps) {
  return guarded([&] {
    if (!(drop > 0.0)) return fail(MCD_ERR_INVALID, "drop must be positive.");
    return debug_eig_host(k, hsub, x, z, xx, xz, drop, 1, dx, new_xx, new_scale, branch, steps);
  });
}

int mcd_debug_eig_method(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                         const double xz[2], int32_t method, double drop, double* dx, double new_xx[2],
                         double new_scale[2], int32_t* branch, int32_t* steps) {
  return guarded([&] {
    if (method < 0 || method > 2) return fail(MCD_ERR_INVALID, "method must be 0, 1 or 2.");
    if (method == 1 && !(drop > 0.0)) return fail(MCD_ERR_INVALID, "drop must be positive for method 1.");
    return debug_eig_host(k, hsub, x, z, xx, xz, method == 1 ? drop : 0.0, method, dx, new_xx, new_scale, branch,
                          steps);
  });
}

int mcd_eig_update_static(int32_t k, const double* hsub, const double* x, const double* z, const double xx[2],
                          const double xz[2], double* dx, double new_xx[2], double new_scale[2], int32_t* branch,
                          void* stream) {
  return guarded([&] {
    if (k < 1 || k > mcd::kStaticEigMaxK)
      return fail(MCD_ERR_UNSUPPORTED, "mcd_eig_update_static: k = " + std::to_string(k) +
                                           " is outside 1..128, the size of its static device scratch.");
    if (!hsub || !x || !z || !xx || !xz || !dx || !new_xx || !new_scale)
      return fail(MCD_ERR_INVALID, "mcd_eig_update_static: NULL argument.");
    mcd::dd out[2];
    int br = 0;
    unsigned err = 0;
    const cudaError_t e = mcd::eig_update_static(k, hsub, x, z, mcd::dd{xx[0], xx[1]}, mcd::dd{xz[0], xz[1]}, dx,
                                                 out, &br, &err, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(MCD_ERR_CUDA, cudaGetErrorString(e));
    new_xx[0] = out[0].hi;
    new_xx[1] = out[0].lo;
    new_scale[0] = out[1].hi;
    new_scale[1] = out[1].lo;
    if (branch) *branch = br;
    if (err) return fail(MCD_ERR_EIG, "The subspace eigenvalue problem failed.");
    return MCD_OK;
  });
}

int mcd_rdm(mcd_solver* s, double* rdm1, double* rdm2) {
  return guarded([&] {
    if (!s || !rdm1 || !rdm2) return fail(MCD_ERR_INVALID, "NULL argument.");
    std::vector<double> g1, g2;
    s->impl->rdm(g1, g2);
    std::copy(g1.begin(), g1.end(), rdm1);
    std::copy(g2.begin(), g2.end(), rdm2);
    return MCD_OK;
  });
}

int mcd_debug_wavefunction(mcd_solver* s, uint64_t* alpha, uint64_t* beta, double* x, int64_t cap, int64_t* n_out) {
  return guarded([&] {
    if (!s || !n_out) return fail(MCD_ERR_INVALID, "NULL argument.");
    std::vector<mcd::Det> d;
    std::vector<double> v;
    s->impl->wavefunction(d, v);
    *n_out = static_cast<int64_t>(d.size());
    const int64_t m = std::min<int64_t>(cap, static_cast<int64_t>(d.size()));
    for (int64_t i = 0; i < m; ++i) {
      if (alpha) alpha[i] = d[static_cast<size_t>(i)].a;
      if (beta) beta[i] = d[static_cast<size_t>(i)].b;
      if (x) x[i] = v[static_cast<size_t>(i)];
    }
    return MCD_OK;
  });
}

int mcd_checkpoint_save(mcd_solver* s, const char* path) {
  return guarded([&] {
    if (!s || !path) return fail(MCD_ERR_INVALID, "NULL argument.");
    s->impl->checkpoint_save(path);
    return MCD_OK;
  });
}

int mcd_checkpoint_load(mcd_solver* s, const char* path) {
  return guarded([&] {
    if (!s || !path) return fail(MCD_ERR_INVALID, "NULL argument.");
    s->impl->checkpoint_load(path);
    return MCD_OK;
  });
}

int mcd_debug_compact(mcd_solver* s, double z_threshold, uint64_t* occupied) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    const unsigned long long occ = s->impl->compact(z_threshold);
    if (occupied) *occupied = occ;
    return MCD_OK;
  });
}

int mcd_debug_grow(mcd_solver* s, int32_t mode, int64_t* wrap_slots) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    long long w = 0;
    if (!s->impl->grow_now(mode, &w)) return fail(MCD_ERR_INVALID, "the table is at its full size.");
    if (wrap_slots) *wrap_slots = w;
    return MCD_OK;
  });
}

int mcd_debug_table_sums(mcd_solver* s, double xx[2], double xz[2], uint64_t* occupied) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    mcd::dd a, b;
    unsigned long long c = 0;
    s->impl->table_sums(&a, &b, &c);
    if (xx) { xx[0] = a.hi; xx[1] = a.lo; }
    if (xz) { xz[0] = b.hi; xz[1] = b.lo; }
    if (occupied) *occupied = c;
    return MCD_OK;
  });
}

int mcd_residual(mcd_solver* s, double* residual) {
  return guarded([&] {
    if (!s || !residual) return fail(MCD_ERR_INVALID, "NULL argument.");
    *residual = s->impl->residual();
    return MCD_OK;
  });
}

int mcd_debug_slots(mcd_solver* s, uint64_t* alpha, uint64_t* beta, double* x, double* z, int64_t cap,
                    int64_t* n_out) {
  return guarded([&] {
    if (!s || !n_out) return fail(MCD_ERR_INVALID, "NULL argument.");
    std::vector<mcd::Slot> v;
    s->impl->slots(v);
    *n_out = static_cast<int64_t>(v.size());
    for (int64_t i = 0; i < cap && i < static_cast<int64_t>(v.size()); ++i) {
      if (alpha) alpha[i] = v[i].a;
      if (beta) beta[i] = v[i].b;
      if (x) x[i] = v[i].x;
      if (z) z[i] = v[i].z;
    }
    return MCD_OK;
  });
}

int mcd_debug_leader_sections(mcd_solver* s, uint64_t* cycles, int32_t n) {
  return guarded([&] {
    if (!s || !cycles) return fail(MCD_ERR_INVALID, "NULL argument.");
    auto v = s->impl->leader_sections();
    for (int32_t i = 0; i < n && i < static_cast<int32_t>(v.size()); ++i) cycles[i] = v[i];
    return MCD_OK;
  });
}

int mcd_debug_column_sections(mcd_solver* s, uint64_t* cycles, int32_t n, int32_t enable) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    auto v = s->impl->column_sections(enable != 0);
    for (int32_t i = 0; cycles && i < n && i < static_cast<int32_t>(v.size()); ++i) cycles[i] = v[i];
    return MCD_OK;
  });
}

int mcd_debug_scatter_rate_mode(mcd_solver* s, int64_t entries, int32_t reps, int32_t ilp, int32_t ctas_per_sm,
                                int32_t mode, double* slots_per_s) {
  return guarded([&] {
    if (!s || !slots_per_s) return fail(MCD_ERR_INVALID, "NULL argument.");
    if (mode < 0 || mode > 3) return fail(MCD_ERR_INVALID, "mode must be 0..3.");
    *slots_per_s = s->impl->scatter_rate(entries, reps, ilp, ctas_per_sm, mode);
    return MCD_OK;
  });
}

int mcd_debug_scatter_rate(mcd_solver* s, int64_t entries, int32_t reps, int32_t ilp, int32_t ctas_per_sm,
                           double* slots_per_s) {
  return guarded([&] {
    if (!s || !slots_per_s) return fail(MCD_ERR_INVALID, "NULL argument.");
    *slots_per_s = s->impl->scatter_rate(entries, reps, ilp, ctas_per_sm);
    return MCD_OK;
  });
}

int mcd_debug_autotune_info(const mcd_solver* s, int32_t* rule, int32_t* chosen, int32_t* trial_groups,
                            double* trial_us, int32_t cap, int32_t* n) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    if (rule) *rule = s->impl->groups_rule();
    if (chosen) *chosen = s->impl->groups();
    const auto& t = s->impl->tune_trials();
    if (n) *n = static_cast<int32_t>(t.size());
    for (int32_t i = 0; i < cap && i < static_cast<int32_t>(t.size()); ++i) {
      if (trial_groups) trial_groups[i] = t[i].first;
      if (trial_us) trial_us[i] = t[i].second;
    }
    return MCD_OK;
  });
}

int mcd_debug_table_info(const mcd_solver* s, uint64_t* capacity, uint64_t* max_capacity, int32_t* growths) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    if (capacity) *capacity = static_cast<uint64_t>(s->impl->table_capacity());
    if (max_capacity) *max_capacity = static_cast<uint64_t>(s->impl->table_max_capacity());
    if (growths) *growths = s->impl->table_growths();
    return MCD_OK;
  });
}

int mcd_debug_setup_times(const mcd_solver* s, double* ms, int32_t n) {
  return guarded([&] {
    if (!s || !ms) return fail(MCD_ERR_INVALID, "NULL argument.");
    for (int32_t i = 0; i < n && i < mcd::GpuSolver::kSetupStages; ++i) ms[i] = s->impl->setup_ms()[i];
    return MCD_OK;
  });
}

int mcd_debug_launch_info(mcd_solver* s, int32_t* groups, int32_t* list_size, int32_t* entries) {
  return guarded([&] {
    if (!s) return fail(MCD_ERR_INVALID, "solver is NULL.");
    if (groups) *groups = s->impl->groups();
    if (list_size) *list_size = s->impl->list_size();
    if (entries) *entries = s->impl->entries_per_column();
    return MCD_OK;
  });
}

int mcd_debug_last_eig(mcd_solver* s, double* hsub, double* x, double* z, double xx[2], double xz[2], int32_t cap,
                       int32_t* k_out) {
  return guarded([&] {
    if (!s || !k_out) return fail(MCD_ERR_INVALID, "NULL argument.");
    *k_out = static_cast<int32_t>(s->impl->last_eig_inputs(hsub, x, z, xx, xz, cap));
    return MCD_OK;
  });
}

int mcd_debug_picked(mcd_solver* s, uint64_t* alpha, uint64_t* beta, double* dx, int32_t cap, int32_t* k_out) {
  return guarded([&] {
    if (!s || !k_out) return fail(MCD_ERR_INVALID, "NULL argument.");
    auto p = s->impl->picked();
    *k_out = static_cast<int32_t>(p.size());
    for (int32_t i = 0; i < cap && i < static_cast<int32_t>(p.size()); ++i) {
      if (alpha) alpha[i] = p[i].first.a;
      if (beta) beta[i] = p[i].first.b;
      if (dx) dx[i] = p[i].second;
    }
    return MCD_OK;
  });
}

}  // extern "C"
