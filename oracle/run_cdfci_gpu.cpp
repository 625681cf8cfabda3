// The reference-side binding of this library, compiled for real: the
// run_cdfci_gpu a maintainer would add to the reference's src/run_wrapper.h
// in place of run_cdfci<N> (src/run_wrapper.h:124-173), with the reference's
// own Option (nlohmann::json), read_input and check_argument, and main as
// src/main.cpp:19-36 with run_cdfci_gpu in place of run_cdfci_wrapper.
//
// Built by `make -C oracle binding REF=<checkout>` into oracle/_ref/run_cdfci_gpu
// (it needs the reference's headers, so it lives with the oracle recipes),
// linked with mcdfci_b200/libmcdfci.so.  Test infrastructure: the library never
// uses it; tests/test_gpu_binding.py runs it on the H2O deck.
#include "run_wrapper.h"

#include "../include/mcdfci.h"

// Drop-in for run_cdfci<N>(option, fci): the same options, the same report
// table on stdout, the same return value (the energy) and error types.
double run_cdfci_gpu(Option& option) {
  const std::string path = option["hamiltonian"]["fcidump_path"];
  mcd_fcidump* f = nullptr;
  if (mcd_fcidump_read(path.c_str(), &f) != MCD_OK) throw std::invalid_argument(mcd_last_error());
  const Option& s = option["solver"]["cdfci"];
  mcd_options o;
  mcd_options_default(&o);  // the defaults of read_input, src/run_wrapper.h:64-80
  o.num_iterations = s["num_iterations"].get<long>();
  o.report_interval = s["report_interval"].get<long>();
  o.num_of_coordinate = s["num_of_coordinate"].get<int>();
  o.estimate = s["estimate"].get<int>();
  o.z_threshold = s["z_threshold"].get<double>();
  o.z_threshold_search = s["z_threshold_search"].get<bool>() ? 1 : 0;
  o.max_memory = s["max_memory"].get<double>();
  o.threshold = option["hamiltonian"]["threshold"].get<double>();
  const std::string update = s["coordinate_update"];
  o.coordinate_update = update == "eig" ? MCD_UPDATE_EIG : MCD_UPDATE_LS;
  std::vector<int32_t> occ;
  for (const auto& v : s["ref_det_occ"]) occ.push_back(v.get<int>());
  o.ref_det_occ = occ.empty() ? nullptr : occ.data();
  o.n_ref_det_occ = static_cast<int32_t>(occ.size());
  o.verbose = 1;  // the report table of CDFCI<N>::solve (src/solver.h:686-798)
  mcd_solver* h = nullptr;
  int rc = mcd_create_from_fcidump(f, &o, &h);  // tables to the GPU, table sized as src/run_wrapper.h:203-213
  mcd_fcidump_free(f);
  if (rc != MCD_OK) throw std::invalid_argument(mcd_last_error());
  rc = mcd_solve(h, nullptr, nullptr);  // CDFCI<N>::solve, z_threshold_search restarts inside
  double e = 0.0;
  if (rc == MCD_OK) mcd_result(h, &e);
  const std::string err = rc == MCD_OK ? "" : mcd_last_error();
  mcd_destroy(h);
  if (rc == MCD_ERR_OVERFLOW) throw std::overflow_error(err);  // "The hash table is full..."
  if (rc == MCD_ERR_INVALID) throw std::invalid_argument(err);
  if (rc != MCD_OK) throw std::runtime_error(err);
  return e;
}

int main(int argc, char* argv[]) {
  try {
    const std::string input_file = check_argument(argc, argv);
    Option option = read_input(input_file);
    const double e = run_cdfci_gpu(option);
    std::cout << "run_cdfci_gpu energy: " << std::fixed << std::setprecision(10) << e << std::endl;
    return 0;
  } catch (const std::exception& e) {
    std::cerr << std::endl << "ERROR: " << e.what() << std::endl;
    return 1;
  }
}
