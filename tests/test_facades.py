"""The C++ facades with the reference's interface names (include/mcdfci.hpp):
a host program written against Fcidump, Determinant, Hamiltonian,
WaveFunction, CoordinatePickGcdGrad, CoordinateUpdateEig and CDFCI compiles
and links with g++ against libmcdfci.so; without a GPU its host-only parts
run (FCIDUMP read, determinant numbering, the error a missing GPU raises), on
a GPU the whole solve runs and ends at the reference's H2O energy."""
import os
import shutil
import subprocess

import pytest

from conftest import REPO, load_golden

LIBDIR = os.path.join(REPO, "mcdfci_b200")

PROGRAM = r'''
#include <cmath>
#include <cstdio>
#include "mcdfci.hpp"
using namespace mcdfci;
int main(int argc, char** argv) {
  Fcidump fci(argv[1]);
  std::printf("norb %d nelec %d\n", fci.norb(), fci.nelec());
  Determinant hf = Determinant::from_occupied({0, 1, 2, 3, 4, 5, 6, 7});
  std::printf("occupied");
  for (int so : hf.occupied_orbitals()) std::printf(" %d", so);
  std::printf("\n");
  if (argc > 2 && std::string(argv[2]) == "host") return 0;
  mcd_options o;
  mcd_options_default(&o);
  o.num_of_coordinate = 8; o.estimate = 8; o.max_memory = 0.005; o.threshold = 0.0;
  o.num_iterations = 20000; o.report_interval = 1000; o.coordinate_update = MCD_UPDATE_EIG;
  try {
    CDFCI solver(fci, o);
    Hamiltonian h = solver.hamiltonian();
    auto col = h.get_column(hf);
    std::printf("column %zu diag %.12f\n", col.size(), h.get_diagonal(hf));
    size_t j = 0;
    while (j < col.size() && col[j].first == hf) ++j;
    const double off = h.get_off_diagonal(hf, col[j].first);
    std::printf("offdiag_matches %d\n", std::fabs(off - col[j].second) <= 1e-12 * (1.0 + std::fabs(off)) ? 1 : 0);
    solver.solve(h, CoordinatePickGcdGrad(), CoordinateUpdateEig(), 8, 8);
    WaveFunction wf = solver.wavefunction();
    std::printf("energy %.10f xz_over_xx %.10f x_size %zu\n", solver.result_energy,
                (double)(wf.xz() / wf.xx()), wf.x_size());
  } catch (const Error& e) {
    std::printf("error %d %s\n", e.code, e.what());
    return 3;
  }
  return 0;
}
'''


def _build(tmp_path):
    if not shutil.which("g++"):
        pytest.skip("g++ is not available")
    src = os.path.join(str(tmp_path), "facade.cpp")
    exe = os.path.join(str(tmp_path), "facade")
    with open(src, "w") as f:
        f.write(PROGRAM)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I" + os.path.join(REPO, "include"), src, "-o", exe,
                    "-L" + LIBDIR, "-lmcdfci", "-Wl,-rpath," + LIBDIR], check=True, capture_output=True)
    return exe


def test_facades_compile_and_run_host_parts(fcidumps, tmp_path):
    exe = _build(tmp_path)
    res = subprocess.run([exe, fcidumps["h2o_sto3g"], "host"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    assert "norb 24 nelec 8" in res.stdout
    assert "occupied 0 1 2 3 4 5 6 7" in res.stdout


@pytest.mark.gpu
def test_facades_solve_h2o(fcidumps, tmp_path):
    exe = _build(tmp_path)
    res = subprocess.run([exe, fcidumps["h2o_sto3g"]], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    out = dict(l.split(" ", 1) for l in res.stdout.strip().splitlines())
    assert out["offdiag_matches"] == "1"
    e, _, rq, _, xs = out["energy"].split()
    assert abs(float(e) - load_golden("energies.json")["h2o_sto3g k8 m8 20000it"]) < 1e-6
    assert abs(float(rq) - float(e)) < 1e-9
    assert int(xs) > 0
