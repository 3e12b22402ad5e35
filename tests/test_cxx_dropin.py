"""The C++ drop-in Solver (neural-pde-surrogate_b200/host/fv_solver2d.hpp) on the CPU: the reference's
own test_solver2d.cpp builds unmodified against the GPU library through it, and the function-pointer
mapping accepts exactly the reference's fluxes and limiters.  Compute needs a GPU: here every run
stops at fv_create's "no CUDA device" error, never in a CPU fallback."""
import subprocess

import pytest

from oracle import build_oracle as bo

ROOT = bo.HERE.parent


@pytest.fixture(scope="module")
def ref_headers():
    if not bo.REF_SRC.is_dir():
        pytest.skip("the reference sources are not present on this machine")
    import importlib
    importlib.import_module("neural-pde-surrogate_b200.build").build()
    return bo.REF_SRC


def test_reference_solver_test_builds_against_the_gpu_library(ref_headers):
    exe = bo.build_ref_on_fv()
    assert exe is not None and exe.exists()
    libs = subprocess.run(["ldd", str(exe)], capture_output=True, text=True, check=True).stdout
    assert "libfv.so" in libs and "not found" not in libs
    import torch
    if not torch.cuda.is_available():
        r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
        assert r.returncode != 0 and "fv_create: no CUDA device available" in r.stderr


PROBE = r"""
#include "fv_solver2d.hpp"
#include <cstdio>
#include <string>
using namespace e2d;
static Conserved my_flux(const Conserved& a, const Conserved&) { return a; }
static double my_limiter(double, double) { return 0.0; }
int main() {
    Grid g = make_grid(8, 8, 0.0, 1.0, 0.0, 1.0, BC::Periodic, BC::Transmissive);
    int rejected = 0, reached_gpu = 0;
    try { Solver s(g, my_flux, van_leer, 0.5); } catch (const std::invalid_argument& e) { ++rejected; std::puts(e.what()); }
    try { Solver s(g, hllc_flux, my_limiter, 0.5); } catch (const std::invalid_argument& e) { ++rejected; std::puts(e.what()); }
    FluxFn fluxes[] = {hllc_flux, rusanov_flux};
    Limiter lims[] = {no_slope, unlimited, minmod, van_leer};
    for (FluxFn f : fluxes)
        for (Limiter l : lims) {
            try { Solver s(g, f, l, 0.5); ++reached_gpu; }
            catch (const std::runtime_error& e) { if (std::string(e.what()).find("CUDA") != std::string::npos) ++reached_gpu; }
        }
    std::printf("rejected %d reached %d\n", rejected, reached_gpu);
    return 0;
}
"""


def test_function_pointer_mapping(ref_headers, tmp_path):
    src = tmp_path / "probe.cpp"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["g++", "-std=gnu++17", "-O1", "-Wall", f"-I{ROOT / 'neural-pde-surrogate_b200' / 'host'}",
                    f"-I{ref_headers}", f"-I{ROOT / 'include'}", str(src), "-o", str(exe),
                    f"-L{bo.LIBFV_DIR}", "-lfv", f"-Wl,-rpath,{bo.LIBFV_DIR}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60, check=True).stdout
    assert "the flux must be hllc_flux or rusanov_flux" in out
    assert "the limiter must be no_slope, unlimited, minmod or van_leer" in out
    assert out.strip().endswith("rejected 2 reached 8")  # all 2 x 4 known pairs get as far as fv_create
