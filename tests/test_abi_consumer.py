"""A compiled C++ consumer of the C ABI: tests/abi_consumer/oclsolve_loop.cpp links
against libgpgmp_b200.so and drives the reference's oclSolve event loop
(DiffusionModel.cpp:1479-1603) through gpgmp_do_reactions / gpgmp_next_diffusion_time /
gpgmp_diffuse, as an adapter in place of the reference's solvers would
(Solver.h:52-100); on a GPU its snapshots must equal gpgmp_solve's bit for bit."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "abi_consumer", "oclsolve_loop.cpp")
LIBDIR = os.path.join(ROOT, "inchman_b200")


def _build(tmp_path):
    from inchman_b200 import build
    build.build()
    exe = str(tmp_path / "oclsolve_loop")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o",
                    exe, "-L", LIBDIR, "-lgpgmp_b200", f"-Wl,-rpath,{LIBDIR}"], check=True)
    return exe


def test_consumer_compiles_and_links_against_the_library(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run(["ldd", exe], capture_output=True, text=True, check=True).stdout
    assert "libgpgmp_b200.so" in out and "not found" not in out


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["homogeneous", "inhomogeneous"])
def test_consumer_event_loop_equals_library_loop(tmp_path, kind):
    exe = _build(tmp_path)
    r = subprocess.run([exe, kind], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "identical to gpgmp_solve" in r.stdout
