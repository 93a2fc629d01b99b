"""The C++ driver shim (include/exafmm_b200.hpp): the reference's own drivers,
3d/fmm.cxx and test/test_fmm.h, compiled unchanged against it
(tests/shim/Makefile, into oracle/_ref/shim).  Linked against an
oracle-backed stand-in of the C entry points they run on the CPU and must
print the reference's own results, which checks the shim's host logic (body
permutation, cell wiring, accumulation of p and F, direct sums on a second
handle); linked against the library they reach the GPU path."""
import os
import re
import subprocess

import pytest

from tests.conftest import ROOT

OUT = os.path.join(ROOT, "oracle", "_ref", "shim")


def binary(name):
    path = os.path.join(OUT, name)
    if not os.path.exists(path):
        pytest.skip("shim checks not built (the reference sources were not found at build time)")
    return path


def errors(text):
    """(p, F) from the 'Rel. L2 Error' lines 3d/fmm.cxx prints."""
    p = re.search(r"Rel\. L2 Error \(p\)\s*:\s*([0-9.eE+-]+)", text)
    f = re.search(r"Rel\. L2 Error \(F\)\s*:\s*([0-9.eE+-]+)", text)
    assert p and f, text[-2000:]
    return float(p.group(1)), float(f.group(1))


def run(path):
    return subprocess.run([path], capture_output=True, text=True, timeout=600, cwd=OUT)


def test_fmm_cxx_through_the_shim_prints_the_reference_results():
    ref, shim = run(binary("fmm_ref")), run(binary("fmm_cpu"))
    assert ref.returncode == 0 and shim.returncode == 0, shim.stderr[-2000:]
    assert errors(shim.stdout) == errors(ref.stdout)


def test_test_fmm_through_the_shim_gives_the_known_answers():
    import numpy as np

    kat = {k: float(v) for k, v in np.load(os.path.join(ROOT, "tests", "golden", "kat.npz")).items()}
    r = run(binary("test_fmm_cpu"))
    assert r.returncode == 0, r.stderr[-2000:]
    e10, e20 = map(float, re.search(r"test_fmm (\S+) (\S+)", r.stdout).groups())
    assert e10 == pytest.approx(kat["fmm_p10"], rel=1e-8) and e20 == pytest.approx(kat["fmm_p20"], rel=1e-8)


def kernel_errors(text):
    """(p, F) of the operator chain from 3d/kernel.cxx's two printed lines."""
    return errors(text)


@pytest.mark.parametrize("P", [10, 20, 30])
def test_kernel_cxx_through_the_shim_prints_the_reference_results(P):
    """The single operators (P2M, M2M, M2L, L2L, L2P, P2P one call each)
    through the shim give the reference's known answers."""
    ref = subprocess.run([binary("kernel_ref"), str(P)], capture_output=True, text=True, timeout=60)
    shim = subprocess.run([binary("kernel_cpu"), str(P)], capture_output=True, text=True, timeout=60)
    assert ref.returncode == 0 and shim.returncode == 0, shim.stderr[-2000:]
    assert kernel_errors(shim.stdout) == kernel_errors(ref.stdout)


def test_test_kernel_through_the_shim_gives_the_known_answers(kat):
    r = run(binary("test_kernel_cpu"))
    assert r.returncode == 0, r.stderr[-2000:]
    e = list(map(float, re.search(r"test_kernel (\S+) (\S+) (\S+)", r.stdout).groups()))
    assert e == pytest.approx([kat["kernel_p10"], kat["kernel_p20"], kat["kernel_p30"]], rel=1e-8)


def test_periodic_fmm_cxx_through_the_shim_prints_the_reference_results():
    """3dp/fmm.cxx (1000 bodies, images = 4, dipole correction, then the Ewald
    parts wavePart, realPart, selfTerm one by one) through the shim."""
    ref, shim = run(binary("fmm3dp_ref")), run(binary("fmm3dp_cpu"))
    assert ref.returncode == 0 and shim.returncode == 0, shim.stderr[-2000:]
    (p, f), (rp, rf) = errors(shim.stdout), errors(ref.stdout)
    assert p == pytest.approx(rp, rel=1e-4) and f == pytest.approx(rf, rel=1e-4)


def test_drivers_linked_against_the_library_reach_it():
    r = run(binary("fmm_gpu"))
    if r.returncode != 0:  # no GPU here: the library's own error, thrown by the shim
        assert "exafmm_b200: no CUDA device" in r.stderr, r.stderr[-2000:]
    else:
        errors(r.stdout)


def test_shim_header_compiles_without_warnings(tmp_path):
    src = tmp_path / "use.cpp"
    src.write_text('#include "exafmm_b200.hpp"\n'
                   "int main() { exafmm::P = 10; exafmm::initKernel(); return exafmm::NTERM == 55 ? 0 : 1; }\n")
    exe = tmp_path / "use"
    c = subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I" + os.path.join(ROOT, "include"),
                        str(src), "-o", str(exe)], capture_output=True, text=True)
    assert c.returncode == 0, c.stderr
    assert subprocess.run([str(exe)]).returncode == 0
