"""The reference's own drivers through the C++ driver shim on the GPU: 3d/fmm.cxx
(100,000 bodies, P=10, ncrit=128, FP64) prints the errors of the reference's
own build, and test/test_fmm.h gives the reference's known answers at P=10
and P=20 (test/test_fmm.cxx:5-6); 3d/kernel.cxx and test/test_kernel.h, which
call the single operators one by one, give the operator chain's known answers
(test/test_kernel.cxx:5-7); 3dp/fmm.cxx (periodic, images = 4, dipole
correction, Ewald parts one by one) prints the errors of the reference's own
build.  The drivers are built by tests/shim/Makefile (oracle/_ref/shim)."""
import subprocess
import os

import pytest

from tests.test_shim import binary, errors, run

pytestmark = pytest.mark.gpu


def test_fmm_cxx_on_the_gpu_through_the_shim():
    ref, gpu = run(binary("fmm_ref")), run(binary("fmm_gpu"))
    assert ref.returncode == 0 and gpu.returncode == 0, gpu.stderr[-2000:]
    (p, f), (rp, rf) = errors(gpu.stdout), errors(ref.stdout)
    assert p == pytest.approx(rp, rel=1e-5) and f == pytest.approx(rf, rel=1e-5)


def test_test_fmm_on_the_gpu_through_the_shim():
    import re

    import numpy as np

    from tests.conftest import ROOT

    kat = {k: float(v) for k, v in np.load(os.path.join(ROOT, "tests", "golden", "kat.npz")).items()}
    r = run(binary("test_fmm_gpu"))
    assert r.returncode == 0, r.stderr[-2000:]
    e10, e20 = map(float, re.search(r"test_fmm (\S+) (\S+)", r.stdout).groups())
    assert e10 == pytest.approx(kat["fmm_p10"], rel=1e-6) and e20 == pytest.approx(kat["fmm_p20"], rel=1e-6)


@pytest.mark.parametrize("P", [10, 20, 30])
def test_kernel_cxx_on_the_gpu_through_the_shim(P):
    ref = subprocess.run([binary("kernel_ref"), str(P)], capture_output=True, text=True, timeout=60)
    gpu = subprocess.run([binary("kernel_gpu"), str(P)], capture_output=True, text=True, timeout=120)
    assert ref.returncode == 0 and gpu.returncode == 0, gpu.stderr[-2000:]
    (p, f), (rp, rf) = errors(gpu.stdout), errors(ref.stdout)
    assert p == pytest.approx(rp, rel=1e-5) and f == pytest.approx(rf, rel=1e-5)


def test_test_kernel_on_the_gpu_through_the_shim(kat):
    import re

    r = run(binary("test_kernel_gpu"))
    assert r.returncode == 0, r.stderr[-2000:]
    e = list(map(float, re.search(r"test_kernel (\S+) (\S+) (\S+)", r.stdout).groups()))
    assert e == pytest.approx([kat["kernel_p10"], kat["kernel_p20"], kat["kernel_p30"]], rel=1e-7)


def test_periodic_fmm_cxx_on_the_gpu_through_the_shim():
    """The GPU's Ewald real part takes every source at its nearest image
    inside the cutoff; the reference's neighbour search picks one image per
    pair of cells, about 1e-6 of the Ewald sum apart, which moves the printed
    errors (~1e-4) by up to a few percent."""
    ref, gpu = run(binary("fmm3dp_ref")), run(binary("fmm3dp_gpu"))
    assert ref.returncode == 0 and gpu.returncode == 0, gpu.stderr[-2000:]
    (p, f), (rp, rf) = errors(gpu.stdout), errors(ref.stdout)
    print("3dp errors gpu", p, f, "reference", rp, rf)
    assert p == pytest.approx(rp, rel=5e-2) and f == pytest.approx(rf, rel=5e-2)
