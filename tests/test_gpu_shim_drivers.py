"""The reference's own drivers through the C++ driver shim on the GPU: 3d/fmm.cxx
(100,000 bodies, P=10, ncrit=128, FP64) prints the errors of the reference's
own build, and test/test_fmm.h gives the reference's known answers at P=10
and P=20 (test/test_fmm.cxx:5-6).  The drivers are built by
tests/shim/Makefile (oracle/_ref/shim)."""
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
