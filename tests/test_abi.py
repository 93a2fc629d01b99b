"""The C-ABI library loads and exports exactly what include/exafmm_b200.h
declares (CPU only: no compute call is made)."""
import ctypes
import os
import re

import pytest

from tests.conftest import ROOT


def declared():
    src = open(os.path.join(ROOT, "include", "exafmm_b200.h")).read()
    return sorted(set(re.findall(r"EXAFMM_API\s+[\w\s\*]+?\b(exafmm_b200_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared()
    assert len(names) >= 20
    import minimal_b200

    assert sorted(minimal_b200.API) == names


def test_library_exports_every_declared_symbol():
    import minimal_b200

    lib = minimal_b200.load_library()
    for name in declared():
        assert hasattr(lib, name), name


def test_library_exports_nothing_else():
    import subprocess

    import minimal_b200

    out = subprocess.run(["nm", "-D", "--defined-only", minimal_b200.LIB_PATH], capture_output=True, text=True).stdout
    exported = sorted(l.split()[-1] for l in out.splitlines() if " T " in l)
    assert exported == declared()


def test_arch_and_argument_checks_without_gpu():
    import minimal_b200

    lib = minimal_b200.load_library()
    assert lib.exafmm_b200_arch() == 100
    h = ctypes.c_void_p()
    bad = minimal_b200.Params(0, 64, 0.4, 0, 0.0, 0, 0)  # P = 0
    assert lib.exafmm_b200_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = minimal_b200.Params(10, 0, 0.4, 0, 0.0, 0, 0)  # ncrit = 0
    assert lib.exafmm_b200_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = minimal_b200.Params(10, 64, 0.4, 2, 0.0, 0, 0)  # images without a period
    assert lib.exafmm_b200_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    assert lib.exafmm_b200_destroy(None) == -1
    # every handle call refuses a null handle without touching the GPU
    one = ctypes.c_double(0.0)
    assert lib.exafmm_b200_set_charges(None, ctypes.byref(one), 0) == -1
    assert lib.exafmm_b200_reevaluate(None) == -1
    assert lib.exafmm_b200_evaluate(None) == -1


def test_no_gpu_is_reported_not_faked():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    import minimal_b200

    with pytest.raises(minimal_b200.FMMError) as e:
        minimal_b200.FMM()
    assert e.value.code == -8
