"""The tensor-core M2L's bounded waits: a stall turns into EXAFMM_ERR_TIMEOUT,
not a hung GPU, and the handle stays usable.

exafmm_b200_test_stall_tc makes the next tensor-core M2L launch wait on a
barrier that nothing arrives at (a short limit, here 2 ms) before its first
group, as if its inputs never came.  The wait runs out; the kernel's other
roles see the abort flag and stop waiting; copies and MMAs already in flight
are drained under their own, long limit; tensor memory is freed.  The host
turns the device flag into EXAFMM_ERR_TIMEOUT (results discarded), and the
next evaluation on the same handle must run normally and give the same
results as a handle that never stalled.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_TIMEOUT = -7


def test_tensor_core_stall_times_out_and_handle_recovers():
    from minimal_b200 import FMM, FMMError, drand48_bodies

    xq = drand48_bodies(20000, 5)
    ref = FMM(P=10, ncrit=64, theta=0.4, precision="mixed")
    ref.set_bodies(xq)
    ref.evaluate()
    want = ref.bodies()

    f = FMM(P=10, ncrit=64, theta=0.4, precision="mixed")
    f.set_bodies(xq)
    f._check(f.lib.exafmm_b200_test_stall_tc(f.h, 2_000_000))
    with pytest.raises(FMMError) as e:
        f.evaluate()
    assert e.value.code == ERR_TIMEOUT
    assert "bounded wait ran out" in str(e.value)
    with pytest.raises(FMMError):  # results were discarded
        f.bodies()
    f.evaluate()  # the hook stalls one launch only
    got = f.bodies()
    assert np.array_equal(got, want)


def test_stall_hook_argument_checks():
    from minimal_b200 import FMM

    f = FMM(P=6, precision="mixed")
    assert f.lib.exafmm_b200_test_stall_tc(f.h, -1) == -1
    assert f.lib.exafmm_b200_test_stall_tc(f.h, 0) == 0
