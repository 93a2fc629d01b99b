"""A whole evaluation runs on three streams (upward pass beside the list
build, near field beside the M2L and L2L); the step calls run the same
kernels one after another on one stream.  Every kernel reads only what the
ones it waits for wrote, so the results must be bit-identical -- a missing
dependency between the streams would show up here as a difference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def stepwise(f):
    f.build_tree()
    f.build_lists()
    f.upward()
    f.horizontal()
    f.downward()
    return f.bodies()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("n,P", [(1 << 20, 10), (50000, 6)])
def test_evaluate_equals_step_calls(prec, n, P):
    from minimal_b200 import FMM, drand48_bodies

    f = FMM(P=P, ncrit=64, theta=0.4, precision=prec)
    f.set_bodies(drand48_bodies(n, 5))
    f.evaluate()
    a = f.bodies()
    f.evaluate()
    b = f.bodies()
    s = stepwise(f)
    f.close()
    assert np.array_equal(a, b)
    assert np.array_equal(a, s)


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_periodic_evaluate_equals_step_calls(prec):
    from minimal_b200 import FMM, drand48_bodies

    cyc = 2 * np.pi
    xq = drand48_bodies(100000, 2, "3dp", cyc)
    f = FMM(P=8, ncrit=64, theta=0.4, precision=prec, images=3, cycle=cyc)
    f.set_bodies(xq)
    f.evaluate()
    a = f.bodies()
    s = stepwise(f)
    f.close()
    assert np.array_equal(a, s)


def test_batch_evaluate_equals_step_calls():
    from minimal_b200 import FMM, drand48_bodies

    systems = [drand48_bodies(m, 10 + q) for q, m in enumerate((3000, 40000, 700, 25000))]
    f = FMM(P=6, ncrit=64, theta=0.5, precision="mixed")
    f.set_batch(systems)
    f.evaluate()
    a = f.bodies()
    s = stepwise(f)
    f.close()
    assert np.array_equal(a, s)
