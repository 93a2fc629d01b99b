"""Leaves of more than 128 bodies (ncrit up to 256, the near-field CTA's
limit): the dense core of a Plummer sphere fills them.  The near-field
kernel has 128 threads and takes two targets each, so these leaves exercise
its second half of targets.  FP64 results must match the oracle within 1e-12;
the mixed form must stay within its accuracy contract."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("ncrit", [129, 192, 256])
def test_leaves_above_128_bodies(port, ncrit):
    from minimal_b200 import FMM, plummer_bodies

    xq = plummer_bodies(40000, 5)
    f = FMM(P=6, ncrit=ncrit, theta=0.4)
    f.set_bodies(xq)
    f.evaluate()
    t = f.tree()
    assert t["nbody"][t["nchild"] == 0].max() > 128  # the case under test occurs
    out = f.bodies()
    ref = port.fmm(xq, 6, ncrit, 0.4)
    assert np.array_equal(out[:, :4], ref[:, :4])
    assert rel(out[:, 4], ref[:, 4]) < 1e-12 and rel(out[:, 5:], ref[:, 5:]) < 1e-12

    m = FMM(P=6, ncrit=ncrit, theta=0.4, precision="mixed")
    m.set_bodies(xq)
    m.evaluate()
    mo = m.bodies()
    assert rel(mo[:, 5:], ref[:, 5:]) < 1e-5
    assert rel(mo[:, 4], ref[:, 4]) < 1e-5
