"""Repeated evaluations on fixed positions: set_charges keeps the tree and
the interaction lists (they depend on the positions only) and reevaluate runs
the passes over them, as the reference's lazy traversal evaluates over its
stored lists (3d/traverse_lazy.h:46-62).  The results must be bit-identical
to a fresh evaluation of the same bodies with the new charges."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def new_charges(n, seed):
    q = np.random.default_rng(seed).uniform(-0.5, 0.5, n)
    return q - q.mean()


def fresh(xq, q, **kw):
    from minimal_b200 import FMM

    b = xq.copy()
    b[:, 3] = q
    f = FMM(**kw)
    f.set_bodies(b)
    f.evaluate()
    out = f.bodies()
    f.close()
    return out


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_set_charges_then_reevaluate_equals_fresh_evaluation(prec):
    from minimal_b200 import FMM, drand48_bodies

    n = 200000
    kw = dict(P=10, ncrit=64, theta=0.4, precision=prec)
    xq = drand48_bodies(n, 4)
    f = FMM(**kw)
    f.set_bodies(xq)
    f.evaluate()
    first = f.bodies()
    for k in range(2):  # twice: the kept lists survive a reevaluation
        q = new_charges(n, 10 + k)
        f.set_charges(q)
        f.reevaluate()
        got = f.bodies()
        assert np.array_equal(got, fresh(xq, q, **kw))
        assert not np.array_equal(got[:, 4:], first[:, 4:])
    f.close()


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_periodic_set_charges_then_reevaluate(prec):
    from minimal_b200 import FMM, drand48_bodies

    n, cyc = 60000, 2 * np.pi
    kw = dict(P=8, ncrit=64, theta=0.4, precision=prec, images=3, cycle=cyc)
    xq = drand48_bodies(n, 6, "3dp", cyc)
    f = FMM(**kw)
    f.set_bodies(xq)
    f.evaluate()
    q = new_charges(n, 21)
    f.set_charges(q)
    f.reevaluate()
    got = f.bodies()
    f.close()
    assert np.array_equal(got, fresh(xq, q, **kw))


def test_batch_set_charges_then_reevaluate():
    from minimal_b200 import FMM, drand48_bodies

    systems = [drand48_bodies(m, 30 + k) for k, m in enumerate((5000, 30000, 900, 12000))]
    f = FMM(P=6, ncrit=64, theta=0.5, precision="mixed")
    f.set_batch(systems)
    f.evaluate()
    q = new_charges(sum(len(x) for x in systems), 22)
    f.set_charges(q)
    f.reevaluate()
    got = f.bodies()
    f.close()
    new = []
    off = 0
    for x in systems:
        y = x.copy()
        y[:, 3] = q[off:off + len(x)]
        off += len(x)
        new.append(y)
    g = FMM(P=6, ncrit=64, theta=0.5, precision="mixed")
    g.set_batch(new)
    g.evaluate()
    want = g.bodies()
    g.close()
    assert np.array_equal(got, want)


def test_reevaluate_and_set_charges_errors():
    import minimal_b200
    from minimal_b200 import FMM, FMMError, drand48_bodies

    n = 20000
    xq = drand48_bodies(n, 7)
    f = FMM(P=6, precision="mixed")
    one = np.zeros(1)
    assert f.lib.exafmm_b200_set_charges(f.h, minimal_b200._p(one), minimal_b200.HOST) == -4  # no bodies
    f.set_bodies(xq)
    with pytest.raises(FMMError) as e:  # no tree and lists yet
        f.reevaluate()
    assert e.value.code == -4
    f.evaluate()
    first = f.bodies()
    q = new_charges(n, 8)
    q[123] = np.nan
    with pytest.raises(FMMError) as e:  # rejected: nothing changes
        f.set_charges(q)
    assert e.value.code == -1
    f.reevaluate()
    assert np.array_equal(f.bodies(), first)
    with pytest.raises(ValueError):
        f.set_charges(q[:-1])
    # the step calls also run over the kept tree and lists after set_charges
    q[123] = 0.0
    f.set_charges(q)
    f.upward()
    f.horizontal()
    f.downward()
    stepped = f.bodies()
    f.reevaluate()
    assert np.array_equal(f.bodies(), stepped)
    f.close()


def test_new_parameters_regroup():
    """The kept grouping belongs to the lists, P and form it was made for:
    after set_params the next evaluation regroups (and reevaluate needs new
    lists first)."""
    from minimal_b200 import FMM, FMMError, drand48_bodies

    xq = drand48_bodies(50000, 9)
    f = FMM(P=10, ncrit=64, theta=0.4, precision="mixed")
    f.set_bodies(xq)
    f.evaluate()
    f.set_params(P=8, theta=0.5)
    with pytest.raises(FMMError):
        f.reevaluate()
    f.evaluate()
    got = f.bodies()
    f.reevaluate()
    again = f.bodies()
    f.close()
    assert np.array_equal(got, again)
    assert np.array_equal(got, fresh(xq, xq[:, 3], P=8, ncrit=64, theta=0.5, precision="mixed"))
