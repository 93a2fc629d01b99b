"""Batches of independent systems on the GPU: one forest, each phase run once
over all systems.  Every system must come out exactly as when it is
evaluated alone: same tree order of its bodies, FP64 results within 1e-12,
mixed-precision results as close to FP64 as a single mixed evaluation."""
import numpy as np
import pytest

from tests.test_gpu_parity import rel_l2

pytestmark = pytest.mark.gpu

SIZES = [1000, 5000, 300, 20000, 64, 1, 65, 7000, 12000, 2500, 100, 40000]


def systems(sizes, seed0=100):
    from minimal_b200 import drand48_bodies

    return [drand48_bodies(n, seed0 + q) for q, n in enumerate(sizes)]


def single(xq, prec, P=6, theta=0.5, ncrit=64):
    from minimal_b200 import FMM

    f = FMM(P=P, ncrit=ncrit, theta=theta, precision=prec)
    f.set_bodies(xq)
    f.evaluate()
    return f.bodies()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_matches_single_systems(prec):
    from minimal_b200 import FMM

    sys_ = systems(SIZES)
    f = FMM(P=6, ncrit=64, theta=0.5, precision=prec)
    f.set_batch(sys_)
    f.evaluate()
    out = f.bodies()
    perm = f.perm()
    off = f.offsets
    for q, xq in enumerate(sys_):
        b = out[off[q]:off[q + 1]]
        ref = single(xq, prec)
        assert np.array_equal(b[:, :4], ref[:, :4]), q  # same tree order
        assert np.all((perm[off[q]:off[q + 1]] >= off[q]) & (perm[off[q]:off[q + 1]] < off[q + 1]))
        if len(xq) == 1:
            continue
        tol = 1e-12 if prec == "fp64" else 2e-6
        assert rel_l2(b[:, 4], ref[:, 4]) < tol, q
        assert rel_l2(b[:, 5:], ref[:, 5:]) < tol, q


def test_batch_mixed_error_vs_fp64():
    from minimal_b200 import FMM

    sys_ = systems(SIZES[:6], 300)
    res = {}
    for prec in ("fp64", "mixed"):
        f = FMM(P=6, ncrit=64, theta=0.5, precision=prec)
        f.set_batch(sys_)
        f.evaluate()
        res[prec] = f.bodies()
    off = f.offsets
    for q in range(len(sys_)):
        a, b = res["mixed"][off[q]:off[q + 1]], res["fp64"][off[q]:off[q + 1]]
        if off[q + 1] - off[q] > 1:
            assert rel_l2(a[:, 5:], b[:, 5:]) < 1e-4


def test_batch_log_uniform_sizes():
    """256 systems with sizes log-uniform in [1000, 65536] (the batched
    configuration's distribution, a smaller count): spot-check systems
    against single evaluations."""
    from minimal_b200 import FMM

    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(np.log(1000), np.log(65536), 256)).astype(int)
    sys_ = systems(sizes, 1000)
    f = FMM(P=6, ncrit=64, theta=0.5, precision="fp64")
    f.set_batch(sys_)
    f.evaluate()
    out = f.bodies()
    off = f.offsets
    for q in (0, 17, 100, 255):
        ref = single(sys_[q], "fp64")
        b = out[off[q]:off[q + 1]]
        assert np.array_equal(b[:, :4], ref[:, :4])
        assert rel_l2(b[:, 5:], ref[:, 5:]) < 1e-12


def test_batch_errors():
    from minimal_b200 import FMM, FMMError

    f = FMM(P=6, ncrit=64, theta=0.5)
    sys_ = systems([100, 200])
    f.set_batch(sys_)
    f.evaluate()
    with pytest.raises(FMMError) as e:
        f.tree()
    assert e.value.code == -4
    with pytest.raises(FMMError) as e:
        f.direct(np.zeros((3, 8)))
    assert e.value.code == -4
    with pytest.raises(FMMError) as e:
        f.set_params(images=2, cycle=6.0)
    assert e.value.code == -4
    bad = np.array([0, 50, 50, 300], dtype=np.int64)
    rec = np.zeros((300, 8))
    rec[:, :3] = np.random.default_rng(1).uniform(-1, 1, (300, 3))
    with pytest.raises(FMMError) as e:
        f._check(f.lib.exafmm_b200_set_batch(f.h, rec.ctypes.data, bad.ctypes.data, 3, 0))
    assert e.value.code == -1
    f.set_bodies(sys_[0])  # back to a single system
    f.evaluate()
    assert len(f.tree()["nchild"]) >= 1


def test_autotune_picks_a_candidate_and_keeps_it():
    """The autotuner times the loaded batch for each candidate ncrit, keeps the
    fastest, and leaves exactly the results of that setting."""
    from minimal_b200 import FMM, FMMError

    sys_ = systems([3000, 20000, 500, 9000], 500)
    f = FMM(P=6, ncrit=64, theta=0.5, precision="mixed")
    f.set_batch(sys_)
    best, ms = f.autotune([32, 64, 128], repeats=2)
    assert best in (32, 64, 128) and ms > 0
    tuned = f.bodies()
    g = FMM(P=6, ncrit=best, theta=0.5, precision="mixed")
    g.set_batch(sys_)
    g.evaluate()
    ref = g.bodies()
    assert np.array_equal(tuned[:, :4], ref[:, :4])
    assert rel_l2(tuned[:, 5:], ref[:, 5:]) < 1e-6
    with pytest.raises(FMMError) as e:
        f.autotune([0, 64])
    assert e.value.code == -1
