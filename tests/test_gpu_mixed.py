"""Mixed-precision form on the GPU: FP32 P2P with compensated accumulation and
tensor-core (tcgen05, split-FP16, FP32 accumulation) M2L.

The form is held to its accuracy contract: its error against FP64 direct
summation must stay within 1.1x of the FP64 form's error at the same P (force)
-- and within 1.5x for the potential, which is dominated by the far field --
while the tree and the lists stay bit-exact (they are shared with FP64).
"""
import numpy as np
import pytest

from tests.conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def errors(fmm, n, nt=1000):
    out = fmm.bodies()
    sample = np.arange(0, n, max(1, n // nt))[:nt]
    tgt = out[sample].copy()
    res = tgt.copy()
    tgt[:, 4:] = 0
    d = fmm.direct(tgt)
    return rel(res[:, 4], d[:, 4]), rel(res[:, 5:], d[:, 5:]), out


def make_bodies(n, dist):
    """uniform: the reference driver's bodies (charges U[-0.5,0.5), neutral);
    uniform_1e-6: the same with every charge times 1e-6; plummer: a Plummer
    sphere with its own equal charges 1/N (the non-uniform benchmark's
    bodies, positions and charges rounded to FP32 values); plummer_pm: the
    same positions with charges U[-0.5,0.5)."""
    from minimal_b200 import drand48_bodies, plummer_bodies

    if dist.startswith("uniform"):
        xq = drand48_bodies(n, 3)
        if dist == "uniform_1e-6":
            xq[:, 3] *= 1e-6
        return xq
    xq = plummer_bodies(n, 3).astype(np.float32).astype(np.float64)
    if dist == "plummer_pm":
        xq[:, 3] = np.random.default_rng(3).uniform(-0.5, 0.5, n)
    return xq


@pytest.mark.parametrize("n,P,theta,ncrit,dist", [
    (10000, 10, 0.4, 64, "uniform"),
    (200000, 10, 0.4, 64, "uniform"),
    (100000, 8, 0.5, 32, "plummer_pm"),
    (60000, 12, 0.4, 64, "uniform"),
    (30000, 6, 0.5, 16, "uniform"),
    (60000, 12, 0.4, 64, "uniform_1e-6"),
    (200000, 10, 0.4, 64, "plummer"),
    (200000, 12, 0.4, 64, "plummer"),
    (100000, 8, 0.4, 64, "plummer"),
    (100000, 6, 0.4, 64, "plummer"),
])
def test_mixed_error_close_to_fp64(n, P, theta, ncrit, dist):
    """Charge scale does not matter: the FP16 split of the tensor-core M2L
    normalises the multipoles by a power of two taken from their largest
    magnitude, so charges of 1/N (or 1e-6 times the usual) keep the same
    relative accuracy as charges of order one."""
    from minimal_b200 import FMM

    xq = make_bodies(n, dist)
    res = {}
    for prec in ("fp64", "mixed"):
        f = FMM(P=P, ncrit=ncrit, theta=theta, precision=prec)
        f.set_bodies(xq)
        f.evaluate()
        res[prec] = errors(f, n)
        if prec == "mixed":
            t = f.tree()
    (p64, f64, o64), (pmx, fmx, omx) = res["fp64"], res["mixed"]
    assert np.array_equal(o64[:, :4], omx[:, :4])  # same tree, same body order
    assert fmx <= 1.1 * f64 + 1e-7, (fmx, f64)
    assert pmx <= 1.5 * p64 + 1e-7, (pmx, p64)
    assert rel(omx[:, 5:], o64[:, 5:]) < 2e-5
    assert len(t["nchild"]) > 1


def test_mixed_full_size_error_target():
    """1M uniform bodies, P=10: the mixed form's force error against direct
    summation on 1000 sampled bodies stays within 1.1x of the FP64 form's
    (3.44e-5, the reference's own error at this configuration)."""
    from minimal_b200 import FMM, drand48_bodies

    g = golden("3d_n1048576_p10_sampled")
    n = int(g["n"])
    f = FMM(P=10, ncrit=64, theta=0.4, precision="mixed")
    f.set_bodies(drand48_bodies(n, 0))
    f.evaluate()
    out = f.bodies()[g["sample"]]
    d = g["direct"]
    ref_f = rel(g["fmm"][:, 5:], d[:, 5:])
    assert rel(out[:, 5:], d[:, 5:]) <= 1.1 * ref_f
    assert rel(out[:, 4], d[:, 4]) <= 1.5 * rel(g["fmm"][:, 4], d[:, 4])


@pytest.mark.parametrize("P", [14, 16, 18])
def test_mixed_high_orders_stay_correct(P):
    """Orders whose operators do not fit the tensor-core tile run the FP64
    contraction; the FP32 near field still applies.  P=14 and 16 take the
    unrolled FP32 P2M/L2P (butterfly sums) and the octant-batched FP32
    shifts, P=18 the runtime-order FP32 P2M/L2P and the per-octant FP64
    shifts."""
    from minimal_b200 import FMM, drand48_bodies

    xq = drand48_bodies(8000, 1)
    f = FMM(P=P, ncrit=64, theta=0.4, precision="mixed")
    f.set_bodies(xq)
    f.evaluate()
    pm, fm, _ = errors(f, 8000, 200)
    g = FMM(P=P, ncrit=64, theta=0.4)
    g.set_bodies(xq)
    g.evaluate()
    p6, f6, _ = errors(g, 8000, 200)
    assert fm <= 2 * f6 + 1e-6 and pm <= 2 * p6 + 1e-6


@pytest.mark.parametrize("P", [10, 16, 18])
@pytest.mark.parametrize("scale", [1e-6, 1e6])
def test_mixed_is_scale_free(P, scale):
    """A domain scaled by s gives potentials scaled by 1/s and forces by
    1/s^2: the FP32 P2M and L2P work in units of each leaf's radius (a power
    of two), so their terms r^n and L_n stay in FP32 range whatever the
    domain's size.  P=10 covers the tensor-core path's FP32 kernels, P=16 the
    unrolled ones and P=18 the runtime-order ones."""
    from minimal_b200 import FMM, drand48_bodies

    n = 20000
    xq = drand48_bodies(n, 8)
    outs = {}
    for prec, s in (("fp64", 1.0), ("mixed", 1.0), ("mixed", scale)):
        x = xq.copy()
        x[:, :3] *= s
        f = FMM(P=P, ncrit=64, theta=0.4, precision=prec)
        f.set_bodies(x)
        f.evaluate()
        outs[prec, s] = f.bodies()
        f.close()
    ref, base, o = outs["fp64", 1.0], outs["mixed", 1.0], outs["mixed", scale]
    assert np.array_equal(o[:, :3], base[:, :3] * scale)  # the same tree
    assert np.isfinite(o[:, 4:]).all()
    # against the unscaled FP64 result, the scaled domain keeps the mixed
    # form's own error (two FP32 roundings of the same sums differ by about
    # sqrt(2) times that error, so they are not compared with each other)
    for k, back in ((4, scale), (slice(5, 8), scale * scale)):
        err0 = rel(base[:, k], ref[:, k])
        assert rel(o[:, k] * back, ref[:, k]) <= 2 * err0 + 1e-7
