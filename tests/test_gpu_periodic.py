"""Periodic systems on the GPU (3dp/): image lists, the far images of
periodic(), the dipole correction, the periodic direct sum and the Ewald
summation that checks them.

FP64 results must match the reference FMM within 1e-12 (fixtures made from
the reference compiled from its own sources); the GPU Ewald must match the
reference's Ewald; the mixed form must stay as close to Ewald as FP64 does.
"""
import numpy as np
import pytest

from tests.conftest import golden
from tests.test_gpu_parity import check_results, make, rel_l2, tree_equal

pytestmark = pytest.mark.gpu

CASES_3DP = ["3dp_n1000_p10_img2", "3dp_n1500_p8_img3"]


@pytest.mark.parametrize("name", CASES_3DP)
def test_periodic_tree_and_lists_bit_exact(name):
    g = golden(name)
    fmm = make(g)
    fmm.set_bodies(g["xq"])
    fmm.build_tree()
    tree_equal(fmm.tree(), g)
    fmm.build_lists()
    lists = fmm.lists()
    for k in ("m2l_off", "m2l_src", "m2l_img", "p2p_off", "p2p_src", "p2p_img"):
        assert np.array_equal(lists[k], g[k]), k


@pytest.mark.parametrize("name", CASES_3DP)
def test_periodic_fmm_fp64_vs_reference(name):
    g = golden(name)
    fmm = make(g)
    fmm.set_bodies(g["xq"])
    fmm.evaluate()
    check_results(fmm.bodies(), g["bodies"])
    M, L = fmm.expansions()
    # the root's L carries the far images of periodic() (3dp/traverse_eager.h:46-93)
    for a, b in ((M, g["M"]), (L, g["L"])):
        assert np.abs(a - b).max() < 1e-12 * np.abs(b).max()
    fmm.dipole_correction()
    check_results(fmm.bodies(), g["bodies_dipole"])


def ewald_min_image(b, cyc, ksize=11, sigma=0.25 / np.pi):
    """Numpy restatement of the GPU Ewald: the wave part and self term of
    3dp/ewald.h (initWaves, dft, idft, selfTerm) and the real part of realP2P
    taken over every source at its nearest image per axis."""
    from scipy.special import erfc

    alpha, cutoff = ksize / cyc, cyc / 2
    d = b[:, None, :3] - b[None, :, :3]
    d = np.where(d < -cyc / 2, d + cyc, d)
    d = np.where(d > cyc / 2, d - cyc, d)
    R2 = (d ** 2).sum(-1)
    ok = (R2 > 0) & (R2 < cutoff ** 2)
    Rs = np.sqrt(np.where(ok, R2, 1.0)) * alpha
    q = b[None, :, 3]
    p = np.where(ok, q * erfc(Rs) / Rs * alpha, 0).sum(1)
    dt = np.where(ok, q * (2 / np.sqrt(np.pi) * np.exp(-Rs ** 2) / Rs ** 2 + erfc(Rs) / Rs ** 3) * alpha ** 3, 0)
    F = -(d * dt[..., None]).sum(1)
    K = np.array([(l, m, n) for l in range(ksize + 1) for m in range(0 if l == 0 else -ksize, ksize + 1)
                  for n in range(1 if l == 0 and m == 0 else -ksize, ksize + 1) if l * l + m * m + n * n <= ksize ** 2],
                 float)
    sc = 2 * np.pi / cyc
    th = (K[:, None, :] * b[None, :, :3] * sc).sum(-1)
    K2 = ((K * sc) ** 2).sum(1)
    fac = 2 / sigma / cyc ** 3 * np.exp(-K2 / (4 * alpha ** 2)) / K2
    re = (b[None, :, 3] * np.cos(th)).sum(1) * fac
    im = (b[None, :, 3] * np.sin(th)).sum(1) * fac
    p += (re[:, None] * np.cos(th) + im[:, None] * np.sin(th)).sum(0)
    dtmp = re[:, None] * np.sin(th) - im[:, None] * np.cos(th)
    F -= (dtmp[..., None] * K[:, None, :]).sum(0) * sc
    p -= 2 / np.sqrt(np.pi) * b[:, 3] * alpha
    return p, F


@pytest.mark.parametrize("name", CASES_3DP)
def test_ewald_vs_reference(name):
    """GPU Ewald (wave + real + self) on every body, with the parameters of
    3dp/fmm.cxx:20-23.  The real part takes every source at its nearest image
    per axis; the reference (3dp/ewald.h:104-119) picks one image per pair of
    cells from the cells' centres and so drops a few pairs inside the cutoff
    whose nearest image differs from their cells' -- a ~1e-6 relative
    difference.  Tight against the restatement, loose against the reference."""
    g = golden(name)
    fmm = make(g)
    fmm.set_bodies(g["xq"])
    fmm.build_tree()
    tgt = np.zeros((len(g["xq"]), 8))
    tgt[:, :4] = g["bodies"][:, :4]  # tree order, as the reference's Ewald output
    e = fmm.ewald(tgt, ksize=11)
    p, F = ewald_min_image(tgt[:, :4], float(g["cycle"]))
    assert rel_l2(e[:, 4], p) < 1e-12
    assert rel_l2(e[:, 5:], F) < 1e-12
    ref = g["ewald"]
    assert np.array_equal(e[:, :4], ref[:, :4])
    assert rel_l2(e[:, 4], ref[:, 4]) < 1e-5
    assert rel_l2(e[:, 5:], ref[:, 5:]) < 1e-5


def energy_and_force_errors(out, ew):
    """The reference's own check (3dp/fmm.cxx:97-108): relative error of the
    energy sum(p q) and relative L2 error of the forces."""
    p = (out[:, 4] * out[:, 3]).sum()
    p2 = (ew[:, 4] * ew[:, 3]).sum()
    ep = abs(p - p2) / abs(p2)
    ef = np.sqrt(((out[:, 5:] - ew[:, 5:]) ** 2).sum() / (ew[:, 5:] ** 2).sum())
    return ep, ef


@pytest.mark.parametrize("name", CASES_3DP)
def test_mixed_periodic_close_to_fp64(name):
    g = golden(name)
    errs = {}
    for prec in ("fp64", "mixed"):
        fmm = make(g, prec)
        fmm.set_bodies(g["xq"])
        fmm.evaluate()
        fmm.dipole_correction()
        errs[prec] = energy_and_force_errors(fmm.bodies(), g["ewald"])
    (p64, f64), (pmx, fmx) = errs["fp64"], errs["mixed"]
    assert fmx <= 1.1 * f64 + 1e-7, (fmx, f64)
    assert pmx <= 1.5 * p64 + 1e-7, (pmx, p64)


def test_periodic_direct_vs_oracle(port):
    """Direct sum over (2r+1)^3 images, r = 1 + 3 (images = 2), against the
    oracle's restatement of the periodic direct() (3dp/traverse_eager.h:131-154)."""
    from minimal_b200 import FMM, drand48_bodies

    cyc = 2 * np.pi
    xq = drand48_bodies(400, 7, "3dp", cyc)
    fmm = FMM(P=6, ncrit=32, theta=0.4, images=2, cycle=cyc)
    fmm.set_bodies(xq)
    fmm.build_tree()
    tgt = np.zeros((40, 8))
    tgt[:, :4] = xq[::10]
    d = fmm.direct(tgt)
    src = np.zeros((len(xq), 8))
    src[:, :4] = xq
    r = port.direct(tgt, src, 2, cyc)
    # 729 images x 400 sources with cancellation: summation order shows at ~1e-12
    assert rel_l2(d[:, 4], r[:, 4]) < 1e-10
    assert rel_l2(d[:, 5:], r[:, 5:]) < 1e-10


def test_periodic_larger_system_vs_ewald():
    """50,000 bodies in a cube of side 2 pi, images = 3: after the dipole
    correction the FMM (FP64 and mixed) agrees with the GPU Ewald sum on 500
    sampled bodies, as the reference's periodic test does for 1,000 bodies."""
    from minimal_b200 import FMM, drand48_bodies

    cyc = 2 * np.pi
    xq = drand48_bodies(50000, 11, "3dp", cyc)
    res = {}
    for prec in ("fp64", "mixed"):
        fmm = FMM(P=10, ncrit=64, theta=0.4, images=3, cycle=cyc, precision=prec)
        fmm.set_bodies(xq)
        fmm.evaluate()
        fmm.dipole_correction()
        res[prec] = fmm.bodies()
    sample = np.arange(0, 50000, 100)
    tgt = res["fp64"][sample].copy()
    tgt[:, 4:] = 0
    ew = fmm.ewald(tgt)
    f64 = rel_l2(res["fp64"][sample, 5:], ew[:, 5:])
    fmx = rel_l2(res["mixed"][sample, 5:], ew[:, 5:])
    assert f64 < 1e-3
    assert fmx <= 1.1 * f64 + 1e-7
    assert np.array_equal(res["fp64"][:, :4], res["mixed"][:, :4])


def test_mixed_periodic_lists_untouched_by_ghosts():
    """The mixed form points image entries with a tiny fractional offset at
    ghost sources; it does so on its own copy of the walk's pairs, so the
    lists exported after a mixed evaluation are the FP64 form's (the
    reference's)."""
    from minimal_b200 import FMM, drand48_bodies

    cyc = 2 * np.pi
    xq = drand48_bodies(20000, 3, "3dp", cyc)
    lists = {}
    for prec in ("fp64", "mixed"):
        fmm = FMM(P=8, ncrit=32, theta=0.4, images=3, cycle=cyc, precision=prec)
        fmm.set_bodies(xq)
        fmm.evaluate()
        lists[prec] = fmm.lists()
        fmm.evaluate()  # the grouping again, on the same lists
        again = fmm.lists()
        for k in again:
            assert np.array_equal(again[k], lists[prec][k]), k
    for k in lists["fp64"]:
        assert np.array_equal(lists["mixed"][k], lists["fp64"][k]), k


def test_far_image_sums_follow_the_parameters():
    """The far images' harmonic sums are kept between evaluations for the
    (P, images, cycle) they were made for: after a change of the period or
    the image count an evaluation gives the same bits as a fresh handle."""
    from minimal_b200 import FMM, drand48_bodies

    xq = drand48_bodies(5000, 4, "3dp", 2 * np.pi)
    f = FMM(P=8, ncrit=32, theta=0.4, images=3, cycle=2 * np.pi)
    f.set_bodies(xq)
    f.evaluate()
    for images, cyc in ((3, 2 * np.pi * 1.25), (4, 2 * np.pi * 1.25), (2, 2 * np.pi)):
        f.set_params(images=images, cycle=cyc)
        f.set_bodies(xq)
        f.evaluate()
        g = FMM(P=8, ncrit=32, theta=0.4, images=images, cycle=cyc)
        g.set_bodies(xq)
        g.evaluate()
        assert np.array_equal(f.bodies(), g.bodies())


def test_mixed_potentials_do_not_drift_with_image_layers():
    """The far images multiply the root's net charge by image shells that grow
    with every layer; the mixed form takes the root's monopole as the FP64
    total charge, so its potentials stay as close to the FP64 form's with 4
    image layers as with 1 (an FP32 root monopole drifted by 7e-4 at 4
    layers)."""
    from minimal_b200 import FMM, drand48_bodies

    cyc = 2 * np.pi
    xq = drand48_bodies(30000, 6, "3dp", cyc)
    diff = {}
    for images in (1, 4):
        out = {}
        for prec in ("fp64", "mixed"):
            f = FMM(P=8, ncrit=64, theta=0.4, images=images, cycle=cyc, precision=prec)
            f.set_bodies(xq)
            f.evaluate()
            f.dipole_correction()
            out[prec] = f.bodies()
        diff[images] = rel_l2(out["mixed"][:, 4], out["fp64"][:, 4])
    assert diff[4] < 3 * diff[1] + 1e-7, diff
