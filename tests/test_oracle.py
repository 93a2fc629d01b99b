"""The oracle pinned against the reference (CPU only).

The C restatement (oracle/fmm_oracle.c) must reproduce, bit for bit, what the
reference's own headers produce: the golden fixtures in tests/golden/ (made
by tests/golden/make_golden.py from oracle/_ref) and the reference tests'
known answers (test/test_kernel.cxx:5-7, test/test_fmm.cxx:5-6).
"""
import os

import numpy as np
import pytest

from tests.conftest import GOLDEN, golden

CASES_3D = ["3d_n2000_p10", "3d_n10000_p10", "3d_n3000_p6_nc16_th05", "3d_clustered_n4000_p8", "3d_n1",
            "3d_n64_single_leaf", "3d_n65"]
CASES_3DP = ["3dp_n1000_p10_img2", "3dp_n1500_p8_img3"]


@pytest.mark.parametrize("P,bound", [(10, 1e-3), (20, 1e-6), (30, 1e-9)])
def test_kernel_chain_known_answer(port, kat, P, bound):
    p_err, f_err = port.kernel_chain(P)
    assert p_err == kat[f"kernel_p{P}"]
    assert p_err < bound  # the reference test's own bound
    assert 0 < f_err < 50 * bound


@pytest.mark.parametrize("name", CASES_3D + CASES_3DP)
def test_port_matches_reference_fixture(port, name):
    g = golden(name)
    images = int(g["images"])
    out = port.fmm(g["xq"], int(g["P"]), int(g["ncrit"]), float(g["theta"]), images,
                   float(g["cycle"]) if images else 0.0)
    c = port.cells()
    for k in ("nchild", "child", "body", "nbody"):
        assert np.array_equal(c[k], g[k]), k
    assert np.array_equal(c["xr"], g["xr"])
    lists = port.lists()
    for k in ("m2l_off", "m2l_src", "m2l_img", "p2p_off", "p2p_src", "p2p_img"):
        assert np.array_equal(lists[k], g[k]), k
    assert np.array_equal(out, g["bodies"], equal_nan=True)  # N=1: the reference divides by r=0
    P = int(g["P"])
    M, L = port.expansions(P * (P + 1) // 2)
    assert np.array_equal(M, g["M"], equal_nan=True) and np.array_equal(L, g["L"], equal_nan=True)
    if "ewald" in g:
        port.dipole_correction(float(g["cycle"]))
        assert np.array_equal(port.bodies(), g["bodies_dipole"])
        ks = 11
        cyc = float(g["cycle"])
        ew = port.ewald(ks, ks / cyc, 0.25 / np.pi, cyc / 2, cyc)
        assert np.allclose(ew, g["ewald"], rtol=1e-13, atol=1e-13 * np.abs(g["ewald"]).max())


def test_port_reproduces_test_fmm(port, kat):
    """test/test_fmm.h:14-90 at P=10: FMM on 10,000 bodies vs direct on 10
    stride-sampled targets (tree order)."""
    xq = port.reference_bodies(10000)
    out = port.fmm(xq, 10, 64, 0.4)
    stride = len(out) // 10
    tgt = out[::stride][:10].copy()
    fmm = tgt.copy()
    tgt[:, 4:] = 0
    d = port.direct(tgt, out)
    err = np.sqrt(((d[:, 4] - fmm[:, 4]) ** 2).sum() / (fmm[:, 4] ** 2).sum())
    assert err == pytest.approx(kat["fmm_p10"], rel=1e-12)
    assert err < 1e-3


def test_port_full_size_lists_match_reference_digest(port):
    """1M uniform bodies: the port's tree and lists hash to the reference's."""
    from tests.golden.make_golden import digest
    from minimal_b200.bodies import drand48_bodies

    g = golden("3d_n1048576_p10_sampled")
    xq = drand48_bodies(int(g["n"]), int(g["seed"]))
    c = port.tree(xq, int(g["ncrit"]))
    assert port.ncells == int(g["ncells"])
    assert digest(c["nchild"], c["child"], c["body"], c["nbody"], c["xr"]) == str(g["tree_digest"])
    lists = port.build_lists(float(g["theta"]))
    assert len(lists["m2l_src"]) == int(g["n_m2l"]) and len(lists["p2p_src"]) == int(g["n_p2p"])
    assert digest(lists["m2l_off"], lists["m2l_src"], lists["m2l_img"], lists["p2p_off"], lists["p2p_src"],
                  lists["p2p_img"]) == str(g["list_digest"])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref",
                                                    "libref3d_lazy.so")), reason="reference not built here")
@pytest.mark.parametrize("seed,ncrit,theta,P", [(11, 20, 0.35, 6), (12, 100, 0.6, 4), (13, 8, 0.3, 5)])
def test_port_matches_compiled_reference_random(port, seed, ncrit, theta, P):
    import oracle
    from minimal_b200.bodies import plummer_bodies

    ref = oracle.Ref("3d", "lazy")
    xq = plummer_bodies(3000, seed)
    xq[:, 3] = np.random.default_rng(seed).uniform(-0.5, 0.5, len(xq))
    a = port.fmm(xq, P, ncrit, theta)
    b = ref.fmm(xq, P, ncrit, theta)
    assert np.array_equal(a, b)
    la, lb = port.lists(), ref.lists()
    for k in la:
        assert np.array_equal(la[k], lb[k])


def test_reference_bodies_generator(port):
    from minimal_b200.bodies import drand48_bodies

    assert np.array_equal(drand48_bodies(5000, 0), port.reference_bodies(5000, 0))
    assert np.array_equal(drand48_bodies(777, 3, kind="3dp"), port.reference_bodies(777, 3, kind=1))
