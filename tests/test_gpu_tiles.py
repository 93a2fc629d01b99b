"""Run-time tile shapes (exafmm_b200_set_tile) and the autotuner's choice of
them: the near-field source tile changes only the grouping of the sums (FP64
results agree to rounding, 1e-13; mixed to FP32 rounding), the M2L flush
interval only the length of the FP32 accumulation windows, and the defaults
are the documented ones."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 2e-6)])
def test_near_field_source_tiles_agree(precision, tol):
    from minimal_b200 import FMM, drand48_bodies

    xq = drand48_bodies(60000, 4)
    f = FMM(P=8, ncrit=64, theta=0.4, precision=precision)
    f.set_bodies(xq)
    assert f.get_tile("p2p_stage") == (1536 if precision == "mixed" else 1024)
    out = {}
    for tile in (1024, 1536, 2048):
        f.set_tile("p2p_stage", tile)
        assert f.get_tile("p2p_stage") == tile
        f.evaluate()
        out[tile] = f.bodies()
    for tile in (1024, 2048):
        assert np.array_equal(out[tile][:, :4], out[1536][:, :4])
        assert rel(out[tile][:, 4], out[1536][:, 4]) < tol
        assert rel(out[tile][:, 5:], out[1536][:, 5:]) < tol


def test_m2l_flush_default_and_range():
    from minimal_b200 import FMM, FMMError, drand48_bodies

    xq = drand48_bodies(30000, 5)
    for P, want in ((8, 2), (10, 2), (11, 1), (12, 1), (14, 4)):
        f = FMM(P=P, precision="mixed")
        assert f.get_tile("m2l_flush") == want
    f = FMM(P=10, precision="mixed")
    f.set_bodies(xq)
    res = {}
    for fl in (1, 16):
        f.set_tile("m2l_flush", fl)
        f.evaluate()
        res[fl] = f.bodies()
    assert rel(res[16][:, 5:], res[1][:, 5:]) < 1e-5
    with pytest.raises(FMMError):
        f.set_tile("m2l_flush", 65)
    with pytest.raises(FMMError):
        f.set_tile("p2p_stage", 777)


def test_autotune_picks_a_source_tile():
    from minimal_b200 import FMM, drand48_bodies

    xq = drand48_bodies(40000, 6)
    f = FMM(P=6, ncrit=64, theta=0.5, precision="mixed")
    f.set_bodies(xq)
    ncrit, ms = f.autotune(candidates=[32, 64], repeats=1)
    assert ncrit in (32, 64) and ms > 0
    assert f.get_tile("p2p_stage") in (1024, 1536, 2048)
    out = f.bodies()
    assert np.isfinite(out[:, 4:]).all()
