"""bench.py's side legs run their Python flow on the CPU against a stand-in
of the FMM class (the GPU numbers come from the real class on a B200): the
keys the JSON line carries, and that every value is JSON-serialisable."""
import json
import types

import numpy as np

from tests.conftest import ROOT  # noqa: F401  (puts the repository on sys.path)


class FakeFMM:
    def __init__(self, P=10, ncrit=64, theta=0.4, precision="fp64", device=0, **kw):
        self.P, self.ncrit, self.precision = P, ncrit, precision
        self.n = 0

    def set_bodies(self, xq):
        self.xq = np.asarray(xq, dtype=np.float64)
        self.n = len(self.xq)

    def set_charges(self, q):
        assert len(q) == self.n and np.all(np.isfinite(q))
        self.xq = self.xq.copy()
        self.xq[:, 3] = q

    def autotune(self, repeats=2):
        return 96, 1.5

    def evaluate(self):
        pass

    def reevaluate(self):
        pass

    def timings(self):
        return {"tree": 0.1, "lists": 0.1, "upward": 0.1, "m2l": 0.5, "p2p": 0.8, "downward": 0.2, "total": 1.25}

    def bodies(self):
        out = np.zeros((self.n, 8))
        out[:, :4] = self.xq[:, :4]
        out[:, 4], out[:, 5:] = 2.0, 0.25
        return out

    def direct(self, targets):
        t = np.array(targets)
        t[:, 4], t[:, 5:] = 2.0 * (1 + 1e-6), 0.25
        return t

    def close(self):
        pass


TORCH = types.SimpleNamespace(cuda=types.SimpleNamespace(synchronize=lambda: None))
FLUSH = types.SimpleNamespace(zero_=lambda: None)


def test_plummer_leg_flow():
    import bench

    r = bench.plummer_leg(FakeFMM, FLUSH, TORCH, 0, n=4096)
    json.dumps(r)
    for P in (6, 8, 10, 12):
        leg = r[f"P{P}"]
        assert leg["ncrit"] == 96 and leg["ms_per_eval"] == 1.25
        assert leg["error_vs_direct"]["targets"] == 1000 and "p" in leg["fp64_error_vs_direct"]


def test_reevaluate_leg_flow():
    import bench

    f = FakeFMM()
    f.set_bodies(np.random.default_rng(0).uniform(-1, 1, (2048, 4)))
    r = bench.reevaluate_leg(f, 2048, FLUSH, TORCH, 2.5)
    json.dumps(r)
    assert r["ms_per_eval"] == 1.25 and r["speedup_vs_full_evaluate"] == 2.0
