"""minimal_b200: B200-native 3D Laplace FMM (minimal ExaFMM `3d/`, `3dp/`).

The product is the C-ABI library ``lib/libexafmm_b200.so`` (declared in
``include/exafmm_b200.h``).  This module is a thin ctypes mirror of the
reference's driver-level interface for Python callers (tests, bench.py):

    fmm = FMM(P=10, ncrit=64, theta=0.4)   # globals of 3d/fmm.cxx:12-15
    fmm.set_bodies(bodies)                  # Body records (N x 8) or x,y,z,q (N x 4)
    fmm.evaluate()                          # buildTree .. downwardPass
    out = fmm.bodies()                      # tree order, like the reference

There is no CPU fallback: without the built library (or without an sm_100
GPU) the calls raise.
"""
import ctypes
import os

import numpy as np

from .bodies import drand48_bodies, plummer_bodies, uniform_bodies  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libexafmm_b200.so")

FP64, MIXED = 0, 1
HOST, DEVICE = 0, 1
ERRORS = {
    -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_NOMEM", -4: "ERR_STATE", -5: "ERR_DEPTH",
    -6: "ERR_CAPACITY", -7: "ERR_TIMEOUT", -8: "ERR_NOGPU",
}

# Every entry point of include/exafmm_b200.h (checked by the tests).
API = [
    "exafmm_b200_create", "exafmm_b200_destroy", "exafmm_b200_last_error", "exafmm_b200_set_params",
    "exafmm_b200_set_bodies", "exafmm_b200_build_tree", "exafmm_b200_build_lists", "exafmm_b200_upward",
    "exafmm_b200_horizontal", "exafmm_b200_downward", "exafmm_b200_evaluate", "exafmm_b200_get_bodies",
    "exafmm_b200_get_perm", "exafmm_b200_num_cells", "exafmm_b200_get_tree", "exafmm_b200_count_lists",
    "exafmm_b200_get_lists", "exafmm_b200_get_expansions", "exafmm_b200_direct", "exafmm_b200_get_timings",
    "exafmm_b200_last_launches", "exafmm_b200_arch", "exafmm_b200_fma_peak", "exafmm_b200_direct_static",
    "exafmm_b200_dipole_correction", "exafmm_b200_ewald", "exafmm_b200_set_batch", "exafmm_b200_autotune",
    "exafmm_b200_set_charges", "exafmm_b200_reevaluate", "exafmm_b200_test_stall_tc",
    "exafmm_b200_set_tile", "exafmm_b200_get_tile", "exafmm_b200_m2l_stats",
    "exafmm_b200_ewald_parts", "exafmm_b200_p2p", "exafmm_b200_p2m", "exafmm_b200_m2m", "exafmm_b200_m2l", "exafmm_b200_l2l", "exafmm_b200_l2p",
]

PHASES = ["tree", "lists", "upward", "m2l", "p2p", "downward", "total"]


class FMMError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("P", ctypes.c_int), ("ncrit", ctypes.c_int), ("theta", ctypes.c_double),
                ("images", ctypes.c_int), ("cycle", ctypes.c_double), ("precision", ctypes.c_int),
                ("device", ctypes.c_int), ("dim", ctypes.c_int)]


_lib = None


def load_library(path=LIB_PATH):
    """Load (once) and type the C ABI.  Raises if the library was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} not built: run `python -m minimal_b200.build`")
    L = ctypes.CDLL(path)
    vp, i, i64, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
    sig = {
        "exafmm_b200_create": (i, [ctypes.POINTER(Params), ctypes.POINTER(vp)]),
        "exafmm_b200_destroy": (i, [vp]),
        "exafmm_b200_last_error": (ctypes.c_char_p, [vp]),
        "exafmm_b200_set_params": (i, [vp, ctypes.POINTER(Params)]),
        "exafmm_b200_set_bodies": (i, [vp, vp, i64, i]),
        "exafmm_b200_build_tree": (i, [vp]),
        "exafmm_b200_build_lists": (i, [vp]),
        "exafmm_b200_upward": (i, [vp]),
        "exafmm_b200_horizontal": (i, [vp]),
        "exafmm_b200_downward": (i, [vp]),
        "exafmm_b200_evaluate": (i, [vp]),
        "exafmm_b200_get_bodies": (i, [vp, vp, i]),
        "exafmm_b200_get_perm": (i, [vp, vp, i]),
        "exafmm_b200_num_cells": (i64, [vp]),
        "exafmm_b200_get_tree": (i, [vp, vp, vp, vp, vp, vp, vp]),
        "exafmm_b200_count_lists": (i, [vp, vp, vp]),
        "exafmm_b200_get_lists": (i, [vp] * 7),
        "exafmm_b200_get_expansions": (i, [vp, vp, vp]),
        "exafmm_b200_direct": (i, [vp, vp, i64, i]),
        "exafmm_b200_get_timings": (i, [vp, vp]),
        "exafmm_b200_last_launches": (i64, [vp]),
        "exafmm_b200_arch": (i, []),
        "exafmm_b200_fma_peak": (i, [vp, i, vp]),
        "exafmm_b200_direct_static": (i, [vp, i64, vp, i64, vp]),
        "exafmm_b200_dipole_correction": (i, [vp]),
        "exafmm_b200_ewald": (i, [vp, i, d, d, d, vp, i64, i]),
        "exafmm_b200_set_batch": (i, [vp, vp, vp, i, i]),
        "exafmm_b200_autotune": (i, [vp, vp, i, i, vp, vp]),
        "exafmm_b200_set_charges": (i, [vp, vp, i]),
        "exafmm_b200_reevaluate": (i, [vp]),
        "exafmm_b200_test_stall_tc": (i, [vp, i64]),
        "exafmm_b200_set_tile": (i, [vp, i, i]),
        "exafmm_b200_m2l_stats": (i, [vp, vp]),
        "exafmm_b200_ewald_parts": (i, [vp, i, i, d, d, d, vp, i64, i]),
        "exafmm_b200_p2p": (i, [vp, vp, i64, vp, i64, vp, i]),
        "exafmm_b200_p2m": (i, [vp, vp, vp, i64, vp, i]),
        "exafmm_b200_m2m": (i, [vp, vp, vp, i, vp, vp, i]),
        "exafmm_b200_m2l": (i, [vp, vp, vp, vp, vp, vp, i]),
        "exafmm_b200_l2l": (i, [vp, vp, vp, i, vp, vp, i]),
        "exafmm_b200_l2p": (i, [vp, vp, vp, vp, i64, i]),
        "exafmm_b200_get_tile": (i, [vp, i, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def as_records(bodies, dim=3):
    """3D: N x 4 (x,y,z,q) or N x 8 Body records -> contiguous N x 8 float64.
    2D: N x 3 (x,y,q) or N x 6 Body records (2d/exafmm.h:14-19) -> N x 6."""
    b = np.asarray(bodies, dtype=np.float64)
    short, full = (3, 6) if dim == 2 else (4, 8)
    if b.ndim != 2 or b.shape[1] not in (short, full):
        raise ValueError(f"bodies must be N x {short} (X, q) or N x {full} (X, q, p, F)")
    if b.shape[1] == short:
        r = np.zeros((len(b), full))
        r[:, :short] = b
        return r
    return np.ascontiguousarray(b)


class FMM:
    """One FMM problem on one GPU (a handle of the C ABI)."""

    def __init__(self, P=10, ncrit=64, theta=0.4, images=0, cycle=0.0, precision="fp64", device=0, dim=3):
        self.lib = load_library()
        self.dim = dim
        self.params = Params(P, ncrit, theta, images, cycle, MIXED if precision == "mixed" else FP64, device, dim)
        h = ctypes.c_void_p()
        rc = self.lib.exafmm_b200_create(ctypes.byref(self.params), ctypes.byref(h))
        if rc != 0:
            raise FMMError(rc, self.lib.exafmm_b200_last_error(None).decode())
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.exafmm_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise FMMError(rc, self.lib.exafmm_b200_last_error(self.h).decode())

    # ---- configuration and input
    def set_params(self, **kw):
        for k, v in kw.items():
            if k == "precision":
                v = MIXED if v == "mixed" else FP64
            setattr(self.params, k, v)
        self._check(self.lib.exafmm_b200_set_params(self.h, ctypes.byref(self.params)))

    def _rec(self, bodies):
        return as_records(bodies, self.dim)

    def _len(self):
        return 6 if self.dim == 2 else 8

    def set_bodies(self, bodies):
        rec = self._rec(bodies)
        self.n = len(rec)
        self._check(self.lib.exafmm_b200_set_bodies(self.h, _p(rec), self.n, HOST))

    def set_bodies_device(self, ptr, n):
        """Body records already in device memory (e.g. a torch tensor's data_ptr())."""
        self.n = int(n)
        self._check(self.lib.exafmm_b200_set_bodies(self.h, ctypes.c_void_p(ptr), self.n, DEVICE))

    def set_batch(self, systems):
        """A batch of independent systems: a list of N_q x 4 (or x 8) arrays.
        evaluate() runs each phase once over all of them; bodies() returns
        every system's bodies in its own tree order, one system after the
        other (split with self.offsets)."""
        recs = [as_records(x) for x in systems]
        offsets = np.zeros(len(recs) + 1, dtype=np.int64)
        offsets[1:] = np.cumsum([len(r) for r in recs])
        rec = np.ascontiguousarray(np.concatenate(recs))
        self.n = len(rec)
        self.offsets = offsets
        self._check(self.lib.exafmm_b200_set_batch(self.h, _p(rec), _p(offsets), len(recs), HOST))

    def set_batch_device(self, ptr, offsets):
        """Batch whose Body records are already in device memory; offsets on the host."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        self.n = int(offsets[-1])
        self.offsets = offsets
        self._check(self.lib.exafmm_b200_set_batch(self.h, ctypes.c_void_p(ptr), _p(offsets), len(offsets) - 1,
                                                   DEVICE))

    # ---- phases (3d/fmm.cxx:40-53)
    def build_tree(self):
        self._check(self.lib.exafmm_b200_build_tree(self.h))

    def build_lists(self):
        self._check(self.lib.exafmm_b200_build_lists(self.h))

    def upward(self):
        self._check(self.lib.exafmm_b200_upward(self.h))

    def horizontal(self):
        self._check(self.lib.exafmm_b200_horizontal(self.h))

    def downward(self):
        self._check(self.lib.exafmm_b200_downward(self.h))

    def evaluate(self):
        self._check(self.lib.exafmm_b200_evaluate(self.h))

    def set_charges(self, q):
        """New charges (N values, input order of set_bodies / set_batch) on
        the same positions: the tree and the interaction lists are kept."""
        q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).ravel())
        if len(q) != self.n:
            raise ValueError(f"need {self.n} charges, got {len(q)}")
        self._check(self.lib.exafmm_b200_set_charges(self.h, _p(q), HOST))

    def reevaluate(self):
        """Upward, horizontal and downward passes over the kept tree and
        lists (after set_charges, or again on the same bodies)."""
        self._check(self.lib.exafmm_b200_reevaluate(self.h))

    # ---- results
    def bodies(self):
        out = np.zeros((self.n, self._len()))
        self._check(self.lib.exafmm_b200_get_bodies(self.h, _p(out), HOST))
        return out

    def bodies_device(self, ptr):
        self._check(self.lib.exafmm_b200_get_bodies(self.h, ctypes.c_void_p(ptr), DEVICE))

    def perm(self):
        out = np.zeros(self.n, np.int64)
        self._check(self.lib.exafmm_b200_get_perm(self.h, _p(out), HOST))
        return out

    def num_cells(self):
        return int(self.lib.exafmm_b200_num_cells(self.h))

    def tree(self):
        c = self.num_cells()
        nchild, child, body, nbody, level = (np.zeros(c, np.int32) for _ in range(5))
        xr = np.zeros((c, 4))
        self._check(self.lib.exafmm_b200_get_tree(self.h, _p(nchild), _p(child), _p(body), _p(nbody), _p(level),
                                                  _p(xr)))
        return dict(nchild=nchild, child=child, body=body, nbody=nbody, level=level, xr=xr)

    def lists(self):
        a, b = np.zeros(1, np.int64), np.zeros(1, np.int64)
        self._check(self.lib.exafmm_b200_count_lists(self.h, _p(a), _p(b)))
        c = self.num_cells()
        na, nb = int(a[0]), int(b[0])
        mo, po = np.zeros(c + 1, np.int32), np.zeros(c + 1, np.int32)
        ms, mi = np.zeros(max(na, 1), np.int32), np.zeros(max(na, 1), np.int32)
        ps, pi = np.zeros(max(nb, 1), np.int32), np.zeros(max(nb, 1), np.int32)
        self._check(self.lib.exafmm_b200_get_lists(self.h, _p(mo), _p(ms), _p(mi), _p(po), _p(ps), _p(pi)))
        return dict(m2l_off=mo, m2l_src=ms[:na], m2l_img=mi[:na], p2p_off=po, p2p_src=ps[:nb], p2p_img=pi[:nb])

    def expansions(self):
        c = self.num_cells()
        nt = self.params.P if self.dim == 2 else self.params.P * (self.params.P + 1) // 2
        M = np.zeros((c, nt, 2))
        L = np.zeros((c, nt, 2))
        self._check(self.lib.exafmm_b200_get_expansions(self.h, _p(M), _p(L)))
        return M[..., 0] + 1j * M[..., 1], L[..., 0] + 1j * L[..., 1]

    def direct(self, targets):
        """FP64 direct sum of all loaded bodies onto targets (Body records; p, F accumulate)."""
        t = self._rec(targets).copy()
        self._check(self.lib.exafmm_b200_direct(self.h, _p(t), len(t), HOST))
        return t

    def dipole_correction(self):
        """Periodic systems: dipole correction of the current results in place
        (3dp/fmm.cxx:63-75)."""
        self._check(self.lib.exafmm_b200_dipole_correction(self.h))

    def ewald(self, targets, ksize=11, alpha=None, sigma=0.25 / np.pi, cutoff=None):
        """FP64 Ewald summation of all loaded bodies onto targets (Body
        records; p, F accumulate).  Defaults follow 3dp/fmm.cxx:20-23:
        alpha = ksize / cycle, cutoff = cycle / 2."""
        cyc = self.params.cycle
        alpha = ksize / cyc if alpha is None else alpha
        cutoff = cyc / 2 if cutoff is None else cutoff
        t = as_records(targets).copy()
        self._check(self.lib.exafmm_b200_ewald(self.h, int(ksize), float(alpha), float(sigma), float(cutoff), _p(t),
                                               len(t), HOST))
        return t

    EWALD_PARTS = {"wave": 1, "real": 2, "self": 4, "all": 7}

    def ewald_parts(self, targets, parts, ksize=11, alpha=None, sigma=0.25 / np.pi, cutoff=None):
        """Some of the Ewald parts ("wave", "real", "self", a list of them, or
        "all") onto targets; defaults as in ewald()."""
        mask = 0
        for p in ([parts] if isinstance(parts, str) else parts):
            mask |= self.EWALD_PARTS[p]
        cyc = self.params.cycle
        alpha = ksize / cyc if alpha is None else alpha
        cutoff = cyc / 2 if cutoff is None else cutoff
        t = as_records(targets).copy()
        self._check(self.lib.exafmm_b200_ewald_parts(self.h, mask, int(ksize), float(alpha), float(sigma),
                                                     float(cutoff), _p(t), len(t), HOST))
        return t

    def autotune(self, candidates=None, repeats=2):
        """Pick the fastest leaf size ncrit for the loaded bodies (one system or
        a batch); returns (ncrit, ms per evaluation) and keeps it."""
        best = np.zeros(1, dtype=np.int32)
        ms = np.zeros(1)
        if candidates is None:
            cand_p, nc = None, 0
        else:
            cand = np.ascontiguousarray(candidates, dtype=np.int32)
            cand_p, nc = _p(cand), len(cand)
        self._check(self.lib.exafmm_b200_autotune(self.h, cand_p, nc, int(repeats), _p(best), _p(ms)))
        self.params.ncrit = int(best[0])
        return int(best[0]), float(ms[0])

    def timings(self):
        t = np.zeros(7)
        self._check(self.lib.exafmm_b200_get_timings(self.h, _p(t)))
        return dict(zip(PHASES, t.tolist()))

    def last_launches(self):
        return int(self.lib.exafmm_b200_last_launches(self.h))

    # ---- single operators (3d/kernel.h:122-323) on explicit cells.  cell:
    # X[3], R; expansions: NTERM complex; bodies: N x 8 Body records.  Each
    # returns the accumulated output as a new array (inputs are not modified).
    def _nt(self):
        return self.params.P * (self.params.P + 1) // 2

    @staticmethod
    def _c2(a, n):
        a = np.zeros(n, complex) if a is None else np.asarray(a, complex).ravel()
        return np.ascontiguousarray(np.stack([a.real, a.imag], -1))

    @staticmethod
    def _cell(c):
        c = np.asarray(c, np.float64).ravel()
        return np.ascontiguousarray(np.concatenate([c, np.zeros(4 - len(c))]) if len(c) < 4 else c[:4])

    # every array handed to the library is bound to a local first: _p() keeps
    # only the address, so an inline temporary could be freed before the call
    def p2p(self, targets, sources, shift=None):
        t = np.array(as_records(targets), order="C")
        s = as_records(sources)
        sh = None if shift is None else np.ascontiguousarray(shift, np.float64)
        self._check(self.lib.exafmm_b200_p2p(self.h, _p(t), len(t), _p(s), len(s), None if sh is None else _p(sh),
                                             HOST))
        return t

    def p2m(self, cell, bodies, M=None):
        m = self._c2(M, self._nt())
        b = as_records(bodies)
        c = self._cell(cell)
        self._check(self.lib.exafmm_b200_p2m(self.h, _p(c), _p(b), len(b), _p(m), HOST))
        return m[:, 0] + 1j * m[:, 1]

    def m2m(self, parent, children, Mchildren, M=None):
        nt = self._nt()
        m = self._c2(M, nt)
        ch = np.ascontiguousarray([self._cell(c) for c in children]).reshape(-1, 4)
        mc = self._c2(Mchildren, nt * len(ch))
        c = self._cell(parent)
        self._check(self.lib.exafmm_b200_m2m(self.h, _p(c), _p(m), len(ch), _p(ch), _p(mc), HOST))
        return m[:, 0] + 1j * m[:, 1]

    def m2l(self, target, source, M, L=None, shift=None):
        nt = self._nt()
        lo, mm = self._c2(L, nt), self._c2(M, nt)
        sh = None if shift is None else np.ascontiguousarray(shift, np.float64)
        t, s = self._cell(target), self._cell(source)
        self._check(self.lib.exafmm_b200_m2l(self.h, _p(t), _p(lo), _p(s), _p(mm), None if sh is None else _p(sh),
                                             HOST))
        return lo[:, 0] + 1j * lo[:, 1]

    def l2l(self, parent, L, children, Lchildren=None):
        nt = self._nt()
        ch = np.ascontiguousarray([self._cell(c) for c in children]).reshape(-1, 4)
        lc = self._c2(Lchildren, nt * len(ch))
        lp = self._c2(L, nt)
        c = self._cell(parent)
        self._check(self.lib.exafmm_b200_l2l(self.h, _p(c), _p(lp), len(ch), _p(ch), _p(lc), HOST))
        return (lc[:, 0] + 1j * lc[:, 1]).reshape(len(ch), nt)

    def l2p(self, cell, L, bodies):
        b = np.array(as_records(bodies), order="C")
        lc = self._c2(L, self._nt())
        c = self._cell(cell)
        self._check(self.lib.exafmm_b200_l2p(self.h, _p(c), _p(lc), _p(b), len(b), HOST))
        return b

    def m2l_stats(self):
        """Grouped M2L of the last evaluation: groups, segments, residual entries, tiles."""
        v = np.zeros(4, dtype=np.int64)
        self._check(self.lib.exafmm_b200_m2l_stats(self.h, _p(v)))
        return dict(zip(("groups", "segments", "residual", "tiles"), v.tolist()))

    TILES = {"m2l_flush": 0, "p2p_stage": 1}

    def set_tile(self, name, value):
        """A run-time tile shape (include/exafmm_b200.h, EXAFMM_TILE_*); 0 = default."""
        self._check(self.lib.exafmm_b200_set_tile(self.h, self.TILES[name], int(value)))

    def get_tile(self, name):
        v = np.zeros(1, dtype=np.int32)
        self._check(self.lib.exafmm_b200_get_tile(self.h, self.TILES[name], _p(v)))
        return int(v[0])

    def fma_peak(self, precision="fp64"):
        """TFLOP/s of FMA chains: "fp64"; "fp32" (the larger of scalar and
        packed FP32x2); "fp32_scalar"; "fp32x2"."""
        kind = {"fp64": 0, "fp32": 1, "mixed": 1, "fp32_scalar": 2, "fp32x2": 3}[precision]
        t = np.zeros(1)
        self._check(self.lib.exafmm_b200_fma_peak(self.h, kind, _p(t)))
        return float(t[0])


def rel_l2(a, b):
    """Relative L2 error of a against b (the reference's verification metric, 3d/fmm.cxx:71-85)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
