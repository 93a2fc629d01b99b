"""Oracle bindings (TEST INFRASTRUCTURE ONLY).

Two CPU checkers for minimal ExaFMM's 3D Laplace FMM, both reached through
ctypes:

* ``Port`` -- ``oracle/_build/liboracle.so``, the plain-C restatement of the
  reference algorithm in ``oracle/fmm_oracle.c`` (every function cites the
  reference lines it restates);
* ``Ref``  -- ``oracle/_ref/libref*.so``, the reference's own headers compiled
  unmodified by ``oracle/Makefile`` around ``oracle/ref/ref_driver.cpp``.

and, for the reference's 2D code (`2d/`), ``Fmm2D("port")`` (the restatement in
``oracle/fmm2d_oracle.c``) and ``Fmm2D("ref")`` (the reference's 2d headers
around ``oracle/ref/ref2d_driver.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
use this package, and only as the checker or the timed CPU baseline.  The
product library (``minimal_b200``) never imports it.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIBS = {
    ("3d", "lazy"): os.path.join(HERE, "_ref", "libref3d_lazy.so"),
    ("3d", "eager"): os.path.join(HERE, "_ref", "libref3d_eager.so"),
    ("3dp", "lazy"): os.path.join(HERE, "_ref", "libref3dp_lazy.so"),
}

_d = ctypes.c_double
_l = ctypes.c_long
_i = ctypes.c_int
_p = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_p)


def build():
    """Compile the port (and, when the reference sources are present, the
    reference libraries) with oracle/Makefile."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE], check=True)


class _Common:
    """Shared result getters: both libraries keep one problem as global state."""

    def _bind_common(self, pre):
        L = self.lib
        self._pre = pre
        getattr(L, pre + "get_bodies").argtypes = [_p]
        getattr(L, pre + "count_lists").argtypes = [_p, _p]
        getattr(L, pre + "get_lists").argtypes = [_p] * 6
        getattr(L, pre + "get_expansions").argtypes = [_p, _p]
        getattr(L, pre + "direct").restype = None

    def bodies(self):
        out = np.zeros((self.n, 8))
        getattr(self.lib, self._pre + "get_bodies")(_ptr(out))
        return out

    def lists(self):
        a = np.zeros(1, np.int64)
        b = np.zeros(1, np.int64)
        getattr(self.lib, self._pre + "count_lists")(_ptr(a), _ptr(b))
        na, nb = int(a[0]), int(b[0])
        mo = np.zeros(self.ncells + 1, np.int32)
        po = np.zeros(self.ncells + 1, np.int32)
        ms, mi = np.zeros(max(na, 1), np.int32), np.zeros(max(na, 1), np.int32)
        ps, pi = np.zeros(max(nb, 1), np.int32), np.zeros(max(nb, 1), np.int32)
        getattr(self.lib, self._pre + "get_lists")(_ptr(mo), _ptr(ms), _ptr(mi), _ptr(po), _ptr(ps), _ptr(pi))
        return dict(m2l_off=mo, m2l_src=ms[:na], m2l_img=mi[:na], p2p_off=po, p2p_src=ps[:nb], p2p_img=pi[:nb])

    def expansions(self, nterm):
        M = np.zeros((self.ncells, nterm, 2))
        L = np.zeros((self.ncells, nterm, 2))
        getattr(self.lib, self._pre + "get_expansions")(_ptr(M), _ptr(L))
        return M[..., 0] + 1j * M[..., 1], L[..., 0] + 1j * L[..., 1]


class Port(_Common):
    """The C restatement (oracle/fmm_oracle.c)."""

    def __init__(self, path=PORT_LIB):
        if not os.path.exists(path):
            build()
        self.lib = L = ctypes.CDLL(path)
        L.orc_tree.restype = _l
        L.orc_tree.argtypes = [_l, _p, _i]
        L.orc_lists.restype = _l
        L.orc_lists.argtypes = [_d, _i, _d]
        L.orc_fmm.restype = _l
        L.orc_fmm.argtypes = [_l, _p, _i, _i, _d, _i, _d]
        L.orc_get_perm.argtypes = [_p]
        L.orc_get_cells.argtypes = [_p] * 6
        L.orc_direct.argtypes = [_l, _p, _l, _p, _i, _d]
        L.orc_dipole_correction.argtypes = [_d]
        L.orc_ewald.argtypes = [_i, _d, _d, _d, _d, _p]
        L.orc_kernel_chain.restype = _d
        L.orc_kernel_chain.argtypes = [_i, _p]
        L.orc_reference_bodies.argtypes = [_l, _l, _i, _d, _p]
        L.orc_op_p2m.argtypes = [_i, _p, _p, _l, _p]
        L.orc_op_m2m.argtypes = [_i, _p, _p, _i, _p, _p]
        L.orc_op_m2l.argtypes = [_i, _p, _p, _p, _p, _p, _d]
        L.orc_op_l2l.argtypes = [_i, _p, _p, _i, _p, _p]
        L.orc_op_l2p.argtypes = [_i, _p, _p, _p, _l]
        L.orc_op_p2p.argtypes = [_p, _l, _p, _l, _p, _d]
        for f in ("p2m", "m2m", "m2l", "l2l", "l2p", "p2p"):
            getattr(L, "orc_op_" + f).restype = None
        self._bind_common("orc_")
        self.n = 0
        self.ncells = 0

    # ---- single operators (3d/kernel.h:122-323) on caller data.  cell: X[3],
    # R; expansions: NTERM complex; bodies: N x 8 Body records.  Each returns
    # the accumulated output (a new array; the inputs are not modified).
    @staticmethod
    def _cplx(a, nt):
        a = np.zeros(nt, complex) if a is None else np.asarray(a, complex).ravel()
        return np.ascontiguousarray(np.stack([a.real, a.imag], -1))

    def op_p2m(self, P, cell, bodies, M=None):
        nt = P * (P + 1) // 2
        m = self._cplx(M, nt)
        b = np.ascontiguousarray(bodies, np.float64)
        self.lib.orc_op_p2m(P, _ptr(np.asarray(cell, np.float64)), _ptr(b), len(b), _ptr(m))
        return m[:, 0] + 1j * m[:, 1]

    def op_m2m(self, P, parent, children, Mchildren, M=None):
        nt = P * (P + 1) // 2
        m = self._cplx(M, nt)
        ch = np.ascontiguousarray(children, np.float64)
        mc = self._cplx(Mchildren, nt * len(ch))
        self.lib.orc_op_m2m(P, _ptr(np.asarray(parent, np.float64)), _ptr(m), len(ch), _ptr(ch), _ptr(mc))
        return m[:, 0] + 1j * m[:, 1]

    def op_m2l(self, P, target, source, M, L=None, ix=None, cycle=0.0):
        nt = P * (P + 1) // 2
        lo = self._cplx(L, nt)
        mm = self._cplx(M, nt)
        ixa = None if ix is None else np.ascontiguousarray(ix, np.int32)
        self.lib.orc_op_m2l(P, _ptr(np.asarray(target, np.float64)), _ptr(lo), _ptr(np.asarray(source, np.float64)),
                            _ptr(mm), None if ixa is None else _ptr(ixa), cycle)
        return lo[:, 0] + 1j * lo[:, 1]

    def op_l2l(self, P, parent, L, children, Lchildren=None):
        nt = P * (P + 1) // 2
        ch = np.ascontiguousarray(children, np.float64)
        lc = self._cplx(Lchildren, nt * len(ch))
        self.lib.orc_op_l2l(P, _ptr(np.asarray(parent, np.float64)), _ptr(self._cplx(L, nt)), len(ch), _ptr(ch),
                            _ptr(lc))
        return (lc[:, 0] + 1j * lc[:, 1]).reshape(len(ch), nt)

    def op_l2p(self, P, cell, L, bodies):
        nt = P * (P + 1) // 2
        b = np.array(bodies, np.float64, order="C")
        self.lib.orc_op_l2p(P, _ptr(np.asarray(cell, np.float64)), _ptr(self._cplx(L, nt)), _ptr(b), len(b))
        return b

    def op_p2p(self, targets, sources, ix=None, cycle=0.0):
        t = np.array(targets, np.float64, order="C")
        s = np.ascontiguousarray(sources, np.float64)
        ixa = None if ix is None else np.ascontiguousarray(ix, np.int32)
        self.lib.orc_op_p2p(_ptr(t), len(t), _ptr(s), len(s), None if ixa is None else _ptr(ixa), cycle)
        return t

    def reference_bodies(self, n, seed=0, kind=0, cycle=2 * np.pi):
        xq = np.zeros((n, 4))
        self.lib.orc_reference_bodies(n, seed, kind, cycle, _ptr(xq))
        return xq

    def tree(self, xq, ncrit):
        xq = np.ascontiguousarray(xq, np.float64)
        self.n = len(xq)
        self.ncells = self.lib.orc_tree(self.n, _ptr(xq), ncrit)
        return self.cells()

    def build_lists(self, theta, images=0, cycle=0.0):
        self.lib.orc_lists(theta, images, cycle)
        return self.lists()

    def fmm(self, xq, P, ncrit, theta, images=0, cycle=0.0):
        xq = np.ascontiguousarray(xq, np.float64)
        self.n = len(xq)
        self.ncells = self.lib.orc_fmm(self.n, _ptr(xq), P, ncrit, theta, images, cycle)
        return self.bodies()

    def perm(self):
        out = np.zeros(self.n, np.int64)
        self.lib.orc_get_perm(_ptr(out))
        return out

    def cells(self):
        c = self.ncells
        nchild, child, body, nbody, level = (np.zeros(c, np.int32) for _ in range(5))
        xr = np.zeros((c, 4))
        self.lib.orc_get_cells(_ptr(nchild), _ptr(child), _ptr(body), _ptr(nbody), _ptr(level), _ptr(xr))
        return dict(nchild=nchild, child=child, body=body, nbody=nbody, level=level, xr=xr)

    def direct(self, targets8, sources8, images=0, cycle=0.0):
        t = np.ascontiguousarray(targets8, np.float64).copy()
        s = np.ascontiguousarray(sources8, np.float64)
        self.lib.orc_direct(len(t), _ptr(t), len(s), _ptr(s), images, cycle)
        return t

    def dipole_correction(self, cycle):
        self.lib.orc_dipole_correction(cycle)

    def ewald(self, ksize, alpha, sigma, cutoff, cycle):
        out = np.zeros((self.n, 8))
        self.lib.orc_ewald(ksize, alpha, sigma, cutoff, cycle, _ptr(out))
        return out

    def kernel_chain(self, P):
        f = np.zeros(1)
        p = self.lib.orc_kernel_chain(P, _ptr(f))
        return p, float(f[0])


class Ref(_Common):
    """The reference's own headers compiled unmodified (oracle/_ref)."""

    def __init__(self, variant="3d", traversal="lazy"):
        path = REF_LIBS[(variant, traversal)]
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (run oracle/Makefile where the reference sources exist)")
        self.variant, self.traversal = variant, traversal
        self.lib = L = ctypes.CDLL(path)
        L.ref_set_threads.argtypes = [_i]
        L.ref_max_threads.restype = _i
        L.ref_build_tree.restype = _l
        L.ref_build_tree.argtypes = [_l, _p, _i]
        L.ref_fmm.restype = _l
        L.ref_fmm.argtypes = [_l, _p, _i, _i, _d, _i, _d, _i]
        L.ref_get_times.argtypes = [_p]
        L.ref_get_cells.argtypes = [_p] * 5
        L.ref_direct.argtypes = [_l, _p, _l, _p]
        L.ref_test_kernel.restype = _d
        L.ref_test_kernel.argtypes = [_i]
        if traversal == "eager" and variant == "3d":
            L.ref_test_fmm.restype = _d
            L.ref_test_fmm.argtypes = [_i]
        if variant == "3dp":
            L.ref_ewald.argtypes = [_i, _d, _d, _d, _p]
        if traversal == "lazy":
            self._bind_common("ref_")
        else:
            L.ref_get_bodies.argtypes = [_p]
            L.ref_get_expansions.argtypes = [_p, _p]
            self._pre = "ref_"
        self.n = 0
        self.ncells = 0

    def set_threads(self, n):
        self.lib.ref_set_threads(int(n))

    def max_threads(self):
        return self.lib.ref_max_threads()

    def tree(self, xq, ncrit):
        xq = np.ascontiguousarray(xq, np.float64)
        self.n = len(xq)
        self.ncells = self.lib.ref_build_tree(self.n, _ptr(xq), ncrit)
        return self.cells()

    def fmm(self, xq, P, ncrit, theta, images=0, cycle=0.0, lists_only=False):
        xq = np.ascontiguousarray(xq, np.float64)
        self.n = len(xq)
        self.ncells = self.lib.ref_fmm(self.n, _ptr(xq), P, ncrit, theta, images, cycle, 2 if lists_only else 1)
        return None if lists_only else self.bodies()

    def times(self):
        t = np.zeros(8)
        self.lib.ref_get_times(_ptr(t))
        return dict(tree=t[0], upward=t[1], lists=t[2], evaluate=t[3], downward=t[4], total=t[5])

    def cells(self):
        c = self.ncells
        nchild, child, body, nbody = (np.zeros(c, np.int32) for _ in range(4))
        xr = np.zeros((c, 4))
        self.lib.ref_get_cells(_ptr(nchild), _ptr(child), _ptr(body), _ptr(nbody), _ptr(xr))
        return dict(nchild=nchild, child=child, body=body, nbody=nbody, xr=xr)

    def direct(self, targets8, sources8):
        t = np.ascontiguousarray(targets8, np.float64).copy()
        s = np.ascontiguousarray(sources8, np.float64)
        self.lib.ref_direct(len(t), _ptr(t), len(s), _ptr(s))
        return t

    def dipole_correction(self):
        self.lib.ref_dipole_correction()

    def ewald(self, ksize, alpha, sigma, cutoff):
        out = np.zeros((self.n, 8))
        self.lib.ref_ewald(ksize, alpha, sigma, cutoff, _ptr(out))
        return out

    def test_kernel(self, P):
        return self.lib.ref_test_kernel(P)

    def test_fmm(self, P):
        return self.lib.ref_test_fmm(P)


# ---------------------------------------------------------------- 2D
REF2D_LIB = os.path.join(HERE, "_ref", "libref2d_lazy.so")
REF2DP_LIB = os.path.join(HERE, "_ref", "libref2dp_lazy.so")


class Fmm2D:
    """A 2D checker (minimal ExaFMM `2d/` and `2dp/`, lazy traversal):
    ``Fmm2D("port")`` is the C restatement in oracle/fmm2d_oracle.c (in
    liboracle.so, both variants), ``Fmm2D("ref")`` / ``Fmm2D("refp")`` the
    reference's own 2d / 2dp headers compiled by oracle/Makefile.  Bodies are
    6 doubles: X[2], q, p, F[2]."""

    def __init__(self, which="port"):
        path, self._pre = {"port": (PORT_LIB, "orc2_"), "ref": (REF2D_LIB, "ref2_"),
                           "refp": (REF2DP_LIB, "ref2_")}[which]
        if not os.path.exists(path):
            build()
        self.lib = L = ctypes.CDLL(path)
        f = lambda name: getattr(L, self._pre + name)  # noqa: E731
        f("tree").restype = _l
        f("tree").argtypes = [_l, _p, _i]
        f("fmm").restype = _l
        f("fmm").argtypes = [_l, _p, _i, _i, _d, _i, _d]
        f("get_bodies").argtypes = [_p]
        f("get_cells").argtypes = [_p] * 5
        f("count_lists").argtypes = [_p, _p]
        f("get_lists").argtypes = [_p] * 6
        f("get_expansions").argtypes = [_p, _p]
        f("direct").argtypes = [_l, _p, _l, _p, _i, _d]
        f("direct").restype = None
        self.n = self.ncells = self.P = 0

    def _f(self, name):
        return getattr(self.lib, self._pre + name)

    def tree(self, xyq, ncrit):
        xyq = np.ascontiguousarray(xyq, dtype=np.float64)
        self.n = len(xyq)
        self.ncells = int(self._f("tree")(self.n, _ptr(xyq), ncrit))
        return self.ncells

    def fmm(self, xyq, P, ncrit, theta, images=0, cycle=0.0):
        xyq = np.ascontiguousarray(xyq, dtype=np.float64)
        self.n, self.P = len(xyq), P
        self.ncells = int(self._f("fmm")(self.n, _ptr(xyq), P, ncrit, theta, images, cycle))
        assert self.ncells > 0, "images > 0 needs the periodic build"
        return self.ncells

    def bodies(self):
        out = np.zeros((self.n, 6))
        self._f("get_bodies")(_ptr(out))
        return out

    def cells(self):
        C = self.ncells
        nchild, child, body, nbody = (np.zeros(C, np.int32) for _ in range(4))
        xr = np.zeros((C, 3))
        self._f("get_cells")(_ptr(nchild), _ptr(child), _ptr(body), _ptr(nbody), _ptr(xr))
        return dict(nchild=nchild, child=child, body=body, nbody=nbody, xr=xr)

    def lists(self):
        a, b = np.zeros(1, np.int64), np.zeros(1, np.int64)
        self._f("count_lists")(_ptr(a), _ptr(b))
        na, nb = int(a[0]), int(b[0])
        mo, po = np.zeros(self.ncells + 1, np.int32), np.zeros(self.ncells + 1, np.int32)
        ms, mi = np.zeros(max(na, 1), np.int32), np.zeros(max(na, 1), np.int32)
        ps, pi = np.zeros(max(nb, 1), np.int32), np.zeros(max(nb, 1), np.int32)
        self._f("get_lists")(_ptr(mo), _ptr(ms), _ptr(mi), _ptr(po), _ptr(ps), _ptr(pi))
        return dict(m2l_off=mo, m2l_src=ms[:na], m2l_img=mi[:na], p2p_off=po, p2p_src=ps[:nb], p2p_img=pi[:nb])

    def expansions(self):
        M = np.zeros((self.ncells, self.P, 2))
        L = np.zeros((self.ncells, self.P, 2))
        self._f("get_expansions")(_ptr(M), _ptr(L))
        return M[..., 0] + 1j * M[..., 1], L[..., 0] + 1j * L[..., 1]

    def direct(self, targets6, sources6, images=0, cycle=0.0):
        t = np.ascontiguousarray(targets6, dtype=np.float64).copy()
        s = np.ascontiguousarray(sources6, dtype=np.float64)
        self._f("direct")(len(t), _ptr(t), len(s), _ptr(s), images, cycle)
        return t


def reference_bodies_2d(n, seed=0):
    """n x 3 (x, y, q) as the reference's 2d driver makes them (2d/fmm.cxx:21-35)."""
    L = ctypes.CDLL(PORT_LIB)
    L.orc2_reference_bodies.argtypes = [_l, _l, _p]
    xyq = np.zeros((n, 3))
    L.orc2_reference_bodies(n, seed, _ptr(xyq))
    return xyq
