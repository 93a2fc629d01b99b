"""Synthetic bodies with the reference drivers' distributions.

``drand48_bodies`` reproduces the reference drivers bit for bit
(3d/fmm.cxx:19-35, 3dp/fmm.cxx:27-44, test/test_fmm.h:23-38): libc's 48-bit
linear congruential generator seeded by srand48(seed), drawn x, y, z, q per
body, then the mean charge removed.  The generator is vectorised by jumping
the LCG ahead (x_{k+s} = A_s x_k + C_s mod 2^48), so a million bodies take a
fraction of a second.  ``plummer_bodies`` and ``uniform_bodies`` are seeded
numpy generators for the workloads the reference has no generator for.
"""
import numpy as np

_A = 0x5DEECE66D
_C = 0xB
_MASK = (1 << 48) - 1


def _drand48_stream(n, seed):
    """First n values of drand48() after srand48(seed), as float64 (exact)."""
    x0 = ((seed & 0xFFFFFFFF) << 16) | 0x330E
    block = 4096
    first = np.empty(min(n, block), dtype=np.uint64)
    x = x0
    for k in range(len(first)):
        x = (_A * x + _C) & _MASK
        first[k] = x
    if n <= block:
        return first[:n].astype(np.float64) / float(1 << 48)
    # jump constants for a stride of `block`
    a_s, c_s = 1, 0
    for _ in range(block):
        a_s, c_s = (_A * a_s) & _MASK, (_A * c_s + _C) & _MASK
    nblk = (n + block - 1) // block
    out = np.empty((nblk, block), dtype=np.uint64)
    out[0] = first
    a_s, c_s = np.uint64(a_s), np.uint64(c_s)
    m = np.uint64(_MASK)
    for b in range(1, nblk):
        out[b] = (out[b - 1] * a_s + c_s) & m  # uint64 wraps mod 2^64; 2^48 divides it
    return out.reshape(-1)[:n].astype(np.float64) / float(1 << 48)


def drand48_bodies(n, seed=0, kind="3d", cycle=2 * np.pi):
    """N x 4 (x, y, z, q) exactly as the reference drivers generate them.

    kind "3d":  x = d*2*M_PI - M_PI           (3d/fmm.cxx:23)
    kind "3dp": x = d*cycle - cycle*.5        (3dp/fmm.cxx:33)
    q = d - .5, then q -= mean (summed in body order, divided by N).
    """
    u = _drand48_stream(4 * n, seed).reshape(n, 4)
    xq = np.empty((n, 4))
    if kind == "3d":
        xq[:, :3] = u[:, :3] * 2 * np.pi - np.pi
    else:
        xq[:, :3] = u[:, :3] * cycle - cycle * .5
    xq[:, 3] = u[:, 3] - .5
    avg = 0.0
    for q in xq[:, 3].tolist():  # sequential sum, as the reference accumulates
        avg += q
    avg /= n
    xq[:, 3] -= avg
    return xq


def uniform_bodies(n, seed=0, lo=-np.pi, hi=np.pi):
    """Seeded uniform cube with charges U[-0.5, 0.5), neutralised."""
    g = np.random.default_rng(seed)
    xq = np.empty((n, 4))
    xq[:, :3] = g.uniform(lo, hi, (n, 3))
    xq[:, 3] = g.uniform(-0.5, 0.5, n)
    xq[:, 3] -= xq[:, 3].mean()
    return xq


def plummer_bodies(n, seed=0, a=1.0, rmax=10.0):
    """Plummer sphere (scale radius a, radii above rmax rejected), charges 1/N.

    r = a / sqrt(u^(-2/3) - 1) with u uniform, isotropic directions.
    """
    g = np.random.default_rng(seed)
    r = np.empty(0)
    while len(r) < n:
        u = g.uniform(1e-12, 1.0, 2 * n)
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = np.concatenate([r, rr[rr <= rmax]])
    r = r[:n]
    cz = g.uniform(-1.0, 1.0, n)
    ph = g.uniform(0.0, 2 * np.pi, n)
    sz = np.sqrt(1.0 - cz * cz)
    xq = np.empty((n, 4))
    xq[:, 0] = r * sz * np.cos(ph)
    xq[:, 1] = r * sz * np.sin(ph)
    xq[:, 2] = r * cz
    xq[:, 3] = 1.0 / n
    return xq
