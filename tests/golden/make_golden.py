"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own headers, compiled unmodified by oracle/Makefile into
oracle/_ref/, on small seeded problems and stores trees, interaction lists,
expansions and potentials/forces as compressed .npz files.  The tests compare
the oracle restatement and the GPU library against these files; the GPU box
has no reference sources, only these fixtures.

    make -C oracle && python tests/golden/make_golden.py       # 3D
    make -C oracle && python tests/golden/make_golden.py 2d    # 2D
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from minimal_b200.bodies import drand48_bodies  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name: (variant, n, seed, P, ncrit, theta, images, body kind, cluster)
CASES = {
    "3d_n2000_p10": ("3d", 2000, 0, 10, 64, 0.4, 0, "3d", False),
    "3d_n10000_p10": ("3d", 10000, 0, 10, 64, 0.4, 0, "3d", False),  # the CPU reference case / test_fmm size
    "3d_n3000_p6_nc16_th05": ("3d", 3000, 7, 6, 16, 0.5, 0, "3d", False),
    "3d_clustered_n4000_p8": ("3d", 4000, 3, 8, 32, 0.4, 0, "3d", True),
    "3d_n1": ("3d", 1, 0, 10, 64, 0.4, 0, "3d", False),
    "3d_n64_single_leaf": ("3d", 64, 0, 10, 64, 0.4, 0, "3d", False),
    "3d_n65": ("3d", 65, 0, 10, 64, 0.4, 0, "3d", False),
    "3dp_n1000_p10_img2": ("3dp", 1000, 0, 10, 64, 0.4, 2, "3dp", False),
    "3dp_n1500_p8_img3": ("3dp", 1500, 5, 8, 32, 0.4, 3, "3dp", False),
}


def bodies_for(n, seed, kind, cluster):
    xq = drand48_bodies(n, seed, kind=kind)
    if cluster:
        # two tight clumps + background: deep, uneven tree
        m = n // 3
        xq[:m, :3] = xq[:m, :3] * 0.01 + 1.0
        xq[m:2 * m, :3] = xq[m:2 * m, :3] * 0.03 - 2.0
    return xq


def digest(*arrays):
    """sha256 over the raw bytes of the arrays (int32 / float64, C order)."""
    import hashlib

    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def full_size():
    """The 1M-body free-space configuration: too big to store, so the tree and
    the lists are kept as counts + sha256 digests, and the reference FMM and
    direct-sum results on 1000 stride-sampled tree positions."""
    n, P, ncrit, theta = 1 << 20, 10, 64, 0.4
    xq = drand48_bodies(n, 0)
    ref = oracle.Ref("3d", "lazy")
    ref.fmm(xq, P, ncrit, theta, lists_only=True)
    cells = ref.cells()
    lists = ref.lists()
    tree_digest = digest(cells["nchild"], cells["child"], cells["body"], cells["nbody"], cells["xr"])
    list_digest = digest(lists["m2l_off"], lists["m2l_src"], lists["m2l_img"], lists["p2p_off"],
                         lists["p2p_src"], lists["p2p_img"])
    out = ref.fmm(xq, P, ncrit, theta)
    sample = np.arange(0, n, n // 1000)[:1000]
    tgt = out[sample].copy()
    tgt[:, 4:] = 0
    direct = ref.direct(tgt, out)
    np.savez_compressed(
        os.path.join(OUT, "3d_n1048576_p10_sampled.npz"),
        n=n, seed=0, P=P, ncrit=ncrit, theta=theta, ncells=ref.ncells, n_m2l=len(lists["m2l_src"]),
        n_p2p=len(lists["p2p_src"]), tree_digest=tree_digest, list_digest=list_digest, sample=sample,
        fmm=out[sample], direct=direct, times=np.array(list(ref.times().values())))
    print("1M cells", ref.ncells, "m2l", len(lists["m2l_src"]), "p2p", len(lists["p2p_src"]), ref.times())


def main():
    for name, (variant, n, seed, P, ncrit, theta, images, kind, cluster) in CASES.items():
        ref = oracle.Ref(variant, "lazy")
        xq = bodies_for(n, seed, kind, cluster)
        cycle = 2 * np.pi
        out = ref.fmm(xq, P, ncrit, theta, images, cycle if images else 0.0)
        cells = ref.cells()
        lists = ref.lists()
        nterm = P * (P + 1) // 2
        M, L = ref.expansions(nterm)
        extra = {}
        if variant == "3dp":
            ref.dipole_correction()
            extra["bodies_dipole"] = ref.bodies()
            ks = 11
            extra["ewald"] = ref.ewald(ks, ks / cycle, 0.25 / np.pi, cycle / 2)
        np.savez_compressed(
            os.path.join(OUT, name + ".npz"),
            xq=xq, P=P, ncrit=ncrit, theta=theta, images=images, cycle=cycle,
            bodies=out, nchild=cells["nchild"], child=cells["child"], body=cells["body"], nbody=cells["nbody"],
            xr=cells["xr"], M=M, L=L, **lists, **extra)
        print(name, "cells", ref.ncells, "m2l", len(lists["m2l_src"]), "p2p", len(lists["p2p_src"]))
    full_size()
    eager = oracle.Ref("3d", "eager")
    kat = {f"kernel_p{p}": eager.test_kernel(p) for p in (10, 20, 30)}
    kat.update({f"fmm_p{p}": eager.test_fmm(p) for p in (10, 20)})
    np.savez(os.path.join(OUT, "kat.npz"), **kat)
    print(kat)


# 2D (minimal ExaFMM `2d/`, and `2dp/` with images > 0):
# name -> (n, seed, P, ncrit, theta, clustered, images)
CASES_2D = {
    "2d_n2000_p10": (2000, 0, 10, 8, 0.4, False, 0),       # the 2d driver's parameters, small N
    "2d_n5000_p14_nc4_th03": (5000, 2, 14, 4, 0.3, False, 0),
    "2d_clustered_n3000_p8": (3000, 5, 8, 8, 0.4, True, 0),
    "2d_n1": (1, 0, 10, 8, 0.4, False, 0),
    "2d_n8_single_leaf": (8, 0, 10, 8, 0.4, False, 0),     # N = ncrit
    "2d_n9": (9, 0, 10, 8, 0.4, False, 0),                 # N = ncrit + 1
    "2dp_n2000_p10_img3": (2000, 0, 10, 8, 0.4, False, 3),  # the 2dp driver's parameters, small N
    "2dp_n1500_p8_img2": (1500, 6, 8, 16, 0.5, False, 2),
}
CYCLE_2D = 2 * np.pi


def bodies_2d(n, seed, clustered):
    """x, y, q: the 2d driver's generator, or three seeded Gaussian clusters."""
    if not clustered:
        return oracle.reference_bodies_2d(n, seed)
    g = np.random.default_rng(seed)
    xy = g.normal(0.0, 0.05, (n, 2)) + g.choice([-1.5, 0.3, 2.0], (n, 1))
    q = g.uniform(-0.5, 0.5, n)
    return np.c_[xy, q - q.mean()]


def main_2d():
    for name, (n, seed, P, ncrit, theta, clustered, images) in CASES_2D.items():
        ref = oracle.Fmm2D("refp" if images else "ref")
        cycle = CYCLE_2D if images else 0.0
        xyq = bodies_2d(n, seed, clustered)
        ref.fmm(xyq, P, ncrit, theta, images, cycle)
        out = ref.bodies()
        cells = ref.cells()
        lists = ref.lists()
        M, L = ref.expansions()
        # direct sum onto up to 20 stride-sampled bodies (tree order, p = F = 0)
        tgt = out[:: max(1, n // 20)][:20].copy()
        tgt[:, 3:] = 0
        direct = ref.direct(tgt, out, images, cycle)
        np.savez_compressed(os.path.join(OUT, name + ".npz"), xyq=xyq, P=P, ncrit=ncrit, theta=theta, images=images,
                            cycle=cycle, bodies=out, M=M, L=L, direct_targets=tgt, direct=direct, **cells, **lists)
        print(name, "cells", ref.ncells, "m2l", len(lists["m2l_src"]), "p2p", len(lists["p2p_src"]))


if __name__ == "__main__":
    # `make_golden.py 2d` writes the 2D fixtures only
    main_2d() if sys.argv[1:] == ["2d"] else main()
