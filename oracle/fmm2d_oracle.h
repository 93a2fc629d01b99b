/* Oracle, 2D: a plain-C CPU restatement of minimal ExaFMM's 2D Laplace FMM
 * (`2d/` free space and `2dp/` periodic: quadtree, logarithmic potential,
 * complex power-series expansions of P terms).  TEST INFRASTRUCTURE ONLY: tests/ use it as the checker; the
 * product library never links or calls it.
 *
 * Pinned against the reference itself: tests/test_oracle2d.py compares it
 * with the reference's 2d headers compiled by oracle/Makefile
 * (oracle/_ref/libref2d_lazy.so) and with the committed fixtures
 * tests/golden/2d_*.npz made from that build.
 *
 * Bodies cross as 6 doubles: X[2], q, p, F[2] (2d/exafmm.h:13-18); input
 * bodies as x, y, q.  One problem at a time (global state), as in the
 * reference.  Cells are reported in the reference's order (children appended
 * as one block when the parent is split, depth first: 2d/build_tree.h:23-86).
 */
#ifndef FMM2D_ORACLE_H
#define FMM2D_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif
/* Quadtree of n bodies (xyq: x, y, q per body), leaves of at most ncrit
 * bodies.  Returns the number of cells. */
long orc2_tree(long n, const double *xyq, int ncrit);
/* Full evaluation: tree, upward pass, lists, M2L + P2P, (images > 0: the
 * 9 first-shell image walks and the far images at the root, period cycle),
 * downward pass.  Returns the number of cells. */
long orc2_fmm(long n, const double *xyq, int P, int ncrit, double theta, int images, double cycle);
void orc2_get_bodies(double *out6); /* tree order */
void orc2_get_cells(int *nchild, int *child, int *body, int *nbody, double *xr); /* xr: x, y, R */
void orc2_count_lists(long *nm2l, long *np2p);
/* per entry its source cell and image periodic1D(iX) = iX0 + 1 + 3 (iX1 + 1) (4 in free space) */
void orc2_get_lists(int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src, int *p2p_img);
void orc2_get_expansions(double *M, double *L); /* P complex per cell, interleaved */
/* Direct summation of sources onto targets (6 doubles per body; p and F
 * accumulate), the reference's direct() (2d/traverse_lazy.h:84-94), over the
 * periodic images when images > 0 (2dp/traverse_lazy.h:154-175). */
void orc2_direct(long nt, double *targets6, long ns, const double *sources6, int images, double cycle);
/* n bodies as 2d/fmm.cxx:21-35 makes them: srand48(seed); per body x, y from
 * drand48() * 2 pi - pi, q = drand48() - 0.5; then q -= mean. */
void orc2_reference_bodies(long n, long seed, double *xyq);
#ifdef __cplusplus
}
#endif
#endif
