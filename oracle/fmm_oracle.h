/* Oracle: a plain-C CPU restatement of minimal ExaFMM's 3D Laplace FMM
 * (`3d/` free space and `3dp/` periodic variants).  TEST INFRASTRUCTURE ONLY:
 * tests/, __graft_entry__.smoke() and bench.py's CPU legs use it as the
 * checker; the product library never links or calls it.
 *
 * Pinned against the reference itself: tests/test_oracle.py compares it with
 * the reference headers compiled by oracle/Makefile (oracle/_ref) and with the
 * reference's own known answers (test/test_kernel.cxx:5-7,
 * test/test_fmm.cxx:5-6) and the committed golden fixtures in tests/golden/.
 *
 * The state is global (one problem at a time), as in the reference.  All
 * arrays in/out are caller-owned.  Cells are reported in the reference's cell
 * order (3d/build_tree.h:69-84: children appended as one block when the
 * parent is visited, depth first).  Bodies are reported in tree order.
 */
#ifndef FMM_ORACLE_H
#define FMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Build the adaptive octree of n bodies (xq: x,y,z,q per body) with leaves of
 * at most ncrit bodies.  Returns the number of cells. */
long orc_tree(long n, const double *xq, int ncrit);

/* Dual-tree interaction lists on the current tree (theta; images>0 adds the
 * 27 first-shell periodic shifts of period cycle).  Returns M2L + P2P count. */
long orc_lists(double theta, int images, double cycle);

/* Full evaluation: tree, upward, lists + M2L/P2P, (3dp: periodic root images),
 * downward.  Returns the number of cells. */
long orc_fmm(long n, const double *xq, int P, int ncrit, double theta, int images, double cycle);

void orc_get_bodies(double *out8);     /* X[3], q, p, F[3] per body, tree order */
void orc_get_perm(long *perm);         /* tree position -> input index */
void orc_get_cells(int *nchild, int *child, int *body, int *nbody, int *level, double *xr);
void orc_count_lists(long *nm2l, long *np2p);
void orc_get_lists(int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src, int *p2p_img);
void orc_get_expansions(double *M, double *L); /* NTERM complex per cell, interleaved */

/* Direct summation of sources onto targets (8 doubles per body, accumulates
 * p and F), summed over the (2*prange+1)^3 periodic images when images>0. */
void orc_direct(long nt, double *targets8, long ns, const double *sources8, int images, double cycle);

/* 3dp dipole correction of the current bodies (3dp/fmm.cxx:63-75). */
void orc_dipole_correction(double cycle);

/* Ewald sum of the current bodies (wave + real + self parts), written as
 * 8 doubles per body in tree order. */
void orc_ewald(int ksize, double alpha, double sigma, double cutoff, double cycle, double *out8);
/* ... only the parts in the mask: 1 wave, 2 real, 4 self (orc_ewald = 7). */
void orc_ewald_parts(int parts, int ksize, double alpha, double sigma, double cutoff, double cycle, double *out8);

/* Operator chain known-answer test (test/test_kernel.h): relative potential
 * error, force error through *ferr. */
double orc_kernel_chain(int P, double *ferr);

/* Single operators on caller data, the reference's kernel functions one call
 * at a time (3d/kernel.h:122-323).  Each replaces the oracle's current
 * problem.  Cells are centre + radius (4 doubles), expansions NTERM complex
 * values (re, im interleaved), bodies Body records; outputs accumulate, as
 * the reference's += does.  ix (3 ints, or NULL) and cycle give the 3dp
 * periodic shift iX * cycle of P2P and M2L (3dp/kernel.h:133,200). */
void orc_op_p2m(int P, const double *cell4, const double *bodies8, long nb, double *M);
void orc_op_m2m(int P, const double *parent4, double *M, int nchild, const double *child4, const double *Mchild);
void orc_op_m2l(int P, const double *target4, double *L, const double *source4, const double *M, const int *ix,
                double cycle);
void orc_op_l2l(int P, const double *parent4, const double *L, int nchild, const double *child4, double *Lchild);
void orc_op_l2p(int P, const double *cell4, const double *L, double *bodies8, long nb);
void orc_op_p2p(double *targets8, long nt, const double *sources8, long ns, const int *ix, double cycle);

/* n bodies as the reference drivers make them: srand48(seed); per body
 * x,y,z from drand48() and q = drand48()-0.5, then q -= mean.  kind 0 is the
 * 3d driver's cube (3d/fmm.cxx:19-35: d*2*M_PI - M_PI), kind 1 the 3dp
 * driver's (3dp/fmm.cxx:30-44: d*cycle - cycle*.5). */
void orc_reference_bodies(long n, long seed, int kind, double cycle, double *xq);

#ifdef __cplusplus
}
#endif
#endif
