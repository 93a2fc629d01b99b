/* TEST INFRASTRUCTURE: the entry points of include/exafmm_b200.h that the
 * C++ driver shim (include/exafmm_b200.hpp) calls, implemented on the CPU
 * oracle (oracle/fmm_oracle.h) instead of the GPU.  tests/test_shim.py links
 * the reference's own drivers (3d/fmm.cxx, test/test_fmm.h) through the shim
 * against this library to check the shim's host logic -- body permutation,
 * cell wiring, accumulation of p and F, direct sums on a second handle --
 * on a machine without a GPU.  The product never links it.
 *
 * The oracle keeps one problem in global state; every call that reads it
 * first makes sure it holds this handle's problem. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "exafmm_b200.h"
#include "fmm_oracle.h"

struct exafmm_b200 {
  exafmm_params prm;
  long n;
  double *xq;      /* x, y, z, q per body, input order */
  long ncells;
  int tree, done;  /* tree built; evaluation done */
  char err[256];
};

static const exafmm_b200 *owner; /* whose problem the oracle holds */
static int owner_done;           /* ... evaluated (not just a tree) */

static int fail(exafmm_b200 *h, int code, const char *msg) {
  if (h) snprintf(h->err, sizeof h->err, "%s", msg);
  return code;
}

static void hold(exafmm_b200 *h, int evaluated) {
  if (owner == h && (owner_done || !evaluated)) return;
  if (evaluated)
    orc_fmm(h->n, h->xq, h->prm.P, h->prm.ncrit, h->prm.theta, h->prm.images, h->prm.cycle);
  else
    orc_tree(h->n, h->xq, h->prm.ncrit);
  owner = h;
  owner_done = evaluated;
}

int exafmm_b200_create(const exafmm_params *p, exafmm_b200 **out) {
  if (!p || !out) return EXAFMM_ERR_ARG;
  exafmm_b200 *h = (exafmm_b200 *)calloc(1, sizeof *h);
  h->prm = *p;
  *out = h;
  return EXAFMM_OK;
}

int exafmm_b200_destroy(exafmm_b200 *h) {
  if (!h) return EXAFMM_ERR_ARG;
  if (owner == h) owner = NULL;
  free(h->xq);
  free(h);
  return EXAFMM_OK;
}

const char *exafmm_b200_last_error(const exafmm_b200 *h) { return h ? h->err : "no handle"; }

int exafmm_b200_set_params(exafmm_b200 *h, const exafmm_params *p) {
  h->prm = *p;
  h->tree = h->done = 0;
  if (owner == h) owner = NULL;
  return EXAFMM_OK;
}

int exafmm_b200_set_bodies(exafmm_b200 *h, const double *rec, int64_t n, int where) {
  if (where != EXAFMM_HOST || !rec || n <= 0) return fail(h, EXAFMM_ERR_ARG, "host bodies, n > 0");
  free(h->xq);
  h->xq = (double *)malloc(sizeof(double) * 4 * n);
  for (int64_t i = 0; i < n; i++) memcpy(h->xq + 4 * i, rec + 8 * i, 4 * sizeof(double));
  h->n = n;
  h->tree = h->done = 0;
  if (owner == h) owner = NULL;
  return EXAFMM_OK;
}

int exafmm_b200_build_tree(exafmm_b200 *h) {
  if (h->n <= 0) return fail(h, EXAFMM_ERR_STATE, "no bodies");
  h->ncells = orc_tree(h->n, h->xq, h->prm.ncrit);
  owner = h;
  owner_done = 0;
  h->tree = 1;
  h->done = 0;
  return EXAFMM_OK;
}

int64_t exafmm_b200_num_cells(exafmm_b200 *h) { return h && h->tree ? h->ncells : -1; }

int exafmm_b200_get_perm(exafmm_b200 *h, int64_t *perm, int where) {
  if (!h->tree || where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_STATE, "no tree");
  hold(h, 0);
  long *p = (long *)malloc(sizeof(long) * h->n);
  orc_get_perm(p);
  for (long i = 0; i < h->n; i++) perm[i] = p[i];
  free(p);
  return EXAFMM_OK;
}

int exafmm_b200_get_tree(exafmm_b200 *h, int *nchild, int *child, int *body, int *nbody, int *level, double *xr) {
  if (!h->tree) return fail(h, EXAFMM_ERR_STATE, "no tree");
  hold(h, 0);
  orc_get_cells(nchild, child, body, nbody, level, xr);
  return EXAFMM_OK;
}

/* the oracle evaluates in one call: the passes only check their order */
int exafmm_b200_upward(exafmm_b200 *h) { return h->tree ? EXAFMM_OK : fail(h, EXAFMM_ERR_STATE, "no tree"); }
int exafmm_b200_horizontal(exafmm_b200 *h) { return h->tree ? EXAFMM_OK : fail(h, EXAFMM_ERR_STATE, "no tree"); }

int exafmm_b200_downward(exafmm_b200 *h) {
  if (!h->tree) return fail(h, EXAFMM_ERR_STATE, "no tree");
  hold(h, 1);
  h->done = 1;
  return EXAFMM_OK;
}

int exafmm_b200_get_bodies(exafmm_b200 *h, double *rec, int where) {
  if (!h->done || where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_STATE, "no completed evaluation");
  hold(h, 1);
  orc_get_bodies(rec);
  return EXAFMM_OK;
}

int exafmm_b200_get_expansions(exafmm_b200 *h, double *M, double *L) {
  if (!h->done) return fail(h, EXAFMM_ERR_STATE, "no completed evaluation");
  hold(h, 1);
  orc_get_expansions(M, L);
  return EXAFMM_OK;
}

int exafmm_b200_direct(exafmm_b200 *h, double *targets8, int64_t nt, int where) {
  if (!h->tree || where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_STATE, "no tree");
  double *src = (double *)calloc(8 * h->n, sizeof(double));
  for (long i = 0; i < h->n; i++) memcpy(src + 8 * i, h->xq + 4 * i, 4 * sizeof(double));
  orc_direct(nt, targets8, h->n, src, h->prm.images, h->prm.cycle);
  free(src);
  return EXAFMM_OK;
}

/* Single operators on the oracle's restated operators (host arrays only). */
/* The shift iX * cycle of a periodic call back to the oracle's (iX, cycle),
 * with the handle's cycle. */
static const int *ix_of(const exafmm_b200 *h, const double *shift3, int ix[3], double *cycle) {
  *cycle = h->prm.cycle;
  if (!shift3 || !(h->prm.cycle > 0)) return NULL;
  for (int d = 0; d < 3; d++) ix[d] = (int)lround(shift3[d] / h->prm.cycle);
  return ix;
}

int exafmm_b200_p2p(exafmm_b200 *h, double *t8, int64_t nt, const double *s8, int64_t ns, const double *shift3,
                    int where) {
  if (where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_ARG, "host arrays only");
  int ix[3];
  double cyc = 0;
  const int *pix = ix_of(h, shift3, ix, &cyc);
  owner = NULL;
  orc_op_p2p(t8, nt, s8, ns, pix, cyc);
  return EXAFMM_OK;
}

int exafmm_b200_p2m(exafmm_b200 *h, const double *cell4, const double *b8, int64_t nb, double *M, int where) {
  if (where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_ARG, "host arrays only");
  owner = NULL;
  orc_op_p2m(h->prm.P, cell4, b8, nb, M);
  return EXAFMM_OK;
}

int exafmm_b200_m2m(exafmm_b200 *h, const double *parent4, double *M, int nchild, const double *child4,
                    const double *Mchild, int where) {
  if (where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_ARG, "host arrays only");
  owner = NULL;
  orc_op_m2m(h->prm.P, parent4, M, nchild, child4, Mchild);
  return EXAFMM_OK;
}

int exafmm_b200_m2l(exafmm_b200 *h, const double *t4, double *L, const double *s4, const double *M,
                    const double *shift3, int where) {
  if (where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_ARG, "host arrays only");
  int ix[3];
  double cyc = 0;
  const int *pix = ix_of(h, shift3, ix, &cyc);
  owner = NULL;
  orc_op_m2l(h->prm.P, t4, L, s4, M, pix, cyc);
  return EXAFMM_OK;
}

int exafmm_b200_l2l(exafmm_b200 *h, const double *parent4, const double *L, int nchild, const double *child4,
                    double *Lchild, int where) {
  if (where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_ARG, "host arrays only");
  owner = NULL;
  orc_op_l2l(h->prm.P, parent4, L, nchild, child4, Lchild);
  return EXAFMM_OK;
}

int exafmm_b200_l2p(exafmm_b200 *h, const double *cell4, const double *L, double *b8, int64_t nb, int where) {
  if (where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_ARG, "host arrays only");
  owner = NULL;
  orc_op_l2p(h->prm.P, cell4, L, b8, nb);
  return EXAFMM_OK;
}

/* Ewald parts of the handle's bodies onto targets.  The oracle evaluates its
 * bodies onto themselves, so the stand-in takes targets that are the
 * handle's bodies in tree order (the periodic driver's case: the same bodies,
 * tree-sorted twice); the self term alone takes any targets. */
int exafmm_b200_ewald_parts(exafmm_b200 *h, int parts, int ksize, double alpha, double sigma, double cutoff,
                            double *t8, int64_t nt, int where) {
  if (where != EXAFMM_HOST) return fail(h, EXAFMM_ERR_ARG, "host arrays only");
  if (parts == EXAFMM_EWALD_SELF) {
    for (int64_t i = 0; i < nt; i++) t8[8 * i + 4] -= M_2_SQRTPI * t8[8 * i + 3] * alpha;
    return EXAFMM_OK;
  }
  if (!h->tree) return fail(h, EXAFMM_ERR_STATE, "no tree");
  hold(h, 0);
  if (nt != h->n) return fail(h, EXAFMM_ERR_ARG, "stand-in: targets must be the handle's bodies");
  double *out = (double *)calloc(8 * nt, sizeof(double));
  orc_ewald_parts(parts, ksize, alpha, sigma, cutoff, h->prm.cycle, out);
  for (int64_t i = 0; i < nt; i++) {
    for (int d = 0; d < 4; d++)
      if (out[8 * i + d] != t8[8 * i + d]) {
        free(out);
        return fail(h, EXAFMM_ERR_ARG, "stand-in: targets must be the handle's bodies in tree order");
      }
    for (int d = 4; d < 8; d++) t8[8 * i + d] += out[8 * i + d];
  }
  free(out);
  return EXAFMM_OK;
}
