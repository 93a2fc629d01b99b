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
