/* Oracle: plain-C CPU restatement of minimal ExaFMM's 3D Laplace FMM.
 * TEST INFRASTRUCTURE ONLY (see fmm_oracle.h).  Every function names the
 * reference lines it restates; paths are relative to the reference project.
 *
 * Layout (own design, not the reference's): bodies are SoA arrays in tree
 * order plus a permutation back to input order; cells are SoA arrays indexed
 * in the reference's cell order; expansions are flat complex arrays
 * [cell][NTERM]; interaction lists are CSR per target cell.
 *
 * Compiled with -ffp-contract=off so that every product and sum rounds as in
 * the reference's x86-64 build (no fused multiply-add).
 */
#define _GNU_SOURCE
#include "fmm_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ------------------------------------------------------------------ state */
static int P_ = 10, NTERM_ = 55, NCRIT_ = 64, IMAGES_ = 0;
static double THETA_ = 0.4, CYCLE_ = 0.0;

static long nb_ = 0;
static double *bx_, *by_, *bz_, *bq_, *bp_, *bf_[3];
static long *perm_;

static long nc_ = 0, cap_ = 0;
static int *nchild_, *child_, *body_, *nbody_, *level_;
static double *cx_, *cy_, *cz_, *cr_;
static double R0_, X0_[3];

static cplx *M_, *L_;

typedef struct { int tgt, src, img; } entry;
static entry *m2l_, *p2p_;
static long nm2l_, np2p_, capm_, capp_;
static int *m2l_off_, *p2p_off_; /* CSR after orc_lists */
static entry *m2l_csr_, *p2p_csr_;

static void *grow(void *p, long *cap, long need, size_t elem) {
  if (need <= *cap) return p;
  long c = *cap ? *cap : 1024;
  while (c < need) c *= 2;
  *cap = c;
  return realloc(p, (size_t)c * elem);
}

/* ------------------------------------------------------------------- tree */

/* Bounding cube: 3d/build_tree.h:7-21 (getBounds). */
static void bounds(void) {
  double lo[3] = {bx_[0], by_[0], bz_[0]}, hi[3] = {bx_[0], by_[0], bz_[0]};
  for (long b = 0; b < nb_; b++) {
    const double x[3] = {bx_[b], by_[b], bz_[b]};
    for (int d = 0; d < 3; d++) lo[d] = fmin(x[d], lo[d]);
    for (int d = 0; d < 3; d++) hi[d] = fmax(x[d], hi[d]);
  }
  for (int d = 0; d < 3; d++) X0_[d] = (hi[d] + lo[d]) / 2;
  R0_ = 0;
  for (int d = 0; d < 3; d++) {
    R0_ = fmax(X0_[d] - lo[d], R0_);
    R0_ = fmax(hi[d] - X0_[d], R0_);
  }
  R0_ *= 1.00001;
}

static long new_cells(int k) {
  long first = nc_;
  nc_ += k;
  if (nc_ > cap_) {
    long c = cap_ ? cap_ : 1024;
    while (c < nc_) c *= 2;
    nchild_ = realloc(nchild_, c * sizeof(int));
    child_ = realloc(child_, c * sizeof(int));
    body_ = realloc(body_, c * sizeof(int));
    nbody_ = realloc(nbody_, c * sizeof(int));
    level_ = realloc(level_, c * sizeof(int));
    cx_ = realloc(cx_, c * sizeof(double));
    cy_ = realloc(cy_, c * sizeof(double));
    cz_ = realloc(cz_, c * sizeof(double));
    cr_ = realloc(cr_, c * sizeof(double));
    cap_ = c;
  }
  return first;
}

static long *ord_, *tmp_;

/* Recursive top-down octree: 3d/build_tree.h:24-86 (buildCells).  Bodies are
 * tracked as an index permutation (ord_) instead of ping-ponged copies; the
 * per-cell stable counting sort by octant (:44-67) gives the same order.  A
 * cell's children are appended as one block when the cell is visited
 * (:70-72), then visited in octant order, so cell indices match the
 * reference's. */
static void split(long cell, long begin, long end, const double X[3], int level) {
  body_[cell] = (int)begin;
  nbody_[cell] = (int)(end - begin);
  nchild_[cell] = 0;
  child_[cell] = -1;
  level_[cell] = level;
  cx_[cell] = X[0];
  cy_[cell] = X[1];
  cz_[cell] = X[2];
  cr_[cell] = R0_ / (1 << level);
  if (end - begin <= NCRIT_) return;
  long count[8] = {0}, start[8], fill[8];
  for (long i = begin; i < end; i++) {
    long b = ord_[i];
    int oct = (bx_[b] > X[0]) + ((by_[b] > X[1]) << 1) + ((bz_[b] > X[2]) << 2);
    count[oct]++;
  }
  long off = begin;
  int kids = 0;
  for (int o = 0; o < 8; o++) {
    start[o] = off;
    off += count[o];
    if (count[o]) kids++;
  }
  memcpy(fill, start, sizeof(fill));
  for (long i = begin; i < end; i++) {
    long b = ord_[i];
    int oct = (bx_[b] > X[0]) + ((by_[b] > X[1]) << 1) + ((bz_[b] > X[2]) << 2);
    tmp_[fill[oct]++] = b;
  }
  memcpy(ord_ + begin, tmp_ + begin, (end - begin) * sizeof(long));
  long first = new_cells(kids);
  nchild_[cell] = kids;
  child_[cell] = (int)first;
  double r = R0_ / (1 << (level + 1));
  int c = 0;
  for (int o = 0; o < 8; o++) {
    double Xc[3];
    for (int d = 0; d < 3; d++) Xc[d] = X[d] + r * (double)((((o >> d) & 1) * 2) - 1);
    if (count[o]) split(first + c++, start[o], start[o] + count[o], Xc, level + 1);
  }
}

static void free_bodies(void) {
  free(bx_); free(by_); free(bz_); free(bq_); free(bp_);
  for (int d = 0; d < 3; d++) free(bf_[d]);
  free(perm_);
}

/* 3d/build_tree.h:88-96 (buildTree): bounds, then the recursive split. */
long orc_tree(long n, const double *xq, int ncrit) {
  free_bodies();
  nb_ = n;
  NCRIT_ = ncrit;
  bx_ = malloc(n * sizeof(double)); by_ = malloc(n * sizeof(double));
  bz_ = malloc(n * sizeof(double)); bq_ = malloc(n * sizeof(double));
  bp_ = calloc(n, sizeof(double));
  for (int d = 0; d < 3; d++) bf_[d] = calloc(n, sizeof(double));
  perm_ = malloc(n * sizeof(long));
  for (long b = 0; b < n; b++) {
    bx_[b] = xq[4 * b]; by_[b] = xq[4 * b + 1]; bz_[b] = xq[4 * b + 2]; bq_[b] = xq[4 * b + 3];
  }
  bounds();
  ord_ = malloc(n * sizeof(long));
  tmp_ = malloc(n * sizeof(long));
  for (long b = 0; b < n; b++) ord_[b] = b;
  nc_ = 0;
  new_cells(1);
  split(0, 0, n, X0_, 0);
  /* apply the permutation: bodies now in tree order */
  double *t[4] = {malloc(n * sizeof(double)), malloc(n * sizeof(double)), malloc(n * sizeof(double)),
                  malloc(n * sizeof(double))};
  for (long i = 0; i < n; i++) {
    long b = ord_[i];
    t[0][i] = bx_[b]; t[1][i] = by_[b]; t[2][i] = bz_[b]; t[3][i] = bq_[b];
    perm_[i] = b;
  }
  free(bx_); free(by_); free(bz_); free(bq_);
  bx_ = t[0]; by_ = t[1]; bz_ = t[2]; bq_ = t[3];
  free(ord_); free(tmp_);
  return nc_;
}

/* ------------------------------------------------------------------ lists */

static void push(entry **arr, long *n, long *cap, int t, int s, int img) {
  *arr = grow(*arr, cap, *n + 1, sizeof(entry));
  (*arr)[*n].tgt = t;
  (*arr)[*n].src = s;
  (*arr)[*n].img = img;
  (*n)++;
}

/* Dual-tree walk recording lists: 3d/traverse_lazy.h:27-44 (getList), with
 * the periodic shift of 3dp/traverse_lazy.h:39-58 (img = periodic1D,
 * 3dp/traverse_lazy.h:27-30). */
static void walk(int i, int j, const int ix[3], int img) {
  double dx = (cx_[i] - cx_[j]) - ix[0] * CYCLE_;
  double dy = (cy_[i] - cy_[j]) - ix[1] * CYCLE_;
  double dz = (cz_[i] - cz_[j]) - ix[2] * CYCLE_;
  double R2 = (dx * dx + dy * dy + dz * dz) * THETA_ * THETA_;
  double Rs = cr_[i] + cr_[j];
  if (R2 > Rs * Rs) {
    push(&m2l_, &nm2l_, &capm_, i, j, img);
  } else if (nchild_[i] == 0 && nchild_[j] == 0) {
    push(&p2p_, &np2p_, &capp_, i, j, img);
  } else if (nchild_[j] == 0 || (cr_[i] >= cr_[j] && nchild_[i] != 0)) {
    for (int c = child_[i]; c < child_[i] + nchild_[i]; c++) walk(c, j, ix, img);
  } else {
    for (int c = child_[j]; c < child_[j] + nchild_[j]; c++) walk(i, c, ix, img);
  }
}

/* Stable bucket by target: per-target order = recording order. */
static void to_csr(const entry *e, long n, int **off, entry **csr) {
  free(*off);
  free(*csr);
  *off = calloc(nc_ + 1, sizeof(int));
  *csr = malloc((n ? n : 1) * sizeof(entry));
  for (long k = 0; k < n; k++) (*off)[e[k].tgt + 1]++;
  for (long c = 0; c < nc_; c++) (*off)[c + 1] += (*off)[c];
  int *fill = malloc((nc_ + 1) * sizeof(int));
  memcpy(fill, *off, (nc_ + 1) * sizeof(int));
  for (long k = 0; k < n; k++) (*csr)[fill[e[k].tgt]++] = e[k];
  free(fill);
}

/* 3dp/traverse_lazy.h:124-141 (horizontalPass list part): with images, one
 * walk per first-shell shift, x outermost. */
long orc_lists(double theta, int images, double cycle) {
  THETA_ = theta;
  IMAGES_ = images;
  CYCLE_ = cycle;
  nm2l_ = np2p_ = 0;
  if (images == 0) {
    int ix[3] = {0, 0, 0};
    walk(0, 0, ix, 13);
  } else {
    int ix[3];
    for (ix[0] = -1; ix[0] <= 1; ix[0]++)
      for (ix[1] = -1; ix[1] <= 1; ix[1]++)
        for (ix[2] = -1; ix[2] <= 1; ix[2]++)
          walk(0, 0, ix, (ix[0] + 1) + 3 * (ix[1] + 1) + 9 * (ix[2] + 1));
  }
  to_csr(m2l_, nm2l_, &m2l_off_, &m2l_csr_);
  to_csr(p2p_, np2p_, &p2p_off_, &p2p_csr_);
  return nm2l_ + np2p_;
}

static void img3(int img, int ix[3]) {
  /* 3dp/traverse_lazy.h:33-37 (periodic3D) */
  ix[0] = (img % 3) - 1;
  ix[1] = ((img / 3) % 3) - 1;
  ix[2] = (img / 9) - 1;
}

/* --------------------------------------------------------------- kernels */

static int sgn(int n) { return (n & 1) ? -1 : 1; }         /* 3d/kernel.h:14-16 */
static int sgn2n(int n) { return n >= 0 ? 1 : sgn(n); }     /* 3d/kernel.h:19-21 */

/* 3d/kernel.h:24-28 (cart2sph) */
static void to_sph(const double d[3], double *r, double *th, double *ph) {
  *r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  *th = *r == 0 ? 0 : acos(d[2] / *r);
  *ph = atan2(d[1], d[0]);
}

/* 3d/kernel.h:31-40 (sph2cart) */
static void to_cart(double r, double th, double ph, const double s[3], double c[3]) {
  c[0] = sin(th) * cos(ph) * s[0] + cos(th) * cos(ph) / r * s[1] - sin(ph) / r / sin(th) * s[2];
  c[1] = sin(th) * sin(ph) * s[0] + cos(th) * sin(ph) / r * s[1] + cos(ph) / r / sin(th) * s[2];
  c[2] = cos(th) * s[0] - sin(th) / r * s[1];
}

/* Regular solid harmonics rho^n Y_n^m and their theta derivative, by the
 * associated-Legendre recurrences of 3d/kernel.h:43-81 (evalMultipole).
 * Y and dY hold P*P entries indexed n*n+n+m, m in [-n,n]. */
static void regular(double rho, double al, double be, cplx *Y, cplx *dY) {
  const double c = cos(al), s = sin(al), is = s == 0 ? 0 : 1 / s;
  double odd = 1, pmm = 1, rm = 1;
  const cplx e1 = CMPLX(cos(be), sin(be));
  cplx em = 1;
  for (int m = 0; m < P_; m++) {
    double p = pmm;
    const int kp = m * m + 2 * m, kn = m * m;
    Y[kp] = rm * p * em;
    Y[kn] = conj(Y[kp]);
    double p1 = p;
    p = c * (2 * m + 1) * p1;
    dY[kp] = rm * (p - (m + 1) * c * p1) * is * em;
    rm *= rho;
    double rn = rm;
    for (int n = m + 1; n < P_; n++) {
      const int np = n * n + n + m, nn = n * n + n - m;
      rn /= -(n + m);
      Y[np] = rn * p * em;
      Y[nn] = conj(Y[np]);
      const double p2 = p1;
      p1 = p;
      p = (c * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      dY[np] = rn * ((n - m + 1) * p - (n + 1) * c * p1) * is * em;
      rn *= rho;
    }
    rm /= -(2 * m + 2) * (2 * m + 1);
    pmm = -pmm * odd * s;
    odd += 2;
    em *= e1;
  }
}

/* Irregular solid harmonics rho^(-n-1) Y_n^m, 3d/kernel.h:83-116
 * (evalLocal).  As in the reference only degrees n < P are formed; the
 * caller's array (4P^2 entries) is zeroed so the higher degrees read as 0,
 * which truncates M2L to j+n < P exactly as the reference does. */
static void irregular(double rho, double al, double be, cplx *Y) {
  const double c = cos(al), s = sin(al);
  double odd = 1, pmm = 1;
  const double inv = -1.0 / rho;
  double rm = -inv;
  const cplx e1 = CMPLX(cos(be), sin(be));
  cplx em = 1;
  for (int m = 0; m < P_; m++) {
    double p = pmm;
    const int kp = m * m + 2 * m, kn = m * m;
    Y[kp] = rm * p * em;
    Y[kn] = conj(Y[kp]);
    double p1 = p;
    p = c * (2 * m + 1) * p1;
    rm *= inv;
    double rn = rm;
    for (int n = m + 1; n < P_; n++) {
      const int np = n * n + n + m, nn = n * n + n - m;
      Y[np] = rn * p * em;
      Y[nn] = conj(Y[np]);
      const double p2 = p1;
      p1 = p;
      p = (c * (2 * n + 1) * p1 - (n + m) * p2) / (n - m + 1);
      rn *= inv * (n - m + 1);
    }
    pmm = -pmm * odd * s;
    odd += 2;
    em *= e1;
  }
}

/* Near field between two body ranges: 3d/kernel.h:122-150 (P2P), periodic
 * shift from 3dp/kernel.h:133. */
static void p2p(long ib, long ni, long jb, long nj, const int ix[3]) {
  for (long i = ib; i < ib + ni; i++) {
    double pot = 0, ax = 0, ay = 0, az = 0;
    for (long j = jb; j < jb + nj; j++) {
      double d[3] = {bx_[i] - bx_[j] - ix[0] * CYCLE_, by_[i] - by_[j] - ix[1] * CYCLE_,
                     bz_[i] - bz_[j] - ix[2] * CYCLE_};
      double R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (R2 != 0) {
        double i2 = 1.0 / R2;
        double iR = bq_[j] * sqrt(i2);
        for (int k = 0; k < 3; k++) d[k] *= i2 * iR;
        pot += iR;
        ax += d[0];
        ay += d[1];
        az += d[2];
      }
    }
    bp_[i] += pot;
    bf_[0][i] -= ax;
    bf_[1][i] -= ay;
    bf_[2][i] -= az;
  }
}

/* 3d/kernel.h:187-202 (P2M): bodies of a leaf into its multipole. */
static void p2m(int c, cplx *Y, cplx *dY) {
  for (long b = body_[c]; b < body_[c] + nbody_[c]; b++) {
    double d[3] = {bx_[b] - cx_[c], by_[b] - cy_[c], bz_[b] - cz_[c]}, r, a, be;
    to_sph(d, &r, &a, &be);
    regular(r, a, -be, Y, dY);
    for (int n = 0; n < P_; n++)
      for (int m = 0; m <= n; m++) M_[(long)c * NTERM_ + n * (n + 1) / 2 + m] += bq_[b] * Y[n * n + n + m];
  }
}

/* 3d/kernel.h:204-231 (M2M): children multipoles shifted to the parent.
 * Generic over (parent centre, child list) so the 3dp periodic super-cell
 * (26 image copies) can use it too. */
static void m2m_into(const double X[3], cplx *Mp, int nkid, const double (*kx)[3], cplx *const *Mk, cplx *Y,
                     cplx *dY) {
  for (int k = 0; k < nkid; k++) {
    double d[3] = {X[0] - kx[k][0], X[1] - kx[k][1], X[2] - kx[k][2]}, r, a, be;
    to_sph(d, &r, &a, &be);
    regular(r, a, be, Y, dY);
    for (int j = 0; j < P_; j++) {
      for (int q = 0; q <= j; q++) {
        cplx acc = 0;
        for (int n = 0; n <= j; n++) {
          int lo = -n > -j + q + n ? -n : -j + q + n, hi = q - 1 < n ? q - 1 : n;
          for (int m = lo; m <= hi; m++) {
            int src = (j - n) * (j - n + 1) / 2 + q - m;
            acc += Mk[k][src] * Y[n * n + n - m] * (double)(sgn2n(m) * sgn(n));
          }
          hi = n < j + q - n ? n : j + q - n;
          for (int m = q; m <= hi; m++) {
            int src = (j - n) * (j - n + 1) / 2 - q + m;
            acc += conj(Mk[k][src]) * Y[n * n + n - m] * (double)sgn(q + n + m);
          }
        }
        Mp[j * (j + 1) / 2 + q] += acc;
      }
    }
  }
}

/* 3d/kernel.h:233-260 (M2L), periodic shift from 3dp/kernel.h:200.  Target
 * centre Xi, source centre Xj, source multipole Mj, into Li. */
static void m2l_into(const double Xi[3], const double Xj[3], const cplx *Mj, cplx *Li, const int ix[3], double cyc,
                     cplx *Y2) {
  double d[3], r, a, be;
  for (int k = 0; k < 3; k++) d[k] = Xi[k] - Xj[k] - ix[k] * cyc;
  to_sph(d, &r, &a, &be);
  memset(Y2, 0, 4 * P_ * P_ * sizeof(cplx));
  irregular(r, a, be, Y2);
  for (int j = 0; j < P_; j++) {
    const double Cj = sgn(j);
    for (int q = 0; q <= j; q++) {
      cplx acc = 0;
      for (int n = 0; n < P_; n++) {
        for (int m = -n; m < 0; m++) {
          int deg = j + n;
          acc += conj(Mj[n * (n + 1) / 2 - m]) * Cj * Y2[deg * deg + deg + m - q];
        }
        for (int m = 0; m <= n; m++) {
          int deg = j + n;
          double C2 = Cj * sgn((q - m) * (q < m) + m);
          acc += Mj[n * (n + 1) / 2 + m] * C2 * Y2[deg * deg + deg + m - q];
        }
      }
      Li[j * (j + 1) / 2 + q] += acc;
    }
  }
}

/* 3d/kernel.h:262-291 (L2L): parent local pushed to each child. */
static void l2l(int c, cplx *Y, cplx *dY) {
  for (int k = child_[c]; k < child_[c] + nchild_[c]; k++) {
    double d[3] = {cx_[k] - cx_[c], cy_[k] - cy_[c], cz_[k] - cz_[c]}, r, a, be;
    to_sph(d, &r, &a, &be);
    regular(r, a, be, Y, dY);
    const cplx *Lp = L_ + (long)c * NTERM_;
    for (int j = 0; j < P_; j++) {
      for (int q = 0; q <= j; q++) {
        cplx acc = 0;
        for (int n = j; n < P_; n++) {
          for (int m = j + q - n; m < 0; m++) {
            int y = (n - j) * (n - j) + n - j + m - q;
            acc += conj(Lp[n * (n + 1) / 2 - m]) * Y[y] * (double)sgn(q);
          }
          for (int m = 0; m <= n; m++) {
            if (n - j >= abs(m - q)) {
              int y = (n - j) * (n - j) + n - j + m - q;
              acc += Lp[n * (n + 1) / 2 + m] * Y[y] * (double)sgn((m - q) * (m < q));
            }
          }
        }
        L_[(long)k * NTERM_ + j * (j + 1) / 2 + q] += acc;
      }
    }
  }
}

/* 3d/kernel.h:293-323 (L2P): local expansion evaluated at the leaf's bodies
 * (potential and spherical gradient, then to Cartesian). */
static void l2p(int c, cplx *Y, cplx *dY) {
  const cplx *Lc = L_ + (long)c * NTERM_;
  for (long b = body_[c]; b < body_[c] + nbody_[c]; b++) {
    double d[3] = {bx_[b] - cx_[c], by_[b] - cy_[c], bz_[b] - cz_[c]}, s[3] = {0, 0, 0}, f[3] = {0, 0, 0};
    double r, th, ph;
    to_sph(d, &r, &th, &ph);
    regular(r, th, ph, Y, dY);
    for (int n = 0; n < P_; n++) {
      int nm = n * n + n, ns = n * (n + 1) / 2;
      bp_[b] += creal(Lc[ns] * Y[nm]);
      s[0] += creal(Lc[ns] * Y[nm]) / r * n;
      s[1] += creal(Lc[ns] * dY[nm]);
      for (int m = 1; m <= n; m++) {
        nm = n * n + n + m;
        ns = n * (n + 1) / 2 + m;
        bp_[b] += 2 * creal(Lc[ns] * Y[nm]);
        s[0] += 2 * creal(Lc[ns] * Y[nm]) / r * n;
        s[1] += 2 * creal(Lc[ns] * dY[nm]);
        s[2] += 2 * creal(Lc[ns] * Y[nm] * I) * m;
      }
    }
    to_cart(r, th, ph, s, f);
    for (int k = 0; k < 3; k++) bf_[k][b] += f[k];
  }
}

/* ------------------------------------------------------------------ passes */

static void alloc_expansions(void) {
  free(M_);
  free(L_);
  M_ = calloc((size_t)nc_ * NTERM_, sizeof(cplx));
  L_ = calloc((size_t)nc_ * NTERM_, sizeof(cplx));
}

/* Post-order upward pass: 3d/traverse_eager.h:127-137. */
static void upward(int c, cplx *Y, cplx *dY) {
  for (int k = child_[c]; k < child_[c] + nchild_[c]; k++) upward(k, Y, dY);
  if (nchild_[c] == 0) p2m(c, Y, dY);
  if (nchild_[c]) {
    double kx[8][3];
    cplx *Mk[8];
    for (int k = 0; k < nchild_[c]; k++) {
      int ck = child_[c] + k;
      kx[k][0] = cx_[ck]; kx[k][1] = cy_[ck]; kx[k][2] = cz_[ck];
      Mk[k] = M_ + (long)ck * NTERM_;
    }
    const double X[3] = {cx_[c], cy_[c], cz_[c]};
    m2m_into(X, M_ + (long)c * NTERM_, nchild_[c], (const double(*)[3])kx, Mk, Y, dY);
  }
}

/* Pre-order downward pass: 3d/traverse_eager.h:175-190. */
static void downward(int c, cplx *Y, cplx *dY) {
  l2l(c, Y, dY);
  if (nchild_[c] == 0) l2p(c, Y, dY);
  for (int k = child_[c]; k < child_[c] + nchild_[c]; k++) downward(k, Y, dY);
}

/* Periodic far field at the root: 3dp/traverse_eager.h:46-93 (periodic).
 * A super-cell (the root's multipole, then 3x3x3 copies of it per level)
 * is M2L'd into the root from the 26*27 image positions of each level. */
static void periodic_root(void) {
  const int nt = NTERM_;
  cplx *Ms = calloc(nt, sizeof(cplx)), *Mk[26], *Y = malloc(P_ * P_ * sizeof(cplx)),
       *dY = malloc(P_ * P_ * sizeof(cplx)), *Y2 = malloc(4 * P_ * P_ * sizeof(cplx));
  memcpy(Ms, M_, nt * sizeof(cplx));
  const double X[3] = {cx_[0], cy_[0], cz_[0]};
  double kx[26][3], cyc = CYCLE_;
  for (int k = 0; k < 26; k++) Mk[k] = malloc(nt * sizeof(cplx));
  for (int lev = 0; lev < IMAGES_ - 1; lev++) {
    for (int a = -1; a <= 1; a++)
      for (int b = -1; b <= 1; b++)
        for (int c = -1; c <= 1; c++) {
          if (a == 0 && b == 0 && c == 0) continue;
          for (int u = -1; u <= 1; u++)
            for (int v = -1; v <= 1; v++)
              for (int w = -1; w <= 1; w++) {
                const int ix[3] = {a * 3 + u, b * 3 + v, c * 3 + w};
                m2l_into(X, X, Ms, L_, ix, cyc, Y2);
              }
        }
    int k = 0;
    for (int a = -1; a <= 1; a++)
      for (int b = -1; b <= 1; b++)
        for (int c = -1; c <= 1; c++) {
          if (a == 0 && b == 0 && c == 0) continue;
          kx[k][0] = X[0] + a * cyc;
          kx[k][1] = X[1] + b * cyc;
          kx[k][2] = X[2] + c * cyc;
          memcpy(Mk[k], Ms, nt * sizeof(cplx));
          k++;
        }
    m2m_into(X, Ms, 26, (const double(*)[3])kx, Mk, Y, dY);
    cyc *= 3;
  }
  for (int k = 0; k < 26; k++) free(Mk[k]);
  free(Ms); free(Y); free(dY); free(Y2);
}

long orc_fmm(long n, const double *xq, int P, int ncrit, double theta, int images, double cycle) {
  P_ = P;
  NTERM_ = P * (P + 1) / 2; /* 3d/kernel.h:118-120 (initKernel) */
  orc_tree(n, xq, ncrit);
  alloc_expansions();
  {
    cplx *Y = malloc(P * P * sizeof(cplx)), *dY = malloc(P * P * sizeof(cplx));
    upward(0, Y, dY);
    free(Y); free(dY);
  }
  orc_lists(theta, images, cycle);
  /* Evaluation of the lists per target cell: 3d/traverse_lazy.h:46-57. */
#pragma omp parallel
  {
    cplx *Y2 = malloc(4 * P * P * sizeof(cplx));
#pragma omp for schedule(dynamic)
    for (long c = 0; c < nc_; c++) {
      const double Xi[3] = {cx_[c], cy_[c], cz_[c]};
      for (int k = m2l_off_[c]; k < m2l_off_[c + 1]; k++) {
        int s = m2l_csr_[k].src, ix[3];
        img3(m2l_csr_[k].img, ix);
        const double Xj[3] = {cx_[s], cy_[s], cz_[s]};
        m2l_into(Xi, Xj, M_ + (long)s * NTERM_, L_ + c * NTERM_, ix, CYCLE_, Y2);
      }
      for (int k = p2p_off_[c]; k < p2p_off_[c + 1]; k++) {
        int s = p2p_csr_[k].src, ix[3];
        img3(p2p_csr_[k].img, ix);
        p2p(body_[c], nbody_[c], body_[s], nbody_[s], ix);
      }
    }
    free(Y2);
  }
  if (images > 0) periodic_root();
  {
    cplx *Y = malloc(P * P * sizeof(cplx)), *dY = malloc(P * P * sizeof(cplx));
    downward(0, Y, dY);
    free(Y); free(dY);
  }
  return nc_;
}

/* ---------------------------------------------------------------- getters */

void orc_get_bodies(double *o) {
  for (long b = 0; b < nb_; b++) {
    double *r = o + 8 * b;
    r[0] = bx_[b]; r[1] = by_[b]; r[2] = bz_[b]; r[3] = bq_[b];
    r[4] = bp_[b]; r[5] = bf_[0][b]; r[6] = bf_[1][b]; r[7] = bf_[2][b];
  }
}

void orc_get_perm(long *perm) { memcpy(perm, perm_, nb_ * sizeof(long)); }

void orc_get_cells(int *nchild, int *child, int *body, int *nbody, int *level, double *xr) {
  for (long c = 0; c < nc_; c++) {
    nchild[c] = nchild_[c];
    child[c] = child_[c];
    body[c] = body_[c];
    nbody[c] = nbody_[c];
    level[c] = level_[c];
    xr[4 * c] = cx_[c]; xr[4 * c + 1] = cy_[c]; xr[4 * c + 2] = cz_[c]; xr[4 * c + 3] = cr_[c];
  }
}

void orc_count_lists(long *a, long *b) {
  *a = nm2l_;
  *b = np2p_;
}

void orc_get_lists(int *mo, int *ms, int *mi, int *po, int *ps, int *pi) {
  memcpy(mo, m2l_off_, (nc_ + 1) * sizeof(int));
  memcpy(po, p2p_off_, (nc_ + 1) * sizeof(int));
  for (long k = 0; k < nm2l_; k++) { ms[k] = m2l_csr_[k].src; mi[k] = m2l_csr_[k].img; }
  for (long k = 0; k < np2p_; k++) { ps[k] = p2p_csr_[k].src; pi[k] = p2p_csr_[k].img; }
}

void orc_get_expansions(double *M, double *L) {
  for (long k = 0; k < nc_ * NTERM_; k++) {
    M[2 * k] = creal(M_[k]); M[2 * k + 1] = cimag(M_[k]);
    L[2 * k] = creal(L_[k]); L[2 * k + 1] = cimag(L_[k]);
  }
}

/* ----------------------------------------------------------------- direct */

/* 3d/traverse_eager.h:193-202 (direct) and, with images, the image sum of
 * 3dp/traverse_eager.h:131-155 (prange = sum of 3^i over the image levels).
 * Targets are independent, so the image loop runs inside the target loop. */
void orc_direct(long nt, double *T, long ns, const double *S, int images, double cycle) {
  int pr = 0;
  for (int i = 0; i < images; i++) pr += (int)powf(3.f, (float)i);
#pragma omp parallel for schedule(dynamic, 4)
  for (long i = 0; i < nt; i++) {
    double *t = T + 8 * i;
    for (int a = -pr; a <= pr; a++)
      for (int b = -pr; b <= pr; b++)
        for (int c = -pr; c <= pr; c++) {
          double pot = 0, ax = 0, ay = 0, az = 0;
          for (long j = 0; j < ns; j++) {
            const double *s = S + 8 * j;
            double d[3] = {t[0] - s[0] - a * cycle, t[1] - s[1] - b * cycle, t[2] - s[2] - c * cycle};
            double R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            if (R2 != 0) {
              double i2 = 1.0 / R2, iR = s[3] * sqrt(i2);
              for (int k = 0; k < 3; k++) d[k] *= i2 * iR;
              pot += iR;
              ax += d[0];
              ay += d[1];
              az += d[2];
            }
          }
          t[4] += pot;
          t[5] -= ax;
          t[6] -= ay;
          t[7] -= az;
        }
  }
}

/* 3dp/fmm.cxx:63-75: dipole correction of the periodic FMM result. */
void orc_dipole_correction(double cycle) {
  double dip[3] = {0, 0, 0};
  for (long b = 0; b < nb_; b++) {
    dip[0] += bx_[b] * bq_[b];
    dip[1] += by_[b] * bq_[b];
    dip[2] += bz_[b] * bq_[b];
  }
  const double coef = 4 * M_PI / (3 * cycle * cycle * cycle);
  for (long b = 0; b < nb_; b++) {
    const double dn = dip[0] * dip[0] + dip[1] * dip[1] + dip[2] * dip[2];
    bp_[b] -= coef * dn / nb_ / bq_[b];
    for (int d = 0; d < 3; d++) bf_[d][b] -= coef * dip[d];
  }
}

/* ------------------------------------------------------------------ Ewald */

/* Real-space pair term: 3dp/ewald.h:82-102 (realP2P). */
static void ewald_real_pair(long ib, long ni, long jb, long nj, const int ix[3], double alpha, double cutoff,
                            double cycle, double *p, double (*f)[3]) {
  for (long i = ib; i < ib + ni; i++) {
    for (long j = jb; j < jb + nj; j++) {
      double d[3] = {bx_[i] - bx_[j] - ix[0] * cycle, by_[i] - by_[j] - ix[1] * cycle,
                     bz_[i] - bz_[j] - ix[2] * cycle};
      double R2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (0 < R2 && R2 < cutoff * cutoff) {
        double R2s = R2 * alpha * alpha, Rs = sqrt(R2s), iRs = 1 / Rs, iR2s = iRs * iRs, iR3s = iR2s * iRs;
        double dt = bq_[j] * (M_2_SQRTPI * exp(-R2s) * iR2s + erfc(Rs) * iR3s);
        dt *= alpha * alpha * alpha;
        p[i] += bq_[j] * erfc(Rs) * iRs * alpha;
        f[i][0] -= d[0] * dt;
        f[i][1] -= d[1] * dt;
        f[i][2] -= d[2] * dt;
      }
    }
  }
}

/* Minimum-image neighbour search: 3dp/ewald.h:104-119 (neighbor). */
static void ewald_neighbor(int ci, int cj, double alpha, double cutoff, double cycle, double *p, double (*f)[3]) {
  double d[3] = {cx_[ci] - cx_[cj], cy_[ci] - cy_[cj], cz_[ci] - cz_[cj]};
  int ix[3];
  for (int k = 0; k < 3; k++) {
    ix[k] = 0;
    if (d[k] < -cycle / 2) ix[k]--;
    if (d[k] > cycle / 2) ix[k]++;
    d[k] -= ix[k] * cycle;
  }
  double R = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (R - cr_[ci] - cr_[cj] < sqrtf(3) * cutoff) {
    if (nchild_[cj] == 0) ewald_real_pair(body_[ci], nbody_[ci], body_[cj], nbody_[cj], ix, alpha, cutoff, cycle, p, f);
    for (int k = child_[cj]; k < child_[cj] + nchild_[cj]; k++) ewald_neighbor(ci, k, alpha, cutoff, cycle, p, f);
  }
}

/* Ewald sum: wave part 3dp/ewald.h:22-79,130-143 (initWaves, dft, idft,
 * wavePart), real part :122-127 (realPart, per target leaf), self term
 * :146-150. */
void orc_ewald(int ksize, double alpha, double sigma, double cutoff, double cycle, double *out) {
  orc_ewald_parts(7, ksize, alpha, sigma, cutoff, cycle, out);
}

/* The parts selected by the mask (1 wave, 2 real, 4 self), as the reference
 * driver calls them one by one (3dp/fmm.cxx:85-93). */
void orc_ewald_parts(int parts, int ksize, double alpha, double sigma, double cutoff, double cycle, double *out) {
  double *p = calloc(nb_, sizeof(double));
  double (*f)[3] = calloc(nb_, sizeof(*f));
  const double scale = 2 * M_PI / cycle;
  /* waves: |k|^2 <= ksize^2 over the half space (l>0, or l=0 and m>0, or l=m=0 and n>0) */
  long nw = 0, capw = 0;
  double *wk = NULL;
  for (int l = 0; l <= ksize; l++) {
    int mmin = l == 0 ? 0 : -ksize;
    for (int m = mmin; m <= ksize; m++) {
      int nmin = (l == 0 && m == 0) ? 1 : -ksize;
      for (int n = nmin; n <= ksize; n++) {
        double ksq = l * l + m * m + n * n;
        if (ksq <= ksize * ksize) {
          wk = grow(wk, &capw, 3 * (nw + 1), sizeof(double));
          wk[3 * nw] = l; wk[3 * nw + 1] = m; wk[3 * nw + 2] = n;
          nw++;
        }
      }
    }
  }
  double *re = calloc(nw, sizeof(double)), *im = calloc(nw, sizeof(double));
  if (!(parts & 1)) nw = 0;  /* no wave part */
#pragma omp parallel for
  for (long w = 0; w < nw; w++) {
    double a = 0, b = 0;
    for (long j = 0; j < nb_; j++) {
      double th = 0;
      th += wk[3 * w] * bx_[j] * scale;
      th += wk[3 * w + 1] * by_[j] * scale;
      th += wk[3 * w + 2] * bz_[j] * scale;
      a += bq_[j] * cos(th);
      b += bq_[j] * sin(th);
    }
    re[w] = a;
    im[w] = b;
  }
  const double coef = 2 / sigma / cycle / cycle / cycle, coef2 = 1 / (4 * alpha * alpha);
  for (long w = 0; w < nw; w++) {
    double K[3] = {wk[3 * w] * scale, wk[3 * w + 1] * scale, wk[3 * w + 2] * scale};
    double K2 = K[0] * K[0] + K[1] * K[1] + K[2] * K[2];
    double fac = coef * exp(-K2 * coef2) / K2;
    re[w] *= fac;
    im[w] *= fac;
  }
#pragma omp parallel for
  for (long i = 0; i < nb_; i++) {
    double pot = 0, F[3] = {0, 0, 0};
    for (long w = 0; w < nw; w++) {
      double th = 0;
      th += wk[3 * w] * bx_[i] * scale;
      th += wk[3 * w + 1] * by_[i] * scale;
      th += wk[3 * w + 2] * bz_[i] * scale;
      double dt = re[w] * sin(th) - im[w] * cos(th);
      pot += re[w] * cos(th) + im[w] * sin(th);
      for (int d = 0; d < 3; d++) F[d] -= dt * wk[3 * w + d];
    }
    for (int d = 0; d < 3; d++) F[d] *= scale;
    p[i] += pot;
    for (int d = 0; d < 3; d++) f[i][d] += F[d];
  }
  /* real part: every target leaf walks the source tree from the root */
  long nleaf = 0;
  for (long c = 0; c < nc_; c++) nleaf += nchild_[c] == 0;
  int *leaves = malloc(nleaf * sizeof(int));
  nleaf = 0;
  for (long c = 0; c < nc_; c++)
    if (nchild_[c] == 0) leaves[nleaf++] = (int)c;
  if (!(parts & 2)) nleaf = 0;  /* no real part */
#pragma omp parallel for schedule(dynamic)
  for (long k = 0; k < nleaf; k++) ewald_neighbor(leaves[k], 0, alpha, cutoff, cycle, p, f);
  if (parts & 4)
    for (long i = 0; i < nb_; i++) p[i] -= M_2_SQRTPI * bq_[i] * alpha;
  for (long b = 0; b < nb_; b++) {
    double *r = out + 8 * b;
    r[0] = bx_[b]; r[1] = by_[b]; r[2] = bz_[b]; r[3] = bq_[b];
    r[4] = p[b]; r[5] = f[b][0]; r[6] = f[b][1]; r[7] = f[b][2];
  }
  free(leaves); free(re); free(im); free(wk); free(p); free(f);
}

/* ------------------------------------------------------------------- KAT */

/* The operator chain of test/test_kernel.h:6-94: one unit charge at (2,2,2),
 * P2M at (3,1,1), M2M to (4,0,0), M2L to (-4,0,0), L2L to (-3,1,1), L2P at
 * (-2,2,2), compared with P2P.  Built on a private 4-cell + 2-body state. */
double orc_kernel_chain(int P, double *ferr) {
  free_bodies();
  P_ = P;
  NTERM_ = P * (P + 1) / 2;
  CYCLE_ = 0;
  nb_ = 3; /* 0: source, 1: target (L2P), 2: target (P2P) */
  bx_ = calloc(3, sizeof(double)); by_ = calloc(3, sizeof(double)); bz_ = calloc(3, sizeof(double));
  bq_ = calloc(3, sizeof(double)); bp_ = calloc(3, sizeof(double));
  for (int d = 0; d < 3; d++) bf_[d] = calloc(3, sizeof(double));
  perm_ = calloc(3, sizeof(long));
  bx_[0] = by_[0] = bz_[0] = 2; bq_[0] = 1;
  for (int t = 1; t < 3; t++) { bx_[t] = -2; by_[t] = 2; bz_[t] = 2; bq_[t] = 1; }
  nc_ = 0;
  new_cells(4);
  const double X[4][3] = {{3, 1, 1}, {4, 0, 0}, {-4, 0, 0}, {-3, 1, 1}};
  const double R[4] = {1, 2, 2, 1};
  for (int c = 0; c < 4; c++) {
    cx_[c] = X[c][0]; cy_[c] = X[c][1]; cz_[c] = X[c][2]; cr_[c] = R[c];
    nchild_[c] = 0; child_[c] = -1; level_[c] = 0; body_[c] = 0; nbody_[c] = 0;
  }
  body_[0] = 0; nbody_[0] = 1;
  nchild_[1] = 1; child_[1] = 0;
  nchild_[2] = 1; child_[2] = 3;
  body_[3] = 1; nbody_[3] = 1;
  alloc_expansions();
  cplx *Y = malloc(P * P * sizeof(cplx)), *dY = malloc(P * P * sizeof(cplx)), *Y2 = malloc(4 * P * P * sizeof(cplx));
  p2m(0, Y, dY);
  {
    double kx[1][3] = {{cx_[0], cy_[0], cz_[0]}};
    cplx *Mk[1] = {M_};
    m2m_into(X[1], M_ + NTERM_, 1, (const double(*)[3])kx, Mk, Y, dY);
  }
  const int ix0[3] = {0, 0, 0};
  m2l_into(X[2], X[1], M_ + NTERM_, L_ + 2 * NTERM_, ix0, 0, Y2);
  l2l(2, Y, dY);
  l2p(3, Y, dY);
  p2p(2, 1, 0, 1, ix0);
  double pd = bp_[1] - bp_[2], pn = bp_[1], fd = 0, fn = 0;
  for (int d = 0; d < 3; d++) {
    fd += (bf_[d][1] - bf_[d][2]) * (bf_[d][1] - bf_[d][2]);
    fn += bf_[d][1] * bf_[d][1];
  }
  free(Y); free(dY); free(Y2);
  if (ferr) *ferr = sqrt(fd / fn);
  return sqrt(pd * pd / (pn * pn));
}

/* ------------------------------------------------------ single operators */

/* A problem of nbodies bodies (Body records, or none) and ncells cells at
 * order P, replacing the current one; cell c gets centre/radius cell4[c]. */
static void op_problem(int P, long nbodies, const double *bodies8, int ncells, const double *cell4) {
  free_bodies();
  P_ = P;
  NTERM_ = P * (P + 1) / 2;
  CYCLE_ = 0;
  nb_ = nbodies;
  long nalloc = nbodies > 0 ? nbodies : 1;
  bx_ = calloc(nalloc, sizeof(double)); by_ = calloc(nalloc, sizeof(double)); bz_ = calloc(nalloc, sizeof(double));
  bq_ = calloc(nalloc, sizeof(double)); bp_ = calloc(nalloc, sizeof(double));
  for (int d = 0; d < 3; d++) bf_[d] = calloc(nalloc, sizeof(double));
  perm_ = calloc(nalloc, sizeof(long));
  for (long b = 0; b < nbodies; b++) {
    const double *r = bodies8 + 8 * b;
    bx_[b] = r[0]; by_[b] = r[1]; bz_[b] = r[2]; bq_[b] = r[3];
    bp_[b] = r[4]; bf_[0][b] = r[5]; bf_[1][b] = r[6]; bf_[2][b] = r[7];
  }
  nc_ = 0;
  new_cells(ncells);
  for (int c = 0; c < ncells; c++) {
    cx_[c] = cell4[4 * c]; cy_[c] = cell4[4 * c + 1]; cz_[c] = cell4[4 * c + 2]; cr_[c] = cell4[4 * c + 3];
    nchild_[c] = 0; child_[c] = -1; level_[c] = 0; body_[c] = 0; nbody_[c] = 0;
  }
  alloc_expansions();
}

static void op_bodies_out(double *bodies8, long nb) {
  for (long b = 0; b < nb; b++) {
    double *r = bodies8 + 8 * b;
    r[4] = bp_[b]; r[5] = bf_[0][b]; r[6] = bf_[1][b]; r[7] = bf_[2][b];
  }
}

/* P2M(C) (3d/kernel.h:187-202) on one cell: M (NTERM complex) accumulates. */
void orc_op_p2m(int P, const double *cell4, const double *bodies8, long nb, double *M) {
  op_problem(P, nb, bodies8, 1, cell4);
  memcpy(M_, M, NTERM_ * sizeof(cplx));
  body_[0] = 0; nbody_[0] = (int)nb;
  cplx *Y = malloc(P * P * sizeof(cplx)), *dY = malloc(P * P * sizeof(cplx));
  p2m(0, Y, dY);
  memcpy(M, M_, NTERM_ * sizeof(cplx));
  free(Y); free(dY);
}

/* M2M(Ci) (3d/kernel.h:204-231): the children's multipoles into the parent's
 * M (accumulates). */
void orc_op_m2m(int P, const double *parent4, double *M, int nchild, const double *child4, const double *Mchild) {
  op_problem(P, 0, NULL, 1, parent4);
  const int nt = P * (P + 1) / 2;
  double (*kx)[3] = malloc((nchild > 0 ? nchild : 1) * sizeof(double[3]));
  cplx **Mk = malloc((nchild > 0 ? nchild : 1) * sizeof(cplx *));
  for (int k = 0; k < nchild; k++) {
    for (int d = 0; d < 3; d++) kx[k][d] = child4[4 * k + d];
    Mk[k] = (cplx *)(Mchild + 2 * (long)k * nt);
  }
  cplx *Y = malloc(P * P * sizeof(cplx)), *dY = malloc(P * P * sizeof(cplx));
  m2m_into(parent4, (cplx *)M, nchild, (const double(*)[3])kx, Mk, Y, dY);
  free(Y); free(dY); free(kx); free(Mk);
}

/* M2L(Ci, Cj) (3d/kernel.h:233-260; 3dp/kernel.h:198-200 with the periodic
 * shift iX * cycle): the source multipole into the target's L (accumulates). */
void orc_op_m2l(int P, const double *target4, double *L, const double *source4, const double *M, const int *ix,
                double cycle) {
  op_problem(P, 0, NULL, 1, target4);
  const int ix0[3] = {0, 0, 0};
  cplx *Y2 = malloc(4 * P * P * sizeof(cplx));
  m2l_into(target4, source4, (const cplx *)M, (cplx *)L, ix ? ix : ix0, ix ? cycle : 0.0, Y2);
  free(Y2);
}

/* L2L(Cj) (3d/kernel.h:262-291): the parent's L into each child's L
 * (Lchild: nchild x NTERM complex, accumulates). */
void orc_op_l2l(int P, const double *parent4, const double *L, int nchild, const double *child4, double *Lchild) {
  double *cells = malloc(4 * (1 + (long)nchild) * sizeof(double));
  memcpy(cells, parent4, 4 * sizeof(double));
  memcpy(cells + 4, child4, 4 * (long)nchild * sizeof(double));
  op_problem(P, 0, NULL, 1 + nchild, cells);
  free(cells);
  nchild_[0] = nchild; child_[0] = 1;
  memcpy(L_, L, NTERM_ * sizeof(cplx));
  memcpy(L_ + NTERM_, Lchild, (long)nchild * NTERM_ * sizeof(cplx));
  cplx *Y = malloc(P * P * sizeof(cplx)), *dY = malloc(P * P * sizeof(cplx));
  l2l(0, Y, dY);
  memcpy(Lchild, L_ + NTERM_, (long)nchild * NTERM_ * sizeof(cplx));
  free(Y); free(dY);
}

/* L2P(C) (3d/kernel.h:293-323): the cell's local expansion at its bodies
 * (Body records; p and F accumulate). */
void orc_op_l2p(int P, const double *cell4, const double *L, double *bodies8, long nb) {
  op_problem(P, nb, bodies8, 1, cell4);
  memcpy(L_, L, NTERM_ * sizeof(cplx));
  body_[0] = 0; nbody_[0] = (int)nb;
  cplx *Y = malloc(P * P * sizeof(cplx)), *dY = malloc(P * P * sizeof(cplx));
  l2p(0, Y, dY);
  op_bodies_out(bodies8, nb);
  free(Y); free(dY);
}

/* P2P(Ci, Cj) (3d/kernel.h:122-150; 3dp/kernel.h:133 with the periodic shift
 * iX * cycle): sources onto targets (Body records; p and F accumulate). */
void orc_op_p2p(double *targets8, long nt, const double *sources8, long ns, const int *ix, double cycle) {
  double *all = malloc(8 * (nt + ns) * sizeof(double));
  memcpy(all, targets8, 8 * nt * sizeof(double));
  memcpy(all + 8 * nt, sources8, 8 * ns * sizeof(double));
  const double c0[4] = {0, 0, 0, 0};
  op_problem(1, nt + ns, all, 1, c0);
  free(all);
  const int ix0[3] = {0, 0, 0};
  CYCLE_ = ix ? cycle : 0.0;
  p2p(0, nt, nt, ns, ix ? ix : ix0);
  CYCLE_ = 0;
  op_bodies_out(targets8, nt);
}

/* --------------------------------------------------------------- bodies */

void orc_reference_bodies(long n, long seed, int kind, double cycle, double *xq) {
  srand48(seed);
  double avg = 0;
  for (long b = 0; b < n; b++) {
    for (int d = 0; d < 3; d++) {
      double u = drand48();
      xq[4 * b + d] = kind == 0 ? u * 2 * M_PI - M_PI : u * cycle - cycle * .5;
    }
    xq[4 * b + 3] = drand48() - .5;
    avg += xq[4 * b + 3];
  }
  avg /= n;
  for (long b = 0; b < n; b++) xq[4 * b + 3] -= avg;
}
