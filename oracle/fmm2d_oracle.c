/* Oracle, 2D: plain-C restatement of minimal ExaFMM's 2D Laplace FMM, free
 * space (`2d/`) and periodic (`2dp/`).  TEST INFRASTRUCTURE ONLY (see
 * fmm2d_oracle.h).  Each function cites the
 * reference lines it restates.  Bit-identity with the reference needs the
 * same operations in the same order: complex products are written out as
 * (ac - bd, ad + bc), a complex times or over a real acts on each part, and
 * complex division and the complex logarithm use C99's (the same runtime
 * routines the reference's std::complex calls).  Compiled with
 * -ffp-contract=off, as the reference is compiled without fused
 * multiply-adds. */
#include "fmm2d_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double r, i;
} cpx;

static cpx cmul(cpx a, cpx b) { return (cpx){a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
static cpx cscale(cpx a, double t) { return (cpx){a.r * t, a.i * t}; }
static cpx cdivr(cpx a, double t) { return (cpx){a.r / t, a.i / t}; }
static cpx cneg(cpx a) { return (cpx){-a.r, -a.i}; }
static void cacc(cpx *d, cpx a) {
  d->r += a.r;
  d->i += a.i;
}
static cpx cdiv(cpx a, cpx b) {
  const double complex q = CMPLX(a.r, a.i) / CMPLX(b.r, b.i);
  return (cpx){creal(q), cimag(q)};
}
static cpx clogc(cpx z) {
  const double complex w = clog(CMPLX(z.r, z.i));
  return (cpx){creal(w), cimag(w)};
}

typedef struct {
  double X[2], q, p, F[2];
} Body2;

typedef struct {
  int nchild, nbody, child, body;  /* child: first child's index (-1: leaf); body: first body */
  double X[2], R;
  int *m2l, nm2l, cm2l;            /* interaction lists, in recording order: */
  int *p2p, np2p, cp2p;            /* source cell, then its image index */
} Cell2;

static Body2 *g_b;
static long g_n;
static Cell2 *g_c;
static long g_nc, g_cap;
static int g_P, g_ncrit, g_images;
static double g_theta, g_cycle;
static int g_iX[2]; /* the image of the current source: a shift of iX * cycle */
static cpx *g_M, *g_L; /* P per cell */

static void free_cells(void) {
  for (long c = 0; c < g_nc; c++) {
    free(g_c[c].m2l);
    free(g_c[c].p2p);
  }
  free(g_c);
  g_c = NULL;
  g_nc = g_cap = 0;
  free(g_M);
  free(g_L);
  g_M = g_L = NULL;
}

static long new_cells(int k) {
  if (g_nc + k > g_cap) {
    g_cap = 2 * (g_nc + k) + 16;
    g_c = (Cell2 *)realloc(g_c, sizeof(Cell2) * g_cap);
  }
  memset(g_c + g_nc, 0, sizeof(Cell2) * k);
  g_nc += k;
  return g_nc - k;
}

/* 2d/build_tree.h:7-21 getBounds */
static void bounds(double *R0, double *X0) {
  double lo[2], hi[2];
  for (int d = 0; d < 2; d++) lo[d] = hi[d] = g_b[0].X[d];
  for (long b = 0; b < g_n; b++)
    for (int d = 0; d < 2; d++) {
      lo[d] = fmin(g_b[b].X[d], lo[d]);
      hi[d] = fmax(g_b[b].X[d], hi[d]);
    }
  for (int d = 0; d < 2; d++) X0[d] = (hi[d] + lo[d]) / 2;
  *R0 = 0;
  for (int d = 0; d < 2; d++) {
    *R0 = fmax(X0[d] - lo[d], *R0);
    *R0 = fmax(hi[d] - X0[d], *R0);
  }
  *R0 *= 1.00001;
}

/* 2d/build_tree.h:23-86 buildCells: the bodies of [begin, end) lie in `src`;
 * split ones are partitioned by quadrant into `dst` (stable) and the children
 * recurse with the roles swapped; a leaf whose bodies lie in the scratch
 * array copies them (X and q only) back.  Every body ends in g_b. */
static void build(Body2 *src, Body2 *dst, long begin, long end, long cell, const double *X, double R, int level,
                  int flip) {
  Cell2 *C = &g_c[cell];
  C->body = (int)begin;
  C->nbody = (int)(end - begin);
  C->nchild = 0;
  C->child = -1;
  for (int d = 0; d < 2; d++) C->X[d] = X[d];
  C->R = R / (1 << level);
  if (end - begin <= g_ncrit) {
    if (flip)
      for (long i = begin; i < end; i++) {
        for (int d = 0; d < 2; d++) dst[i].X[d] = src[i].X[d];
        dst[i].q = src[i].q;
      }
    return;
  }
  long size[4] = {0, 0, 0, 0}, off[4], cnt[4], o = begin;
  for (long i = begin; i < end; i++) size[(src[i].X[0] > X[0]) + ((src[i].X[1] > X[1]) << 1)]++;
  int nchild = 0;
  for (int q = 0; q < 4; q++) {
    off[q] = o;
    o += size[q];
    if (size[q]) nchild++;
  }
  for (int q = 0; q < 4; q++) cnt[q] = off[q];
  for (long i = begin; i < end; i++) {
    const int q = (src[i].X[0] > X[0]) + ((src[i].X[1] > X[1]) << 1);
    for (int d = 0; d < 2; d++) dst[cnt[q]].X[d] = src[i].X[d];
    dst[cnt[q]].q = src[i].q;
    cnt[q]++;
  }
  const long first = new_cells(nchild);  /* may move g_c */
  g_c[cell].nchild = nchild;
  g_c[cell].child = (int)first;
  int c = 0;
  for (int q = 0; q < 4; q++) {
    double Xc[2] = {X[0], X[1]};
    const double r = R / (1 << (level + 1));
    for (int d = 0; d < 2; d++) Xc[d] += r * (((q & 1 << d) >> d) * 2 - 1);
    if (size[q]) {
      build(dst, src, off[q], off[q] + size[q], first + c, Xc, R, level + 1, !flip);
      c++;
    }
  }
}

long orc2_tree(long n, const double *xyq, int ncrit) {
  free_cells();
  free(g_b);
  g_n = n;
  g_ncrit = ncrit;
  g_b = (Body2 *)calloc(n, sizeof(Body2));
  for (long b = 0; b < n; b++) {
    g_b[b].X[0] = xyq[3 * b];
    g_b[b].X[1] = xyq[3 * b + 1];
    g_b[b].q = xyq[3 * b + 2];
  }
  Body2 *buf = (Body2 *)malloc(sizeof(Body2) * n);
  memcpy(buf, g_b, sizeof(Body2) * n);
  double R0, X0[2];
  bounds(&R0, X0);
  new_cells(1);
  build(g_b, buf, 0, n, 0, X0, R0, 0, 0);
  free(buf);
  return g_nc;
}

/* 2d/kernel.h:12-31 P2P; 2dp/kernel.h:12-35 with the source image shifted
 * by iX * cycle (zero in free space: x - 0.0 is x) */
static void p2p(Body2 *Bi, long ni, const Body2 *Bj, long nj) {
  for (long i = 0; i < ni; i++) {
    double p = 0, F[2] = {0, 0};
    for (long j = 0; j < nj; j++) {
      double dX[2];
      for (int d = 0; d < 2; d++) dX[d] = Bi[i].X[d] - Bj[j].X[d] - g_iX[d] * g_cycle;
      const double R2 = dX[0] * dX[0] + dX[1] * dX[1];
      if (R2 != 0) {
        const double invR = 1 / sqrt(R2);
        p += Bj[j].q * log(invR);
        for (int d = 0; d < 2; d++) F[d] += dX[d] * Bj[j].q / R2;
      }
    }
    Bi[i].p += p;
    for (int d = 0; d < 2; d++) Bi[i].F[d] -= F[d];
  }
}

/* 2d/kernel.h:33-44 P2M */
static void p2m(long c) {
  const Cell2 *C = &g_c[c];
  cpx *M = g_M + c * g_P;
  for (long b = C->body; b < C->body + C->nbody; b++) {
    const cpx Z = {g_b[b].X[0] - C->X[0], g_b[b].X[1] - C->X[1]};
    cpx pw = {1.0, 0.0};
    M[0].r += g_b[b].q;
    for (int n = 1; n < g_P; n++) {
      pw = cmul(pw, cdivr(Z, (double)n));
      cacc(&M[n], cscale(pw, g_b[b].q));
    }
  }
}

/* 2d/kernel.h:46-59 M2M: one child's multipole Mj (centre Xj) into the
 * parent's Mi (centre Xi) */
static void m2m_one(const double *Xi, cpx *Mi, const double *Xj, const cpx *Mj) {
  const cpx Z = {Xj[0] - Xi[0], Xj[1] - Xi[1]};
  for (int k = 0; k < g_P; k++) {
    cpx pw = {1.0, 0.0};
    cacc(&Mi[k], Mj[k]);
    for (int n = 1; n <= k; n++) {
      pw = cmul(pw, cdivr(Z, (double)n));
      cacc(&Mi[k], cmul(Mj[k - n], pw));
    }
  }
}

static void m2m(long ci) {
  for (long cj = g_c[ci].child; cj < g_c[ci].child + g_c[ci].nchild; cj++)
    m2m_one(g_c[ci].X, g_M + ci * g_P, g_c[cj].X, g_M + cj * g_P);
}

/* 2d/kernel.h:61-89 M2L (2dp/kernel.h:65-93: source shifted by iX * cycle),
 * from the multipole M to the local expansion L */
static void m2l_at(const double *Xi, const double *Xj, const cpx *M, cpx *L) {
  const cpx Z = {Xi[0] - Xj[0] - g_iX[0] * g_cycle, Xi[1] - Xj[1] - g_iX[1] * g_cycle};
  const cpx one = {1.0, 0.0}, invZ = cdiv(one, Z);
  cpx pzn, pznk = one;
  cacc(&L[0], cmul(cneg(M[0]), clogc(Z)));
  cacc(&L[0], cmul(M[1], invZ));
  pzn = invZ;
  for (int k = 2; k < g_P; k++) {
    pzn = cmul(pzn, cscale(invZ, (double)(k - 1)));
    cacc(&L[0], cmul(M[k], pzn));
  }
  cacc(&L[1], cmul(cneg(M[0]), invZ));
  pzn = invZ;
  for (int k = 1; k < g_P; k++) {
    pzn = cmul(pzn, cscale(invZ, (double)k));
    cacc(&L[1], cmul(cneg(M[k]), pzn));
  }
  double Cnk = -1;
  for (int n = 2; n < g_P; n++) {
    Cnk *= -1;
    pznk = cmul(pznk, invZ);
    pzn = cscale(pznk, Cnk);
    for (int k = 0; k < g_P; k++) {
      pzn = cmul(pzn, cscale(invZ, (double)(n + k - 1)));
      cacc(&L[n], cmul(M[k], pzn));
    }
    pznk = cscale(pznk, (double)(n - 1));
  }
}

static void m2l(long ci, long cj) { m2l_at(g_c[ci].X, g_c[cj].X, g_M + cj * g_P, g_L + ci * g_P); }

/* 2d/kernel.h:91-105 L2L */
static void l2l(long cj) {
  const Cell2 *Cj = &g_c[cj];
  const cpx *Lj = g_L + cj * g_P;
  for (long ci = Cj->child; ci < Cj->child + Cj->nchild; ci++) {
    const cpx Z = {g_c[ci].X[0] - Cj->X[0], g_c[ci].X[1] - Cj->X[1]};
    cpx *Li = g_L + ci * g_P;
    for (int l = 0; l < g_P; l++) {
      cpx pw = {1.0, 0.0};
      cacc(&Li[l], Lj[l]);
      for (int k = 1; k < g_P - l; k++) {
        pw = cmul(pw, cdivr(Z, (double)k));
        cacc(&Li[l], cmul(Lj[l + k], pw));
      }
    }
  }
}

/* 2d/kernel.h:107-124 L2P */
static void l2p(long c) {
  const Cell2 *C = &g_c[c];
  const cpx *L = g_L + c * g_P;
  for (long b = C->body; b < C->body + C->nbody; b++) {
    Body2 *B = &g_b[b];
    const cpx Z = {B->X[0] - C->X[0], B->X[1] - C->X[1]};
    cpx pw = {1.0, 0.0};
    B->p += L[0].r;
    B->F[0] += L[1].r;
    B->F[1] -= L[1].i;
    for (int n = 1; n < g_P; n++) {
      pw = cmul(pw, cdivr(Z, (double)n));
      B->p += cmul(L[n], pw).r;
      if (n < g_P - 1) {
        const cpx t = cmul(L[n + 1], pw);
        B->F[0] += t.r;
        B->F[1] -= t.i;
      }
    }
  }
}

/* 2d/traverse_lazy.h:5-17 upwardPass (children first, then P2M / M2M) */
static void upward(long c) {
  for (long k = g_c[c].child; k < g_c[c].child + g_c[c].nchild; k++) upward(k);
  if (g_c[c].nchild == 0) p2m(c);
  m2m(c);
}

static void push(int **a, int *n, int *cap, int v) {
  if (*n == *cap) {
    *cap = 2 * *cap + 8;
    *a = (int *)realloc(*a, sizeof(int) * *cap);
  }
  (*a)[(*n)++] = v;
}

/* 2d/traverse_lazy.h:26-43 getList: the MAC, then the branch rules
 * (2dp/traverse_lazy.h:33-52: source image iX, recorded per entry as
 * periodic1D = iX0 + 1 + 3 (iX1 + 1)) */
static void get_list(long ci, long cj) {
  Cell2 *Ci = &g_c[ci];
  const Cell2 *Cj = &g_c[cj];
  const double dX[2] = {Ci->X[0] - Cj->X[0] - g_iX[0] * g_cycle, Ci->X[1] - Cj->X[1] - g_iX[1] * g_cycle};
  const double R2 = (dX[0] * dX[0] + dX[1] * dX[1]) * g_theta * g_theta;
  const int img = g_iX[0] + 1 + 3 * (g_iX[1] + 1);
  if (R2 > (Ci->R + Cj->R) * (Ci->R + Cj->R)) {
    push(&Ci->m2l, &Ci->nm2l, &Ci->cm2l, (int)cj);
    push(&Ci->m2l, &Ci->nm2l, &Ci->cm2l, img);
  } else if (Ci->nchild == 0 && Cj->nchild == 0) {
    push(&Ci->p2p, &Ci->np2p, &Ci->cp2p, (int)cj);
    push(&Ci->p2p, &Ci->np2p, &Ci->cp2p, img);
  } else if (Cj->nchild == 0 || (Ci->R >= Cj->R && Ci->nchild != 0)) {
    for (long k = Ci->child; k < Ci->child + Ci->nchild; k++) get_list(k, cj);
  } else {
    for (long k = Cj->child; k < Cj->child + Cj->nchild; k++) get_list(ci, k);
  }
}

/* 2d/traverse_lazy.h:59-71 downwardPass (L2L to the children, L2P at a leaf,
 * then the children) */
static void downward(long c) {
  l2l(c);
  if (g_c[c].nchild == 0) l2p(c);
  for (long k = g_c[c].child; k < g_c[c].child + g_c[c].nchild; k++) downward(k);
}

/* 2dp/traverse_lazy.h:79-122 periodic: the far images as a hierarchy of 3 x 3
 * super-cells around the root.  Per image level: M2L into the root from the
 * 72 cells of the level's ring (8 neighbours x 9 sub-cells), then the
 * super-cell's multipole from its 8 neighbour copies (M2M), cycle x 3. */
static void periodic(void) {
  cpx *Mp = (cpx *)malloc(sizeof(cpx) * g_P), *Mc = (cpx *)malloc(sizeof(cpx) * 8 * g_P);
  memcpy(Mp, g_M, sizeof(cpx) * g_P);
  const double Xp[2] = {g_c[0].X[0], g_c[0].X[1]};
  for (int level = 0; level < g_images - 1; level++) {
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++) {
        if (ix == 0 && iy == 0) continue;
        for (int cx = -1; cx <= 1; cx++)
          for (int cy = -1; cy <= 1; cy++) {
            g_iX[0] = ix * 3 + cx;
            g_iX[1] = iy * 3 + cy;
            m2l_at(g_c[0].X, Xp, Mp, g_L);
          }
      }
    double Xc[8][2];
    int c = 0;
    for (int ix = -1; ix <= 1; ix++)
      for (int iy = -1; iy <= 1; iy++) {
        if (ix == 0 && iy == 0) continue;
        Xc[c][0] = Xp[0] + ix * g_cycle;
        Xc[c][1] = Xp[1] + iy * g_cycle;
        memcpy(Mc + c * g_P, Mp, sizeof(cpx) * g_P);
        c++;
      }
    for (c = 0; c < 8; c++) m2m_one(Xp, Mp, Xc[c], Mc + c * g_P);
    g_cycle *= 3;
  }
  free(Mp);
  free(Mc);
}

long orc2_fmm(long n, const double *xyq, int P, int ncrit, double theta, int images, double cycle) {
  orc2_tree(n, xyq, ncrit);
  g_P = P;
  g_theta = theta;
  g_images = images;
  g_cycle = cycle;
  g_M = (cpx *)calloc((size_t)g_nc * P, sizeof(cpx));
  g_L = (cpx *)calloc((size_t)g_nc * P, sizeof(cpx));
  upward(0);
  /* 2dp/traverse_lazy.h:124-141 horizontalPass: one walk per image of the
   * first shell (iX0 outer, iX1 inner), or the plain walk */
  if (images == 0) {
    g_iX[0] = g_iX[1] = 0;
    get_list(0, 0);
  } else {
    for (g_iX[0] = -1; g_iX[0] <= 1; g_iX[0]++)
      for (g_iX[1] = -1; g_iX[1] <= 1; g_iX[1]++) get_list(0, 0);
  }
  /* 2d/traverse_lazy.h:45-56 evaluate: per target cell, its M2L then its P2P
   * list, each entry at its image (2dp/traverse_lazy.h:54-65) */
  for (long c = 0; c < g_nc; c++) {
    for (int k = 0; k < g_c[c].nm2l; k += 2) {
      g_iX[0] = g_c[c].m2l[k + 1] % 3 - 1;
      g_iX[1] = g_c[c].m2l[k + 1] / 3 - 1;
      m2l(c, g_c[c].m2l[k]);
    }
    for (int k = 0; k < g_c[c].np2p; k += 2) {
      const Cell2 *S = &g_c[g_c[c].p2p[k]];
      g_iX[0] = g_c[c].p2p[k + 1] % 3 - 1;
      g_iX[1] = g_c[c].p2p[k + 1] / 3 - 1;
      p2p(g_b + g_c[c].body, g_c[c].nbody, g_b + S->body, S->nbody);
    }
  }
  if (images > 0) periodic();
  g_cycle = cycle;
  downward(0);
  return g_nc;
}

void orc2_get_bodies(double *out) {
  for (long b = 0; b < g_n; b++) {
    double *o = out + 6 * b;
    o[0] = g_b[b].X[0];
    o[1] = g_b[b].X[1];
    o[2] = g_b[b].q;
    o[3] = g_b[b].p;
    o[4] = g_b[b].F[0];
    o[5] = g_b[b].F[1];
  }
}

void orc2_get_cells(int *nchild, int *child, int *body, int *nbody, double *xr) {
  for (long c = 0; c < g_nc; c++) {
    nchild[c] = g_c[c].nchild;
    child[c] = g_c[c].child;
    body[c] = g_c[c].body;
    nbody[c] = g_c[c].nbody;
    xr[3 * c] = g_c[c].X[0];
    xr[3 * c + 1] = g_c[c].X[1];
    xr[3 * c + 2] = g_c[c].R;
  }
}

void orc2_count_lists(long *nm2l, long *np2p) {
  *nm2l = *np2p = 0;
  for (long c = 0; c < g_nc; c++) {
    *nm2l += g_c[c].nm2l / 2;
    *np2p += g_c[c].np2p / 2;
  }
}

void orc2_get_lists(int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src, int *p2p_img) {
  int a = 0, b = 0;
  for (long c = 0; c < g_nc; c++) {
    m2l_off[c] = a;
    p2p_off[c] = b;
    for (int k = 0; k < g_c[c].nm2l; k += 2, a++) {
      m2l_src[a] = g_c[c].m2l[k];
      m2l_img[a] = g_c[c].m2l[k + 1];
    }
    for (int k = 0; k < g_c[c].np2p; k += 2, b++) {
      p2p_src[b] = g_c[c].p2p[k];
      p2p_img[b] = g_c[c].p2p[k + 1];
    }
  }
  m2l_off[g_nc] = a;
  p2p_off[g_nc] = b;
}

void orc2_get_expansions(double *M, double *L) {
  memcpy(M, g_M, sizeof(cpx) * g_nc * g_P);
  memcpy(L, g_L, sizeof(cpx) * g_nc * g_P);
}

/* 2d/traverse_lazy.h:84-94 direct; 2dp/traverse_lazy.h:154-175 over the
 * (2 prange + 1)^2 images, prange = sum_{i < images} 3^i (ix outer) */
void orc2_direct(long nt, double *t6, long ns, const double *s6, int images, double cycle) {
  Body2 *T = (Body2 *)malloc(sizeof(Body2) * nt), *S = (Body2 *)malloc(sizeof(Body2) * ns);
  memcpy(T, t6, sizeof(Body2) * nt);
  memcpy(S, s6, sizeof(Body2) * ns);
  int prange = 0;
  for (int i = 0, p3 = 1; i < images; i++, p3 *= 3) prange += p3;
  const double save = g_cycle;
  g_cycle = cycle;
  for (int ix = -prange; ix <= prange; ix++)
    for (int iy = -prange; iy <= prange; iy++) {
      g_iX[0] = ix;
      g_iX[1] = iy;
      p2p(T, nt, S, ns);
    }
  g_cycle = save;
  memcpy(t6, T, sizeof(Body2) * nt);
  free(T);
  free(S);
}

void orc2_reference_bodies(long n, long seed, double *xyq) {
  srand48(seed);
  double avg = 0;
  for (long b = 0; b < n; b++) {
    for (int d = 0; d < 2; d++) xyq[3 * b + d] = drand48() * 2 * M_PI - M_PI;
    xyq[3 * b + 2] = drand48() - .5;
    avg += xyq[3 * b + 2];
  }
  avg /= n;
  for (long b = 0; b < n; b++) xyq[3 * b + 2] -= avg;
}
