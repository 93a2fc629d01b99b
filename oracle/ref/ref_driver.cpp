// Test infrastructure only: a C-ABI wrapper around the reference's OWN headers
// (minimal ExaFMM `3d/` or `3dp/`), compiled from where they lie by
// oracle/Makefile into oracle/_ref/.  Nothing here restates the algorithm; it
// calls the reference's buildTree / upwardPass / getList / evaluate /
// horizontalPass / downwardPass / direct / Ewald functions and copies their
// results out for the parity tests, the golden-fixture generator and the CPU
// baseline leg of bench.py.  The product library never links this file.
//
// Build-time macros: REF_PERIODIC (3dp headers), EXAFMM_LAZY or EXAFMM_EAGER.
#ifndef REF_PERIODIC
#define REF_PERIODIC 0
#endif
#include <chrono>
#include <cmath>
#include <cstring>
#include <omp.h>
#include "build_tree.h"
#include "kernel.h"
#if REF_PERIODIC
#include "ewald.h"
#endif
#if EXAFMM_EAGER
#include "traverse_eager.h"
#else
#include "traverse_lazy.h"
#endif
#include "timer.h"
#include "test_kernel.h"
#if EXAFMM_EAGER && !REF_PERIODIC
#include "test_fmm.h"
#endif

using namespace exafmm;

#if !REF_PERIODIC
// 3d has no periodic globals; keep one driver body for both variants.
static int images = 0;
static double cycle = 0;
#endif

namespace {
Bodies g_bodies;
Cells g_cells;
double g_times[8];

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void load_bodies(long n, const double *xq) {
  g_bodies.assign(n, Body());
  for (long b = 0; b < n; b++) {
    for (int d = 0; d < 3; d++) g_bodies[b].X[d] = xq[4 * b + d];
    g_bodies[b].q = xq[4 * b + 3];
    g_bodies[b].p = 0;
    for (int d = 0; d < 3; d++) g_bodies[b].F[d] = 0;
  }
}
}  // namespace

extern "C" {

// 0 = 3d, 1 = 3dp; +2 when built lazy (lists available).
int ref_variant() {
  int v = REF_PERIODIC ? 1 : 0;
#if EXAFMM_LAZY
  v += 2;
#endif
  return v;
}

void ref_set_threads(int n) { omp_set_num_threads(n); }
int ref_max_threads() { return omp_get_max_threads(); }

// Build the tree only (buildTree).  Returns the number of cells.
long ref_build_tree(long n, const double *xq, int nc) {
  ncrit = nc;
  load_bodies(n, xq);
  g_cells = buildTree(g_bodies);
  return (long)g_cells.size();
}

// Full evaluation on n bodies (xq: x,y,z,q per body).  phases bit 0: run the
// far field + near field (upward, horizontal, downward); bit 1: only build the
// tree and the lists (lazy builds only).  Timings (s) land in g_times:
// [tree, upward, lists, evaluate(M2L+P2P), downward, total].
long ref_fmm(long n, const double *xq, int p, int nc, double th, int img, double cyc, int phases) {
  P = p;
  ncrit = nc;
  theta = th;
  images = img;
  cycle = cyc;
  std::memset(g_times, 0, sizeof(g_times));
  load_bodies(n, xq);
  double t0 = now();
  g_cells = buildTree(g_bodies);
  double t1 = now();
  initKernel();
  if (phases & 2) {
#if EXAFMM_LAZY
    for (auto &c : g_cells) { c.M.resize(NTERM, 0.0); c.L.resize(NTERM, 0.0); }
#if REF_PERIODIC
    if (images == 0) {
      iX[0] = iX[1] = iX[2] = 0;
      getList(&g_cells[0], &g_cells[0]);
    } else {
      for (iX[0] = -1; iX[0] <= 1; iX[0]++)
        for (iX[1] = -1; iX[1] <= 1; iX[1]++)
          for (iX[2] = -1; iX[2] <= 1; iX[2]++) getList(&g_cells[0], &g_cells[0]);
    }
#else
    getList(&g_cells[0], &g_cells[0]);
#endif
#endif
    g_times[0] = t1 - t0;
    return (long)g_cells.size();
  }
  upwardPass(g_cells);
  double t2 = now();
#if EXAFMM_LAZY && !REF_PERIODIC
  getList(&g_cells[0], &g_cells[0]);
  double t3 = now();
  evaluate(g_cells);
  double t4 = now();
#else
  double t3 = t2;
  horizontalPass(g_cells, g_cells);
  double t4 = now();
#endif
  downwardPass(g_cells);
  double t5 = now();
  g_times[0] = t1 - t0;
  g_times[1] = t2 - t1;
  g_times[2] = t3 - t2;
  g_times[3] = t4 - t3;
  g_times[4] = t5 - t4;
  g_times[5] = t5 - t0;
  return (long)g_cells.size();
}

void ref_get_times(double *t) { std::memcpy(t, g_times, sizeof(g_times)); }

// Bodies in tree order: X[3], q, p, F[3] per body.
void ref_get_bodies(double *out) {
  for (size_t b = 0; b < g_bodies.size(); b++) {
    const Body &B = g_bodies[b];
    double *o = out + 8 * b;
    o[0] = B.X[0]; o[1] = B.X[1]; o[2] = B.X[2]; o[3] = B.q;
    o[4] = B.p; o[5] = B.F[0]; o[6] = B.F[1]; o[7] = B.F[2];
  }
}

// Cell table in the reference's own order: NCHILD, first-child index,
// first-body index, NBODY; centre and radius as X[3], R.
void ref_get_cells(int *nchild, int *child, int *body, int *nbody, double *xr) {
  for (size_t c = 0; c < g_cells.size(); c++) {
    const Cell &C = g_cells[c];
    nchild[c] = C.NCHILD;
    child[c] = C.NCHILD ? (int)(C.CHILD - &g_cells[0]) : -1;
    body[c] = (int)(C.BODY - &g_bodies[0]);
    nbody[c] = C.NBODY;
    for (int d = 0; d < 3; d++) xr[4 * c + d] = C.X[d];
    xr[4 * c + 3] = C.R;
  }
}

// Multipole/local coefficients (complex, interleaved re/im), NTERM per cell.
void ref_get_expansions(double *M, double *L) {
  for (size_t c = 0; c < g_cells.size(); c++) {
    for (int t = 0; t < NTERM; t++) {
      complex_t m = t < (int)g_cells[c].M.size() ? g_cells[c].M[t] : 0.0;
      complex_t l = t < (int)g_cells[c].L.size() ? g_cells[c].L[t] : 0.0;
      M[2 * (c * NTERM + t)] = m.real(); M[2 * (c * NTERM + t) + 1] = m.imag();
      L[2 * (c * NTERM + t)] = l.real(); L[2 * (c * NTERM + t) + 1] = l.imag();
    }
  }
}

#if EXAFMM_LAZY
void ref_count_lists(long *nm2l, long *np2p) {
  long a = 0, b = 0;
  for (auto &c : g_cells) { a += c.listM2L.size(); b += c.listP2P.size(); }
  *nm2l = a;
  *np2p = b;
}

// Per-target lists in recording order as CSR (offsets have ncells+1 entries).
// img is the 3dp periodic index periodic1D(iX) (13 = no shift) or 13 for 3d.
void ref_get_lists(int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src, int *p2p_img) {
  long a = 0, b = 0;
  for (size_t c = 0; c < g_cells.size(); c++) {
    const Cell &C = g_cells[c];
    m2l_off[c] = (int)a;
    p2p_off[c] = (int)b;
    for (size_t j = 0; j < C.listM2L.size(); j++, a++) {
      m2l_src[a] = (int)(C.listM2L[j] - &g_cells[0]);
#if REF_PERIODIC
      m2l_img[a] = C.periodicM2L[j];
#else
      m2l_img[a] = 13;
#endif
    }
    for (size_t j = 0; j < C.listP2P.size(); j++, b++) {
      p2p_src[b] = (int)(C.listP2P[j] - &g_cells[0]);
#if REF_PERIODIC
      p2p_img[b] = C.periodicP2P[j];
#else
      p2p_img[b] = 13;
#endif
    }
  }
  m2l_off[g_cells.size()] = (int)a;
  p2p_off[g_cells.size()] = (int)b;
}
#endif

// Reference direct() (free space): targets/sources as 8 doubles per body;
// accumulates into the targets' p and F.
void ref_direct(long nt, double *targets, long ns, const double *sources) {
  Bodies t(nt), s(ns);
  for (long i = 0; i < nt; i++) std::memcpy(&t[i], targets + 8 * i, sizeof(Body));
  for (long j = 0; j < ns; j++) std::memcpy(&s[j], sources + 8 * j, sizeof(Body));
#if REF_PERIODIC
  int saved = images;
  images = 0;  // the periodic direct() races across images; keep it to one image
  iX[0] = iX[1] = iX[2] = 0;
  direct(t, s);
  images = saved;
#else
  direct(t, s);
#endif
  for (long i = 0; i < nt; i++) std::memcpy(targets + 8 * i, &t[i], sizeof(Body));
}

#if REF_PERIODIC
// Dipole correction exactly as the 3dp driver applies it (3dp/fmm.cxx:63-75),
// on the bodies of the last ref_fmm call.
void ref_dipole_correction() {
  real_t dipole[3] = {0, 0, 0};
  for (size_t b = 0; b < g_bodies.size(); b++)
    for (int d = 0; d < 3; d++) dipole[d] += g_bodies[b].X[d] * g_bodies[b].q;
  real_t coef = 4 * M_PI / (3 * cycle * cycle * cycle);
  for (size_t b = 0; b < g_bodies.size(); b++) {
    real_t dnorm = dipole[0] * dipole[0] + dipole[1] * dipole[1] + dipole[2] * dipole[2];
    g_bodies[b].p -= coef * dnorm / g_bodies.size() / g_bodies[b].q;
    for (int d = 0; d != 3; d++) g_bodies[b].F[d] -= coef * dipole[d];
  }
}

// Ewald sum (wavePart + realPart + selfTerm) of the bodies of the last
// ref_fmm call, as the 3dp driver runs it (3dp/fmm.cxx:77-94).  Writes
// 8 doubles per body (X,q,p,F) in the same (tree) order into out.
void ref_ewald(int ks, double alph, double sig, double cut, double *out) {
  ksize = ks;
  alpha = alph;
  sigma = sig;
  cutoff = cut;
  Bodies jbodies = g_bodies;
  for (auto &B : jbodies) { B.p = 0; for (int d = 0; d < 3; d++) B.F[d] = 0; }
  Cells jcells = buildTree(jbodies);
  // realPart walks the FMM tree, whose BODY pointers alias g_bodies: swap the
  // zeroed copy in so the result lands there, then restore.
  Bodies saved = g_bodies;
  for (auto &B : g_bodies) { B.p = 0; for (int d = 0; d < 3; d++) B.F[d] = 0; }
  wavePart(g_bodies, jbodies);
  realPart(&g_cells[0], &jcells[0]);
  selfTerm(g_bodies);
  for (size_t b = 0; b < g_bodies.size(); b++) {
    const Body &B = g_bodies[b];
    double *o = out + 8 * b;
    o[0] = B.X[0]; o[1] = B.X[1]; o[2] = B.X[2]; o[3] = B.q;
    o[4] = B.p; o[5] = B.F[0]; o[6] = B.F[1]; o[7] = B.F[2];
  }
  g_bodies = saved;
}
#endif

// The reference's own known-answer tests, compiled unmodified from test/:
// test_kernel(p) (operator chain P2M->M2M->M2L->L2L->L2P vs P2P, relative
// potential error) and, in eager builds, test_fmm(p) (10,000-body FMM vs
// direct on 10 targets, relative potential error).
double ref_test_kernel(int p) { return test_kernel(p); }
#if EXAFMM_EAGER && !REF_PERIODIC
double ref_test_fmm(int p) { return test_fmm(p); }
#endif

}  // extern "C"
