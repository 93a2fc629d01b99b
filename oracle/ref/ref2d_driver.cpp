// Test infrastructure only: a C-ABI wrapper around the reference's OWN 2d or
// 2dp headers (minimal ExaFMM `2d/` / `2dp/` with REF_PERIODIC, lazy
// traversal), compiled from where they lie by oracle/Makefile into
// oracle/_ref/libref2d_lazy.so and libref2dp_lazy.so.  Nothing here restates
// the algorithm: it calls the reference's buildTree / upwardPass /
// horizontalPass / downwardPass / direct and copies the results out for the
// 2D oracle's parity tests and fixtures.  The product library never links it.
#ifndef REF_PERIODIC
#define REF_PERIODIC 0
#endif
#include <cstring>
#include <omp.h>

#include "build_tree.h"
#include "kernel.h"
#include "traverse_lazy.h"

using namespace exafmm;

namespace {
Bodies g_bodies;
Cells g_cells;

void load(long n, const double *xyq) {
  g_bodies.assign(n, Body());
  for (long b = 0; b < n; b++) {
    g_bodies[b].X[0] = xyq[3 * b];
    g_bodies[b].X[1] = xyq[3 * b + 1];
    g_bodies[b].q = xyq[3 * b + 2];
    g_bodies[b].p = 0;
    g_bodies[b].F[0] = g_bodies[b].F[1] = 0;
  }
}

void to6(const Body &b, double *o) {
  o[0] = b.X[0];
  o[1] = b.X[1];
  o[2] = b.q;
  o[3] = b.p;
  o[4] = b.F[0];
  o[5] = b.F[1];
}
}  // namespace

extern "C" {

void ref2_set_threads(int n) { omp_set_num_threads(n); }

long ref2_tree(long n, const double *xyq, int nc) {
  ncrit = nc;
  load(n, xyq);
  g_cells = buildTree(g_bodies);
  return (long)g_cells.size();
}

long ref2_fmm(long n, const double *xyq, int p, int nc, double th, int img, double cyc) {
  P = p;
  theta = th;
#if REF_PERIODIC
  images = img;
  cycle = cyc;
#else
  if (img != 0) return -1;  // free-space build
  (void)cyc;
#endif
  ref2_tree(n, xyq, nc);
  upwardPass(g_cells);
  horizontalPass(g_cells, g_cells);
  downwardPass(g_cells);
  return (long)g_cells.size();
}

void ref2_get_bodies(double *out) {
  for (size_t b = 0; b < g_bodies.size(); b++) to6(g_bodies[b], out + 6 * b);
}

void ref2_get_cells(int *nchild, int *child, int *body, int *nbody, double *xr) {
  for (size_t c = 0; c < g_cells.size(); c++) {
    const Cell &C = g_cells[c];
    nchild[c] = C.NCHILD;
    child[c] = C.NCHILD ? (int)(C.CHILD - &g_cells[0]) : -1;
    body[c] = (int)(C.BODY - &g_bodies[0]);
    nbody[c] = C.NBODY;
    xr[3 * c] = C.X[0];
    xr[3 * c + 1] = C.X[1];
    xr[3 * c + 2] = C.R;
  }
}

void ref2_count_lists(long *nm2l, long *np2p) {
  *nm2l = *np2p = 0;
  for (const Cell &C : g_cells) {
    *nm2l += (long)C.listM2L.size();
    *np2p += (long)C.listP2P.size();
  }
}

void ref2_get_lists(int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src, int *p2p_img) {
  int a = 0, b = 0;
  for (size_t c = 0; c < g_cells.size(); c++) {
    const Cell &C = g_cells[c];
    m2l_off[c] = a;
    p2p_off[c] = b;
    for (size_t k = 0; k < C.listM2L.size(); k++, a++) {
      m2l_src[a] = (int)(C.listM2L[k] - &g_cells[0]);
#if REF_PERIODIC
      m2l_img[a] = C.periodicM2L[k];
#else
      m2l_img[a] = 4;  // the central image
#endif
    }
    for (size_t k = 0; k < C.listP2P.size(); k++, b++) {
      p2p_src[b] = (int)(C.listP2P[k] - &g_cells[0]);
#if REF_PERIODIC
      p2p_img[b] = C.periodicP2P[k];
#else
      p2p_img[b] = 4;
#endif
    }
  }
  m2l_off[g_cells.size()] = a;
  p2p_off[g_cells.size()] = b;
}

void ref2_get_expansions(double *M, double *L) {
  for (size_t c = 0; c < g_cells.size(); c++) {
    std::memcpy(M + 2 * P * c, g_cells[c].M.data(), sizeof(complex_t) * P);
    std::memcpy(L + 2 * P * c, g_cells[c].L.data(), sizeof(complex_t) * P);
  }
}

// one thread: the periodic direct sum adds the images in parallel otherwise,
// and its summation order (ix outer, iy inner) is only fixed on one thread
void ref2_direct(long nt, double *t6, long ns, const double *s6, int img, double cyc) {
#if REF_PERIODIC
  images = img;
  cycle = cyc;
#else
  (void)img;
  (void)cyc;
#endif
  const int threads = omp_get_max_threads();
  omp_set_num_threads(1);
  Bodies t(nt), s(ns);
  for (long i = 0; i < nt; i++) {
    t[i].X[0] = t6[6 * i];
    t[i].X[1] = t6[6 * i + 1];
    t[i].q = t6[6 * i + 2];
    t[i].p = t6[6 * i + 3];
    t[i].F[0] = t6[6 * i + 4];
    t[i].F[1] = t6[6 * i + 5];
  }
  for (long j = 0; j < ns; j++) {
    s[j].X[0] = s6[6 * j];
    s[j].X[1] = s6[6 * j + 1];
    s[j].q = s6[6 * j + 2];
    s[j].p = s[j].F[0] = s[j].F[1] = 0;
  }
  direct(t, s);
  omp_set_num_threads(threads);
  for (long i = 0; i < nt; i++) to6(t[i], t6 + 6 * i);
}
}
