/* C++ names of minimal ExaFMM's driver API on top of the exafmm_b200 C ABI.
 *
 * The reference's "API" is a set of header-inlined functions and globals in
 * namespace exafmm (3d/exafmm.h:8-44, 3d/build_tree.h:88-96,
 * 3d/kernel.h:118-120, 3d/traverse_eager.h:140-202, 3d/timer.h:9-22) that its
 * drivers call: 3d/fmm.cxx and test/test_fmm.h.  This header gives the same
 * names, types and call sequence, backed by one exafmm_b200 handle per
 * process, so those drivers compile unchanged: put include/exafmm_shim/ (its
 * files are named like the reference's headers and include this one) and
 * include/ on the include path, and link -lexafmm_b200.
 *
 *   Body, Bodies, Cell, Cells, real_t, complex_t   as in 3d/exafmm.h
 *   P, NTERM, ncrit, theta (+ images, cycle)        globals read at buildTree
 *   buildTree(bodies)       uploads the bodies, builds the octree on the GPU,
 *                           permutes `bodies` into tree order in place and
 *                           returns the cells (reference cell order; CHILD and
 *                           BODY point into the returned vector and `bodies`)
 *   initKernel()            NTERM = P(P+1)/2
 *   upwardPass(cells)       P2M + M2M on the GPU
 *   horizontalPass(ci, cj)  interaction lists + M2L + P2P on the GPU
 *   downwardPass(cells)     L2L + L2P on the GPU; p and F are added into the
 *                           bodies given to buildTree (the reference
 *                           accumulates, callers zero them first)
 *   direct(targets, sources) FP64 direct sum on the GPU, added into targets
 *   P2P(Ci, Cj), P2M(C), M2M(Ci), M2L(Ci, Cj), L2L(Cj), L2P(C)
 *                           the single operators of 3d/kernel.h:122-323 on the
 *                           GPU (exafmm_b200_p2p ...), for drivers that call
 *                           them one by one (3d/kernel.cxx, test/test_kernel.h);
 *                           the 3dp shift iX * cycle is applied to P2P and M2L
 *   wavePart(bodies, jbodies), realPart(Ci, Cj), selfTerm(bodies)
 *                           the Ewald parts of 3dp/ewald.h:122-150 on the GPU
 *                           (exafmm_b200_ewald_parts), with the globals ksize,
 *                           alpha, sigma, cutoff
 *   start(event), stop(event) wall-clock timers printing as 3d/timer.h does
 *
 * Differences, by design: the handle keeps its own copy of the bodies from
 * buildTree (the passes do not read the caller's vector again); Cell::M and
 * Cell::L are filled after downwardPass only when `keep_expansions` is set
 * (they are large and no driver reads them); the single operators run on a
 * second handle, so they never disturb the tree of the first; realPart takes
 * each source at its nearest periodic image inside the cutoff (the
 * reference's neighbour search picks one image per pair of cells).  Errors
 * of the C ABI are thrown as exafmm::Error.
 */
#ifndef EXAFMM_B200_HPP
#define EXAFMM_B200_HPP

#include <chrono>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "exafmm_b200.h"

namespace exafmm {

typedef double real_t;
typedef std::complex<real_t> complex_t;

// 8 doubles, the record the C ABI takes (3d/exafmm.h:14-19)
struct Body {
  real_t X[3];
  real_t q;
  real_t p;
  real_t F[3];
};
typedef std::vector<Body> Bodies;

struct Cell {
  int NCHILD;
  int NBODY;
  Cell *CHILD;  // first child (nullptr for a leaf)
  Body *BODY;   // first body, in the tree-ordered bodies
  real_t X[3];
  real_t R;
  std::vector<complex_t> M;  // filled by downwardPass with keep_expansions
  std::vector<complex_t> L;
};
typedef std::vector<Cell> Cells;

// globals of 3d/exafmm.h:39-42, the periodic ones of 3dp/exafmm.h, and the
// two choices the GPU adds (FP64 is the drop-in form)
inline int P = 10;
inline int NTERM = 0;
inline int ncrit = 64;
inline real_t theta = 0.4;
inline int images = 0;
inline real_t cycle = 0;
inline int precision = EXAFMM_FP64;
inline int device = 0;
inline bool keep_expansions = false;
// 3dp: the periodic image of the current P2P / M2L source (3dp/exafmm.h:46)
// and the Ewald parameters (3dp/ewald.h:13-16)
inline int iX[3] = {0, 0, 0};
inline int ksize = 0;
inline real_t alpha = 0;
inline real_t sigma = 0;
inline real_t cutoff = 0;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

namespace shim {

inline exafmm_params params() {
  exafmm_params p{};
  p.dim = 3;
  p.P = P;
  p.ncrit = ncrit;
  p.theta = theta;
  p.images = images;
  p.cycle = cycle;
  p.precision = precision;
  p.device = device;
  return p;
}

inline void check(int rc, exafmm_b200 *h) {
  if (rc != EXAFMM_OK) throw Error(rc, std::string("exafmm_b200: ") + exafmm_b200_last_error(h));
}

inline exafmm_b200 *create() {
  const exafmm_params p = params();
  exafmm_b200 *h = nullptr;
  const int rc = exafmm_b200_create(&p, &h);
  if (rc != EXAFMM_OK) throw Error(rc, std::string("exafmm_b200: ") + exafmm_b200_last_error(nullptr));
  return h;
}

// the process's handle and the bodies the current tree was built from
struct State {
  exafmm_b200 *h = nullptr;
  Bodies *bodies = nullptr;
  ~State() {
    if (h) exafmm_b200_destroy(h);
  }
};
inline State &state() {
  static State s;
  return s;
}

inline exafmm_b200 *handle() {
  State &s = state();
  if (!s.h) {
    s.h = create();
  } else {
    const exafmm_params p = params();
    check(exafmm_b200_set_params(s.h, &p), s.h);
  }
  return s.h;
}

inline exafmm_b200 *current() {
  if (!state().h || !state().bodies) throw Error(EXAFMM_ERR_STATE, "exafmm: buildTree() has not run");
  return state().h;
}

// The handle of the single operators and the self term (no bodies needed):
// its own, so that they never reset the tree of the handle above.
struct OpState {
  exafmm_b200 *h = nullptr;
  exafmm_params prm{};
  ~OpState() {
    if (h) exafmm_b200_destroy(h);
  }
};
inline exafmm_b200 *op_handle() {
  static OpState s;
  const exafmm_params p = params();
  if (!s.h) {
    s.h = create();
  } else if (p.P != s.prm.P || p.images != s.prm.images || p.cycle != s.prm.cycle || p.precision != s.prm.precision) {
    check(exafmm_b200_set_params(s.h, &p), s.h);
  }
  s.prm = p;
  return s.h;
}

inline void cell4(const Cell *c, double *x) {
  for (int d = 0; d < 3; d++) x[d] = c->X[d];
  x[3] = c->R;
}

// the 3dp source shift iX * cycle (3dp/kernel.h:133, :200)
inline const double *image_shift(double *s) {
  for (int d = 0; d < 3; d++) s[d] = iX[d] * cycle;
  return s;
}

inline complex_t *terms(std::vector<complex_t> &v, const char *what) {
  if (v.size() < (size_t)(P * (P + 1) / 2))
    throw Error(EXAFMM_ERR_ARG, std::string("exafmm: ") + what + " needs NTERM coefficients (resize it first)");
  return v.data();
}

}  // namespace shim

inline Cells buildTree(Bodies &bodies) {
  exafmm_b200 *h = shim::handle();
  const int64_t n = (int64_t)bodies.size();
  shim::check(exafmm_b200_set_bodies(h, (const double *)bodies.data(), n, EXAFMM_HOST), h);
  shim::check(exafmm_b200_build_tree(h), h);
  // bodies into tree order, as the reference's in-place partition leaves them
  std::vector<int64_t> perm(n);
  shim::check(exafmm_b200_get_perm(h, perm.data(), EXAFMM_HOST), h);
  const Bodies in(bodies);
  for (int64_t i = 0; i < n; i++) bodies[i] = in[perm[i]];
  // cells in the reference's order
  const int64_t C = exafmm_b200_num_cells(h);
  if (C <= 0) throw Error(EXAFMM_ERR_STATE, "exafmm: no cells after buildTree()");
  std::vector<int> nchild(C), child(C), body(C), nbody(C), level(C);
  std::vector<double> xr(4 * C);
  shim::check(exafmm_b200_get_tree(h, nchild.data(), child.data(), body.data(), nbody.data(), level.data(),
                                   xr.data()),
              h);
  Cells cells(C);
  for (int64_t c = 0; c < C; c++) {
    Cell &cell = cells[c];
    cell.NCHILD = nchild[c];
    cell.NBODY = nbody[c];
    cell.CHILD = child[c] >= 0 ? &cells[child[c]] : nullptr;
    cell.BODY = bodies.data() + body[c];
    for (int d = 0; d < 3; d++) cell.X[d] = xr[4 * c + d];
    cell.R = xr[4 * c + 3];
  }
  shim::state().bodies = &bodies;
  return cells;
}

inline void initKernel() { NTERM = P * (P + 1) / 2; }

inline void upwardPass(Cells &) {
  exafmm_b200 *h = shim::current();
  shim::check(exafmm_b200_upward(h), h);
}

inline void horizontalPass(Cells &, Cells &) {
  exafmm_b200 *h = shim::current();
  shim::check(exafmm_b200_horizontal(h), h);
}

inline void downwardPass(Cells &cells) {
  exafmm_b200 *h = shim::current();
  shim::check(exafmm_b200_downward(h), h);
  Bodies &bodies = *shim::state().bodies;
  Bodies out(bodies.size());
  shim::check(exafmm_b200_get_bodies(h, (double *)out.data(), EXAFMM_HOST), h);
  for (size_t i = 0; i < bodies.size(); i++) {
    bodies[i].p += out[i].p;
    for (int d = 0; d < 3; d++) bodies[i].F[d] += out[i].F[d];
  }
  if (keep_expansions) {
    const size_t nt = (size_t)P * (P + 1) / 2;
    std::vector<complex_t> M(cells.size() * nt), L(cells.size() * nt);
    shim::check(exafmm_b200_get_expansions(h, (double *)M.data(), (double *)L.data()), h);
    for (size_t c = 0; c < cells.size(); c++) {
      cells[c].M.assign(M.begin() + c * nt, M.begin() + (c + 1) * nt);
      cells[c].L.assign(L.begin() + c * nt, L.begin() + (c + 1) * nt);
    }
  }
}

// a handle of its own holds the sources, so the FMM handle keeps its tree
inline void direct(Bodies &targets, Bodies &sources) {
  if (targets.empty() || sources.empty()) return;
  exafmm_b200 *h = shim::create();
  try {
    shim::check(exafmm_b200_set_bodies(h, (const double *)sources.data(), (int64_t)sources.size(), EXAFMM_HOST), h);
    shim::check(exafmm_b200_build_tree(h), h);
    shim::check(exafmm_b200_direct(h, (double *)targets.data(), (int64_t)targets.size(), EXAFMM_HOST), h);
  } catch (...) {
    exafmm_b200_destroy(h);
    throw;
  }
  exafmm_b200_destroy(h);
}

// ---- single operators (3d/kernel.h:122-323)
inline void P2P(Cell *Ci, Cell *Cj) {
  exafmm_b200 *h = shim::op_handle();
  double s[3];
  shim::check(exafmm_b200_p2p(h, (double *)Ci->BODY, Ci->NBODY, (const double *)Cj->BODY, Cj->NBODY,
                              shim::image_shift(s), EXAFMM_HOST),
              h);
}

inline void P2M(Cell *C) {
  exafmm_b200 *h = shim::op_handle();
  double c[4];
  shim::cell4(C, c);
  shim::check(exafmm_b200_p2m(h, c, (const double *)C->BODY, C->NBODY, (double *)shim::terms(C->M, "P2M: Cell::M"),
                              EXAFMM_HOST),
              h);
}

inline void M2M(Cell *Ci) {
  exafmm_b200 *h = shim::op_handle();
  const size_t nt = (size_t)P * (P + 1) / 2;
  double c[4];
  shim::cell4(Ci, c);
  std::vector<double> kids(4 * (size_t)Ci->NCHILD);
  std::vector<complex_t> Mk(nt * Ci->NCHILD);
  for (int k = 0; k < Ci->NCHILD; k++) {
    Cell *Cj = Ci->CHILD + k;
    shim::cell4(Cj, &kids[4 * k]);
    const complex_t *m = shim::terms(Cj->M, "M2M: child Cell::M");
    for (size_t t = 0; t < nt; t++) Mk[k * nt + t] = m[t];
  }
  shim::check(exafmm_b200_m2m(h, c, (double *)shim::terms(Ci->M, "M2M: Cell::M"), Ci->NCHILD, kids.data(),
                              (const double *)Mk.data(), EXAFMM_HOST),
              h);
}

inline void M2L(Cell *Ci, Cell *Cj) {
  exafmm_b200 *h = shim::op_handle();
  double ci[4], cj[4], s[3];
  shim::cell4(Ci, ci);
  shim::cell4(Cj, cj);
  shim::check(exafmm_b200_m2l(h, ci, (double *)shim::terms(Ci->L, "M2L: Cell::L"), cj,
                              (const double *)shim::terms(Cj->M, "M2L: Cell::M"), shim::image_shift(s), EXAFMM_HOST),
              h);
}

inline void L2L(Cell *Cj) {
  exafmm_b200 *h = shim::op_handle();
  const size_t nt = (size_t)P * (P + 1) / 2;
  double c[4];
  shim::cell4(Cj, c);
  std::vector<double> kids(4 * (size_t)Cj->NCHILD);
  std::vector<complex_t> Lk(nt * Cj->NCHILD);
  for (int k = 0; k < Cj->NCHILD; k++) {
    Cell *Ci = Cj->CHILD + k;
    shim::cell4(Ci, &kids[4 * k]);
    const complex_t *l = shim::terms(Ci->L, "L2L: child Cell::L");
    for (size_t t = 0; t < nt; t++) Lk[k * nt + t] = l[t];
  }
  shim::check(exafmm_b200_l2l(h, c, (const double *)shim::terms(Cj->L, "L2L: Cell::L"), Cj->NCHILD, kids.data(),
                              (double *)Lk.data(), EXAFMM_HOST),
              h);
  for (int k = 0; k < Cj->NCHILD; k++)
    for (size_t t = 0; t < nt; t++) Cj->CHILD[k].L[t] = Lk[k * nt + t];
}

inline void L2P(Cell *Ci) {
  exafmm_b200 *h = shim::op_handle();
  double c[4];
  shim::cell4(Ci, c);
  shim::check(exafmm_b200_l2p(h, c, (const double *)shim::terms(Ci->L, "L2P: Cell::L"), (double *)Ci->BODY,
                              Ci->NBODY, EXAFMM_HOST),
              h);
}

// ---- Ewald parts (3dp/ewald.h:122-150): sources on a handle of their own
namespace shim {
inline void ewald_part(int part, const Body *sources, int64_t ns, Body *targets, int64_t nt) {
  if (nt <= 0) return;
  exafmm_b200 *h = create();
  try {
    check(exafmm_b200_set_bodies(h, (const double *)sources, ns, EXAFMM_HOST), h);
    check(exafmm_b200_build_tree(h), h);
    check(exafmm_b200_ewald_parts(h, part, ksize, alpha, sigma, cutoff, (double *)targets, nt, EXAFMM_HOST), h);
  } catch (...) {
    exafmm_b200_destroy(h);
    throw;
  }
  exafmm_b200_destroy(h);
}
}  // namespace shim

inline void wavePart(Bodies &bodies, Bodies &jbodies) {
  shim::ewald_part(EXAFMM_EWALD_WAVE, jbodies.data(), (int64_t)jbodies.size(), bodies.data(), (int64_t)bodies.size());
}

inline void realPart(Cell *Ci, Cell *Cj) {
  shim::ewald_part(EXAFMM_EWALD_REAL, Cj->BODY, Cj->NBODY, Ci->BODY, Ci->NBODY);
}

inline void selfTerm(Bodies &bodies) {
  if (bodies.empty()) return;
  exafmm_b200 *h = shim::op_handle();
  shim::check(exafmm_b200_ewald_parts(h, EXAFMM_EWALD_SELF, ksize, alpha, sigma, cutoff, (double *)bodies.data(),
                                      (int64_t)bodies.size(), EXAFMM_HOST),
              h);
}

namespace shim {
inline std::map<std::string, std::chrono::steady_clock::time_point> &timers() {
  static std::map<std::string, std::chrono::steady_clock::time_point> t;
  return t;
}
}  // namespace shim

inline void start(std::string event) { shim::timers()[event] = std::chrono::steady_clock::now(); }

inline void stop(std::string event) {
  const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - shim::timers()[event]).count();
  printf("%-20s : %f s\n", event.c_str(), s);
}

}  // namespace exafmm

#endif
