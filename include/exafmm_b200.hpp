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
 *   start(event), stop(event) wall-clock timers printing as 3d/timer.h does
 *
 * Differences, by design: the handle keeps its own copy of the bodies from
 * buildTree (the passes do not read the caller's vector again); Cell::M and
 * Cell::L are filled after downwardPass only when `keep_expansions` is set
 * (they are large and no driver reads them); the operator-level kernels
 * (P2M(Cell*), M2L(Cell*, Cell*), ...) and the periodic Ewald parts
 * (wavePart, realPart, selfTerm) are not provided -- the GPU runs whole
 * passes, and exafmm_b200_ewald() sums all Ewald parts at once.  Errors of
 * the C ABI are thrown as exafmm::Error.
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

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

namespace shim {

inline exafmm_params params() {
  exafmm_params p;
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
