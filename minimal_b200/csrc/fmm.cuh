// Internal definitions of the exafmm_b200 library: the handle, device buffer
// management, error plumbing and the launchers each .cu file provides.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/exafmm_b200.h"

namespace fmm {

typedef unsigned long long u64;
typedef unsigned int u32;

struct Error {
  int code;
  std::string msg;
};

#define FMM_CUDA(call)                                                                                     \
  do {                                                                                                     \
    cudaError_t e_ = (call);                                                                               \
    if (e_ != cudaSuccess)                                                                                 \
      throw ::fmm::Error{EXAFMM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + " at " +   \
                                              __FILE__ + ":" + std::to_string(__LINE__)};                  \
  } while (0)

#define FMM_LAUNCH()                                                                                       \
  do {                                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                                   \
    if (e_ != cudaSuccess)                                                                                 \
      throw ::fmm::Error{EXAFMM_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_) + " at " + \
                                              __FILE__ + ":" + std::to_string(__LINE__)};                  \
  } while (0)

// A device allocation that grows on demand and is kept between evaluations.
struct Buf {
  void *p = nullptr;
  size_t bytes = 0;
  template <class T>
  T *as() const { return (T *)p; }
  void need(size_t b) {
    if (b <= bytes) return;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    size_t nb = b + b / 4 + 256;
    if (cudaMalloc(&p, nb) != cudaSuccess) {
      cudaGetLastError();
      throw Error{EXAFMM_ERR_NOMEM, "cudaMalloc of " + std::to_string(nb) + " bytes failed"};
    }
    bytes = nb;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
};

// Geometry of the root cell, computed on the device (bounds kernel).
struct RootGeom {
  double X0[3];
  double R0;
};

// Counters written by device code and read once per phase by the host.
struct DevCounters {
  int ncells;          // cells in the tree
  int level_count[EXAFMM_MAX_LEVEL + 2];
  int overflow;        // a cell at the deepest key level still had > ncrit bodies
  int nleaves;
  unsigned long long n_m2l, n_p2p;  // emitted list entries (may exceed capacity)
  unsigned long long frontier[3];   // BFS pair frontier sizes (rotating over the steps)
  int list_overflow;   // an emission or the frontier exceeded its capacity
  int walk_resid;      // M2L entries the walk found without a group key
  int max_m2l_seg, max_p2p_seg;
  int gcounts[4];      // grouped M2L: residual entries, flagged targets, groups, segments
  unsigned long long gfill;
  int tc_error;        // a bounded tensor-core wait ran out
  // largest |scaled multipole| over the possible M2L sources, as the bits of
  // a non-negative double (the FP16 split's power-of-two normalisation)
  unsigned long long m16_max;
  int nghost;  // ghost sources of image entries (mixed form, periodic)
};

// Per-phase timing slots (CUDA events on the handle stream).
enum Phase { PH_TREE = 0, PH_LISTS, PH_UP, PH_M2L, PH_P2P, PH_DOWN, PH_COUNT };

struct Handle {
  exafmm_params prm{};
  int nterm = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  // a whole evaluation runs the near field on `side` (lower priority), from
  // the lists until the downward pass, beside the far field on `stream`
  cudaStream_t side = nullptr;
  // ... and the upward pass on `aux` (top priority) or `aux_lo` (one level
  // below the list build), beside the dual-tree walk
  cudaStream_t aux = nullptr, aux_lo = nullptr;
  cudaEvent_t fork_ev = nullptr, up_ev = nullptr, lists_ev = nullptr, join_ev = nullptr;
  int64_t launches = 0;

  // bodies; a batch holds nsys independent systems, system q owning input
  // bodies [sys_off[q], sys_off[q+1])
  int64_t n = 0;
  int nsys = 1;
  Buf sys_off;                        // long long [nsys + 1] (device)
  std::vector<int64_t> sys_off_host;
  Buf in;      // double4 (x,y,z,q), caller order
  Buf src;     // double4 (x,y,z,q), tree order
  Buf out;     // double4 (p,Fx,Fy,Fz), tree order
  Buf perm;    // int, tree position -> input index
  Buf srcf;    // float4 (x,y,z rel. to leaf centre, q), tree order (mixed form)
  Buf body_leaf;  // int, tree order: the leaf slot (index into `leaves`) of each body (mixed form)
  Buf l2p_f;      // mixed-form L2P: FP32 local expansions of the leaves in leaf units, then their scales
  bool srcf_ready = false;  // srcf matches the current tree
  Buf stage;   // staging for Body records crossing the boundary

  // tree build scratch
  Buf keys[2], vals[2];  // radix sort ping-pong (u64 keys, u32 values)
  Buf lfirst, chain, prebase, scan_tmp, hist;
  int key_levels = 0;

  // tree (BFS order: by level, then first body)
  int ncells = 0, nleaves = 0, depth = 0;
  int level_base[EXAFMM_MAX_LEVEL + 3] = {0};
  Buf c_begin, c_count, c_child, c_nchild, c_parent, c_level, c_xr, c_pre, c_ref, c_leaf_of_body;
  Buf leaves;  // BFS indices of leaves
  Buf pre_tmp; // preorder tables
  Buf ctmp;    // cell-count scratch (level sort, index maps)
  Buf geom;    // RootGeom
  Buf counters;  // DevCounters
  DevCounters hc{};  // host copy

  // lists (CSR by target, BFS indices)
  Buf frontier[2];
  size_t frontier_cap = 0;
  Buf m2l_raw, p2p_raw;  // emitted (tgt, src|img) pairs
  Buf m2l_key;           // group key of each raw M2L entry (-1: none)
  size_t m2l_cap = 0, p2p_cap = 0;
  Buf m2l_off, m2l_ent, p2p_off, p2p_ent, fill;
  int64_t n_m2l = 0, n_p2p = 0;
  bool m2l_ordered = false;  // m2l_off/m2l_ent built: per-target CSR in the reference's recording order

  // expansions
  Buf M, L;   // double2 [ncells][nterm]
  Buf shift_ops;   // M2M / L2L harmonics of the unit child offsets (expansions.cu)
  Buf shift_terms; // M2M / L2L term tables (expansions.cu)
  size_t shift_at[4] = {0, 0, 0, 0};  // offsets of the four term tables
  int shift_P = -1;
  Buf m2l_units;  // balanced contraction table for the M2L kernel (per P)
  int m2l_units_P = -1;

  // grouped M2L (m2l_group.cu)
  Buf g_mt, g_ekey, g_occ, g_cnt, g_keyof, g_ops, g_tk, g_tile, g_seg, g_tg, g_m16, g_slot, g_pairs;
  Buf g_gmark;      // ghost slots: marks, their scan, the slot of every ghost
  int g_nghost = 0;  // ghost multipole rows after the cells' in g_m16
  // operator cache: group key -> slot in g_ops, for order op_P and layout
  // op_layout (0: FP64 row blocks, 1: tensor-core FP16 images)
  std::unordered_map<int, int> op_slot;
  int op_P = -1, op_layout = -1;
  double op_cycle = 0, op_R0 = 0;  // image-key operators: the geometry they were built for
  int op_depth = -1;
  std::vector<int> op_host_keys, op_host_slots, op_host_new_keys, op_host_new_slots;
  int *keys_host = nullptr;  // pinned: the group keys read with the counts
  int g_ntiles = 0, g_ngroups = 0, g_nseg = 0;
  bool g_used_tc = false;
  // the grouping of the last grouped M2L (tiles, segments, operator slots),
  // valid for the same lists, P and form: a reevaluation contracts directly
  struct {
    bool valid = false, tcore = false, ordered = false;
    int P = 0, nres = 0;
  } g_plan;
  bool force_direct_m2l = false;  // diagnostic: per-pair direct-form M2L only
  Buf op_scratch;  // single-operator entry points (ops.cu): staged arrays
  // far-image harmonic sums (periodic.cu), kept for the (P, images, cycle)
  // they were made for
  Buf per_harm;
  Buf per_part;  // partial charge sums (the mixed form's root monopole)
  Buf g_gharm;  // harmonics of the ghost shifts, per (image, finer level)
  Buf g_part;   // tensor-core M2L: partial local expansions of tiles split between CTAs
  int nsm = 0;  // streaming multiprocessors of the device (0: not read yet)
  int per_P = 0, per_images = 0;
  double per_cycle = 0;
  // tile shapes chosen at run time (exafmm_b200_set_tile; the autotuner)
  int tile_m2l_flush = 0;  // tensor-core M2L groups per FP32 accumulator window (0: default)
  int tile_p2p_stage = 0;  // near-field source tile: bodies staged per chunk (0: default)
  // test hook (exafmm_b200_test_stall_tc): the next tensor-core M2L launch
  // waits this long on a barrier nothing arrives at, then times out
  long tc_stall_ns = 0;

  // phase state
  bool have_tree = false, have_lists = false, have_up = false, have_horiz = false, have_down = false;

  // device error flags copied back on the stream (pinned), checked after
  // each synchronisation: [0] a bounded tensor-core wait ran out
  int *flags_host = nullptr;

  cudaEvent_t ev[PH_COUNT + 1][2];
  float ms[PH_COUNT + 1] = {0};
  bool ev_ok = false;
};

// ---- launchers (each .cu file) ----
// scan.cu / sort.cu
void scan_exclusive_int(Handle &h, const int *in, int *out, long n, int *total_dev);
void radix_sort_pairs(Handle &h, u64 *&k, u32 *&v, u64 *&k2, u32 *&v2, long n, int lo_bit, int hi_bit);
// tree.cu
void build_tree(Handle &h);
// lists.cu
void build_lists(Handle &h);
void export_lists(Handle &h, int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src, int *p2p_img);
void order_m2l_lists(Handle &h);
// expansions.cu
void upward_pass(Handle &h, cudaStream_t s);
// before_l2p: an event the stream waits for before L2P (or nullptr)
void downward_pass(Handle &h, cudaStream_t s, cudaEvent_t before_l2p);
// m2l.cu
void m2l_pass(Handle &h);
// p2p.cu
void p2p_pass(Handle &h, cudaStream_t s);  // s: h.stream, or h.side once the FP32 sources are made
void make_srcf(Handle &h);
void direct_sum(Handle &h, double4 *targets_pq /*x,y,z,q*/, double4 *out, long nt);
// periodic.cu
void periodic_set_attributes();
void periodic_pass(Handle &h);
void dipole_correction(Handle &h);
// fmm2d.cu: the 2D variants (dim = 2) of the passes above
void flatten_tree_2d(Handle &h);
void upward_pass_2d(Handle &h, cudaStream_t s);
void m2l_pass_2d(Handle &h);
void periodic_pass_2d(Handle &h);
void p2p_pass_2d(Handle &h, cudaStream_t s);
void downward_pass_2d(Handle &h, cudaStream_t s, cudaEvent_t before_l2p);
void direct_sum_2d(Handle &h, double4 *targets, double4 *out, long nt);
void ewald(Handle &h, int parts, int ksize, double alpha, double sigma, double cutoff, double cycle, double *rec_dev,
           long nt);

inline int nterm_of(int P) { return P * (P + 1) / 2; }
inline unsigned grid_for(long n, int block) { return (unsigned)((n + block - 1) / block); }

}  // namespace fmm
