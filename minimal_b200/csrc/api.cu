// The C ABI (include/exafmm_b200.h): argument checking, phase ordering,
// per-phase CUDA-event timing and the host<->device copies at the boundary.
// Every entry point turns internal errors into a status code plus a message.
#include <cstring>
#include <new>

#include <algorithm>

#include <nvtx3/nvToolsExt.h>

#include "fmm.cuh"

namespace fmm {
double fma_peak_tflops(int precision);
int m2l_flush_interval(const Handle &h);
int p2p_tile(const Handle &h);
void ops_set_attributes();
void op_p2p_call(Handle &h, double *t8, long nt, const double *s8, long ns, const double *shift3, int where);
void op_p2m_call(Handle &h, const double *cell4, const double *b8, long nb, double *M, int where);
void op_l2p_call(Handle &h, const double *cell4, const double *L, double *b8, long nb, int where);
void op_shift_call(Handle &h, int kind, const double *parent4, const double *in, int nkid, const double *kids4,
                   double *out, int where);
void op_m2l_call(Handle &h, const double *t4, double *L, const double *s4, const double *M, const double *shift3,
                 int where);
void m2l_set_attributes();
void m2l_grouped_set_attributes();
void p2p_set_attributes();
void expansions_set_attributes();
}  // namespace fmm

using namespace fmm;

struct exafmm_b200 {
  Handle h;
};

// Message of the last failed call on this thread that had no handle to hold
// it (create, direct_static); read back through exafmm_b200_last_error(NULL).
thread_local std::string exafmm_b200_static_err;

namespace {


// The handle's device for the duration of a call, whichever device the
// calling thread has current (a new thread starts on device 0); the
// caller's device is put back afterwards.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      prev = -1;
    }
    if (prev != dev) FMM_CUDA(cudaSetDevice(dev));
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

template <class F>
int guarded(exafmm_b200 *H, F f) {
  if (!H) return EXAFMM_ERR_ARG;
  try {
    DeviceScope scope(H->h.prm.device);
    f(H->h);
    H->h.err.clear();
    return EXAFMM_OK;
  } catch (const Error &e) {
    H->h.err = e.msg;
    return e.code;
  } catch (const std::bad_alloc &) {
    H->h.err = "host allocation failed";
    return EXAFMM_ERR_NOMEM;
  }
}

void check_params(const exafmm_params &p) {
  if (p.P < 1 || p.P > EXAFMM_MAX_P) throw Error{EXAFMM_ERR_ARG, "P must be in [1, 32]"};
  if (p.ncrit < 1) throw Error{EXAFMM_ERR_ARG, "ncrit must be >= 1"};
  if (!(p.theta > 0) || !(p.theta < 1e6)) throw Error{EXAFMM_ERR_ARG, "theta must be positive and finite"};
  if (p.images < 0 || p.images > 12) throw Error{EXAFMM_ERR_ARG, "images must be in [0, 12]"};
  if (p.images > 0 && !(p.cycle > 0)) throw Error{EXAFMM_ERR_ARG, "cycle must be positive when images > 0"};
  if (p.precision != EXAFMM_FP64 && p.precision != EXAFMM_MIXED) throw Error{EXAFMM_ERR_ARG, "unknown precision"};
  if (p.dim != 0 && p.dim != 2 && p.dim != 3) throw Error{EXAFMM_ERR_ARG, "dim must be 2 or 3 (0 = 3)"};
  if (p.dim == 2 && p.precision != EXAFMM_FP64) throw Error{EXAFMM_ERR_ARG, "the 2D variants are FP64 only"};
  if (p.dim == 2 && p.P < 2) throw Error{EXAFMM_ERR_ARG, "the 2D variants need P >= 2"};
}

bool is2d(const Handle &h) { return h.prm.dim == 2; }
int rec_len(const Handle &h) { return is2d(h) ? 6 : 8; }  // doubles per Body record

void need_3d(Handle &h, const char *what) {
  if (is2d(h)) throw Error{EXAFMM_ERR_STATE, std::string(what) + " is for the 3D variants (dim = 3)"};
}

// Body records (8 doubles in 3D, 6 in 2D: X[dim], q, p, F[dim]) -> x, y, z, q
// (z = 0 in 2D).
__global__ void k_pack_in(const double *rec, long n, int len, double4 *in, int *bad) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *r = rec + len * i;
  const double4 v = len == 8 ? make_double4(r[0], r[1], r[2], r[3]) : make_double4(r[0], r[1], 0.0, r[2]);
  if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z) || !isfinite(v.w)) *bad = 1;
  in[i] = v;
}

__global__ void k_check_finite(const double *q, long n, int *bad) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && !isfinite(q[i])) *bad = 1;
}

// New charges in input order: the caller-order bodies, and (once a tree
// exists) the tree-order bodies through the permutation.
__global__ void k_set_charges(const double *q, long n, double4 *in, const int *perm, double4 *src) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  in[i].w = q[i];
  if (src) src[i].w = q[perm[i]];
}

__global__ void k_unpack_out(const double4 *src, const double4 *out, long n, int len, double *rec) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 a = src[i], b = out[i];
  double *r = rec + len * i;
  if (len == 8) {
    r[0] = a.x; r[1] = a.y; r[2] = a.z; r[3] = a.w;
    r[4] = b.x; r[5] = b.y; r[6] = b.z; r[7] = b.w;
  } else {
    r[0] = a.x; r[1] = a.y; r[2] = a.w;
    r[3] = b.x; r[4] = b.y; r[5] = b.z;
  }
}

__global__ void k_direct_prep(const double *rec, long n, int len, double4 *xq, double4 *pf) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *r = rec + len * i;
  if (len == 8) {
    xq[i] = make_double4(r[0], r[1], r[2], r[3]);
    pf[i] = make_double4(r[4], r[5], r[6], r[7]);
  } else {
    xq[i] = make_double4(r[0], r[1], 0.0, r[2]);
    pf[i] = make_double4(r[3], r[4], r[5], 0.0);
  }
}

__global__ void k_direct_back(const double4 *pf, long n, int len, double *rec) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double *r = rec + len * i;
  if (len == 8) {
    r[4] = pf[i].x; r[5] = pf[i].y; r[6] = pf[i].z; r[7] = pf[i].w;
  } else {
    r[3] = pf[i].x; r[4] = pf[i].y; r[5] = pf[i].z;
  }
}

// A phase: CUDA events on its stream (the timings), and an NVTX range on
// the host around its launches (named in a profiler's timeline; no cost
// without one).
const char *const kPhaseNames[PH_COUNT] = {"tree", "lists", "upward", "m2l", "p2p", "downward"};

struct Timer {
  Handle &h;
  int ph;
  cudaStream_t s;
  Timer(Handle &h_, int p, cudaStream_t s_ = nullptr) : h(h_), ph(p), s(s_ ? s_ : h_.stream) {
    nvtxRangePushA(kPhaseNames[ph]);
    if (h.ev_ok) cudaEventRecord(h.ev[ph][0], s);
  }
  ~Timer() {
    if (h.ev_ok) cudaEventRecord(h.ev[ph][1], s);
    nvtxRangePop();
  }
};

void need_tree(Handle &h) {
  if (!h.have_tree) throw Error{EXAFMM_ERR_STATE, "build_tree() has not run on the current bodies"};
}

// Tree and list exports, direct sums and the periodic tools address one
// system; a batch only evaluates and returns bodies.
void need_single(Handle &h, const char *what) {
  if (h.nsys > 1) throw Error{EXAFMM_ERR_STATE, std::string(what) + " is not available for a batch of systems"};
}

void do_tree(Handle &h) {
  if (h.n <= 0) throw Error{EXAFMM_ERR_STATE, "no bodies loaded"};
  Timer t(h, PH_TREE);
  build_tree(h);  // sets srcf_ready: the mixed form's FP32 sources come with the gathered bodies
  h.have_tree = true;
  h.have_lists = h.have_up = h.have_horiz = h.have_down = false;
}

void do_lists(Handle &h) {
  need_tree(h);
  Timer t(h, PH_LISTS);
  build_lists(h);
  h.have_lists = true;
}

void do_up(Handle &h) {
  need_tree(h);
  Timer t(h, PH_UP);
  upward_pass(h, h.stream);
  h.have_up = true;
}

void do_horiz(Handle &h) {
  if (!h.have_up) throw Error{EXAFMM_ERR_STATE, "upward() must run before horizontal()"};
  if (!h.have_lists) do_lists(h);
  {
    Timer t(h, PH_M2L);
    m2l_pass(h);
    periodic_pass(h);  // far images beyond the first layer (images >= 2)
  }
  {
    Timer t(h, PH_P2P);
    p2p_pass(h, h.stream);
  }
  h.have_horiz = true;
}

void do_down(Handle &h) {
  if (!h.have_horiz) throw Error{EXAFMM_ERR_STATE, "horizontal() must run before downward()"};
  Timer t(h, PH_DOWN);
  downward_pass(h, h.stream, nullptr);
  h.have_down = true;
}

void sync(Handle &h);

// A whole evaluation on three streams.  The upward pass needs only the tree
// and the FP32 sources, so it runs on `aux` beside the dual-tree walk.  The
// near field needs the tree, the lists and the bodies, and only L2P reads
// what it writes (L2P adds into the near-field sums), so it runs on `side`
// from the lists until L2P, filling the SMs that the far field's per-level
// launches and its host read of the group counts leave idle.  The far field
// and the upward pass have the higher stream priority.
void run_all(Handle &h, bool rebuild) {
  if (rebuild) {
    do_tree(h);
  } else {
    if (!h.have_lists) throw Error{EXAFMM_ERR_STATE, "reevaluate() needs the tree and lists of an earlier evaluation"};
    if (h.ev_ok)  // tree and lists kept: zero time, and the total starts here
      for (int p : {PH_TREE, PH_LISTS})
        for (int k = 0; k < 2; k++) cudaEventRecord(h.ev[p][k], h.stream);
  }
  if (h.prm.precision == EXAFMM_MIXED) make_srcf(h);  // read by P2M and the near field
  // the mixed form's upward pass is shorter than the list build and yields
  // to it; the FP64 one is longer and keeps the top priority
  cudaStream_t up = h.prm.precision == EXAFMM_MIXED ? h.aux_lo : h.aux;
  FMM_CUDA(cudaEventRecord(h.fork_ev, h.stream));
  try {
    FMM_CUDA(cudaStreamWaitEvent(up, h.fork_ev, 0));
    {
      Timer t(h, PH_UP, up);
      upward_pass(h, up);
    }
    FMM_CUDA(cudaEventRecord(h.up_ev, up));
    h.have_up = true;
    if (rebuild) do_lists(h);
    FMM_CUDA(cudaEventRecord(h.lists_ev, h.stream));
    FMM_CUDA(cudaStreamWaitEvent(h.side, h.lists_ev, 0));
    {
      Timer t(h, PH_P2P, h.side);
      p2p_pass(h, h.side);
    }
    FMM_CUDA(cudaEventRecord(h.join_ev, h.side));
    FMM_CUDA(cudaStreamWaitEvent(h.stream, h.up_ev, 0));
    Timer t(h, PH_M2L);
    m2l_pass(h);
    periodic_pass(h);
  } catch (...) {
    // nothing of this evaluation stays in flight
    cudaStreamSynchronize(up);
    cudaStreamSynchronize(h.side);
    throw;
  }
  h.have_horiz = true;
  {
    Timer t(h, PH_DOWN);
    downward_pass(h, h.stream, h.join_ev);
  }
  h.have_down = true;
  sync(h);
}

void sync(Handle &h) {
  FMM_CUDA(cudaStreamSynchronize(h.stream));
  if (h.flags_host && h.flags_host[0]) {
    h.flags_host[0] = 0;
    h.have_horiz = h.have_down = false;
    throw Error{EXAFMM_ERR_TIMEOUT, "tensor-core M2L: a bounded wait ran out (results discarded)"};
  }
  if (h.ev_ok) {
    for (int p = 0; p < PH_COUNT; p++) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, h.ev[p][0], h.ev[p][1]) == cudaSuccess) h.ms[p] = ms;
      else { cudaGetLastError(); h.ms[p] = 0; }
    }
    float tot = 0;
    if (cudaEventElapsedTime(&tot, h.ev[PH_TREE][0], h.ev[PH_DOWN][1]) == cudaSuccess) h.ms[PH_COUNT] = tot;
    else cudaGetLastError();
  }
}

}  // namespace

extern "C" {

int exafmm_b200_arch(void) { return 100; }

int exafmm_b200_create(const exafmm_params *params, exafmm_b200 **out) {
  if (!params || !out) return EXAFMM_ERR_ARG;
  *out = nullptr;
  exafmm_b200 *H = new (std::nothrow) exafmm_b200();
  if (!H) return EXAFMM_ERR_NOMEM;
  try {
    check_params(*params);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw Error{EXAFMM_ERR_NOGPU, "no CUDA device"};
    }
    if (params->device < 0 || params->device >= ndev) throw Error{EXAFMM_ERR_ARG, "device ordinal out of range"};
    cudaDeviceProp prop;
    FMM_CUDA(cudaGetDeviceProperties(&prop, params->device));
    if (prop.major != 10) throw Error{EXAFMM_ERR_NOGPU, std::string("needs an sm_100 GPU, found ") + prop.name};
    FMM_CUDA(cudaSetDevice(params->device));
    Handle &h = H->h;
    h.prm = *params;
    h.nterm = params->dim == 2 ? params->P : nterm_of(params->P);
    int least = 0, greatest = 0;
    FMM_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    FMM_CUDA(cudaStreamCreateWithPriority(&h.stream, cudaStreamNonBlocking, greatest));
    FMM_CUDA(cudaStreamCreateWithPriority(&h.side, cudaStreamNonBlocking, least));
    FMM_CUDA(cudaStreamCreateWithPriority(&h.aux, cudaStreamNonBlocking, greatest));
    FMM_CUDA(cudaStreamCreateWithPriority(&h.aux_lo, cudaStreamNonBlocking, greatest < least ? greatest + 1 : greatest));
    for (cudaEvent_t *e : {&h.fork_ev, &h.up_ev, &h.lists_ev, &h.join_ev})
      FMM_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    FMM_CUDA(cudaMallocHost(&h.flags_host, 4 * sizeof(int)));
    h.flags_host[0] = 0;
    h.ev_ok = true;
    for (int p = 0; p < PH_COUNT + 1; p++)
      for (int k = 0; k < 2; k++)
        if (cudaEventCreate(&h.ev[p][k]) != cudaSuccess) h.ev_ok = false;
    m2l_set_attributes();
    m2l_grouped_set_attributes();
    p2p_set_attributes();
    expansions_set_attributes();
    periodic_set_attributes();
    ops_set_attributes();
    FMM_CUDA(cudaGetLastError());
  } catch (const Error &e) {
    exafmm_b200_static_err = e.msg;
    delete H;
    return e.code;
  }
  *out = H;
  return EXAFMM_OK;
}

int exafmm_b200_destroy(exafmm_b200 *H) {
  if (!H) return EXAFMM_ERR_ARG;
  Handle &h = H->h;
  cudaSetDevice(h.prm.device);
  if (h.stream) cudaStreamSynchronize(h.stream);
  if (h.side) cudaStreamSynchronize(h.side);
  if (h.aux) cudaStreamSynchronize(h.aux);
  if (h.aux_lo) cudaStreamSynchronize(h.aux_lo);
  Buf *bufs[] = {&h.in, &h.src, &h.out, &h.perm, &h.srcf, &h.keys[0], &h.keys[1], &h.vals[0], &h.vals[1],
                 &h.lfirst, &h.chain, &h.prebase, &h.scan_tmp, &h.hist, &h.c_begin, &h.c_count, &h.c_child,
                 &h.c_nchild, &h.c_parent, &h.c_level, &h.c_xr, &h.c_pre, &h.c_ref, &h.c_leaf_of_body,
                 &h.leaves, &h.pre_tmp, &h.ctmp, &h.geom, &h.counters, &h.frontier[0], &h.frontier[1],
                 &h.m2l_raw, &h.m2l_key, &h.p2p_raw, &h.m2l_off, &h.m2l_ent, &h.p2p_off, &h.p2p_ent, &h.fill, &h.M, &h.L,
                 &h.m2l_units, &h.stage, &h.g_mt, &h.g_ekey, &h.g_occ, &h.g_cnt, &h.g_keyof, &h.g_ops,
                 &h.g_tk, &h.g_tile, &h.g_seg, &h.g_tg, &h.g_m16, &h.g_slot, &h.g_pairs, &h.shift_ops, &h.shift_terms,
                 &h.op_scratch, &h.g_gmark, &h.per_harm, &h.g_gharm, &h.per_part,
                 &h.g_part, &h.body_leaf, &h.l2p_f};
  for (Buf *b : bufs) b->release();
  if (h.ev_ok)
    for (int p = 0; p < PH_COUNT + 1; p++)
      for (int k = 0; k < 2; k++) cudaEventDestroy(h.ev[p][k]);
  if (h.stream) cudaStreamDestroy(h.stream);
  if (h.side) cudaStreamDestroy(h.side);
  if (h.aux) cudaStreamDestroy(h.aux);
  if (h.aux_lo) cudaStreamDestroy(h.aux_lo);
  for (cudaEvent_t e : {h.fork_ev, h.up_ev, h.lists_ev, h.join_ev})
    if (e) cudaEventDestroy(e);
  if (h.flags_host) cudaFreeHost(h.flags_host);
  if (h.keys_host) cudaFreeHost(h.keys_host);
  delete H;
  return EXAFMM_OK;
}

const char *exafmm_b200_last_error(const exafmm_b200 *H) {
  if (!H) return exafmm_b200_static_err.c_str();
  return H->h.err.c_str();
}

int exafmm_b200_set_params(exafmm_b200 *H, const exafmm_params *params) {
  return guarded(H, [&](Handle &h) {
    if (!params) throw Error{EXAFMM_ERR_ARG, "null params"};
    check_params(*params);
    if (h.nsys > 1 && params->images != 0)
      throw Error{EXAFMM_ERR_STATE, "batches of systems are free-space only (images = 0)"};
    if (params->device != h.prm.device) throw Error{EXAFMM_ERR_ARG, "a handle stays on its device"};
    if ((params->dim == 2) != is2d(h) && h.n > 0)
      throw Error{EXAFMM_ERR_STATE, "dim changes the Body record: load the bodies again after set_params"};
    if (params->dim == 2 && h.nsys > 1) throw Error{EXAFMM_ERR_STATE, "batches of systems are 3D only"};
    h.prm = *params;
    h.nterm = params->dim == 2 ? params->P : nterm_of(params->P);
    h.have_tree = h.have_lists = h.have_up = h.have_horiz = h.have_down = false;
  });
}

int exafmm_b200_set_bodies(exafmm_b200 *H, const double *rec, int64_t n, int where) {
  return guarded(H, [&](Handle &h) {
    if (!rec || n <= 0) throw Error{EXAFMM_ERR_ARG, "need a body array with n > 0"};
    if (n >= (1ll << 31)) throw Error{EXAFMM_ERR_ARG, "n must be below 2^31"};
    if (where != EXAFMM_HOST && where != EXAFMM_DEVICE) throw Error{EXAFMM_ERR_ARG, "where must be HOST or DEVICE"};
    FMM_CUDA(cudaSetDevice(h.prm.device));
    h.n = n;
    h.in.need(n * sizeof(double4));
    h.counters.need(sizeof(DevCounters));
    const double *drec = rec;
    const int len = rec_len(h);
    int *bad = &h.counters.as<DevCounters>()->overflow;
    FMM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), h.stream));
    // whole records cross the bus (a strided copy of only X and q, half the
    // bytes, measured slower: the copy engine moves 32-byte rows poorly)
    if (where == EXAFMM_HOST) {
      h.stage.need(n * len * sizeof(double));
      FMM_CUDA(cudaMemcpyAsync(h.stage.p, rec, n * len * sizeof(double), cudaMemcpyHostToDevice, h.stream));
      drec = h.stage.as<double>();
    }
    k_pack_in<<<grid_for(n, 256), 256, 0, h.stream>>>(drec, n, len, h.in.as<double4>(), bad);
    h.launches++;
    FMM_LAUNCH();
    int hb = 0;
    FMM_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    FMM_CUDA(cudaStreamSynchronize(h.stream));
    if (hb) throw Error{EXAFMM_ERR_ARG, "non-finite body position or charge"};
    h.have_tree = h.have_lists = h.have_up = h.have_horiz = h.have_down = false;
    h.nsys = 1;
    h.sys_off_host.clear();
  });
}

int exafmm_b200_set_batch(exafmm_b200 *H, const double *rec, const int64_t *offsets, int nsys, int where) {
  if (!H) return EXAFMM_ERR_ARG;
  if (!offsets || nsys < 1 || nsys > (1 << 20)) {
    H->h.err = "need offsets for 1 <= nsys <= 2^20 systems";
    return EXAFMM_ERR_ARG;
  }
  if (offsets[0] != 0) {
    H->h.err = "offsets[0] must be 0";
    return EXAFMM_ERR_ARG;
  }
  for (int q = 0; q < nsys; q++)
    if (offsets[q + 1] <= offsets[q]) {
      H->h.err = "every system needs at least one body (offsets strictly increasing)";
      return EXAFMM_ERR_ARG;
    }
  if (H->h.prm.images != 0) {
    H->h.err = "batches of systems are free-space only (images = 0)";
    return EXAFMM_ERR_STATE;
  }
  if (is2d(H->h)) {
    H->h.err = "batches of systems are for the 3D variants (dim = 3)";
    return EXAFMM_ERR_STATE;
  }
  const int rc = exafmm_b200_set_bodies(H, rec, offsets[nsys], where);
  if (rc != EXAFMM_OK) return rc;
  return guarded(H, [&](Handle &h) {
    h.sys_off.need((size_t)(nsys + 1) * sizeof(long long));
    FMM_CUDA(cudaMemcpyAsync(h.sys_off.p, offsets, (nsys + 1) * sizeof(long long), cudaMemcpyHostToDevice,
                             h.stream));
    h.sys_off_host.assign(offsets, offsets + nsys + 1);
    h.nsys = nsys;
    h.key_levels = 0;
  });
}

int exafmm_b200_build_tree(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) { do_tree(h); sync(h); });
}
int exafmm_b200_build_lists(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) { do_lists(h); sync(h); });
}
int exafmm_b200_upward(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) { do_up(h); sync(h); });
}
int exafmm_b200_horizontal(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) { do_horiz(h); sync(h); });
}
int exafmm_b200_downward(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) { do_down(h); sync(h); });
}

int exafmm_b200_evaluate(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) {
    h.launches = 0;
    run_all(h, true);
  });
}

int exafmm_b200_reevaluate(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) {
    h.launches = 0;
    run_all(h, false);
  });
}

int exafmm_b200_set_charges(exafmm_b200 *H, const double *q, int where) {
  return guarded(H, [&](Handle &h) {
    if (!q) throw Error{EXAFMM_ERR_ARG, "null charges"};
    if (where != EXAFMM_HOST && where != EXAFMM_DEVICE) throw Error{EXAFMM_ERR_ARG, "where must be HOST or DEVICE"};
    if (h.n <= 0) throw Error{EXAFMM_ERR_STATE, "no bodies loaded"};
    FMM_CUDA(cudaSetDevice(h.prm.device));
    const double *dq = q;
    if (where == EXAFMM_HOST) {
      h.stage.need(h.n * sizeof(double));
      FMM_CUDA(cudaMemcpyAsync(h.stage.p, q, h.n * sizeof(double), cudaMemcpyHostToDevice, h.stream));
      dq = h.stage.as<double>();
    }
    int *bad = &h.counters.as<DevCounters>()->overflow;
    FMM_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), h.stream));
    k_check_finite<<<grid_for(h.n, 256), 256, 0, h.stream>>>(dq, h.n, bad);
    h.launches++;
    FMM_LAUNCH();
    int hb = 0;
    FMM_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
    FMM_CUDA(cudaStreamSynchronize(h.stream));
    if (hb) throw Error{EXAFMM_ERR_ARG, "non-finite charge"};  // nothing changed
    k_set_charges<<<grid_for(h.n, 256), 256, 0, h.stream>>>(dq, h.n, h.in.as<double4>(), h.perm.as<int>(),
                                                           h.have_tree ? h.src.as<double4>() : nullptr);
    h.launches++;
    FMM_LAUNCH();
    FMM_CUDA(cudaStreamSynchronize(h.stream));
    // the tree and the lists depend on the positions only; everything after them is redone
    h.srcf_ready = false;
    h.have_up = h.have_horiz = h.have_down = false;
  });
}

int exafmm_b200_autotune(exafmm_b200 *H, const int *candidates, int ncand, int repeats, int *best_ncrit,
                         double *best_ms) {
  return guarded(H, [&](Handle &h) {
    if (h.n <= 0) throw Error{EXAFMM_ERR_STATE, "autotune() needs bodies (set_bodies or set_batch)"};
    static const int defaults[] = {32, 48, 64, 96, 128, 192, 256};
    if (!candidates) {
      candidates = defaults;
      ncand = (int)(sizeof(defaults) / sizeof(defaults[0]));
    }
    if (ncand < 1 || ncand > 64) throw Error{EXAFMM_ERR_ARG, "autotune(): 1 to 64 candidates"};
    for (int k = 0; k < ncand; k++)
      if (candidates[k] < 1) throw Error{EXAFMM_ERR_ARG, "autotune(): ncrit candidates must be >= 1"};
    if (repeats < 1 || repeats > 100) throw Error{EXAFMM_ERR_ARG, "autotune(): repeats in [1, 100]"};
    auto run = [&]() {
      h.launches = 0;
      run_all(h, true);
      return (double)h.ms[PH_COUNT];
    };
    int best = -1;
    double tbest = 0;
    for (int k = 0; k < ncand; k++) {
      h.prm.ncrit = candidates[k];
      h.key_levels = 0;  // the key depth follows ncrit
      run();             // warm-up: buffers grow to this tree's size
      double t = run();
      for (int r = 1; r < repeats; r++) t = std::min(t, run());
      if (best < 0 || t < tbest) {
        best = candidates[k];
        tbest = t;
      }
    }
    h.prm.ncrit = best;
    h.key_levels = 0;
    // then the near-field source tile at that leaf size (a speed choice:
    // the sums change only by rounding)
    if (best <= 256) {
      const int saved = h.tile_p2p_stage;
      int best_tile = saved;
      for (int tile : {1024, 1536, 2048}) {
        h.tile_p2p_stage = tile;
        run();
        double t = run();
        for (int r = 1; r < repeats; r++) t = std::min(t, run());
        if (t < tbest) {
          tbest = t;
          best_tile = tile;
        }
      }
      h.tile_p2p_stage = best_tile;
    }
    run();  // leave the results of the chosen setting
    if (best_ncrit) *best_ncrit = best;
    if (best_ms) *best_ms = tbest;
  });
}

int exafmm_b200_get_bodies(exafmm_b200 *H, double *rec, int where) {
  return guarded(H, [&](Handle &h) {
    if (!rec) throw Error{EXAFMM_ERR_ARG, "null output"};
    if (!h.have_down) throw Error{EXAFMM_ERR_STATE, "no completed evaluation"};
    double *drec = rec;
    const int len = rec_len(h);
    if (where == EXAFMM_HOST) {
      h.stage.need(h.n * len * sizeof(double));
      drec = h.stage.as<double>();
    }
    k_unpack_out<<<grid_for(h.n, 256), 256, 0, h.stream>>>(h.src.as<double4>(), h.out.as<double4>(), h.n, len, drec);
    FMM_LAUNCH();
    if (where == EXAFMM_HOST)
      FMM_CUDA(cudaMemcpyAsync(rec, drec, h.n * len * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    FMM_CUDA(cudaStreamSynchronize(h.stream));
  });
}

int exafmm_b200_get_perm(exafmm_b200 *H, int64_t *perm, int where) {
  return guarded(H, [&](Handle &h) {
    need_tree(h);
    if (!perm) throw Error{EXAFMM_ERR_ARG, "null output"};
    std::vector<int> p(h.n);
    FMM_CUDA(cudaMemcpy(p.data(), h.perm.p, h.n * 4, cudaMemcpyDeviceToHost));
    std::vector<int64_t> q(p.begin(), p.end());
    FMM_CUDA(cudaMemcpy(perm, q.data(), h.n * 8, where == EXAFMM_HOST ? cudaMemcpyHostToHost : cudaMemcpyHostToDevice));
  });
}

int64_t exafmm_b200_num_cells(exafmm_b200 *H) { return H && H->h.have_tree ? H->h.ncells : -1; }

int exafmm_b200_get_tree(exafmm_b200 *H, int *nchild, int *child, int *body, int *nbody, int *level, double *xr) {
  return guarded(H, [&](Handle &h) {
    need_tree(h);
    need_single(h, "get_tree()");
    const int C = h.ncells;
    std::vector<int> nc(C), ch(C), bg(C), ct(C), lv(C), rf(C);
    std::vector<double4> x(C);
    FMM_CUDA(cudaMemcpy(nc.data(), h.c_nchild.p, C * 4, cudaMemcpyDeviceToHost));
    FMM_CUDA(cudaMemcpy(ch.data(), h.c_child.p, C * 4, cudaMemcpyDeviceToHost));
    FMM_CUDA(cudaMemcpy(bg.data(), h.c_begin.p, C * 4, cudaMemcpyDeviceToHost));
    FMM_CUDA(cudaMemcpy(ct.data(), h.c_count.p, C * 4, cudaMemcpyDeviceToHost));
    FMM_CUDA(cudaMemcpy(lv.data(), h.c_level.p, C * 4, cudaMemcpyDeviceToHost));
    FMM_CUDA(cudaMemcpy(rf.data(), h.c_ref.p, C * 4, cudaMemcpyDeviceToHost));
    FMM_CUDA(cudaMemcpy(x.data(), h.c_xr.p, C * sizeof(double4), cudaMemcpyDeviceToHost));
    for (int b = 0; b < C; b++) {
      const int r = rf[b];
      if (r < 0 || r >= C) throw Error{EXAFMM_ERR_STATE, "corrupt cell numbering"};
      if (nchild) nchild[r] = nc[b];
      if (child) child[r] = nc[b] ? rf[ch[b]] : -1;
      if (body) body[r] = bg[b];
      if (nbody) nbody[r] = ct[b];
      if (level) level[r] = lv[b];
      if (xr) { xr[4 * r] = x[b].x; xr[4 * r + 1] = x[b].y; xr[4 * r + 2] = x[b].z; xr[4 * r + 3] = x[b].w; }
    }
  });
}

int exafmm_b200_count_lists(exafmm_b200 *H, int64_t *a, int64_t *b) {
  return guarded(H, [&](Handle &h) {
    if (!h.have_lists) throw Error{EXAFMM_ERR_STATE, "lists not built"};
    if (a) *a = h.n_m2l;
    if (b) *b = h.n_p2p;
  });
}

int exafmm_b200_get_lists(exafmm_b200 *H, int *mo, int *ms, int *mi, int *po, int *ps, int *pi) {
  return guarded(H, [&](Handle &h) {
    if (!h.have_lists) throw Error{EXAFMM_ERR_STATE, "lists not built"};
    need_single(h, "get_lists()");
    if (!mo || !ms || !mi || !po || !ps || !pi) throw Error{EXAFMM_ERR_ARG, "null output"};
    export_lists(h, mo, ms, mi, po, ps, pi);
  });
}

int exafmm_b200_get_expansions(exafmm_b200 *H, double *M, double *L) {
  return guarded(H, [&](Handle &h) {
    if (!h.have_up) throw Error{EXAFMM_ERR_STATE, "upward() has not run"};
    need_single(h, "get_expansions()");
    const int C = h.ncells, nt = h.nterm;
    std::vector<int> rf(C);
    std::vector<double2> m((size_t)C * nt), l((size_t)C * nt);
    FMM_CUDA(cudaMemcpy(rf.data(), h.c_ref.p, C * 4, cudaMemcpyDeviceToHost));
    FMM_CUDA(cudaMemcpy(m.data(), h.M.p, (size_t)C * nt * 16, cudaMemcpyDeviceToHost));
    if (h.have_horiz) FMM_CUDA(cudaMemcpy(l.data(), h.L.p, (size_t)C * nt * 16, cudaMemcpyDeviceToHost));
    for (int b = 0; b < C; b++)
      for (int k = 0; k < nt; k++) {
        const size_t d = ((size_t)rf[b] * nt + k) * 2, s = (size_t)b * nt + k;
        if (M) { M[d] = m[s].x; M[d + 1] = m[s].y; }
        if (L) { L[d] = l[s].x; L[d + 1] = l[s].y; }
      }
  });
}

int exafmm_b200_direct(exafmm_b200 *H, double *targets, int64_t nt, int where) {
  return guarded(H, [&](Handle &h) {
    need_tree(h);
    need_single(h, "direct()");
    if (!targets || nt <= 0) throw Error{EXAFMM_ERR_ARG, "need targets"};
    const int len = rec_len(h);
    const size_t bytes = (size_t)nt * len * sizeof(double);
    Buf rec, xq, pf;
    rec.need(bytes);
    xq.need(nt * sizeof(double4));
    pf.need(nt * sizeof(double4));
    FMM_CUDA(cudaMemcpyAsync(rec.p, targets, bytes, where == EXAFMM_HOST ? cudaMemcpyHostToDevice
                                                                        : cudaMemcpyDeviceToDevice, h.stream));
    k_direct_prep<<<grid_for(nt, 256), 256, 0, h.stream>>>(rec.as<double>(), nt, len, xq.as<double4>(),
                                                          pf.as<double4>());
    FMM_LAUNCH();
    if (is2d(h)) direct_sum_2d(h, xq.as<double4>(), pf.as<double4>(), nt);
    else direct_sum(h, xq.as<double4>(), pf.as<double4>(), nt);
    k_direct_back<<<grid_for(nt, 256), 256, 0, h.stream>>>(pf.as<double4>(), nt, len, rec.as<double>());
    FMM_LAUNCH();
    FMM_CUDA(cudaMemcpyAsync(targets, rec.p, bytes, where == EXAFMM_HOST ? cudaMemcpyDeviceToHost
                                                                        : cudaMemcpyDeviceToDevice, h.stream));
    FMM_CUDA(cudaStreamSynchronize(h.stream));
    rec.release();
    xq.release();
    pf.release();
  });
}

int exafmm_b200_dipole_correction(exafmm_b200 *H) {
  return guarded(H, [&](Handle &h) {
    need_single(h, "dipole_correction()");
    need_3d(h, "dipole_correction()");
    if (!h.have_down) throw Error{EXAFMM_ERR_STATE, "dipole_correction() needs the results of evaluate()"};
    if (h.prm.images <= 0) throw Error{EXAFMM_ERR_STATE, "dipole_correction() is for periodic systems (images > 0)"};
    dipole_correction(h);
  });
}

int exafmm_b200_ewald(exafmm_b200 *H, int ksize, double alpha, double sigma, double cutoff, double *targets,
                      int64_t nt, int where) {
  return exafmm_b200_ewald_parts(H, EXAFMM_EWALD_ALL, ksize, alpha, sigma, cutoff, targets, nt, where);
}

int exafmm_b200_ewald_parts(exafmm_b200 *H, int parts, int ksize, double alpha, double sigma, double cutoff,
                            double *targets, int64_t nt, int where) {
  return guarded(H, [&](Handle &h) {
    if (parts <= 0 || parts > EXAFMM_EWALD_ALL) throw Error{EXAFMM_ERR_ARG, "ewald: parts is a nonzero mask of WAVE, REAL, SELF"};
    need_3d(h, "ewald()");
    if (parts != EXAFMM_EWALD_SELF) {  // the self term reads only the targets
      need_tree(h);
      need_single(h, "ewald()");
    }
    if (!targets || nt <= 0) throw Error{EXAFMM_ERR_ARG, "need targets"};
    if (where != EXAFMM_HOST && where != EXAFMM_DEVICE) throw Error{EXAFMM_ERR_ARG, "where must be HOST or DEVICE"};
    FMM_CUDA(cudaSetDevice(h.prm.device));
    if (ksize < 1 || ksize > 64 || !(alpha > 0) || !(sigma > 0) || !(cutoff > 0))
      throw Error{EXAFMM_ERR_ARG, "ewald: ksize in [1, 64] and positive alpha, sigma, cutoff required"};
    if (!(h.prm.cycle > 0)) throw Error{EXAFMM_ERR_STATE, "ewald() needs a periodic handle (cycle > 0)"};
    Buf rec;
    rec.need(nt * 64);
    FMM_CUDA(cudaMemcpyAsync(rec.p, targets, nt * 64, where == EXAFMM_HOST ? cudaMemcpyHostToDevice
                                                                          : cudaMemcpyDeviceToDevice, h.stream));
    ewald(h, parts, ksize, alpha, sigma, cutoff, h.prm.cycle, rec.as<double>(), nt);
    FMM_CUDA(cudaMemcpyAsync(targets, rec.p, nt * 64, where == EXAFMM_HOST ? cudaMemcpyDeviceToHost
                                                                          : cudaMemcpyDeviceToDevice, h.stream));
    FMM_CUDA(cudaStreamSynchronize(h.stream));
    rec.release();
  });
}

int exafmm_b200_get_timings(exafmm_b200 *H, double *ms7) {
  return guarded(H, [&](Handle &h) {
    if (!ms7) throw Error{EXAFMM_ERR_ARG, "null output"};
    for (int p = 0; p <= PH_COUNT; p++) ms7[p] = h.ms[p];
  });
}

int64_t exafmm_b200_last_launches(exafmm_b200 *H) { return H ? H->h.launches : -1; }

int exafmm_b200_fma_peak(exafmm_b200 *H, int precision, double *tflops) {
  return guarded(H, [&](Handle &h) {
    if (!tflops) throw Error{EXAFMM_ERR_ARG, "null output"};
    if (precision < 0 || precision > 3) throw Error{EXAFMM_ERR_ARG, "fma_peak: kind in [0, 3]"};
    FMM_CUDA(cudaSetDevice(h.prm.device));
    *tflops = fma_peak_tflops(precision);
  });
}

int exafmm_b200_p2p(exafmm_b200 *H, double *targets8, int64_t nt, const double *sources8, int64_t ns,
                    const double *shift3, int where) {
  return guarded(H, [&](Handle &h) {
    need_3d(h, "the single operators");
    FMM_CUDA(cudaSetDevice(h.prm.device));
    op_p2p_call(h, targets8, nt, sources8, ns, shift3, where);
  });
}

int exafmm_b200_p2m(exafmm_b200 *H, const double *cell4, const double *bodies8, int64_t nb, double *M, int where) {
  return guarded(H, [&](Handle &h) {
    need_3d(h, "the single operators");
    FMM_CUDA(cudaSetDevice(h.prm.device));
    op_p2m_call(h, cell4, bodies8, nb, M, where);
  });
}

int exafmm_b200_m2m(exafmm_b200 *H, const double *parent4, double *M, int nchild, const double *children4,
                    const double *Mchildren, int where) {
  return guarded(H, [&](Handle &h) {
    need_3d(h, "the single operators");
    FMM_CUDA(cudaSetDevice(h.prm.device));
    op_shift_call(h, 0, parent4, Mchildren, nchild, children4, M, where);
  });
}

int exafmm_b200_m2l(exafmm_b200 *H, const double *target4, double *L, const double *source4, const double *M,
                    const double *shift3, int where) {
  return guarded(H, [&](Handle &h) {
    need_3d(h, "the single operators");
    FMM_CUDA(cudaSetDevice(h.prm.device));
    op_m2l_call(h, target4, L, source4, M, shift3, where);
  });
}

int exafmm_b200_l2l(exafmm_b200 *H, const double *parent4, const double *L, int nchild, const double *children4,
                    double *Lchildren, int where) {
  return guarded(H, [&](Handle &h) {
    need_3d(h, "the single operators");
    FMM_CUDA(cudaSetDevice(h.prm.device));
    op_shift_call(h, 1, parent4, L, nchild, children4, Lchildren, where);
  });
}

int exafmm_b200_l2p(exafmm_b200 *H, const double *cell4, const double *L, double *bodies8, int64_t nb, int where) {
  return guarded(H, [&](Handle &h) {
    need_3d(h, "the single operators");
    FMM_CUDA(cudaSetDevice(h.prm.device));
    op_l2p_call(h, cell4, L, bodies8, nb, where);
  });
}

int exafmm_b200_set_tile(exafmm_b200 *H, int which, int value) {
  return guarded(H, [&](Handle &h) {
    if (which == EXAFMM_TILE_M2L_FLUSH) {
      if (value < 0 || value > 64) throw Error{EXAFMM_ERR_ARG, "set_tile: M2L flush interval in [1, 64] (0: default)"};
      h.tile_m2l_flush = value;
    } else if (which == EXAFMM_TILE_P2P_STAGE) {
      if (value != 0 && value != 1024 && value != 1536 && value != 2048)
        throw Error{EXAFMM_ERR_ARG, "set_tile: near-field source tile 1024, 1536 or 2048 (0: default)"};
      h.tile_p2p_stage = value;
    } else {
      throw Error{EXAFMM_ERR_ARG, "set_tile: unknown tile parameter"};
    }
  });
}

int exafmm_b200_get_tile(exafmm_b200 *H, int which, int *value) {
  return guarded(H, [&](Handle &h) {
    if (!value) throw Error{EXAFMM_ERR_ARG, "null output"};
    if (which == EXAFMM_TILE_M2L_FLUSH) *value = m2l_flush_interval(h);
    else if (which == EXAFMM_TILE_P2P_STAGE) *value = p2p_tile(h);
    else throw Error{EXAFMM_ERR_ARG, "get_tile: unknown tile parameter"};
  });
}

int exafmm_b200_m2l_stats(exafmm_b200 *H, int64_t *stats4) {
  return guarded(H, [&](Handle &h) {
    if (!stats4) throw Error{EXAFMM_ERR_ARG, "null output"};
    stats4[0] = h.g_ngroups;
    int nseg = 0;  // the exact count, from the segment scan's total
    if (h.g_plan.valid && h.g_ngroups > 0)
      FMM_CUDA(cudaMemcpy(&nseg, &h.counters.as<DevCounters>()->gcounts[3], sizeof(int), cudaMemcpyDeviceToHost));
    stats4[1] = nseg;
    stats4[2] = h.g_plan.valid ? h.g_plan.nres : 0;
    stats4[3] = h.g_ntiles;
  });
}

int exafmm_b200_test_stall_tc(exafmm_b200 *H, int64_t ns) {
  return guarded(H, [&](Handle &h) {
    if (ns < 0 || ns > 1000000000LL) throw Error{EXAFMM_ERR_ARG, "test_stall_tc: ns in [0, 1e9]"};
    h.tc_stall_ns = (long)ns;
  });
}

}  // extern "C"
