/* exafmm_b200: B200-native 3D Laplace FMM (free space and periodic), C ABI.
 *
 * Drop-in for the evaluation path of minimal ExaFMM's `3d/` and `3dp/`
 * variants: the same bodies, adaptive octree, dual-tree interaction lists and
 * P2P/P2M/M2M/M2L/L2L/L2P operators with complex spherical-harmonic expansions
 * of order P, computed by hand-written sm_100a CUDA kernels on one GPU.
 * Interface citations name the reference function each entry point replaces
 * (paths relative to the reference project).
 *
 * Conventions
 *  - Every function returns an int status: EXAFMM_OK (0) or a negative
 *    EXAFMM_ERR_* code; exafmm_b200_last_error() gives the message.
 *  - Bodies cross the boundary as the reference's Body record, 8 doubles per
 *    body: X[3], q, p, F[3] (3d/exafmm.h:14-19).  Host or device pointers are
 *    accepted where a `where` argument says so.
 *  - A handle owns its device buffers and one CUDA stream; calls on a handle
 *    must not overlap in time (the reference is not reentrant either:
 *    3d/exafmm.h:40-45 keeps its state in globals).  Separate handles are
 *    independent.
 *  - Results are in tree order (the order buildTree leaves the bodies in,
 *    3d/build_tree.h:88-96), and exafmm_b200_get_perm() maps tree positions
 *    back to input positions.
 */
#ifndef EXAFMM_B200_H
#define EXAFMM_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define EXAFMM_API __attribute__((visibility("default")))
#else
#define EXAFMM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
  EXAFMM_OK = 0,
  EXAFMM_ERR_ARG = -1,       /* invalid argument (N, P, ncrit, theta, pointer) */
  EXAFMM_ERR_CUDA = -2,      /* a CUDA call failed */
  EXAFMM_ERR_NOMEM = -3,     /* device allocation failed */
  EXAFMM_ERR_STATE = -4,     /* call out of order (e.g. lists before tree) */
  EXAFMM_ERR_DEPTH = -5,     /* tree deeper than EXAFMM_MAX_LEVEL (coincident bodies) */
  EXAFMM_ERR_CAPACITY = -6,  /* a device buffer stayed too small after retries */
  EXAFMM_ERR_TIMEOUT = -7,   /* a bounded device-side wait ran out */
  EXAFMM_ERR_NOGPU = -8      /* no usable sm_100 device */
};

enum { EXAFMM_FP64 = 0, EXAFMM_MIXED = 1 };
enum { EXAFMM_HOST = 0, EXAFMM_DEVICE = 1 };

#define EXAFMM_MAX_P 32     /* largest expansion order accepted */
#define EXAFMM_MAX_LEVEL 21 /* deepest octree level (3 bits per level in a 64-bit key) */

/* Global configuration of the reference (3d/exafmm.h:40-45 P, ncrit, theta;
 * 3dp/exafmm.h:45-47 images, cycle) plus the arithmetic form. */
typedef struct exafmm_params {
  int P;           /* expansion order (NTERM = P(P+1)/2 coefficients) */
  int ncrit;       /* max bodies per leaf */
  double theta;    /* multipole acceptance criterion */
  int images;      /* 0: free space (3d); >0: periodic image levels (3dp) */
  double cycle;    /* period of the periodic box (3dp) */
  int precision;   /* EXAFMM_FP64 or EXAFMM_MIXED */
  int device;      /* CUDA device ordinal */
  int dim;         /* 3 (or 0): the 3d/3dp variants; 2: the 2d/2dp variants */
} exafmm_params;

/* The 2D variants (2d/, 2dp/: the log kernel, complex power series of P
 * terms, quadtree; 2d/kernel.h:12-126) run on the same handle with dim = 2,
 * FP64 only, P >= 2.  What changes at the boundary: bodies are the 2D Body
 * record, 6 doubles X[2], q, p, F[2] (2d/exafmm.h:14-19), in set_bodies,
 * get_bodies, set_charges (N doubles, as in 3D) and direct; get_tree's xr is
 * x, y, 0, R; expansions are P complex coefficients per cell
 * (2d/kernel.h:34-45); list image indices are the 2D periodic1D
 * (ix+1) + 3 (iy+1) (2dp/traverse_lazy.h:27-30; 4 = no shift); with
 * images > 0 the walk repeats over the 9 in-plane images and the root adds
 * the far images of 2dp/traverse_eager.h:46-93; direct() sums the
 * (2r+1)^2 images of 2dp/traverse_eager.h:124-143.  Batches, the mixed form,
 * the single operators, the dipole correction and Ewald are 3D only. */

typedef struct exafmm_b200 exafmm_b200;

/* Handle lifecycle.  exafmm_b200_create replaces the reference's global
 * set-up (3d/fmm.cxx:12-15 parameter globals, 3d/kernel.h:118-120
 * initKernel). */
EXAFMM_API int exafmm_b200_create(const exafmm_params *params, exafmm_b200 **out);
EXAFMM_API int exafmm_b200_destroy(exafmm_b200 *h);
EXAFMM_API const char *exafmm_b200_last_error(const exafmm_b200 *h);
EXAFMM_API int exafmm_b200_set_params(exafmm_b200 *h, const exafmm_params *params);

/* Load N bodies (Body records, 8 doubles each; p and F are ignored).
 * where = EXAFMM_HOST or EXAFMM_DEVICE.  The caller's copy is not modified. */
EXAFMM_API int exafmm_b200_set_bodies(exafmm_b200 *h, const double *bodies8, int64_t n, int where);

/* Phases of one evaluation, replacing the reference's buildTree
 * (3d/build_tree.h:88-96), the list recording of the lazy traversal
 * (3d/traverse_lazy.h:27-44 getList; 3dp/traverse_lazy.h:124-141 image loop),
 * upwardPass (3d/traverse_eager.h:127-144), horizontalPass
 * (3d/traverse_eager.h:147-172 M2L + P2P; 3dp/traverse_eager.h:95-110 with the
 * periodic root, :46-93) and downwardPass (3d/traverse_eager.h:175-190). */
EXAFMM_API int exafmm_b200_build_tree(exafmm_b200 *h);
EXAFMM_API int exafmm_b200_build_lists(exafmm_b200 *h);
EXAFMM_API int exafmm_b200_upward(exafmm_b200 *h);
EXAFMM_API int exafmm_b200_horizontal(exafmm_b200 *h);
EXAFMM_API int exafmm_b200_downward(exafmm_b200 *h);

/* All phases: tree, lists, upward, horizontal, downward (3d/fmm.cxx:40-53).
 * The handle runs them on three streams: the upward pass beside the list
 * build, the near field beside the M2L and L2L; the results are those of
 * the calls above made one after another. */
EXAFMM_API int exafmm_b200_evaluate(exafmm_b200 *h);

/* Repeated evaluations on fixed positions (an FMM matrix-vector product with
 * new charges each time).  set_charges replaces the charges (N doubles in
 * the input order of set_bodies / set_batch; a non-finite value is rejected
 * and nothing changes) and keeps the tree and the interaction lists, which
 * depend on the positions only.  reevaluate then runs upward, horizontal and
 * downward over the kept tree and lists: the lazy traversal's evaluate()
 * over its stored lists (3d/traverse_lazy.h:46-62).  Results are those of
 * evaluate() on the same bodies; reevaluate needs a tree and lists from an
 * earlier evaluate() or build_lists(). */
EXAFMM_API int exafmm_b200_set_charges(exafmm_b200 *h, const double *q, int where);
EXAFMM_API int exafmm_b200_reevaluate(exafmm_b200 *h);

/* Results.  get_bodies writes N Body records in tree order (X,q as sorted,
 * p,F = FMM result) to host or device memory.  get_perm writes, per tree
 * position, the input index of that body. */
EXAFMM_API int exafmm_b200_get_bodies(exafmm_b200 *h, double *bodies8, int where);
EXAFMM_API int exafmm_b200_get_perm(exafmm_b200 *h, int64_t *perm, int where);

/* Tree in the reference's cell order (3d/build_tree.h:69-84): per cell
 * NCHILD, index of the first child (-1 for a leaf), index of the first body
 * in tree order, NBODY, level, and centre+radius as 4 doubles.  Host arrays
 * of exafmm_b200_num_cells() entries. */
EXAFMM_API int64_t exafmm_b200_num_cells(exafmm_b200 *h);
EXAFMM_API int exafmm_b200_get_tree(exafmm_b200 *h, int *nchild, int *child, int *body, int *nbody, int *level, double *xr);

/* Interaction lists per target cell, reference cell indices, in the
 * reference's recording order (3d/traverse_lazy.h:27-44): CSR offsets
 * (num_cells+1), source cells, and the periodic index periodic1D(iX)
 * (3dp/traverse_lazy.h:27-30; 13 = no shift).  Counts first, then arrays. */
EXAFMM_API int exafmm_b200_count_lists(exafmm_b200 *h, int64_t *n_m2l, int64_t *n_p2p);
EXAFMM_API int exafmm_b200_get_lists(exafmm_b200 *h, int *m2l_off, int *m2l_src, int *m2l_img, int *p2p_off, int *p2p_src,
                          int *p2p_img);

/* Multipole and local expansions (complex, re/im interleaved, NTERM per cell)
 * in the reference's cell order.  Host arrays. */
EXAFMM_API int exafmm_b200_get_expansions(exafmm_b200 *h, double *M, double *L);

/* Direct summation of all current bodies onto nt targets (Body records in
 * host or device memory; p and F accumulate), FP64: replaces direct()
 * (3d/traverse_eager.h:193-202).  With images > 0 the sources repeat over
 * (2r+1)^3 copies shifted by multiples of cycle, r = sum_{i<images} 3^i, as
 * in the periodic direct() (3dp/traverse_eager.h:131-154). */
EXAFMM_API int exafmm_b200_direct(exafmm_b200 *h, double *targets8, int64_t nt, int where);

/* Periodic systems (images > 0).  Dipole correction of the current results
 * in place (3dp/fmm.cxx:63-75): with d = sum q X, coef = 4 pi / (3 cycle^3),
 * p -= coef |d|^2 / N / q and F -= coef d; FP64. */
EXAFMM_API int exafmm_b200_dipole_correction(exafmm_b200 *h);

/* Ewald summation of the current bodies (all sources, FP64) onto nt targets
 * (Body records in host or device memory; p and F accumulate): wave part over
 * the integer wave vectors 0 < |k| <= ksize of initWaves, real part with the
 * nearest image per axis inside `cutoff`, and the self term, with the
 * parameters of 3dp/ewald.h (alpha, sigma, cutoff; cycle from the handle).
 * Replaces wavePart + realPart + selfTerm (3dp/ewald.h:83-149). */
EXAFMM_API int exafmm_b200_ewald(exafmm_b200 *h, int ksize, double alpha, double sigma, double cutoff,
                                 double *targets8, int64_t nt, int where);

/* The Ewald parts one at a time (or any mask of them), as the reference's
 * periodic driver calls them (3dp/fmm.cxx:85-93): EXAFMM_EWALD_WAVE replaces
 * wavePart (3dp/ewald.h:130-143), EXAFMM_EWALD_REAL realPart
 * (3dp/ewald.h:122-127; nearest image per axis, as above), EXAFMM_EWALD_SELF
 * selfTerm (3dp/ewald.h:146-150: p -= 2/sqrt(pi) q alpha, which needs no
 * loaded bodies).  Sources are the handle's bodies; p and F of the targets
 * accumulate; exafmm_b200_ewald() is EXAFMM_EWALD_ALL. */
enum { EXAFMM_EWALD_WAVE = 1, EXAFMM_EWALD_REAL = 2, EXAFMM_EWALD_SELF = 4, EXAFMM_EWALD_ALL = 7 };
EXAFMM_API int exafmm_b200_ewald_parts(exafmm_b200 *h, int parts, int ksize, double alpha, double sigma,
                                       double cutoff, double *targets8, int64_t nt, int where);

/* Single operators: the reference's kernel functions one call at a time, on
 * cells the caller describes (3d/kernel.h:122-323; the kernel test and the
 * operator chain of 3d/kernel.cxx:4-91 and test/test_kernel.h:6-94 call them
 * this way).  The order P is the handle's; no bodies need to be loaded.  A
 * cell is its centre and radius, 4 doubles X[3], R (the layout of
 * exafmm_b200_get_tree's xr; R is not read); an expansion is NTERM complex
 * coefficients, re and im interleaved, index n(n+1)/2+m (3d/kernel.h:197);
 * bodies are Body records.  Outputs accumulate, as the reference's += does.
 * `where` says whether all the call's arrays are in host or device memory.
 * shift3 (3 doubles, or NULL for none) is the periodic source offset iX*cycle
 * of the 3dp variants: the pair offset is (Xi - Xj) - shift3
 * (3dp/kernel.h:133, :200).  FP64, the same arithmetic as the FP64 form.
 *   p2p  P2P(Ci, Cj) (3d/kernel.h:122-150): sources onto targets' p and F.
 *   p2m  P2M(C) (3d/kernel.h:187-202): the cell's bodies into its M.
 *   m2m  M2M(Ci) (3d/kernel.h:204-231): nchild children (centres
 *        children4, multipoles Mchildren, nchild x NTERM) into the parent's M.
 *   m2l  M2L(Ci, Cj) (3d/kernel.h:233-260): the source's M into the target's L.
 *   l2l  L2L(Cj) (3d/kernel.h:262-291): the parent's L into each child's L
 *        (Lchildren, nchild x NTERM).
 *   l2p  L2P(C) (3d/kernel.h:293-323): the cell's L into its bodies' p and F. */
EXAFMM_API int exafmm_b200_p2p(exafmm_b200 *h, double *targets8, int64_t nt, const double *sources8, int64_t ns,
                               const double *shift3, int where);
EXAFMM_API int exafmm_b200_p2m(exafmm_b200 *h, const double *cell4, const double *bodies8, int64_t nb, double *M,
                               int where);
EXAFMM_API int exafmm_b200_m2m(exafmm_b200 *h, const double *parent4, double *M, int nchild, const double *children4,
                               const double *Mchildren, int where);
EXAFMM_API int exafmm_b200_m2l(exafmm_b200 *h, const double *target4, double *L, const double *source4,
                               const double *M, const double *shift3, int where);
EXAFMM_API int exafmm_b200_l2l(exafmm_b200 *h, const double *parent4, const double *L, int nchild,
                               const double *children4, double *Lchildren, int where);
EXAFMM_API int exafmm_b200_l2p(exafmm_b200 *h, const double *cell4, const double *L, double *bodies8, int64_t nb,
                               int where);

/* Batch of independent free-space systems (no reference counterpart: the
 * reference evaluates one system per process).  bodies8 holds the systems'
 * Body records one after the other; system q owns records
 * [offsets[q], offsets[q+1]) (offsets: nsys+1 values, offsets[0] = 0, each
 * system at least one body).  evaluate() then builds one forest -- every
 * system with its own bounds and tree, exactly as if built alone -- and runs
 * each phase once over all systems; get_bodies() returns every system's
 * bodies in its own tree order, systems in input order, and get_perm() the
 * input record of each.  Exports of trees, lists and expansions, direct(),
 * ewald() and dipole_correction() address a single system and return
 * EXAFMM_ERR_STATE for a batch; set_bodies() returns to a single system. */
EXAFMM_API int exafmm_b200_set_batch(exafmm_b200 *h, const double *bodies8, const int64_t *offsets, int nsys,
                                     int where);

/* Autotuner (no reference counterpart: the reference hard-codes ncrit,
 * 3d/fmm.cxx:14).  Times evaluate() on the bodies now loaded (one system or a
 * batch) for each candidate leaf size ncrit (NULL = 32, 48, 64, 96, 128,
 * 192, 256), `repeats` timed runs each after one warm-up, keeps the fastest
 * in the handle's parameters, then at that leaf size times the near-field
 * source tiles (EXAFMM_TILE_P2P_STAGE 1024, 1536, 2048) and keeps the
 * fastest, and leaves the results of the chosen setting in the handle.  ncrit
 * shapes the tree, so results after tuning are those of the chosen ncrit,
 * not of the reference's; the plain drop-in configuration keeps ncrit = 64. */
EXAFMM_API int exafmm_b200_autotune(exafmm_b200 *h, const int *ncrit_candidates, int ncand, int repeats,
                                    int *best_ncrit, double *best_ms);

/* Per-phase device times of the last evaluation in milliseconds, measured
 * with CUDA events on the stream each phase ran on: tree, lists, upward, m2l,
 * p2p, downward, total (7 values).  In evaluate() phases overlap, so the
 * phase times add up to more than the total. */
EXAFMM_API int exafmm_b200_get_timings(exafmm_b200 *h, double *ms7);

/* Library information: number of kernel launches issued by the last
 * evaluate(), and the build's compute capability target (100 = sm_100a). */
EXAFMM_API int64_t exafmm_b200_last_launches(exafmm_b200 *h);
EXAFMM_API int exafmm_b200_arch(void);

/* Diagnostic with no reference counterpart: FMA-pipe throughput of the
 * handle's device in TFLOP/s, measured with independent FMA chains; the
 * denominator of the FP64 and FP32 rooflines.  precision EXAFMM_FP64: scalar
 * FP64 FMAs; EXAFMM_MIXED: FP32, the larger of scalar FMAs and packed FP32x2
 * FMAs (fma.rn.f32x2, two lanes per instruction); 2: scalar FP32 only; 3:
 * packed FP32x2 only. */
EXAFMM_API int exafmm_b200_fma_peak(exafmm_b200 *h, int precision, double *tflops);

/* Tile shapes chosen at run time (no reference counterpart; the reference has
 * no kernels to tile).  EXAFMM_TILE_M2L_FLUSH: groups of the tensor-core M2L
 * (mixed form) accumulated in FP32 in tensor memory before the partial sum is
 * folded into the compensated running sum: fewer groups per window means
 * fewer FP32 additions between folds (a smaller accumulation error) and more
 * fold work (the default: 2 for P <= 10, 1 for P = 11 and 12, 4 above).  Values 1-64; 0 restores
 * the default.  EXAFMM_TILE_P2P_STAGE: bodies of source leaves the near-field
 * kernel stages in shared memory per chunk (the source tile), 1024, 1536 or
 * 2048 (default: 1536 mixed, 1024 FP64); a speed choice: the sums change only
 * by rounding (the chunks group the sources differently).  get_tile returns the value in effect.  exafmm_b200_autotune()
 * chooses the source tile after the leaf size. */
enum { EXAFMM_TILE_M2L_FLUSH = 0, EXAFMM_TILE_P2P_STAGE = 1 };
EXAFMM_API int exafmm_b200_set_tile(exafmm_b200 *h, int which, int value);
EXAFMM_API int exafmm_b200_get_tile(exafmm_b200 *h, int which, int *value);

/* Diagnostic with no reference counterpart: the grouped M2L of the last
 * evaluation -- operator groups, (tile, group) segments contracted, entries
 * left to the direct-form kernel, target tiles (4 values). */
EXAFMM_API int exafmm_b200_m2l_stats(exafmm_b200 *h, int64_t *stats4);

/* Test hook with no reference counterpart: the next launch of the
 * tensor-core M2L kernel on this handle (mixed form) first waits `ns`
 * nanoseconds on a barrier that nothing arrives at, as if its inputs never
 * came.  The wait runs out, the kernel's other roles stop waiting, copies and
 * MMAs in flight are drained, tensor memory is freed, and the evaluation
 * returns EXAFMM_ERR_TIMEOUT with its results discarded; the handle stays
 * usable and the next evaluation runs normally.  ns = 0 clears the hook. */
EXAFMM_API int exafmm_b200_test_stall_tc(exafmm_b200 *h, int64_t ns);

/* Direct summation that allocates nothing.  No counterpart in the reference:
 * it exists for callers that may not allocate device memory -- programs that
 * hand all of HBM to their own pool at start-up, or loops that must never
 * enter the CUDA allocator -- and so cannot create a handle.  sources8 (ns
 * Body records) and targets8 (nt Body records) are device pointers owned by
 * the caller; p and F of the targets accumulate, in FP64, as in
 * exafmm_b200_direct().  The only other memory used is a fixed scratch array
 * built into the library (two 32-byte records per target, 4 MiB per GPU that
 * loads the library, kept until exit), so nt may not exceed
 * EXAFMM_DIRECT_STATIC_MAX_TARGETS (larger nt returns EXAFMM_ERR_ARG).  The
 * work is queued on `stream` (a cudaStream_t; NULL = default stream) and the
 * call returns without waiting.  All calls share the scratch: calls that
 * overlap on the GPU race and must be serialised by the caller.  The first
 * call on each device looks up the scratch address; make it before any
 * stream capture.  Errors: exafmm_b200_last_error(NULL). */
#define EXAFMM_DIRECT_STATIC_MAX_TARGETS 65536
EXAFMM_API int exafmm_b200_direct_static(const double *sources8, int64_t ns, double *targets8, int64_t nt,
                                         void *stream);

#ifdef __cplusplus
}
#endif
#endif
