/*
 * pfblob.h -- C ABI of the B200 vortex-blob hot path (libpfblob.so).
 *
 * Drop-in boundary for pHyFlow's blob velocity, panel velocity and remesh
 * extension functions.  Plain pointers and sizes only.  Unless stated
 * otherwise every array argument is a DEVICE pointer (cudaMalloc'd or from a
 * caller-owned allocator such as torch), FP64, contiguous, and every call is
 * asynchronous on the CUDA stream passed as `stream` (NULL = legacy default
 * stream).  Calls never abort and never reset the device: failures are
 * reported as a pf_status and a message retrievable with pf_last_error().
 *
 * Ownership: the caller owns inputs and outputs; the library owns scratch in
 * a per-context, grow-only device arena (pf_mem_usage reports its size).  A
 * context may be used from one host thread at a time; use one context per
 * thread for concurrency.
 */
#ifndef PFBLOB_H
#define PFBLOB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pf_status {
    PF_OK = 0,
    PF_ERR_INVALID_ARG = 1, /* bad size, NULL pointer, unsupported option */
    PF_ERR_OOM = 2,         /* device arena could not grow */
    PF_ERR_CUDA = 3,        /* a CUDA runtime call failed (message has the name) */
    PF_ERR_TIMEOUT = 4,     /* a bounded device wait ran out */
    PF_ERR_NAN_INPUT = 5,   /* NaN/Inf in coordinates (checked where stated) */
    PF_ERR_CAPACITY = 6,    /* output capacity too small; *_needed says how much */
    PF_ERR_NOT_BUILT = 7    /* the library was built without the requested path */
} pf_status;

/* Method / hardware / kernel constants, same values as pHyFlow's
 * src/python/blobs/blobOptions.py:53-66. */
#define PF_FMM_METHOD 0
#define PF_DIRECT_METHOD 1
#define PF_CUTOFF_KERNEL 0
#define PF_GAUSS_KERNEL 1

typedef struct pf_ctx pf_ctx;

/* Create a context bound to CUDA device `device`.  Allocates nothing on the
 * device until the first call that needs scratch. */
pf_status pf_create(int device, pf_ctx **out);
pf_status pf_destroy(pf_ctx *ctx);
/* Message of the last failing call on this host thread ("" if none). */
const char *pf_last_error(void);
/* Bytes currently held by the context's scratch arena. */
pf_status pf_mem_usage(const pf_ctx *ctx, size_t *bytes);
/* Release the context's scratch arena (it regrows on demand). */
pf_status pf_trim(pf_ctx *ctx);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int pf_version(void);
/* Process-wide count of kernels this library has launched (all contexts,
 * all threads; a step-graph launch adds its kernel nodes).  Diagnostic: the
 * difference across a region is the number of library kernels enqueued in it. */
uint64_t pf_kernel_launches(void);
/* 1 in the bounds-checked build (libpfblob_checked.so, compiled with
 * -DPF_BOUNDS_CHECK), else 0.  In that build the kernels test their
 * data-dependent indices; a failed test records the first (site, index,
 * limit) on the device and skips the access instead of trapping. */
int pf_bounds_checked(void);
/* Checked build: synchronise `device` (-1: the current device), read and
 * clear every recorded bounds failure; PF_ERR_CUDA with the site, index and
 * limit in pf_last_error() if there was one.  Normal build: PF_OK, no work.
 * (No reference counterpart: the reference has no sanitizer build.) */
pf_status pf_check_bounds(int device);

/* ---------------------------------------------------------------------------
 * Gaussian-blob Biot-Savart velocity by direct summation, FP32 arithmetic with
 * hi/lo-split coordinates and compensated accumulation, FP64 in and out.
 *
 *   v_k = 1/(2 pi) sum_m g_m (-dy, dx) / r2 * (1 - exp(-r2/ksigmasqr)),
 *   r2 = dx^2 + dy^2 + 1e-12,  (dx, dy) = target_k - blob_m
 *
 * Replaces vv2parGauss_gpu  (src/cpp/blobs/cuda/vv2parGauss_gpu/
 *   vv2parGauss_py_gpu.cu:104-206, kernel vv2parGauss_device.cu:107-162) and
 *   vv2parGauss_C_cpu (src/cpp/blobs/c/vv2parGauss_C/vv2parGauss_C_cpu.c:89-160),
 * reached from _velocity_direct_{cpu,gpu}_gauss
 *   (src/python/blobs/base/induced/_induced.py:339-518).
 * No padding to a block size is required. n_src or n_tgt may be 0.
 * ------------------------------------------------------------------------- */
pf_status pf_velocity_direct(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                             const double *g, int64_t n_tgt, const double *xt,
                             const double *yt, double ksigmasqr, double *vx, double *vy,
                             void *stream);

/* Cutoff (Rosenhead-Krasny) kernel by direct summation, same arithmetic
 * scheme as pf_velocity_direct:
 *   v_k = 1/(2 pi) sum_m g_m (-dy, dx) / (dx^2 + dy^2 + sigmasqr).
 * Replaces vv2par_C_cpu (src/cpp/blobs/c/vv2par_C/vv2par_C_cpu.c:88-161) and
 * vv2par_gpu (src/cpp/blobs/cuda/vv2par_gpu/vv2par_device.cu:59-70), reached
 * from _velocity_direct_{cpu,gpu}_cutoff (src/python/blobs/base/induced/
 * _induced.py:521-699) with sigmasqr = sigma^2.  The reference has no FMM for
 * this kernel (_induced.py:159-163). */
pf_status pf_velocity_direct_cutoff(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                                    const double *g, int64_t n_tgt, const double *xt,
                                    const double *yt, double sigmasqr, double *vx, double *vy,
                                    void *stream);

/* ---------------------------------------------------------------------------
 * Induced vorticity of Gaussian blobs by direct summation (same FP32
 * hi/lo + compensated scheme as pf_velocity_direct), FP64 in and out:
 *
 *   w_k = 1/(pi ksigmasqr) sum_m g_m exp(-r2/ksigmasqr),  r2 = dx^2 + dy^2 + 1e-12
 *
 * Replaces ww2parGauss_C_cpu (src/cpp/blobs/c/ww2parGauss_C/
 * ww2parGauss_C_cpu.c:89-150) and ww2parGauss_gpu
 * (src/cpp/blobs/cuda/ww2parGauss_gpu/ww2parGauss_py_gpu.cu), reached from
 * vorticity (src/python/blobs/base/induced/_induced.py:702-963).
 * ------------------------------------------------------------------------- */
pf_status pf_vorticity_direct(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                              const double *g, int64_t n_tgt, const double *xt,
                              const double *yt, double ksigmasqr, double *w, void *stream);

/* Induced vorticity of the cutoff kernel as the reference computes it,
 *   w_k = 1/(2 pi) sum_m g_m / sqrt(dx^2 + dy^2 + sigmasqr).
 * Replaces ww2par_C_cpu (src/cpp/blobs/c/ww2par_C/ww2par_C_cpu.c:88-150) and
 * ww2par_gpu (src/cpp/blobs/cuda/ww2par_gpu/ww2par_device.cu:59-70), reached
 * from _vorticity_direct_{cpu,gpu}_cutoff (_induced.py:969-1123). */
pf_status pf_vorticity_direct_cutoff(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                                     const double *g, int64_t n_tgt, const double *xt,
                                     const double *yt, double sigmasqr, double *w, void *stream);

/* ---------------------------------------------------------------------------
 * Blob velocity by the 2D fast multipole method (uniform quadtree, FP64
 * multipole/local expansions, FP32-compensated near field with the Gaussian
 * kernel).  Arguments as fmm2d_py: sigma-derived xopt/cutoff are computed by
 * the caller as the reference Python layer does (xopt = sqrt(1.2564312086261697
 * * k sigma^2), cutoff = 5 xopt by default); the velocity is returned directly
 * (vx, vy), i.e. already mapped as (-qi/2pi, -qr/2pi).
 * `ndirect` is the target mean leaf occupancy; `tol` the requested accuracy;
 * tol == 0 computes the direct sum.
 *
 * Replaces fmm2d_py (src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm2d_py.cpp:59-186
 *   GPU, :189-316 CPU) -> fmm2dInteract (fmm.cpp:88-304), reached from
 *   _velocity_fmm_{cpu,gpu}_gauss (src/python/blobs/base/induced/_induced.py:169-336).
 * ------------------------------------------------------------------------- */
pf_status pf_velocity_fmm(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                          const double *g, int64_t n_tgt, const double *xt, const double *yt,
                          double ksigmasqr, double xopt, double cutoff, double tol,
                          int ndirect, double *vx, double *vy, void *stream);

/* pf_velocity_fmm with the tree's bounding box given by the caller:
 * box = {xmin, xmax, ymin, ymax} (host array) must contain every source and
 * target (points outside are clamped into the edge leaves, which voids the
 * error bound).  Skips the device bounding-box pass and its read-back, so the
 * call never synchronises once the FMM plan for the box is cached (for
 * resident blob sets whose box is known, e.g. a serving loop).  No NaN check.
 * Results equal pf_velocity_fmm's when box is the exact bounding box. */
pf_status pf_velocity_fmm_box(pf_ctx *ctx, int64_t n_src, const double *x, const double *y,
                              const double *g, int64_t n_tgt, const double *xt, const double *yt,
                              double ksigmasqr, double xopt, double cutoff, double tol,
                              int ndirect, const double *box, double *vx, double *vy,
                              void *stream);

/* Number of FMM plans (interaction tables and operators on the device) built
 * by this process so far.  Plans are cached by leaf level, block size,
 * expansion order and the separation key of the cutoff / root-width ratio (the
 * smallest well-separated squared box offset per level), so a blob set whose
 * box drifts from step to step reuses its plan until a list changes.  No
 * counterpart in the reference (its fmm2dInteract rebuilds its tree and lists
 * on every call, src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm.cpp:88-304). */
uint64_t pf_fmm_plan_builds(void);

/* Tuning of the FMM for the calling host thread (0 = automatic):
 * leaf_level in [2, 11]; expansion_terms (p+1) in {16, 20, 24, 28, 32};
 * block_level_drop in [0, 2] (P2P blocks of 2^drop x 2^drop leaves).  The
 * reference fixes these at build time (FMM_THETA, Ndirect-based level count,
 * p from tol: src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm.cpp:538-555); here the
 * autotuner and experiments set them at run time. */
pf_status pf_fmm_set_tuning(int leaf_level, int expansion_terms, int block_level_drop);

/* Statistics of the last pf_velocity_fmm call on a context.  Counters are
 * always collected (one atomic per CTA/warp); phase times only while
 * profiling is enabled with pf_fmm_profile (CUDA events recorded on the
 * call's stream around each phase; -1 otherwise).  pf_fmm_last_stats waits
 * for the last call's stream. */
typedef struct pf_fmm_stats {
    int32_t leaf_level;       /* L (leaves are 2^L x 2^L) */
    int32_t expansion_terms;  /* p + 1 */
    int32_t block_level_drop; /* P2P blocks of 2^kb x 2^kb leaves */
    int32_t used_direct;      /* 1 if the call fell back to the direct sum */
    int64_t n_src, n_tgt;
    int64_t p2p_pairs;        /* near-field pair interactions evaluated */
    int64_t m2l_translations; /* multipole-to-local translations */
    float ms_sort, ms_upward, ms_m2l, ms_downward, ms_p2p, ms_l2p, ms_total;
    float reserved;
    int64_t p2p_pairs_far;    /* of p2p_pairs, those whose source lies beyond the
                                 Gaussian's reach of every target of its group
                                 (no exponential evaluated) */
} pf_fmm_stats;
pf_status pf_fmm_profile(pf_ctx *ctx, int enable);
pf_status pf_fmm_last_stats(pf_ctx *ctx, pf_fmm_stats *out);

/* Leaf Morton keys of points for a tree with origin (x0, y0), leaf width
 * `leaf_width` and leaf level `leaf_level` (<= 15): key = interleave(qx, qy)
 * with qx = clamp(floor((x - x0)/leaf_width), 0, 2^L - 1), x in the even
 * bits.  The same kernel sorts the FMM's particles; exported so the integer
 * keys can be checked bit for bit.  keys: device uint32 array of n entries. */
pf_status pf_fmm_tree_keys(pf_ctx *ctx, int64_t n, const double *x, const double *y, double x0,
                           double y0, double leaf_width, int leaf_level, uint32_t *keys,
                           void *stream);

/* ---------------------------------------------------------------------------
 * Host-only (no device work): the interaction offset tables of the FMM tree
 * for leaf level `leaf_level` (root box width `root_width`, boxes at level l
 * of width root_width/2^l), P2P blocks of 2^block_level_drop leaves a side,
 * separation parameter `theta` and Gaussian `cutoff`.  Two same-level boxes
 * at integer offset (i, j) are well separated when (i^2+j^2) theta^2 >= 2 and
 * (sqrt(i^2+j^2) - sqrt 2) w >= cutoff -- the two connectivity checks of the
 * reference FMM (src/cpp/blobs/c++/fmm2d_py_cpu_gpu/fmm.cpp:1735-1835,
 * THETACUTOFFCHECK), which replaces its per-box list build
 * (MPexp_connect_CPU_, fmmsort.cpp:792-910) for a uniform tree.
 * Flattened int32 layout:
 *   L, kb; for l = 0..L: n, n (i, j) pairs (near); for l = 1..L: npos, then per
 *   position n, n (i, j) pairs (M2L); then n, n (i, j) pairs (P2P block list).
 * *needed receives the length; PF_ERR_CAPACITY if `capacity` is smaller.
 * ------------------------------------------------------------------------- */
pf_status pf_fmm_lists(int leaf_level, int block_level_drop, double root_width, double cutoff,
                       double theta, int32_t *buf, int64_t capacity, int64_t *needed);

/* ---------------------------------------------------------------------------
 * Constant-strength straight vortex panels -> induced velocity at points,
 * accumulated into (vx, vy) when `accumulate` != 0 (the blob + panel sum of
 * LagrangianSolver.evaluateVelocity, src/python/lagrangian/
 * __lagrangianSolverClass.py:257-263), else overwritten.
 *
 * Replaces _vortexPanel_Cython_cpu.inducedVelocity (src/cpp/panels/cython/
 *   vortexPanel_Cython/_vortexPanel_Cython_cpu.pyx:243-396), reached from
 *   panelSolver.inducedVelocity (src/python/panels/base/panelSolver.py:148-262),
 *   whose GPU branch is not implemented in the reference (:257-258).
 * Panel arrays have m entries (m <= 65536); evaluation arrays n entries.
 * The sum is taken over groups of 16 consecutive panels: a point at least two
 * group radii from a group's centre takes the group's FP64 Laurent series
 * (remainder <= 1e-10 of the group's share), nearer points the pair formula
 * for each panel.  Any panel order gives the same sum to that tolerance; a
 * boundary given as a chain (consecutive panels adjacent) gives the fastest.
 * Scratch: 608 B per group + 48 B per panel from the context's arena.
 * ------------------------------------------------------------------------- */
pf_status pf_panel_velocity(pf_ctx *ctx, int64_t m, const double *gamma, const double *xs,
                            const double *ys, const double *xe, const double *ye,
                            const double *cosa, const double *sina, int64_t n,
                            const double *xv, const double *yv, double *vx, double *vy,
                            int accumulate, void *stream);

/* Constant-strength source panels (strengths sigma), otherwise as
 * pf_panel_velocity: in the panel frame vxP = s/(4 pi) log(r1^2/r2^2),
 * vyP = s/(2 pi) (atan2(yP, xP-x2) - atan2(yP, xP)).  Replaces
 * _sourcePanel_Cython_cpu.inducedVelocity (src/cpp/panels/cython/
 * sourcePanel_Cython/_sourcePanel_Cython_cpu.pyx:244-393, formula :368-390), reached from
 * panelSolver.inducedVelocity with panelKernel = 0 (panelSolver.py:252-253). */
pf_status pf_source_panel_velocity(pf_ctx *ctx, int64_t m, const double *sigma, const double *xs,
                                   const double *ys, const double *xe, const double *ye,
                                   const double *cosa, const double *sina, int64_t n,
                                   const double *xv, const double *yv, double *vx, double *vy,
                                   int accumulate, void *stream);

/* Influence matrix of M vortex panels on their collocation points, FP64:
 * A[i*M + j] = (velocity at (xcp_i, ycp_i) of panel j at unit strength) .
 * (cos_i, sin_i), row-major, device array of M*M.  Replaces
 * assemble_influenceMatrix (src/cpp/panels/cython/vortexPanel_Cython/
 * _vortexPanel_Cython_cpu.pyx:81-236), reached from influenceMatrix
 * (src/python/panels/base/panelSolver.py:31-144) and Panels
 * (src/python/panels/__panelsClass.py:872-962). */
pf_status pf_panel_influence_matrix(pf_ctx *ctx, int64_t m, const double *xcp, const double *ycp,
                                    const double *xs, const double *ys, const double *xe,
                                    const double *ye, const double *cosa, const double *sina,
                                    double *A, void *stream);

/* Influence matrix of source panels: the velocity of panel j at unit
 * strength at collocation point i projected on the normal (-sin_i, cos_i).
 * Replaces _sourcePanel_Cython_cpu.assemble_influenceMatrix (src/cpp/panels/
 * cython/sourcePanel_Cython/_sourcePanel_Cython_cpu.pyx:82-237, formula :209-234), reached from
 * panelSolver.influenceMatrix with panelKernel = 0 (panelSolver.py:133-134). */
pf_status pf_source_panel_influence_matrix(pf_ctx *ctx, int64_t m, const double *xcp,
                                           const double *ycp, const double *xs, const double *ys,
                                           const double *xe, const double *ye, const double *cosa,
                                           const double *sina, double *A, void *stream);

/* Dense LU factorisation with partial pivoting of the row-major m x m FP64
 * device matrix `a`, in place: P a = L U, L unit lower; ipiv[k] (device
 * int32) is the row exchanged with row k at step k.  The DEVICE int32
 * *info_dev receives 0, or k+1 if U[k][k] is exactly zero (the factorisation
 * still completes, as LAPACK getrf).  pf_dense_lu_solve overwrites the device
 * vector b with the solution.  No host synchronisation.  Replaces the
 * scipy.linalg lu_factor / lu_solve pair of the panel solve
 * (src/python/panels/__panelsClass.py:782, :960-962). */
pf_status pf_dense_lu_factor(pf_ctx *ctx, int64_t m, double *a, int32_t *ipiv,
                             int32_t *info_dev, void *stream);
pf_status pf_dense_lu_solve(pf_ctx *ctx, int64_t m, const double *lu, const int32_t *ipiv,
                            double *b, void *stream);

/* ---------------------------------------------------------------------------
 * M4' remesh onto the lattice x_i = i h + h/2 + xb0 (same in y), h = sigma *
 * overlap.  Every cell touched by a blob's 4x4 window is emitted, including
 * cells whose summed weight is exactly zero, in (ix, iy) lexicographic order;
 * duplicates are summed in FP64.  `c` is the Wee diffusion coefficient of the
 * M4' weights (0 = plain remesh).
 *
 * Output capacity: the caller passes arrays of `capacity` entries; *n_out
 * (host pointer) receives the number of new blobs.  If capacity is too small
 * the call returns PF_ERR_CAPACITY with *n_out set to the size needed and
 * writes nothing.  ix_out / iy_out (optional, may be NULL) receive the int64
 * lattice indices.  The lattice window is found on the device; the call
 * synchronises `stream` once, at its end, to read the output count.  Its
 * scratch is sized for the context's previous window plus 25% (at least n
 * base cells); a larger window is detected on the device and costs one more
 * pass on the exact window.  The context's scratch arena is
 * shared by all calls on that context: calls issued on different streams with
 * one context must be ordered by the caller.
 *
 * Replaces Regrid (src/python/blobs/base/regrid/_regridding.py:36-222) with
 * m4kernel_1d (src/cpp/blobs/c++/interpolation_kernels_1d/
 * _interpolation_kernels_1d.cpp:21-93), reached from Blobs.redistribute
 * (src/python/blobs/__blobsClass.py:828-897) and diffusion_wee
 * (src/python/blobs/base/evolution/_evolution.py:138-235).
 * ------------------------------------------------------------------------- */
pf_status pf_remesh(pf_ctx *ctx, int64_t n, const double *x, const double *y, const double *g,
                    double h, double xb0, double yb0, double c, int64_t capacity,
                    double *x_out, double *y_out, double *g_out, int64_t *ix_out,
                    int64_t *iy_out, int64_t *n_out, void *stream);

/* Remesh with Tutty's diffusive redistribution weights instead of M4':
 * reference node i = xL + 1, Delta = (x - x_i)/h, q = 1 - 2 (hnu/h)^2 and the
 * four weights of nodes i-1..i+2 built from f = q - Delta^2 and
 * g = q - (Delta - 1)^2, hnu = sqrt(dt nu) (0 = plain Tutty redistribution).
 * Lattice, output order, explicit zeros and arguments as pf_remesh.
 * Replaces diffusion_tutty (src/python/blobs/base/evolution/_evolution.py:
 * 238-445), called from Blobs._diffusion (src/python/blobs/__blobsClass.py:
 * 1073-1111). */
pf_status pf_remesh_tutty(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                          const double *g, double h, double xb0, double yb0, double hnu,
                          int64_t capacity, double *x_out, double *y_out, double *g_out,
                          int64_t *ix_out, int64_t *iy_out, int64_t *n_out, void *stream);

/* Remesh onto a caller-given lattice window, with no host synchronisation
 * (for stream-ordered pipelines and CUDA-graph capture).  The window holds the
 * base cells ix in [ixmin, ixmin + nbx), iy in [iymin, iymin + nby) (a blob's
 * base cell is its window-left index, as in pf_remesh); outputs span
 * (nbx + 3) x (nby + 3) cells.  The output count is written to the DEVICE
 * int64 *n_out_dev; if it exceeds `capacity` nothing is written.  The DEVICE
 * int32 *status_dev (may be NULL) receives 0, or 4 if some blob lay outside
 * the window (such blobs are skipped).  Same values and order as pf_remesh.
 * ------------------------------------------------------------------------- */
pf_status pf_remesh_window(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                           const double *g, double h, double xb0, double yb0, double c,
                           int64_t ixmin, int64_t iymin, int64_t nbx, int64_t nby,
                           int64_t capacity, double *x_out, double *y_out, double *g_out,
                           int64_t *ix_out, int64_t *iy_out, int64_t *n_out_dev,
                           int32_t *status_dev, void *stream);

/* ---------------------------------------------------------------------------
 * Remesh with the window computed on the device and no host synchronisation
 * (resident blob sets in stream-ordered pipelines).  The scratch is sized for
 * windows of at most `max_base_cells` base cells (nbx nby); a larger window
 * does nothing and sets bit 8 of the DEVICE int32 *status_dev (may be NULL);
 * bits 1 and 2 report a NaN/Inf coordinate and a lattice index beyond
 * +-2^30 (nothing done either).  The DEVICE int64 *n_out_dev receives the
 * output count (0 when nothing was done; if it exceeds `capacity` nothing is
 * written), the DEVICE int64 window_dev[4] (may be NULL) the window
 * {ixmin, iymin, nbx, nby} of the blobs, so that a caller can retry with
 * max_base_cells = nbx nby.  The DEVICE double moments_dev[8] (may be NULL)
 * receives the FP64 moments {sum g, sum g x, sum g y, sum |g|} of the input
 * blobs, then of the new blobs, each summed in a fixed order (the
 * circulation and linear-impulse check of the step, no extra pass).  Same
 * values and order as pf_remesh.
 * Replaces Regrid (src/python/blobs/base/regrid/_regridding.py:36-222) for
 * callers that keep blobs on the device, as Blobs.redistribute
 * (src/python/blobs/__blobsClass.py:828-897) does between steps.
 * ------------------------------------------------------------------------- */
pf_status pf_remesh_async(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                          const double *g, double h, double xb0, double yb0, double c,
                          int64_t max_base_cells, int64_t capacity, double *x_out, double *y_out,
                          double *g_out, int64_t *ix_out, int64_t *iy_out, int64_t *n_out_dev,
                          int32_t *status_dev, int64_t *window_dev, double *moments_dev,
                          void *stream);

/* ---------------------------------------------------------------------------
 * One step of a resident blob set in one call, with no host synchronisation:
 * the induced velocity at the blobs -- FMM on the given tree box (as
 * pf_velocity_fmm_box, Ndirect 35, leaf level `leaf_level` or automatic) or
 * the direct sum (as pf_velocity_direct) -- written to vx, vy, then the M4'
 * remesh of the same blobs with the window found on the device (as
 * pf_remesh_async: count, status word and the 8 FP64 moments to device
 * memory).  All arrays are DEVICE arrays.  Replaces the pair of calls a
 * stepping loop makes, Blobs.evaluateVelocity then Blobs.redistribute
 * (src/python/blobs/__blobsClass.py:546-626, 828-897), for a serving loop that
 * issues one call per request.
 * ------------------------------------------------------------------------- */
typedef struct pf_step {
    int64_t n;                 /* blobs */
    const double *x, *y, *g;   /* blob positions and circulations */
    double ksigmasqr, xopt, cutoff, tol;
    int32_t method;            /* PF_FMM_METHOD or PF_DIRECT_METHOD */
    int32_t leaf_level;        /* 0 = automatic */
    double box[4];             /* FMM tree box {xmin, xmax, ymin, ymax} holding the blobs */
    double *vx, *vy;           /* velocity out, n entries */
    double h, xb0, yb0, c;     /* remesh lattice and Wee coefficient */
    int64_t max_base_cells;    /* remesh window bound (pf_remesh_async) */
    int64_t capacity;          /* entries of x_out, y_out, g_out */
    double *x_out, *y_out, *g_out;
    int64_t *n_out_dev;        /* output count */
    int32_t *status_dev;       /* may be NULL */
    double *moments_dev;       /* 8 doubles, may be NULL */
} pf_step;
pf_status pf_blob_step(pf_ctx *ctx, const pf_step *step, void *stream);

/* ---------------------------------------------------------------------------
 * pf_blob_step as one CUDA graph, for a resident set stepped many times.
 * pf_step_graph_create waits for the device, runs the step once (sizing the
 * scratch, building or finding the FMM plan), then captures the same call;
 * the graph owns a private context, so its scratch and FMM plan stay fixed
 * while it lives.  pf_step_graph_launch enqueues the whole step on `stream`
 * with one graph launch, ordered after prior work there.  The step's arrays
 * may change in value between launches, not in address or size; the box,
 * lattice and window bound are those of `step`.  Results are bitwise those
 * of pf_blob_step.  No reference counterpart (the reference issues every
 * kernel of a step separately, src/python/blobs/__blobsClass.py:546-626,
 * 828-897).
 * ------------------------------------------------------------------------- */
typedef struct pf_step_graph pf_step_graph;
pf_status pf_step_graph_create(pf_ctx *ctx, const pf_step *step, pf_step_graph **out);
pf_status pf_step_graph_launch(pf_step_graph *graph, void *stream);
/* Kernel nodes of the captured step (each launch adds them to
 * pf_kernel_launches). */
pf_status pf_step_graph_kernels(const pf_step_graph *graph, int64_t *kernels);
pf_status pf_step_graph_destroy(pf_step_graph *graph);

/* ---------------------------------------------------------------------------
 * pf_remesh_window without any device allocation, for callers that cannot
 * allocate: a process whose device memory is already committed to another
 * allocator (e.g. a serving loop that gives all free HBM to its own pool), or
 * a latency-critical thread that must not trigger the device-wide
 * synchronisation cudaMalloc/cudaFree can cause.  No counterpart in the
 * reference (its Regrid allocates new arrays on every call).
 *
 * Scratch is one fixed buffer of PF_NOALLOC_SCRATCH_BYTES per GPU, held until
 * the process exits; no pf_ctx is needed and none is created.  The call works
 * on the current device.  Its first call on a device does the set-up: it
 * looks up the buffer's device address, and with lazy module loading (the
 * CUDA default; CUDA_MODULE_LOADING=EAGER loads at start-up instead) that
 * lookup loads the library's device code, which is when the driver commits
 * the buffer's memory.  So make that first call early: before handing the
 * device's free memory to another allocator, and before any stream capture.
 * The address is kept per device for the process: do not use the entry point
 * across a cudaDeviceReset.  Blob sets needing more scratch than the buffer
 * holds (about 90 bytes per blob plus 8 bytes per base cell and 5 bytes per
 * output cell of the window, and 66 KB) are rejected with
 * PF_ERR_INVALID_ARG.  Every
 * call shares the buffer, which keeps the last call's contents (the call
 * clears what must start at zero): calls that overlap on the GPU (different
 * streams, or different host threads) race and must be serialised by the
 * caller.  Arguments and results as pf_remesh_window.
 * ------------------------------------------------------------------------- */
#define PF_NOALLOC_SCRATCH_BYTES (32u << 20)
pf_status pf_remesh_window_noalloc(int64_t n, const double *x, const double *y, const double *g,
                                   double h, double xb0, double yb0, double c, int64_t ixmin,
                                   int64_t iymin, int64_t nbx, int64_t nby, int64_t capacity,
                                   double *x_out, double *y_out, double *g_out, int64_t *ix_out,
                                   int64_t *iy_out, int64_t *n_out_dev, int32_t *status_dev,
                                   void *stream);

/* ---------------------------------------------------------------------------
 * Population control: drop the blobs with |g| < thr, where thr starts at
 * g_threshold_local and is divided by 10 (each division rounded, as the
 * reference's loop) until the dropped circulation sum(|g|) is below
 * g_threshold_global; the kept blobs keep their input order.  The threshold
 * search runs on the device (FP64 sums in a fixed order; a dropped sum within
 * rounding of g_threshold_global may be decided differently from numpy's
 * pairwise sum).  g_threshold_global must be positive and finite (the
 * reference loops forever otherwise).  Outputs hold n entries and must not
 * alias the inputs; the DEVICE int64 *n_out_dev receives the kept count, the
 * DEVICE double *threshold_dev (may be NULL) the threshold used.  No host
 * synchronisation.
 *
 * Replaces PopulationControl (src/python/blobs/base/regrid/_regridding.py:
 * 226-330), called from Blobs.populationControl
 * (src/python/blobs/__blobsClass.py:783-825).
 * ------------------------------------------------------------------------- */
pf_status pf_population_control(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                const double *g, double g_threshold_local,
                                double g_threshold_global, double *x_out, double *y_out,
                                double *g_out, int64_t *n_out_dev, double *threshold_dev,
                                void *stream);

/* pf_remesh followed by population control of the remeshed blobs in the same
 * pass: the dropped cells are never emitted.  Results equal pf_remesh then
 * pf_population_control on its output.  *threshold_used (host, may be NULL)
 * receives the threshold used; *n_out and capacity as pf_remesh (capacity
 * covers the kept blobs).  Replaces the redistribute + populationControl
 * pair of Blobs.evolve (src/python/blobs/__blobsClass.py:768-781). */
pf_status pf_remesh_population_control(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                                       const double *g, double h, double xb0, double yb0,
                                       double c, double g_threshold_local,
                                       double g_threshold_global, int64_t capacity,
                                       double *x_out, double *y_out, double *g_out,
                                       int64_t *ix_out, int64_t *iy_out, int64_t *n_out,
                                       double *threshold_used, void *stream);

/* ---------------------------------------------------------------------------
 * FP64 moments of a blob set, written to the DEVICE array out4:
 * out4 = {sum g, sum g x, sum g y, sum |g|}, in a fixed reduction order
 * (deterministic).  Used for the circulation / linear impulse conservation
 * checks after remesh.  No reference counterpart (the reference checks
 * nothing); listed for the conservation gate.
 * ------------------------------------------------------------------------- */
pf_status pf_moments(pf_ctx *ctx, int64_t n, const double *x, const double *y,
                     const double *g, double *out4, void *stream);

/* ---------------------------------------------------------------------------
 * Batched execution: many independent blob simulations (uneven sizes) per
 * launch.  No reference counterpart: the reference evaluates one blob set per
 * call (src/python/blobs/__blobsClass.py:546-628, :828-897).
 *
 * pf_batch_create plans every instance (FMM tree or direct sum, remesh
 * lattice window), allocates all buffers and captures the whole step --
 * velocity of every instance at its own blobs, then optionally its remesh --
 * into one CUDA graph; pf_batch_run replays it with one graph launch on
 * `stream`.  Direct-sum instances run together in one persistent kernel;
 * FMM and remesh jobs run on library streams inside the graph.  The batch
 * keeps the instance pointers: inputs may change in value between runs but
 * not in size (create a new batch when sizes change).  Results are the same
 * as the single-instance calls with the same method and tree.
 * ------------------------------------------------------------------------- */
typedef struct pf_batch_instance {
    int64_t n;                      /* blobs */
    const double *x, *y, *g;        /* device, n entries */
    double *vx, *vy;                /* device, n entries: velocity at the blobs */
    double ksigmasqr;               /* k sigma^2 */
    double cutoff;                  /* FMM Gaussian cutoff (reference: 5 xopt) */
    double box[4];                  /* xmin, xmax, ymin, ymax containing every blob */
    int32_t method;                 /* PF_FMM_METHOD or PF_DIRECT_METHOD */
    int32_t leaf_level;             /* FMM leaf level, 0 = automatic */
    int32_t expansion_terms;        /* FMM p+1, 0 = from tol */
    int32_t remesh;                 /* nonzero: M4' remesh after the velocity */
    double h, xb0, yb0, c;          /* remesh lattice spacing, origin, Wee coefficient */
    int64_t capacity;               /* remesh output capacity */
    double *x_out, *y_out, *g_out;  /* remesh outputs, capacity entries (device) */
} pf_batch_instance;

typedef struct pf_batch pf_batch;

pf_status pf_batch_create(pf_ctx *ctx, int32_t n, const pf_batch_instance *inst, double tol,
                          int32_t n_streams, pf_batch **out);
/* One graph launch: the whole batch step, ordered after prior work on stream. */
pf_status pf_batch_run(pf_batch *b, void *stream);
/* Waits for the last run; per instance: remesh output count (n_out) and
 * status (0, or 4 if a blob lay outside its box).  Host arrays of n entries,
 * either may be NULL. */
pf_status pf_batch_results(pf_batch *b, int64_t *n_out, int32_t *status);
/* Resolved method and FMM leaf level (0 for direct) per instance, and the
 * number of kernel nodes in the captured graph (any pointer may be NULL). */
pf_status pf_batch_info(const pf_batch *b, int32_t *methods, int32_t *leaf_levels,
                        int64_t *kernel_nodes);
pf_status pf_batch_destroy(pf_batch *b);

#ifdef __cplusplus
}
#endif

#endif /* PFBLOB_H */
