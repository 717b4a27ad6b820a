/*
 * rdcu.h -- C ABI of librdcu, a B200 (sm_100a) FP64 solver for dictionary
 * reaction-diffusion equations
 *
 *     du_i/dt = sum_j Sigma_ij Theta_j,   Theta_j = prod_k Y_k^eta_jk,
 *
 * where Y = (u_i, d_a u_i, d_a d_b u_i) on a periodic uniform grid in 1-3 dimensions.
 *
 * Two methods, as in the reference rdcu:
 *   RDCU_METHOD_DP45  explicit Dormand-Prince 4(5) with pseudospectral derivatives;
 *   RDCU_METHOD_BDF   implicit variable-order NDF/BDF with 2nd-order finite differences.
 *
 * The reference has no library boundary: its CLI (rdcu.cu main) calls file-static
 * steppers through function-pointer callbacks (dp45.h:7-11, bdf.h:9-13).  This ABI
 * replaces that stepper <-> problem callback boundary with one opaque, re-entrant
 * handle that owns its CUDA stream and device buffers.  Every entry point returns an
 * int status: RDCU_OK (0) or a negative RDCU_ERR_* code; rdcu_last_error() gives the
 * message.  Plain pointers and sizes only; no CUDA or C++ types in the signatures.
 *
 * Memory conventions: "device" pointers are CUDA device (or managed) addresses on the
 * handle's device; entry points that accept "host or device" detect the kind.
 * A state vector y has n*N doubles, field-major, each field a C-order grid with the
 * last axis fastest (N = Ns[0]*...*Ns[ndim-1]).
 */
#ifndef RDCU_H
#define RDCU_H

#ifdef __cplusplus
extern "C" {
#endif

#define RDCU_OK 0
#define RDCU_ERR_INVALID -1     /* bad argument or specification */
#define RDCU_ERR_CUDA -2        /* a CUDA runtime call failed */
#define RDCU_ERR_UNSUPPORTED -3 /* size or option outside what the library implements */
#define RDCU_ERR_TIMEOUT -4     /* a bounded device loop gave up */
#define RDCU_ERR_NOMEM -5       /* device or host allocation failed */
#define RDCU_ERR_NUMERIC -6     /* linear solve or iteration failed to converge */
#define RDCU_ERR_STATE -7       /* call out of order (e.g. eval before any step) */
#define RDCU_ERR_CALLBACK -8    /* the output callback returned non-zero */

#define RDCU_METHOD_DP45 0
#define RDCU_METHOD_BDF 1

typedef struct rdcu_handle rdcu_t;

/* Problem specification.  Mirrors the reference's option values (rdcu.cu:603-607,
 * 612-731) and its coupling-term table (rdcu.cu:606, 654-660, 822-837): term i has
 * coefficient C[i] and the integer list c[i][0..nprods[i]-1] = field, then
 * (Y index, power) pairs, Y index k = Yind*n + field with Yind 0 (u), 1..ndim (d_a u),
 * ndim+1+a*ndim+b (d_a d_b u).  A list of odd length reads the missing last power as 0,
 * as the reference's calloc'ed buffer does. */
typedef struct rdcu_spec {
  int n;                 /* number of fields (-n) */
  int ndim;              /* 1..3 (number of -N values) */
  int Ns[3];             /* grid points per axis (-N) */
  double Ls[3];          /* domain length per axis (-L) */
  int nterms;            /* number of coupling terms */
  const double *C;       /* [nterms] coefficients */
  const int *nprods;     /* [nterms] length of each integer list */
  const int *const *c;   /* [nterms] integer lists (field, Yidx, pow, Yidx, pow, ...) */
  int method;            /* RDCU_METHOD_DP45 or RDCU_METHOD_BDF (-S) */
  int fixed;             /* fixed time step (-F) */
  double rtol, atol;     /* -r, -a */
  int device;            /* CUDA device ordinal (-g) */
} rdcu_spec;

/* Sizes and resources of a handle. */
typedef struct rdcu_info {
  long long state_len;   /* n*N */
  long long Y_len;       /* n*(1+ndim+ndim^2)*N complex values written by rdcu_rhs's Y */
  long long nnz_max;     /* capacity needed for rdcu_jac's cols/vals */
  int n_channels;        /* inverse spectral channels of the fused RHS (DP45) */
  int order;             /* current BDF order (0 for DP45) */
  void *stream;          /* the handle's cudaStream_t */
  long long device_bytes;/* device memory held by the handle */
} rdcu_info;

/* ---- lifecycle -------------------------------------------------------------------
 * Replaces dp45_init (dp45.h:8) / bdf_init (bdf.h:10) together with the problem set-up
 * in rdcu.cu main (plans rdcu.cu:899-900, device buffers rdcu.cu:1065-1088, stencils
 * init_dY rdcu.cu:1147).  Allocates all device memory once. */
int rdcu_create(rdcu_t **out, const rdcu_spec *spec);
/* Replaces dp45_destroy (dp45.h:10) / bdf_destroy (bdf.h:12) and main's cleanup. */
int rdcu_destroy(rdcu_t *h);

/* State (t, h, y) and, for BDF, the order and backward differences D_1..D_order as
 * fs.dat stores them (rdcu.cu:944-990).  y and D may be host or device pointers;
 * D may be NULL when order == 0.  Replaces the initial-value copy of
 * dp45_init/bdf_init (dp45.cu:207, bdf.cu:449). */
int rdcu_set_state(rdcu_t *h, double t, double hstep, const double *y, int order,
                   const double *D);
/* Reads the state back; y (n*N) and D (order*n*N) may be host or device pointers or
 * NULL.  This is what fs.dat holds (rdcu.cu:320-339). */
int rdcu_get_state(rdcu_t *h, double *t, double *hstep, int *order, double *y, double *D);

int rdcu_get_info(rdcu_t *h, rdcu_info *info);

/* ---- problem evaluations ---------------------------------------------------------
 * f = dydt(t, y) (rdcu.cu:167-184).  y, f: host or device pointers (n*N).  If Y is not NULL
 * it receives every Y block as complex128 pairs, n*(1+ndim+ndim^2)*N of them, the
 * layout of Y.dat (rdcu.cu:287-291): for DP45 the full complex inverse transform of
 * each block (real and imaginary parts, makeY rdcu.cu:151-164); for BDF the real
 * finite-difference blocks with zero imaginary parts (rdcu.cu:122-149). */
int rdcu_rhs(rdcu_t *h, double t, const double *y, double *f, double *Y);

/* CSR Jacobian of the finite-difference RHS at y (rdcu.cu:186-250): rows (n*N+1),
 * cols/vals (capacity rdcu_info.nnz_max) and *nnz; host or device pointers.
 * Column order and explicit zeros follow the csrgeam2 accumulation of the reference.
 * For DP45 handles the reference has no stencils; the result is nnz = 0 with all-zero
 * row pointers, which is what the reference's -D4 dump of a non-stiff run holds. */
int rdcu_jac(rdcu_t *h, double t, const double *y, int *nnz, int *rows, int *cols,
             double *vals);

/* ---- stepping --------------------------------------------------------------------
 * One step attempt from the current state: dp45_step (dp45.h:7, dp45.cu:87-147) or
 * bdf_step (bdf.h:9, bdf.cu:135-323).  On return *t and *hstep are the updated time
 * and step size and *accepted is 1 (accepted) or 0 (rejected).  The incoming *t and
 * *hstep must equal the handle's state (they are the reference's in/out pointers). */
int rdcu_step(rdcu_t *h, double *t, double *hstep, double hmin, double hmax, int *accepted);

/* Dense output at t_eval within the last accepted step: dp45_eval (dp45.cu:149-152)
 * or bdf_eval (bdf.cu:325-328).  y_eval: host or device pointer (n*N). */
int rdcu_eval(rdcu_t *h, double t_eval, double *y_eval);

/* ---- whole integration -----------------------------------------------------------
 * Events delivered by rdcu_solve, in the order the reference's step_eval
 * (rdcu.cu:252-341) acts on them. */
#define RDCU_EV_ATTEMPT 0    /* after every attempt: t, h, accepted (steps.dat) */
#define RDCU_EV_EVAL 1       /* one per output time passed: t_eval, y = dense output */
#define RDCU_EV_CHECKPOINT 2 /* after the evals of one step: t, h, y = D (fs.dat) */

typedef struct rdcu_event {
  int kind;
  int accepted;      /* ATTEMPT */
  int steps;         /* accepted steps so far */
  int eval_index;    /* EVAL: index into t_eval */
  int order;         /* BDF order after the step (0 for DP45) */
  double t, h;       /* time and step size after the attempt */
  double t_eval;     /* EVAL */
  const double *y;   /* EVAL: device pointer to y(t_eval) (n*N);
                        CHECKPOINT: device pointer to the state y (n*N), followed for
                        BDF by D_1..D_order (each n*N) */
} rdcu_event;

typedef int (*rdcu_out_cb)(void *user, const rdcu_event *ev);

/* Integrates while t < t1 and h > hmin: dp45_run (dp45.h:9, dp45.cu:154-169) or
 * bdf_run (bdf.h:11, bdf.cu:330-389), with the output logic of step_eval: after each
 * accepted step, one EVAL per t_eval[i] <= t not yet output, then a CHECKPOINT if any
 * EVAL was delivered.  Steps run on the device without host round trips between
 * output times.  cb may be NULL.  t_eval: host array of n_eval increasing times. */
int rdcu_solve(rdcu_t *h, double t1, double hmin, double hmax, const double *t_eval,
               int n_eval, rdcu_out_cb cb, void *user);

/* Runs exactly n_attempts step attempts from the current state with the controller on
 * the device and no host round trip between them (the loop body of dp45_run,
 * dp45.cu:159-168, without outputs); the stepping-only workload of the benchmark.
 * *accepted receives how many were accepted.  DP45 handles only. */
int rdcu_advance(rdcu_t *h, int n_attempts, double hmin, double hmax, long long *accepted);

/* Per-kernel timing of one fused RHS stage for roofline reporting: each pass kernel of
 * DP45 stage 4 (forward x transform with the stage combination, strided transforms,
 * axis-0 pass with the derivative multipliers, inverse x transform with the dictionary)
 * is launched `reps` times between CUDA events on the handle's stream, then stage 7's
 * forward pass ("fwd_x_stage7", six slopes) and inverse pass ("inv_x_stage7", with the
 * error estimate's reads on adaptive handles).  Fills up to max_passes entries with the
 * pass name, its average time in ms and the bytes the pass must read and write per
 * launch.  Leaves y and k1 untouched.  DP45 handles only. */
typedef struct rdcu_pass_timing {
  const char *name;
  double ms;
  double bytes;
} rdcu_pass_timing;
int rdcu_profile_passes(rdcu_t *h, int reps, rdcu_pass_timing *out, int max_passes, int *npass);

/* Accepted steps and attempts counted by the last rdcu_solve. */
int rdcu_get_counters(rdcu_t *h, long long *accepted, long long *attempts);

/* Linear-solver statistics of a BDF handle since its creation: GMRES iterations, linear
 * solves (one per Newton iteration, where the reference calls cudssExecute SOLVE,
 * bdf.cu:176-180) and GMRES(40) restart cycles.  Zeros for DP45 handles.  Any output
 * pointer may be NULL. */
int rdcu_get_linear_stats(rdcu_t *h, long long *iterations, long long *solves, long long *cycles);

/* Uniform random initial condition of the reference CLI (rdcu.cu:898,991-1001):
 * srand(seed); y[N*i+j] = A0 + A/2*(2.0/RAND_MAX*rand()-1), field loop outer, with the
 * C library's own rand().  y: host array of n*N doubles.  No handle needed. */
int rdcu_random_ic(double *y, int n, long long N, double A, double A0, int seed);

/* Synchronous copy of `bytes` bytes between any host/device pointers on the handle's
 * device (the reference's cudaMemcpy calls around step_eval, rdcu.cu:277-320). */
int rdcu_memcpy(rdcu_t *h, void *dst, const void *src, unsigned long long bytes);

/* ---- coefficients and the discrete adjoint ----------------------------------------
 * No counterpart in the reference (its coefficients are fixed when FILEBASEcoupling.dat
 * is read, rdcu.cu:606-662, and it has no gradients).
 *
 * rdcu_set_coefficients: replaces the coefficient of every coupling term (C[nterms], in
 * the order of rdcu_spec.c) without rebuilding the plan.  Pseudospectral handles only;
 * call rdcu_set_state afterwards (the cached slope k1 of the old coefficients is
 * dropped). */
int rdcu_set_coefficients(rdcu_t *h, const double *C);

/* rdcu_adjoint_forward: the DP45 map y0 -> yT over the step sizes hs[0..nsteps) (host
 * array; one value repeated for fixed steps, or an accepted-step sequence recorded from
 * an adaptive run), as fixed steps (no error control).  Keeps the state every K steps
 * on the device for rdcu_adjoint_backward.  y0 and yT (may be NULL) are host or device
 * arrays of n*N doubles.  The handle's state afterwards is yT at t = sum(hs).  Needs a
 * pseudospectral handle created with fixed = 1.  Device memory: one state per
 * checkpoint plus 6*K states of stage storage and about 10 states of work space.
 *
 * rdcu_adjoint_backward: the discrete adjoint of the last rdcu_adjoint_forward: given
 * lambdaT = dL/dyT (host or device), writes dL/dy0 to grad_y0 (host or device, n*N;
 * may be NULL) and dL/dC_t for every coupling term to grad_C (host, nterms; may be
 * NULL).  Stage states are recomputed segment by segment from the checkpoints.  The
 * result is the exact derivative of the discrete map (Dormand-Prince tableau of
 * dp45.cu:6-11), up to rounding.  It can be called again with another lambdaT; the
 * handle's state (t, h, y) afterwards is unspecified: set it before stepping again. */
int rdcu_adjoint_forward(rdcu_t *h, const double *y0, const double *hs, int nsteps, int K,
                         double *yT);
int rdcu_adjoint_backward(rdcu_t *h, const double *lambdaT, double *grad_y0, double *grad_C);

/* ---- ensembles ---------------------------------------------------------------------
 * No counterpart in the reference (one problem per process).  Many independent 2D
 * pseudospectral DP45 problems -- each with its own grid, lengths, coupling terms and
 * tolerances -- stepped together: every FFT pass of a stage is one persistent launch over
 * all members' tiles, each member keeps its own adaptive step control on the device,
 * and one ensemble attempt is replayed as a CUDA graph.  A member's trajectory is
 * bitwise the one a single handle with the same spec produces (same accepted and
 * rejected steps, same states).
 *
 * rdcu_ensemble_create: specs[0..count) as for rdcu_create, with method DP45, ndim 2 and
 *   fixed 0; every spec names the same device.
 * rdcu_ensemble_set_state / get_state: (t, h, y) of member i (y host or device).
 * rdcu_ensemble_solve: every member from its state until its first accepted step at or
 *   past t1 (the end condition of rdcu_solve without outputs); synchronous.
 * rdcu_ensemble_counters: accepted steps and attempts of member i since its set_state.
 * rdcu_ensemble_tune: times one batched RHS stage for a few tile sizes (complex values
 *   per CTA) and keeps the fastest; *tile_elems receives it.  States are kept.
 * rdcu_ensemble_info: member count, the stream (cudaStream_t) and device bytes. */
typedef struct rdcu_ensemble rdcu_ensemble_t;
int rdcu_ensemble_create(rdcu_ensemble_t **out, const rdcu_spec *specs, int count);
int rdcu_ensemble_destroy(rdcu_ensemble_t *e);
int rdcu_ensemble_set_state(rdcu_ensemble_t *e, int i, double t, double hstep, const double *y);
int rdcu_ensemble_get_state(rdcu_ensemble_t *e, int i, double *t, double *hstep, double *y);
int rdcu_ensemble_solve(rdcu_ensemble_t *e, double t1, double hmin, double hmax);
int rdcu_ensemble_counters(rdcu_ensemble_t *e, int i, long long *accepted, long long *attempts);
int rdcu_ensemble_tune(rdcu_ensemble_t *e, int *tile_elems);
int rdcu_ensemble_info(rdcu_ensemble_t *e, int *count, void **stream, long long *device_bytes);
/* Last error message of the ensemble (or of the last failed rdcu_ensemble_create when
 * e is NULL). */
const char *rdcu_ensemble_last_error(rdcu_ensemble_t *e);

/* ---- allocation-free RHS ----------------------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot allocate device
 * memory.  Examples: code that runs under a device-memory budget owned by another
 * framework (a caching allocator that already holds the GPU's memory, so a raw
 * cudaMalloc fails or fragments it), and real-time loops that cannot afford the device-
 * wide synchronisation cudaMalloc/cudaFree may imply.
 *
 * f = dydt(t, y) of a pseudospectral (RDCU_METHOD_DP45) problem, like rdcu_rhs, with
 * no handle and no allocation: no cudaMalloc, cudaFree or allocating library call.
 * Its working memory (FFT tables, dictionary tables, spectra) lives in one file-scope
 * __device__ array of RDCU_NOALLOC_SCRATCH_BYTES (64 MiB) that every GPU which loads
 * librdcu holds until the process exits.  A problem needs about
 * (n_fields + n_channels) * N * 8 bytes of it for the half spectra, n_channels being the
 * dictionary's inverse transforms (one per field for the CGLE, up to one per distinct
 * derivative factor), plus a few KB of tables: the 2-field CGLE fits up to ~2M grid
 * points.  Larger problems are rejected with RDCU_ERR_UNSUPPORTED.
 *   - y and f are device pointers of n*N doubles; spec->device selects the GPU, which is
 *     made current for the call; the caller's current device is restored on return.
 *   - The work is queued on `stream` (a cudaStream_t; NULL for the default stream) and
 *     the call returns after that stream has finished it.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress); make that first call before any stream capture.
 *   - All calls share the one array, which keeps the last call's contents (each call
 *     overwrites everything it reads).  Calls that overlap on the GPU race with each
 *     other: issue them on one stream, or otherwise one at a time. */
#define RDCU_NOALLOC_SCRATCH_BYTES (64ull << 20)
int rdcu_rhs_noalloc(const rdcu_spec *spec, const double *y, double *f, void *stream);

/* ---- defect lines -----------------------------------------------------------------
 * The reference's post-processing of 3D CGLE states (makelines.py) on the GPU: the
 * phase theta = atan2(v, u) + pi of a 2-field state, the winding of every grid
 * plaquette (wloop, makelines.py:19-24), the "line cubes" on either side of each
 * winding plaquette, their periodic face-neighbour graph and its connected components
 * (findlines, makelines.py:26-57), and the minimum periodic L1 distance between the
 * components of two frames (correlate, makelines.py:112-144).  The reference's Python
 * functions are the interface these entry points replace; its graph is built by an
 * all-pairs distance test and numbered by networkx, here by a grid lookup and a
 * union-find on the device.  3D grids only, every axis >= 2, at most 2^29 points.
 *
 * rdcu_lines_create: workspace for one grid (Ns, Ls as the reference's --Ns/--Ls) on
 *   `device`; the handle owns a stream and keeps the results of its last frame.
 * rdcu_lines_find: one frame.  src (host or device) is the state -- u block then v block,
 *   2*N doubles, C order, as one frame of states.dat (makelines.py:60-65) -- when kind is
 *   RDCU_LINES_STATE, or the phase field theta (N doubles) when RDCU_LINES_PHASE.  src
 *   NULL takes the frame staged by rdcu_lines_prefetch (same kind).
 * rdcu_lines_prefetch: starts copying a host frame (pinned memory, for the copy to
 *   overlap other work) into the handle's staging buffer on a copy stream and returns;
 *   the handle's current results stay valid (a two-handle sequence stages frame k+1 in
 *   the previous frame's handle while frame k is found in the other).  The host array
 *   must stay unchanged until the rdcu_lines_find that uses it.
 *   Outputs the number of line cubes, edges and components.  Components are numbered
 *   by their smallest cube (networkx's connected_components order).
 * rdcu_lines_edges / rdcu_lines_cubes write arrays sized by the counts of the handle's
 *   last frame (rdcu_lines_find's outputs; rdcu_lines_profile finds the same frame).
 * rdcu_lines_edges: xyz[n_edges][2][3] (host or device) -- edge (u, v), u < v, of every
 *   component as cube coordinates c scaled (c * L) / (N - 1), components in order, each
 *   component's edges in ascending (u, v) order -- and comp_offsets[n_components + 1]
 *   into them.  Either pointer may be NULL.
 * rdcu_lines_cubes: the cube indices (C order) grouped by component, ascending within
 *   each, and comp_offsets[n_components + 1].  Either pointer may be NULL.
 * rdcu_lines_correlate: diffs[n_cur][n_prev] (int64, host or device) between the last
 *   frames of two handles on the same grid: the minimum over cubes a of component i of
 *   `prev` and b of component j of `cur` of sum_axis |((a - b + N/2) mod N) - N/2|, with
 *   the cube coordinates recovered from the scaled edge coordinates as the reference
 *   does (rounded for prev, truncated toward zero for cur).
 * rdcu_lines_correlate_sets: the same matrix for explicit cube sets (C-order indices
 *   grouped by component, offsets n + 1 starting at 0, host or device), on l's grid.
 * rdcu_lines_profile: one rdcu_lines_find on src, then `reps` runs of its launches with
 *   CUDA events between the pass groups (phase, faces, mark, compact, components, sort,
 *   edges; phase only for RDCU_LINES_STATE): mean ms and algorithmic bytes of each, as
 *   rdcu_profile_passes reports them.  The handle keeps that frame's results.
 * rdcu_lines_info: the handle's stream (cudaStream_t), device bytes and the number of
 *   kernels it has launched. */
#define RDCU_LINES_STATE 0
#define RDCU_LINES_PHASE 1
typedef struct rdcu_lines rdcu_lines_t;
int rdcu_lines_create(rdcu_lines_t **out, const int Ns[3], const double Ls[3], int device);
int rdcu_lines_destroy(rdcu_lines_t *l);
int rdcu_lines_find(rdcu_lines_t *l, const double *src, int kind, long long *n_cubes, long long *n_edges,
                    long long *n_components);
int rdcu_lines_prefetch(rdcu_lines_t *l, const double *src, int kind);
int rdcu_lines_edges(rdcu_lines_t *l, double *xyz, long long *comp_offsets);
int rdcu_lines_cubes(rdcu_lines_t *l, long long *cubes, long long *comp_offsets);
int rdcu_lines_correlate(rdcu_lines_t *prev, rdcu_lines_t *cur, long long *diffs);
int rdcu_lines_correlate_sets(rdcu_lines_t *l, const long long *prev_cubes, const long long *prev_offsets,
                              long long n_prev, const long long *cur_cubes, const long long *cur_offsets,
                              long long n_cur, long long *diffs);
int rdcu_lines_profile(rdcu_lines_t *l, const double *src, int kind, int reps, rdcu_pass_timing *out, int max_passes,
                       int *npass);
int rdcu_lines_info(rdcu_lines_t *l, void **stream, long long *device_bytes, long long *launches);
/* Last error message of the handle (or of the last failed rdcu_lines_create when l is
 * NULL). */
const char *rdcu_lines_last_error(rdcu_lines_t *l);

/* ---- errors ----------------------------------------------------------------------- */
const char *rdcu_error_string(int code);
/* Last error message of the handle (or of the last failed rdcu_create when h is NULL). */
const char *rdcu_last_error(rdcu_t *h);

#ifdef __cplusplus
}
#endif
#endif /* RDCU_H */
