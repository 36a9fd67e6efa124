/*
 * brdc.h -- C ABI of the B200 boundary-row (BR) values-only
 * divide-and-conquer symmetric tridiagonal eigensolver.
 *
 * Every entry point replaces one interface of the reference artifact
 * (Ruinique/PPoPP27-BRDC-AE); the citation beside each declaration names
 * the reference file:line it stands in for.  Plain C types only: device
 * pointers are passed as typed pointers, sizes as int64_t/size_t, the CUDA
 * stream as an opaque pointer that is ABI-identical to cudaStream_t.
 *
 * Conventions shared by all device entry points
 *  - The caller owns D, E, W and the workspace (device memory).  D and E
 *    are read only.  No entry point on the solve path allocates memory.
 *  - Work is enqueued on the handle's stream and returns without a host
 *    synchronisation, so a solve can be captured in a CUDA graph.
 *    brdc_get_info() / brdc_get_diagnostics() synchronise the stream.
 *  - A handle is not thread safe (it records the last error); use one
 *    handle per host thread.
 */
#ifndef BRDC_H
#define BRDC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Values 0-8 mirror evd_status
 * (gpu/include/evd/status.h:8-18) one for one; NOT_CONVERGED is new: the
 * reference records a secular non-convergence only in a debug array and
 * still returns success (gpu/src/tridiag_solver.cu:2351-2370). */
typedef enum brdc_status {
    BRDC_STATUS_SUCCESS = 0,
    BRDC_STATUS_INVALID_HANDLE = 1,
    BRDC_STATUS_INVALID_POINTER = 2,
    BRDC_STATUS_INVALID_VALUE = 3,
    BRDC_STATUS_INVALID_WORKSPACE = 4,
    BRDC_STATUS_ALLOC_FAILED = 5,
    BRDC_STATUS_CUDA_ERROR = 6,
    BRDC_STATUS_INTERNAL_ERROR = 7,
    BRDC_STATUS_NOT_IMPLEMENTED = 8,
    BRDC_STATUS_NOT_CONVERGED = 9
} brdc_status;

/* Error source of the last failure (gpu/include/evd/types.h:24-29). */
typedef enum brdc_error_source {
    BRDC_ERROR_SRC_NONE = 0,
    BRDC_ERROR_SRC_CUDA = 1,
    BRDC_ERROR_SRC_DEVICE = 2 /* a status word written by a kernel */
} brdc_error_source;

typedef struct CUstream_st *brdc_stream_t; /* == cudaStream_t */
typedef struct brdc_handle_struct *brdc_handle;

/* Handle life cycle: replaces evd_create_handle / evd_destroy_handle
 * (gpu/include/evd/handle.h:13-14, gpu/src/handle.cu:76-150).  Like the
 * reference, a new handle owns a non-blocking stream (handle.cu:95). */
brdc_status brdc_create(brdc_handle *handle);
brdc_status brdc_destroy(brdc_handle handle);

/* Run on a caller-owned stream instead of the handle's own one.  As in the
 * CUDA runtime, NULL names the legacy default stream.  No reference
 * counterpart: the reference always uses its own stream. */
brdc_status brdc_set_stream(brdc_handle handle, brdc_stream_t stream);
brdc_status brdc_get_stream(brdc_handle handle, brdc_stream_t *stream);

/* Last error (code, source, call site): replaces evd_get_last_error
 * (gpu/include/evd/handle.h:15, gpu/src/handle.cu:152-168). */
brdc_status brdc_get_last_error(brdc_handle handle, int *code,
                                brdc_error_source *source, const char **site);

/* Status names: replaces evd_status_to_string (gpu/src/handle.cu:198-221). */
const char *brdc_status_to_string(brdc_status status);

/* Workspace query for one solve of order n: replaces
 * evd::internal::tridiag_solver_workspace_size
 * (gpu/src/syev2stage_pipeline.hpp:70-71, gpu/src/tridiag_solver.cu:2373).
 * flags: 0, or BRDC_FLAG_KEEP_CHECKPOINTS to reserve the per-level records
 * that brdc_dstebr_backward() reads.  Bytes are O(n) (every slot 256-byte
 * aligned, gpu/src/workspace_align.hpp:9); the reference reserves an
 * n x min(n,4096) delta slab on top (gpu/src/tridiag_solver_dc.cuh:183-199).
 * n <= 0 -> BRDC_STATUS_INVALID_VALUE (tridiag_solver_dc.cuh:284-286). */
#define BRDC_FLAG_KEEP_CHECKPOINTS 1
brdc_status brdc_dstebr_workspace_size(int64_t n, int flags, size_t *bytes);

/* Values-only BR solve: D[n], E[n-1] (device, read only) -> W[n] ascending
 * (device).  Replaces evd::internal::tridiag_solver_run_from_device_tridiagonal
 * (gpu/src/syev2stage_pipeline.hpp:74-77, gpu/src/tridiag_solver.cu:2541-2583)
 * with the same argument meaning and checks: NULL handle ->
 * INVALID_HANDLE; NULL D or W, or NULL E with n > 1 -> INVALID_POINTER;
 * n <= 0 -> INVALID_VALUE; workspace smaller than the query or NULL ->
 * INVALID_WORKSPACE; CUDA launch failure -> CUDA_ERROR with the last error
 * recorded.  The sign of E is ignored (|E| is used, tridiag_solver.cu:1308).
 * The call is asynchronous: a secular iteration that fails to converge is
 * reported by brdc_get_info(). */
brdc_status brdc_dstebr(brdc_handle handle, int64_t n, const double *d_D,
                        const double *d_E, double *d_W, void *workspace,
                        size_t workspace_size);

/* Allocation-free variant of brdc_dstebr, for callers that cannot allocate
 * device memory when they solve (work inside host callbacks or
 * stream-ordered sections where cudaMalloc would synchronise or is not
 * allowed, plug-ins whose host owns every device allocation, paths that
 * must not meet an allocation failure).  No reference counterpart: the
 * reference solve always takes a caller-allocated workspace.
 *  - Scratch is one static device array of 6 MiB inside the library,
 *    present on every GPU that loads it until the process exits; it bounds
 *    n to 16384.  Larger n returns BRDC_STATUS_INVALID_VALUE and records
 *    the reason as the last error.
 *  - The first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before any stream capture.  The handle must belong to the current
 *    device.  No cudaMalloc or cudaFree is ever called.
 *  - All calls share the one array: calls whose solves overlap on the GPU
 *    (other streams, other host threads) race and corrupt each other.
 *    Serialise them on one stream.  The array keeps the last call's data;
 *    every solve writes what it reads, so nothing needs clearing.
 *  - The device-side status of the last solve (unconverged roots, non-finite
 *    input, a wait that ran out) is read by brdc_dstebr_noalloc_get_info. */
brdc_status brdc_dstebr_noalloc(brdc_handle handle, int64_t n,
                                const double *d_D, const double *d_E,
                                double *d_W);

/* brdc_get_info for the allocation-free entry: the status word that the
 * last brdc_dstebr_noalloc solve on the handle's device left in the static
 * scratch array (synchronises the handle's stream; same info and return
 * values as brdc_get_info).  INVALID_VALUE when no such solve ran yet on
 * that device.  No reference counterpart. */
brdc_status brdc_dstebr_noalloc_get_info(brdc_handle handle, int *info);

/* Adjoint of brdc_dstebr for the loss L = sum_i G[i] * W[i]: writes
 * dL/dD[n] and dL/dE[n-1] (device) without forming eigenvectors, by
 * running back through the merge tree.  The workspace must come from a
 * brdc_dstebr() call with the same n, D, E made with a workspace sized for
 * BRDC_FLAG_KEEP_CHECKPOINTS (the call re-runs the forward solve itself
 * when keep_forward is 0).  No reference counterpart (values-only
 * reference has no derivative). */
brdc_status brdc_dstebr_backward(brdc_handle handle, int64_t n,
                                 const double *d_D, const double *d_E,
                                 const double *d_G, double *d_gD,
                                 double *d_gE, void *workspace,
                                 size_t workspace_size, int keep_forward);

/* Device status of the last solve on this workspace; synchronises the
 * stream.  *info = 0 on success, > 0 = number of secular roots that did
 * not converge (BRDC_STATUS_NOT_CONVERGED), < 0 = the solve stopped early
 * (BRDC_STATUS_INTERNAL_ERROR, the code also recorded as the last error
 * with source BRDC_ERROR_SRC_DEVICE):
 *   -1  a wait for a tile copy into shared memory ran out (wait limit)
 *   -3  a wait at a grid-wide barrier ran out (wait limit)
 *   -4  D or E holds a NaN or an infinity: nothing was solved.
 * After a negative info W (or dL/dD, dL/dE) holds no result. */
brdc_status brdc_get_info(brdc_handle handle, const void *workspace,
                          int *info);

/* Per-level deflation and iteration counters of the last solve on this
 * workspace (synchronises).  Mirrors the values-only fields of the
 * reference's TridiagMergeLevelDiagnostics (gpu/src/handle_impl.hpp:16-77)
 * which are compared level by level with the reference prototype. */
typedef struct brdc_level_diagnostics {
    int level;               /* 0 = merges of leaves */
    int merge_count;         /* merges at this level */
    int size_sum;            /* sum of merged node sizes (= n) */
    int dd_before_sum;       /* active poles after the small-z test */
    int dd_after_sum;        /* K: poles left after close-pole deflation */
    int dd_after_max;        /* largest K of one merge */
    int zero_deflated_total; /* size_sum - dd_before_sum */
    int close_deflated_total;/* dd_before_sum - dd_after_sum */
    int secular_iter_sum;    /* secular iterations summed over roots */
    int secular_iter_max;
    int secular_iter_failed; /* roots that hit the iteration cap */
    int threads_per_root;    /* lanes that shared one root's sums */
    long long dd_after_sq_sum; /* sum of K^2: pole-root pairs of the level */
} brdc_level_diagnostics;

#define BRDC_MAX_LEVELS 40
typedef struct brdc_diagnostics {
    int n;
    int levels;
    int leaf_count;
    int leaf_sweeps_max;     /* Jacobi sweeps of the slowest leaf */
    int leaf_sweeps_sum;     /* Jacobi sweeps summed over the leaves */
    brdc_level_diagnostics level[BRDC_MAX_LEVELS];
} brdc_diagnostics;

brdc_status brdc_get_diagnostics(brdc_handle handle, const void *workspace,
                                 brdc_diagnostics *out);

/* Deflation record of one merge level of the last solve of order n on a
 * checkpointing workspace (BRDC_FLAG_KEEP_CHECKPOINTS; synchronises the
 * stream; one matrix, not a batch).  Host arrays of n entries, indexed by
 * the row's position in its node's merged list (the two children's
 * eigenvalues in ascending order; the nodes' slices in row order):
 *   d, z     the pole and its weight as the merge formed them
 *            (z = child boundary row / sqrt(2))
 *   row      the pole's row within its node before the merge
 *            (row < floor(size/2): from the left child)
 *   state    0 secular pole, 1 deflated by the small-z test |rho z| <= tol,
 *            2 rotated out by close-pole deflation
 *   link     state 0: its index among the node's K poles (ascending d);
 *            state 2: merged position of the chain base it was rotated
 *            into; state 1: -1
 *   c, s     state 2: the Givens pair that zeroed its z (else 0)
 * and, per node of the level (2^(levels-1-level) of them, in row order),
 * K, rho and tol.  The record of the reference's merge kernels (mask, map,
 * dcount, cc, ss: gpu/src/tridiag_solver_merge_kernels.cuh:143-290), which
 * the tests compare with the reference's own decisions on the same data. */
brdc_status brdc_get_merge_trace(brdc_handle handle, const void *workspace,
                                 size_t workspace_size, int64_t n, int level,
                                 double *d, double *z, int *row, int *state, int *link,
                                 double *c, double *s, int *node_K, double *node_rho,
                                 double *node_tol);

/* Per-phase device timings of the last solve enqueued with timing on,
 * measured with CUDA events on the handle's stream between the kernels.
 * Replaces evd_get_last_stage_timings (gpu/include/evd/evd.h:27-29,
 * gpu/src/handle.cu:170-196) and the per-level slot timers of the
 * reference's diagnostics (gpu/src/tridiag_solver.cu:158-359).  Timing adds
 * one event record per kernel; leave it off for headline measurements.
 * brdc_get_last_timings synchronises the stream. */
typedef struct brdc_timings {
    float total_ms;
    float init_ms;
    float leaf_ms;       /* leaves, with the fused_levels solved alongside them */
    float merge_ms;      /* merge + deflation, all levels */
    float secular_ms;    /* secular roots, all levels */
    float lowner_ms;     /* Loewner z, all levels */
    float rows_ms;       /* boundary rows + placement, all levels */
    int launches;        /* kernels enqueued by the solve */
    int levels;
    float level_ms[BRDC_MAX_LEVELS][4]; /* merge, secular, lowner, rows */
    int fused_levels;    /* lowest merge levels solved by the subtree kernel
                            (their level_ms rows are empty) */
} brdc_timings;

/* Launch-shape parameters of a handle's solves.  None changes a result
 * beyond rounding: deflation decisions, roots and ordering follow the
 * same rules under every setting.  No reference counterpart (the
 * prototype's shapes are compile-time constants).
 *   subtree_levels      merge levels solved inside the per-subtree kernel (-1: auto),
 *                       with its leaves, in shared memory (0..5; 0 runs the
 *                       leaves alone and every level with per-level kernels;
 *                       up to 4 levels a CTA holds 256 rows, 5 levels 512)
 *   deflate_cluster     largest thread-block cluster that deflates one big
 *                       merge (1, 2, 4, 8 or 16; 1 = one CTA per merge; the
 *                       per-level deflation kernel uses at most 8)
 *   sweep_lanes_target  threads the per-level root sweeps aim to keep busy
 *                       (lanes per root = smallest power of two reaching it)
 *   fused_level_rows    levels above the subtree whose largest merge has at
 *                       most this many rows run as one fused kernel per level
 *                       (merge, deflation, roots of merges with <= 1024
 *                       poles, placement; larger merges continue in the
 *                       sweep kernel); 0 disables it
 * brdc_autotune picks them by timing; defaults: subtree_levels = -1 (5 for
 * a batch of at least 1024 rows per SM, else by tree height: 3 up to
 * n = 32768, 5 above), 16, 303104,
 * fused_level_rows = 2^30 (every level). */
typedef struct brdc_tuning {
    int subtree_levels;
    int deflate_cluster;
    int sweep_lanes_target;
    int fused_level_rows;
} brdc_tuning;

brdc_status brdc_set_tuning(brdc_handle handle, const brdc_tuning *tuning);
brdc_status brdc_get_tuning(brdc_handle handle, brdc_tuning *tuning);

/* Failure limits of a handle's solves, stored in the workspace by each
 * solve.  No reference counterpart: the reference caps the secular
 * iteration at a compile-time 50 (gpu/src/tridiag_solver_secular.cuh:12)
 * and its waits are host synchronisations.
 *   secular_max_iter  iterations of one secular root before it stops and is
 *                     counted as not converged (brdc_get_info > 0);
 *                     1..1000, default 64
 *   wait_limit_ns     bound of every device-side wait: the grid-wide
 *                     barriers of the per-level sweep kernel and the waits
 *                     for tile copies into shared memory.  A wait that runs
 *                     out stops the solve (brdc_get_info < 0); a block whose
 *                     tile wait ran out first waits up to 2 s more for its
 *                     copies in flight.  0..1e12, default 2e10 (20 s).
 * Out-of-range values -> BRDC_STATUS_INVALID_VALUE. */
typedef struct brdc_limits {
    int secular_max_iter;
    int reserved;            /* 0 */
    long long wait_limit_ns;
} brdc_limits;

brdc_status brdc_set_limits(brdc_handle handle, const brdc_limits *limits);
brdc_status brdc_get_limits(brdc_handle handle, brdc_limits *limits);

/* Autotuner: times the batched solve of this exact input (count = 1 is the
 * plain solve) under candidate tunings on the handle's stream -- coordinate
 * descent over subtree depth, deflation cluster and sweep lanes, median of
 * three runs each (one for solves above 50 ms) -- then leaves the fastest
 * on the handle and copies it to *best (may be NULL).  Uses the caller's
 * workspace, sized as for brdc_dstebr_batched; allocates no device memory;
 * synchronizes the stream, so it cannot be captured.  W receives the
 * eigenvalues.  No reference counterpart. */
brdc_status brdc_autotune(brdc_handle handle, int64_t count, const int64_t *offsets,
                          const double *d_D, const double *d_E, double *d_W,
                          void *workspace, size_t workspace_size, brdc_tuning *best);

brdc_status brdc_set_timing(brdc_handle handle, int enable);
brdc_status brdc_get_last_timings(brdc_handle handle, brdc_timings *out);

/* Graph replay of repeated solves (on by default).  A call of brdc_dstebr
 * or brdc_dstebr_backward (timing off, the stream not being captured by the
 * caller) that repeats the previous call's signature for that entry --
 * order, D, E, W (G, gD, gE and keep_forward for the adjoint), workspace and
 * its size, tuning and limits -- is captured as a CUDA graph on that second
 * call and replayed from then on: the same kernels with the same
 * arguments, less launch processing.  One graph is kept for the forwards
 * (plain, checkpointing, and the solve of brdc_dstebr_host) and one for the
 * adjoint, so a loop of forward and adjoint replays both.  New values in
 * the same buffers are read by the replay; any other change of the
 * signature drops that graph.  A failed capture falls back to ordinary
 * launches for that signature.  brdc_set_graphs(handle, 0) turns replay off
 * and drops the graphs.  brdc_get_last_launches: kernels the last forward
 * ran, and whether the last solve was a graph replay (replayed may be
 * NULL).  No reference counterpart: the reference launches every kernel
 * from the host and synchronises on each level's deflation count
 * (gpu/src/tridiag_solver.cu:624-630). */
brdc_status brdc_set_graphs(brdc_handle handle, int enable);
brdc_status brdc_get_last_launches(brdc_handle handle, int *launches, int *replayed);

/* brdc_dstebr on host buffers: D[n], E[n-1] in host memory -> W[n] in host
 * memory, through device images of D, E and W kept in the caller's
 * workspace after the solve's own (brdc_dstebr_host_workspace_size; the
 * workspace takes no checkpoints).  Same checks and statuses as
 * brdc_dstebr.  Page-locked D and E are read by the solve's first kernel
 * through their device addresses (it writes the device images as it takes
 * the norm); others are copied in first (one copy when E lies right after
 * D in one host buffer, h_E == h_D + n; else two).  A page-locked W is
 * written by the solve itself through its device address, any other W by
 * a copy out after it.  Everything is enqueued on the handle's stream; W
 * is valid once the stream has synchronised.  With
 * page-locked buffers (cudaMallocHost, cudaHostAlloc, cudaHostRegister)
 * the call does not block the host; pageable buffers are staged by the
 * runtime, which blocks it.  The solve itself is brdc_dstebr's on the
 * device images, so a repeated call with the same workspace replays its
 * graph.  No reference counterpart: the reference's LAPACK-style host
 * entry allocates and frees device memory on every call
 * (cpu/src/dstedc_dc_br.f:7-75 has the interface; brdc_dstedc_dc_br_ below
 * keeps that behaviour). */
brdc_status brdc_dstebr_host_workspace_size(int64_t n, size_t *bytes);
brdc_status brdc_dstebr_host(brdc_handle handle, int64_t n, const double *h_D,
                             const double *h_E, double *h_W, void *workspace,
                             size_t workspace_size);

/* LAPACK-style host entry with the argument list and workspace-query
 * semantics of DSTEDC_DC_BR (cpu/src/dstedc_dc_br.f:7-75): LWORK = -1 or
 * LIWORK = -1 returns LWMIN = max(1,(16+2*NTHR)*N) in WORK(1) and
 * LIWMIN = max(1,7*N) in IWORK(1) (NTHR as BRDC_WPROD_NTHREADS,
 * dstedc_dc_br.f:153-213); INFO = -1/-5/-7 for a bad N/LWORK/LIWORK.  The
 * solve itself runs on the GPU (host D, E copied in, D overwritten by the
 * ascending eigenvalues, E destroyed); INFO > 0 if a root did not converge.
 * Fortran calling convention (all arguments by reference). */
void brdc_dstedc_dc_br_(const int *n, double *d, double *e, double *work,
                        const int *lwork, int *iwork, const int *liwork,
                        int *info);

/* Batched solve of `count` independent tridiagonals of uneven order packed
 * back to back: instance b has order n_b = offsets[b+1]-offsets[b] and
 * occupies D[offsets[b] .. offsets[b+1]), E[offsets[b] .. offsets[b+1]-1)
 * (the E slot at offsets[b+1]-1 is ignored), W likewise.  offsets is a host
 * array of count+1 int64 values (offsets[0] = 0).  All levels of all
 * instances run in one pass of kernels per level.  No reference
 * counterpart (the reference solves one matrix per call).
 * Per-instance tables: a batched call made outside a stream capture copies
 * small per-instance tables (offsets, levels, prefixes) into the workspace
 * ahead of its kernels, so the workspace may be used for anything between
 * calls.  A call made while the stream is being captured copies nothing
 * (the graph holds kernels only): it needs the previous non-captured
 * batched call (or backward) on this handle to have used the same
 * workspace, offsets and checkpoint size, otherwise it returns
 * BRDC_STATUS_INVALID_VALUE; and the workspace then belongs to the graph
 * until the graph's last replay. */
brdc_status brdc_dstebr_batched_workspace_size(int64_t count,
                                               const int64_t *offsets,
                                               size_t *bytes);
brdc_status brdc_dstebr_batched(brdc_handle handle, int64_t count,
                                const int64_t *offsets, const double *d_D,
                                const double *d_E, double *d_W,
                                void *workspace, size_t workspace_size);

/* Batched adjoint, the batch form of brdc_dstebr_backward: dL/dD and dL/dE
 * of L = sum G_i W_i over all instances, packed like D and E (the ignored E
 * slot of each instance gets 0).  The workspace must have the size from
 * brdc_dstebr_batched_checkpoint_workspace_size; brdc_dstebr_batched run
 * with such a workspace records the checkpoints (keep_forward = 1 reuses
 * them), otherwise the forward solve is re-run first.  No reference
 * counterpart. */
brdc_status brdc_dstebr_batched_checkpoint_workspace_size(int64_t count,
                                                          const int64_t *offsets,
                                                          size_t *bytes);
brdc_status brdc_dstebr_batched_backward(brdc_handle handle, int64_t count,
                                         const int64_t *offsets, const double *d_D,
                                         const double *d_E, const double *d_G,
                                         double *d_gD, double *d_gE, void *workspace,
                                         size_t workspace_size, int keep_forward);

/* Eigenvalues and eigenvectors: the vector path of the reference's solver
 * (compute_eigenvectors = 1, gpu/src/tridiag_solver.cu:848-1071).  A
 * checkpointing values solve records every merge; each node's eigenvector
 * matrix is then assembled from its children's: the deflated eigenvectors
 * are children's eigenvectors (or short rotation combinations of them),
 * the K root eigenvectors blockdiag(Q_left, Q_right) * M_node[:, :K], M
 * built from the recorded permutations, rotations and secular vectors
 * (Loewner weights), the products by the library's own FP64 tensor-core
 * kernel, which writes each root eigenvector straight to its place.
 * W[n] ascending, Z column-major n x n (ld ldz >= n), column j the unit
 * eigenvector of W[j].  The workspace (query below) holds the checkpoints,
 * M and two levels of eigenvector blocks, about 16 n^2 bytes; n <= 32768.
 * It reads each level's largest K back once (a stream synchronisation) to
 * size the level's M; inside a graph capture it reads nothing and sizes it
 * by the level's largest node instead (the same result). */
brdc_status brdc_dstebr_vectors_workspace_size(int64_t n, size_t *bytes);
brdc_status brdc_dstebr_vectors(brdc_handle handle, int64_t n, const double *d_D,
                                const double *d_E, double *d_W, double *d_Z,
                                int64_t ldz, void *workspace, size_t workspace_size);

/* Library version string. */
const char *brdc_version(void);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* BRDC_H */
