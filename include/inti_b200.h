/*
 * inti_b200.h — C ABI of libinti_b200.so, the B200 (sm_100a) implementation
 * of Inti.jl's Nyström operator application.
 *
 * The library replaces, for one GPU, the product that Inti.jl evaluates on
 * the CPU:
 *
 *     y = alpha * (A_K * x + C * x) + beta * y,
 *     (A_K)_ij = K(x_i, y_j) * w_j        (src/nystrom.jl:93-96)
 *
 * with K one of the Laplace / Helmholtz single-layer, double-layer,
 * adjoint-double-layer or hypersingular kernels (src/kernels.jl:137-204,
 * 347-413) evaluated on the fly over all target/source node pairs (never
 * stored), and C a sparse DIM/BDIM/VDIM correction (src/bdim.jl:193-194,
 * src/vdim.jl:127) applied as a CSR SpMV.  It also builds the BDIM
 * correction on the GPU, runs GMRES (plain FP64 or FP32-inner / FP64-outer
 * refinement) and evaluates adjoints and shape gradients.
 *
 * Conventions
 *  - Every entry point returns an int status (INTI_OK = 0).  On failure
 *    inti_last_error(ctx) returns a message; no C++ exception crosses this
 *    boundary.  Error categories mirror the ArgumentError / ErrorException
 *    split of the Julia side (src/nystrom.jl:81-84, src/utils.jl:192-194).
 *  - Arrays are plain host pointers unless `on_device` is set, in which case
 *    they are device pointers on the context's device.  The library never
 *    keeps a caller's pointer past the call.
 *  - Coordinates / normals: dim x n, column-major (= array-of-structs
 *    x0 y0 [z0] x1 y1 ...), the layout of Julia's Matrix{Float64}(dim, n) and
 *    of Vector{SVector{dim,Float64}}.
 *  - Complex data (Helmholtz) is interleaved (re, im) doubles: ComplexF64.
 *  - Indices are 0-based.  inti_csr_create_from_csc accepts Julia's 1-based
 *    SparseMatrixCSC arrays directly.
 *  - One context per device and stream.  Calls on one context are serialised
 *    by an internal lock; different contexts are independent.
 */
#ifndef INTI_B200_H
#define INTI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define INTI_B200_ABI_VERSION 1

typedef struct inti_ctx inti_ctx;
typedef struct inti_quad inti_quad;
typedef struct inti_csr inti_csr;
typedef struct inti_op inti_op;

/* status codes */
enum {
  INTI_OK = 0,
  INTI_E_ARG = 1,         /* invalid argument (ArgumentError) */
  INTI_E_SHAPE = 2,       /* dimension mismatch (DimensionMismatch) */
  INTI_E_CUDA = 3,        /* CUDA runtime failure */
  INTI_E_NONFINITE = 4,   /* NaN/Inf found in an input */
  INTI_E_TIMEOUT = 5,     /* a device-side bounded wait ran out */
  INTI_E_NOMEM = 6,       /* device allocation failed */
  INTI_E_UNSUPPORTED = 7, /* combination not implemented */
  INTI_E_NOCONV = 8,      /* iterative solver did not reach tolerance */
  INTI_E_STATE = 9        /* handle used with the wrong context/state */
};

/* differential operators (src/kernels.jl:118, 310) */
enum { INTI_LAPLACE = 0, INTI_HELMHOLTZ = 1 };
/* kernels (src/kernels.jl:52-112) */
enum { INTI_SL = 0, INTI_DL = 1, INTI_ADL = 2, INTI_HS = 3 };
/* arithmetic of the pair evaluation */
enum {
  INTI_FP64 = 0,  /* FP64 pairs and accumulation */
  INTI_FP32C = 1, /* FP32 pairs, compensated (two-sum) accumulation; FP64 correction SpMV */
  INTI_TF32 = 2   /* batches only: kernel tile x density block on the tensor cores (TF32 in,
                     FP32 accumulate); FP64 correction SpMV */
};
/* element type of densities / correction values */
enum { INTI_F64 = 0, INTI_C128 = 1 };
/* inti_memcpy directions */
enum { INTI_H2D = 0, INTI_D2H = 1, INTI_D2D = 2 };
/* GMRES modes */
enum { INTI_GMRES_FP64 = 0, INTI_GMRES_MIXED = 1 };

int inti_version(void);

/* ---- context ----------------------------------------------------------- */
/* stream: a cudaStream_t to run on, or NULL for a library-owned stream.
 * The library's device buffers come from a per-device memory pool for blocks
 * under 64 MB (made by the first context on a device, 256 MB reserved then,
 * released memory kept up to 8 GB for reuse; the pool lives until exit) and
 * from cudaMalloc for larger blocks. */
int inti_ctx_create(int device, void* stream, inti_ctx** out);
int inti_ctx_destroy(inti_ctx* ctx);
/* Message of the last failure on ctx (or of the calling thread when ctx is
 * NULL, e.g. after inti_ctx_create failed).  Valid until the next call. */
const char* inti_last_error(const inti_ctx* ctx);
int inti_ctx_synchronize(inti_ctx* ctx);
/* The cudaStream_t every launch of ctx goes to. */
void* inti_ctx_stream(inti_ctx* ctx);
/* Number of library kernels launched on ctx so far. */
int64_t inti_ctx_launch_count(const inti_ctx* ctx);
/* Per-kernel device timing with CUDA events recorded on ctx's stream around
 * each launch (off by default; enabling clears earlier records). */
int inti_ctx_set_profiling(inti_ctx* ctx, int enable);
/* Total device milliseconds and launch count recorded for one kernel class
 * ("pack", "pair", "epilogue", "csr", "transpose", "dim", "gmres") since
 * profiling was enabled.  Synchronises the stream. */
int inti_ctx_profile(inti_ctx* ctx, const char* kernel, double* total_ms, int64_t* launches);

/* ---- device buffers, for callers without a CUDA allocator --------------- */
int inti_dev_alloc(inti_ctx* ctx, int64_t bytes, void** ptr);
int inti_dev_free(inti_ctx* ctx, void* ptr);
/* Stream-ordered copy on ctx's stream; synchronous when host memory is
 * involved. */
int inti_memcpy(inti_ctx* ctx, void* dst, const void* src, int64_t bytes, int direction);

/* ---- quadrature (replaces Inti.Quadrature's node arrays,
 *      src/quadrature.jl:7-11, 65-70) ------------------------------------ */
/* normals may be NULL (bare target points, src/quadrature.jl:50); weights may
 * be NULL for target-only sets (taken as 1).  nq > 0 declares that element e
 * owns the contiguous nodes e*nq .. e*nq+nq-1 (etype2qtags,
 * src/quadrature.jl:160); 0 means no element structure. */
int inti_quad_create(inti_ctx* ctx, int dim, int64_t n, const double* coords,
                     const double* normals, const double* weights, int32_t nq,
                     inti_quad** out);
int inti_quad_destroy(inti_quad* q);
int64_t inti_quad_size(const inti_quad* q);

/* ---- sparse correction (replaces SparseMatrixCSC δS/δD,
 *      src/bdim.jl:193-194, src/api.jl:170-185) -------------------------- */
int inti_csr_create(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz, const int64_t* rowptr,
                    const int32_t* col, const double* val, int dtype, inti_csr** out);
/* From Julia's 1-based CSC arrays (colptr length n+1, rowval/nzval length
 * nnz); the transposition to CSR keeps the pattern bit-exactly. */
int inti_csr_create_from_csc(inti_ctx* ctx, int64_t m, int64_t n, int64_t nnz,
                             const int64_t* colptr1, const int64_t* rowval1,
                             const double* nzval, int dtype, inti_csr** out);
int inti_csr_info(const inti_csr* c, int64_t* m, int64_t* n, int64_t* nnz, int* dtype);
/* Copies the CSR arrays to host buffers sized m+1, nnz, nnz*(1|2). */
int inti_csr_download(const inti_csr* c, int64_t* rowptr, int32_t* col, double* val);
/* y = alpha*C*x + beta*y (alpha/beta: 2 doubles, re and im). */
int inti_csr_apply(inti_csr* c, const double* x, double* y, const double* alpha,
                   const double* beta, int on_device);
int inti_csr_destroy(inti_csr* c);

/* ---- operator (replaces IntegralOperator + its LinearMap sum with the
 *      correction, src/nystrom.jl:67-96, src/api.jl:179-184) ------------- */
/* k_re/k_im: Helmholtz wavenumber (ignored for Laplace).  correction may be
 * NULL.  The operator keeps references to target, source and correction:
 * destroy it before them. */
int inti_op_create(inti_ctx* ctx, int pde, int kernel, double k_re, double k_im,
                   const inti_quad* target, const inti_quad* source,
                   const inti_csr* correction, int precision, inti_op** out);
/* A = c_dl*(D + C_dl) + c_sl*(S + C_sl) (3D) evaluated in ONE pass over the
 * pairs: the combined-field operator the reference composes as a LinearMap
 * sum (docs/src/examples/helmholtz_scattering.jl:485-486,
 * L = I/2 + D - i*k*S).  c_dl, c_sl: 2 doubles each (re, im; real for
 * Laplace).  The corrections (either may be NULL) are merged once into
 * c_dl*C_dl + c_sl*C_sl.  inti_gmres fuses DL + SL terms into this operator
 * by itself. */
int inti_op_create_combined(inti_ctx* ctx, int pde, double k_re, double k_im,
                            const inti_quad* target, const inti_quad* source,
                            const inti_csr* corr_dl, const inti_csr* corr_sl, const double* c_dl,
                            const double* c_sl, int precision, inti_op** out);
int inti_op_info(const inti_op* op, int64_t* m, int64_t* n, int* dtype);
/* Y = alpha*(A*X + C*X) + beta*Y for nrhs columns (leading dimensions ldx,
 * ldy in elements).  alpha, beta: 2 doubles each (re, im); NULL means 1, 0.
 * beta = 0 does not read Y.  FP64 3D operators (every kernel) apply 8 or
 * more columns in one pass that evaluates each kernel value once
 * per 64 columns (16 complex / 32 real when all columns fit), the pair tile
 * multiplied with the columns on the FP64 MMA path; other operators and
 * fewer columns run one pair product per column.  Results agree to rounding
 * (the summation order differs). */
int inti_op_apply(inti_op* op, const double* x, int64_t ldx, double* y, int64_t ldy,
                  int32_t nrhs, const double* alpha, const double* beta, int on_device);
/* Y = alpha*(A^T*X + C^T*X) + beta*Y: the transpose (not conjugate) apply,
 * the density gradient of the adjoint method. */
int inti_op_apply_transpose(inti_op* op, const double* x, int64_t ldx, double* y,
                            int64_t ldy, int32_t nrhs, const double* alpha,
                            const double* beta, int on_device);
/* Dense column-major m x n matrix of A (without the correction), the GPU
 * counterpart of assemble_matrix (src/nystrom.jl:103-124). */
int inti_op_assemble(inti_op* op, double* out, int on_device);
int inti_op_destroy(inti_op* op);
/* Launch shape of the operator's pair kernel: targets per thread (2 or 4)
 * and the number of source chunks (split).  Operators created through
 * inti_op_create / inti_op_create_combined with more than 2^26 pairs pick
 * them by timing the candidates once, on a zero density, at creation (the
 * choice is cached per context and problem shape, and reused by operators
 * the library derives internally); smaller ones, or a context with
 * autotuning off, keep the occupancy heuristic.  No counterpart in the
 * reference (launch configuration). */
int inti_op_tuning(const inti_op* op, int32_t* targets_per_thread, int32_t* split);
int inti_ctx_set_autotune(inti_ctx* ctx, int enable);  /* default on */
/* Square operators (target === source, the same inti_quad) of every kernel
 * (single layer, double layer, combined field, adjoint double layer,
 * hypersingular; 3D and the 2D Laplace kernels) use a symmetric pair kernel: each unordered pair's distance,
 * reciprocal square root and phase are computed once and serve both
 * y_i += K(x_i, x_j) w_j x_j and y_j += K(x_j, x_i) w_i x_i (G(x, y) =
 * G(y, x); the double-layer and adjoint-double-layer radial factors are shared
 * and only the dipole or the normal changes; the hypersingular kernel is
 * symmetric in the pair).  The partial sums are reduced in a fixed order, so results
 * are deterministic; they differ from the one-sided kernel's by rounding.
 * The row and column partials take up to N^2 / (256 or 512) values.  While
 * they fit the partial budget (2e9 bytes, or a quarter of the device memory
 * free at creation if less) the work runs in one launch; beyond it the work
 * items are grouped into panels of source blocks, run one after another with
 * the partials of one panel at a time, so the operator's memory stays O(N)
 * plus the budget (inti_op_panels reports the panel count, 1 for one
 * launch).  inti_ctx_set_partial_budget sets the budget for operators
 * created afterwards (bytes; 0 restores 2e9).  For symmetric operators
 * inti_op_tuning reports the targets per thread and the source blocks per
 * work item.  inti_ctx_set_symmetric(ctx, 0) makes operators created
 * afterwards use the one-sided kernel; inti_op_symmetric returns 1 when an
 * operator uses the symmetric form, 0 otherwise.  No counterpart in the
 * reference, which evaluates every ordered pair (src/nystrom.jl:117-124). */
int inti_ctx_set_symmetric(inti_ctx* ctx, int enable);  /* default on */
int inti_op_symmetric(const inti_op* op);
int inti_ctx_set_partial_budget(inti_ctx* ctx, double bytes);
int inti_op_panels(const inti_op* op);
/* Small FP64 operators (at most 2^20 target-source pairs and 65,536 sources,
 * e.g. the 1,000-node kite) apply in a single-launch form: one kernel per product builds the
 * source records, forms the pair sums (a cluster of up to 8 CTAs per 32
 * targets, the CTAs and their warps splitting the sources, sums in a fixed
 * order), adds the correction rows and applies alpha/beta.  Transposed
 * products of small square operators run the same kernel with the transposed
 * kernel and the transposed correction; item-sharded applies keep the tiled
 * kernels.  inti_ctx_set_single_launch(ctx,
 * 0) makes operators created afterwards use the tiled kernels;
 * inti_op_single_launch returns 1 when an operator uses the form.  No
 * counterpart in the reference. */
int inti_ctx_set_single_launch(inti_ctx* ctx, int enable);  /* default on */
int inti_op_single_launch(const inti_op* op);
/* Item shard of a symmetric operator for one process per GPU: after
 * inti_op_set_shard(op, r, P), inti_op_apply on rank r computes this rank's
 * share of the unordered node pairs (every P-th work item, largest first,
 * so the shares balance) as a partial y over all rows; rank 0 adds the
 * correction and beta*y.  The sum of the P partials (one all-reduce) is
 * alpha*(A + C)x + beta*y.  nranks = 1 restores the whole operator.
 * Multi-column applies of a shard run column by column; transposes and
 * GMRES refuse shards.  Operators without the symmetric form return
 * INTI_E_UNSUPPORTED (shard them by target rows: an operator on a row block
 * of targets).  No counterpart in the reference (single process). */
int inti_op_set_shard(inti_op* op, int rank, int nranks);

/* ---- BDIM correction on the GPU (src/bdim.jl:50-196) ------------------- */
/* green_multiplier: n values or NULL for -1/2 (on the surface,
 * src/nystrom.jl:196-207).  derivative = 1 builds the ADL/HS corrections.
 * Outputs two CSR handles (δS, δD) with the element-block pattern of
 * src/quadrature.jl:250-256. */
int inti_dim_correction(inti_ctx* ctx, int pde, double k_re, double k_im,
                        const inti_quad* q, int derivative, const double* green_multiplier,
                        inti_csr** dS, inti_csr** dD);
/* The same for targets other than the source nodes (src/api.jl:105-148 and
 * bdim.jl:50-196 with etype_to_nearest_points, src/quadrature.jl:264-286):
 * each target is assigned to the element of its nearest source node (ties to
 * the lowest node index) when that distance is <= maxdist (INFINITY: every
 * target); green_multiplier (m values, required) is -1 inside, 0 outside,
 * -1/2 on the surface (src/nystrom.jl:196-207).  Outputs m x n CSR handles
 * whose row i holds the nq nodes of target i's element, or nothing.
 * derivative = 1 needs target normals. */
int inti_dim_correction_targets(inti_ctx* ctx, int pde, double k_re, double k_im,
                                const inti_quad* target, const inti_quad* source, int derivative,
                                const double* green_multiplier, double maxdist, inti_csr** dS,
                                inti_csr** dD);

/* ---- GMRES on L = shift*I + sum_t coef_t * op_t ------------------------- */
typedef struct {
  int32_t iterations;       /* total Krylov iterations (all restarts, all solves) */
  int32_t outer;            /* refinement steps (MIXED) or restarts + 1 (FP64) */
  int32_t fp64_applies;     /* applications of the FP64 operator */
  int32_t fp32_applies;     /* applications of the FP32C operator */
  int32_t converged;        /* 1 if relres <= rtol */
  int32_t reserved;
  double relres;            /* ||b - L x|| / ||b||, FP64 residual */
  double seconds;           /* wall time of the whole call: operator set-up it
                               triggers (fused combined field, FP32C twins and
                               their timed launch shapes), copies of b and x
                               in, the solve, and x back (host clock) */
  double setup_seconds;     /* the operator set-up part of seconds (0 when
                               cached from an earlier solve) */
} inti_gmres_stats;

/* coefs: nterms complex pairs; shift: one complex pair.  All ops must share
 * the same source/target quadrature and be FP64 operators; MIXED mode runs
 * the inner solves with FP32C twins built internally.  b/x: n values
 * (complex if any operator or coefficient is).  x is the initial guess on
 * input.  history (nullable, maxiter+1 doubles) receives relative residuals
 * per iteration. */
int inti_gmres(inti_ctx* ctx, int32_t nterms, inti_op* const* ops, const double* coefs,
               const double* shift, const double* b, double* x, double rtol,
               int32_t restart, int32_t maxiter, int32_t mode, int on_device,
               double* history, inti_gmres_stats* stats);
/* Systems of at most max_unknowns unknowns (default 8192) run each Arnoldi
 * step's orthogonalisation (both Gram-Schmidt passes), the new basis vector
 * and the Givens update in one single-CTA kernel after the operator
 * application, and the host checks the residual once per four steps (the
 * steps enqueued after convergence leave the iterate alone; their operator
 * applications still run and are counted); larger systems use the multi-CTA
 * kernels and read the Hessenberg column back every step.  0 turns the
 * small-system form off.  Both forms give the same iterates up to rounding.
 * No counterpart in the reference (its examples call IterativeSolvers). */
int inti_ctx_set_gmres_small(inti_ctx* ctx, int64_t max_unknowns);

/* ---- adjoint: gradients of J(u), u = A sigma (Laplace, on-the-fly) ------ */
/* Given the cotangent g = dJ/du (m values) and the density sigma (n values),
 * returns dJ/dsigma (n), dJ/dcoords (dim x n), dJ/dnormals (dim x n) and
 * dJ/dweights (n) of the source quadrature; any output may be NULL.  Tiles
 * of the kernel are recomputed, nothing m x n is stored. */
int inti_op_grad_sources(inti_op* op, const double* g, const double* sigma, double* dsigma,
                         double* dcoords, double* dnormals, double* dweights, int on_device);

/* ---- measured peaks for the roofline ------------------------------------ */
/* Sustained throughput of dependent-free FP64 FMA, FP32 FMA and MUFU rsqrt
 * on this device, in operations per second (FMA counted as 2 flops). */
int inti_measure_peaks(inti_ctx* ctx, double* fp64_flops, double* fp32_flops,
                       double* mufu_ops);
/* Tensor-core throughput (flop/s) of back-to-back tcgen05.mma kind::tf32,
 * M = N = 128, K = 8, on every SM: the shape the batched kernel issues.
 * No counterpart in the reference (measurement support for the roofline). */
int inti_measure_peak_tf32(inti_ctx* ctx, double* tf32_flops);

/* ---- batches: many surfaces, many right-hand sides, one launch ----------
 * The block-diagonal operator diag(A_1 + C_1, ..., A_S + C_S) over S
 * quadratures of uneven size (the batching form of the workloads: plane
 * waves on a batch of star-shaped surfaces).  kernel: INTI_SL, INTI_DL or
 * 4 (combined field c_dl*DL + c_sl*SL, coefficients as 2 doubles each).
 * corr_dl / corr_sl: per-surface corrections (arrays of S handles, entries
 * or arrays may be NULL); they are merged with the coefficients.  Densities
 * are column-major over the concatenated nodes (surface s occupies rows
 * off_s .. off_s + n_s - 1 of every column). */
typedef struct inti_batch inti_batch;
int inti_batch_create(inti_ctx* ctx, int32_t nsurf, const inti_quad* const* quads, int pde, int kernel,
                      double k_re, double k_im, const double* c_dl, const double* c_sl,
                      const inti_csr* const* corr_dl, const inti_csr* const* corr_sl,
                      inti_batch** out);
/* Y = alpha*(A X + C X) + beta*Y for nrhs columns.  precision INTI_FP64
 * (CUDA cores) or INTI_TF32 (Helmholtz: kernel tiles x density blocks on the
 * tcgen05 tensor cores, FP32 accumulation, FP64 correction).  With
 * on_device = 1, a TF32 apply after a first one with the same nrhs only
 * enqueues work on the context's stream (no allocation, no synchronisation),
 * so it can be captured into a CUDA graph and replayed. */
int inti_batch_apply(inti_batch* b, int precision, const double* x, int64_t ldx, double* y, int64_t ldy,
                     int32_t nrhs, const double* alpha, const double* beta, int on_device);
/* GMRES on every (surface, column) system shift*I + A_s + C_s at once, in
 * lockstep: one batched operator launch per Krylov step (Helmholtz).
 * mode INTI_GMRES_FP64, or INTI_GMRES_MIXED: inner solves on the TF32
 * tensor-core operator, FP64 residuals.  B/X: ld x nrhs complex, X is the
 * initial guess on input.  relres (nullable, S*nrhs doubles, index
 * s*nrhs + r) receives each system's final FP64 relative residual; stats
 * report the worst. */
int inti_batch_gmres(inti_batch* b, const double* shift, const double* B, double* X, int64_t ld,
                     int32_t nrhs, double rtol, int32_t restart, int32_t maxiter, int32_t mode,
                     int on_device, double* relres, inti_gmres_stats* stats);
int64_t inti_batch_size(const inti_batch* b);
int inti_batch_destroy(inti_batch* b);

/* ---- allocation-free apply ------------------------------------------------
 * No counterpart in the reference: Inti.jl's operators allocate freely.
 * For callers that cannot call cudaMalloc when they apply the operator (a
 * framework's caching allocator owns the device memory, a solver loop that
 * must not pay for allocation).
 *
 * y = alpha*(A x + C x) + beta*y with the same kernels as inti_op_apply, but
 * every array is a caller-owned DEVICE pointer on the current device:
 * target coords/normals (dim x m), source coords/normals/weights (dim x n,
 * n), the optional CSR correction (rowptr m+1, col, val; all NULL for none),
 * x (n) and y (m) — complex data interleaved for Helmholtz.  alpha/beta are
 * host pairs (re, im) or NULL for 1, 0.  Work goes to `stream` (NULL: the
 * legacy default stream); synchronize != 0 waits and reports device-side
 * timeouts as INTI_E_TIMEOUT.  With synchronize = 0 no status reports a
 * timeout: a timed-out call leaves NaN in every entry of y.
 *
 * Scratch lives in a fixed 32 MiB static device array that every GPU loading
 * the library holds until exit; problems whose packed sources plus one
 * partial vector exceed it are rejected with INTI_E_ARG.  The first call on a
 * device sets that array up (address lookup, phase tables): make it before
 * any stream capture.  All calls on a device share the array, so calls that
 * overlap on the GPU race.  Errors: inti_last_error(NULL). */
int inti_apply_noalloc(int pde, int kernel, int dim, double k, int precision, int64_t m,
                       const double* tcoords, const double* tnormals, int64_t n,
                       const double* scoords, const double* snormals, const double* sweights,
                       const int64_t* rowptr, const int32_t* col, const double* val,
                       const double* x, double* y, const double* alpha, const double* beta,
                       void* stream, int synchronize);

/* Accuracy of the pair loops' fast special functions on this device, against
 * extended-precision host values: out[0] max relative error of the FP64
 * reciprocal square root over [1e-27, 1e27]; out[1], out[2] max absolute
 * error of the FP64 e^{i theta} for theta <= 25 and theta <= 1000; out[3]
 * the same for the FP32 form, theta <= 25; out[4] max relative error of the
 * FP64 x^{-3/2} over [1e-27, 1e27]; out[5] max relative error of the FP64
 * reciprocal over [1e-27, 1e27].  out holds 6 doubles. */
int inti_selftest_math(inti_ctx* ctx, double* out);
/* Runs the device-side bounded wait of the pair kernels on an mbarrier that
 * nothing arrives at: the wait gives up after its poll limit, records the
 * timeout in the context's flag and the kernel returns, so this returns
 * INTI_E_TIMEOUT and the context stays usable (the flag is cleared).  For
 * tests of the timeout path; no counterpart in the reference. */
int inti_selftest_wait_timeout(inti_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* INTI_B200_H */
