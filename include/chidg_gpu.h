/*
 * chidg_gpu.h -- C ABI of the B200-native implicit linear-solve path for ChiDG.
 *
 * The entry points are what ChiDG's Fortran host code binds through
 * iso_c_binding when the container backend is 'cuda' (a third option next to
 * 'native' and 'petsc', selected by mod_io::backend).  Each group below names
 * the reference interface it replaces (paths relative to the ChiDG source
 * tree).  The Fortran binding module is interfaces/chidg_gpu_mod.f90.
 *
 * Conventions
 *  - Every function returns an int status: CHIDG_GPU_OK (0) or an error code.
 *    Nothing here aborts; the Fortran shim maps a nonzero code onto
 *    chidg_signal(FATAL, ...) exactly where the reference would stop
 *    (src/tools/messenger.f90:968-977).
 *  - Host arrays are owned by the caller and only read (or written, for
 *    outputs) during the call: uploads return once the copy has left the host
 *    array, whether it is pageable or page-locked.  Device objects are opaque library handles,
 *    released by the matching _destroy call (the reference's tear_down/release).
 *  - Handles are not thread safe.  A context owns one CUDA stream (the caller
 *    may pass its own, which must then outlive the context and everything
 *    made from it); all work of objects made from that context is ordered on
 *    it.  Concurrency comes from several contexts.
 *  - Element numbering is 0-based over all domains of the mesh (flattened
 *    reference element order).  The vector of an element holds ntime levels
 *    of nvars fields x nterms modes: time-major, then field, then mode
 *    (densevector_t%get_time_start, src/containers/type_densevector.f90:208).
 *  - A block couples row (element, time) to column (element, time); it is an
 *    nrows x ncols column-major FP64 array (Fortran storage of
 *    densematrix_t%mat), nrows = nvars*nterms of the row element.
 */
#ifndef CHIDG_GPU_H
#define CHIDG_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define CHIDG_GPU_OK            0
#define CHIDG_GPU_EINVAL        1  /* bad argument / inconsistent pattern            */
#define CHIDG_GPU_ENOMEM        2  /* device or pinned host allocation failed        */
#define CHIDG_GPU_ESINGULAR     3  /* zero pivot in a block inverse (mod_inv::inv)   */
#define CHIDG_GPU_ENONFINITE    4  /* NaN/Inf residual (type_newton.f90:197-200)     */
#define CHIDG_GPU_ETIMEOUT      5  /* a bounded device wait ran out                  */
#define CHIDG_GPU_ENOTCONVERGED 6  /* iteration cap reached before tol/rtol          */
#define CHIDG_GPU_ECUDA         7  /* CUDA runtime error (message via last_error)    */
#define CHIDG_GPU_ESTATE        8  /* object used in the wrong state                 */

/* ---- block kinds: the four storage groups of domain_matrix_t
 *      (src/containers/type_domain_matrix.f90:32-40) ---------------------- */
#define CHIDG_BLK_LOCAL   0   /* lblks: interior face neighbours + DIAG      */
#define CHIDG_BLK_CHIMERA 1   /* chi_blks                                    */
#define CHIDG_BLK_BC      2   /* bc_blks                                     */
#define CHIDG_BLK_HB      3   /* hb_blks (cross time-level coupling)         */

/* ---- preconditioner kinds: names of create_preconditioner
 *      (src/preconditioners/mod_preconditioner.f90:49-108) ---------------- */
#define CHIDG_PRECON_IDENTITY 0   /* 'identity' */
#define CHIDG_PRECON_JACOBI   1   /* 'jacobi'   */
#define CHIDG_PRECON_ILU0     2   /* 'ilu0'     */
#define CHIDG_PRECON_RASILU0  3   /* 'rasilu0'  */
#define CHIDG_PRECON_HB       4   /* 'HB' (precon_HB.f90): per element the inverse of its block over all time
                                     levels (DIAG blocks and hb_blks); element blocks up to 1024 rows */

/* ---- precision modes ----------------------------------------------------- */
#define CHIDG_GPU_FP64        0   /* everything FP64 (the plain GPU path)               */
#define CHIDG_GPU_MIXED_FP32  1   /* FP64 outer FGMRES; FP32 inner FGMRES, matvec and
                                     ILU factors with FP32 accumulation                 */
#define CHIDG_GPU_MIXED_BF16  2   /* as MIXED_FP32 but the ILU factors stored in BF16   */
#define CHIDG_GPU_MIXED_PRECON_FP32 3  /* FP64 FGMRES (vectors, matvec, residuals); the ILU0
                                     apply reads FP32 factors and an FP32 copy of the
                                     U blocks, with FP64 vectors and accumulation      */

#define CHIDG_ORTH_CGS 0
#define CHIDG_ORTH_MGS 1

typedef struct chidg_gpu_ctx    chidg_gpu_ctx;
typedef struct chidg_gpu_matrix chidg_gpu_matrix;
typedef struct chidg_gpu_vector chidg_gpu_vector;
typedef struct chidg_gpu_precon chidg_gpu_precon;

/* Block pattern of a chidg_matrix_t.  Blocks are listed row by row in the
 * reference storage order: for each (element, time) row the lblks in face
 * order XI_MIN, XI_MAX, ETA_MIN, ETA_MAX, ZETA_MIN, ZETA_MAX, DIAG (boundary
 * faces absent), then chi_blks, bc_blks, hb_blks
 * (type_domain_matrix.f90:102-632).  elem_proc gives the MPI rank that owns
 * each element (its RAS subdomain); NULL means every element on rank 0. */
typedef struct {
    int32_t        nelem;
    int32_t        ntime;
    const int32_t* elem_nvars;     /* [nelem] */
    const int32_t* elem_nterms;    /* [nelem] */
    const int32_t* elem_proc;      /* [nelem] or NULL */
    int64_t        nblocks;
    const int32_t* blk_row_elem;   /* [nblocks] */
    const int32_t* blk_row_time;   /* [nblocks] */
    const int32_t* blk_col_elem;   /* [nblocks] eparent */
    const int32_t* blk_col_time;   /* [nblocks] tparent */
    const int32_t* blk_kind;       /* [nblocks] CHIDG_BLK_* */
} chidg_gpu_pattern;

/* Options of linear_solver_t (src/linear_solvers/type_linear_solver.f90:21-40,
 * set by linear_solver%set :113-131). */
typedef struct {
    double  tol;                      /* absolute, |p(j+1)| < tol            */
    double  rtol;                     /* relative to the first r0 norm       */
    int32_t nmax;                     /* iteration cap, <= 0 = unlimited     */
    int32_t nkrylov;                  /* restart length                      */
    int32_t orthogonalization;        /* CHIDG_ORTH_CGS / CHIDG_ORTH_MGS     */
    int32_t inner_fgmres;             /* 1 = inner FGMRES correction         */
    double  inner_tol;
    double  inner_rtol;
    int32_t inner_nmax;
    int32_t inner_nkrylov;
    int32_t inner_orthogonalization;
    int32_t use_controller;           /* 1 = refresh M only if A's stamp changed
                                         (solver_controller%update_preconditioner);
                                         0 = refresh on every call, as without a
                                         controller (type_fgmres.f90:118-122)   */
    int32_t precision;                /* CHIDG_GPU_FP64 / _MIXED_FP32 / _MIXED_BF16 / _MIXED_PRECON_FP32 */
    int32_t mixed_inner_nkrylov;      /* mixed: Krylov length of the FP32 inner solve */
    double  mixed_inner_rtol;         /* mixed: relative tolerance of the inner solve */
    int32_t mixed_inner_nmax;         /* mixed: iteration cap of the inner solve      */
} chidg_gpu_fgmres_opts;

/* Result of one solve: fgmres_t%niter, %residual_norm and the |p(j+1)|
 * history the reference prints at verbosity >= 4. */
typedef struct {
    int32_t niter;           /* outer iterations (fgmres_t%niter)               */
    int32_t nrestart;
    int32_t inner_iters;     /* total inner iterations (inner FGMRES / mixed)   */
    int32_t nhist;           /* entries written into hist                       */
    double  residual_norm;   /* true ||b - A x|| in FP64 (print_report)         */
    double  res_estimate;    /* |p(j+1)| at exit                                */
    double  r0norm_initial;
    double  seconds;         /* wall time of the call                           */
} chidg_gpu_fgmres_result;

/* ---- context ------------------------------------------------------------ */
/* Create a context on `device`.  `stream` is a cudaStream_t to order work on,
 * or NULL to let the library create one. */
int chidg_gpu_ctx_create(int device, void* stream, chidg_gpu_ctx** out);
int chidg_gpu_ctx_destroy(chidg_gpu_ctx* ctx);
int chidg_gpu_ctx_sync(chidg_gpu_ctx* ctx);
/* Copy the last error message (NUL-terminated) into buf. */
int chidg_gpu_last_error(chidg_gpu_ctx* ctx, char* buf, int32_t buflen);
/* Element id (0-based) of the last ESINGULAR / ENONFINITE, or -1. */
int chidg_gpu_error_element(chidg_gpu_ctx* ctx, int32_t* elem);
/* Number of kernels this context has launched so far. */
int chidg_gpu_launch_count(chidg_gpu_ctx* ctx, int64_t* count);
/* Time kernel classes with CUDA events on the context's stream (off by
 * default; switching resets the totals).  Classes: 0 FP64 matvec, 1 ILU
 * forward sweep, 2 ILU backward sweep (FP64), 3 factorisation (whole
 * precon update), 4 FP32 matvec, 5 low-precision ILU apply, 6 and 7 the
 * GEMM and inverse launches of one factorisation level, 8 the FP64 backward
 * sweep with FGMRES's following matvec (w = A z) run in the same launch.
 * One count is one matvec launch, one full sweep, one factorisation, or one
 * level. */
int chidg_gpu_ctx_set_profiling(chidg_gpu_ctx* ctx, int32_t on);
int chidg_gpu_ctx_kernel_time(chidg_gpu_ctx* ctx, int32_t kernel_class, double* total_ms, int64_t* count);
/* Page-locked host memory for the upload / download calls. */
int chidg_gpu_host_alloc(size_t bytes, void** out);
int chidg_gpu_host_free(void* p);

/* ---- chidg_matrix_t (src/containers/type_chidg_matrix.f90) --------------- */
/* replaces chidg_matrix%init (:221-248) for backend='cuda' */
int chidg_gpu_matrix_create(chidg_gpu_ctx* ctx, const chidg_gpu_pattern* pat,
                            chidg_gpu_matrix** out);
int chidg_gpu_matrix_destroy(chidg_gpu_matrix* A);
/* Number of FP64 values of the packed block array (sum of nrows*ncols). */
int chidg_gpu_matrix_nvalues(chidg_gpu_matrix* A, int64_t* nvalues);
/* Vector length (sum over elements of ntime*nvars*nterms). */
int chidg_gpu_matrix_nvec(chidg_gpu_matrix* A, int64_t* n);
/* Upload all blocks, packed in pattern order, each column-major (the
 * storage that chidg_matrix%store* fills, :575-747).  `host` may be pageable
 * or pinned host memory.  Updates the stamp (chidg_matrix_t%stamp). */
int chidg_gpu_matrix_upload(chidg_gpu_matrix* A, const double* host);
/* Same, one host pointer per block (each densematrix_t%mat allocation). */
int chidg_gpu_matrix_upload_blocks(chidg_gpu_matrix* A, const double* const* block_ptrs);
/* Same, from a packed device array already resident on this GPU. */
int chidg_gpu_matrix_upload_device(chidg_gpu_matrix* A, const double* dev);
/* Part of the packed values: host[0..count) into values first..first+count-1
 * (no counterpart in the reference: a caller that packs several systems into
 * one matrix uploads each from its own array).  Bumps the stamp. */
int chidg_gpu_matrix_upload_range(chidg_gpu_matrix* A, const double* host, int64_t first, int64_t count);
/* Download the packed blocks into host memory. */
int chidg_gpu_matrix_download(chidg_gpu_matrix* A, double* host);
/* chidg_matrix%clear (:841): zero all blocks, bump the stamp. */
int chidg_gpu_matrix_clear(chidg_gpu_matrix* A);
/* chidg_matrix%scale_diagonal (:769-792), the pseudo-transient term: for
 * every element e, field f and time t, add scale[e,f] * mass_e to field f's
 * nterms x nterms diagonal sub-block of the DIAG block.  mass is packed per
 * element, nterms*nterms column-major; scale holds nvars(e) entries per
 * element, elements in order; bump the stamp. */
int chidg_gpu_matrix_scale_diagonal(chidg_gpu_matrix* A, const double* mass,
                                    const double* scale);
int chidg_gpu_matrix_stamp(chidg_gpu_matrix* A, int64_t* stamp);
/* chidg_matrix_t%transposed (:49; set by solverdata%init for the adjoint,
 * type_solverdata.f90:242).  While set, chidg_gpu_matvec computes A^T x
 * (operator_chidg_mv.f90:46-60, 692-1049), ILU0 and Jacobi factor A^T
 * (precon_ILU0.f90:148-207, precon_jacobi.f90:121-125), the FGMRES entry
 * points solve A^T x = b, and RASILU0 update/apply return CHIDG_GPU_EINVAL
 * (precon_RASILU0.f90:254,494).  The first set builds A^T in block-row
 * storage on the device (as much memory again as A's values); its values are
 * re-transposed from A when A's stamp has changed.  The packed values of A
 * (upload, download) stay in A's own layout.  A preconditioner built before the
 * flag changed rebuilds its programme at its next update. */
int chidg_gpu_matrix_set_transposed(chidg_gpu_matrix* A, int32_t transposed);
int chidg_gpu_matrix_get_transposed(chidg_gpu_matrix* A, int32_t* transposed);
/* chidg_matrix%to_file (:1451-1507): the LOCAL blocks as text, one line per
 * entry, " irow,icol,nblk,value" with each field centred in 25 columns as
 * messenger%write_line writes them (integers in I10, values in F24.14 for
 * 0.1 < |v| < 1e9 and in E24.14 otherwise), 1-based irow = b (ielem-1) + i,
 * icol = b (ielement_g-1) + j with b the block's row count, nblk the row's
 * LOCAL block count; time levels, elements and blocks in storage order, each
 * block column by column.  Like the reference it assumes one block size for
 * all elements and writes no time offset. */
int chidg_gpu_matrix_to_file(chidg_gpu_matrix* A, const char* path);
/* No counterpart in the reference: a binary image of the matrix (pattern,
 * transposed flag and packed FP64 values, little-endian) that
 * chidg_gpu_matrix_load reads back without loss into a new matrix. */
int chidg_gpu_matrix_save(chidg_gpu_matrix* A, const char* path);
int chidg_gpu_matrix_load(chidg_gpu_ctx* ctx, const char* path, chidg_gpu_matrix** out);
/* The pattern the matrix was created with (arrays sized nelem / nblocks;
 * any output may be NULL). */
int chidg_gpu_matrix_get_pattern(chidg_gpu_matrix* A, int32_t* nelem, int32_t* ntime, int64_t* nblocks,
                                 int32_t* elem_nvars, int32_t* elem_nterms, int32_t* elem_proc,
                                 int32_t* blk_row_elem, int32_t* blk_row_time, int32_t* blk_col_elem,
                                 int32_t* blk_col_time, int32_t* blk_kind);

/* ---- chidg_vector_t (src/containers/type_chidg_vector.f90) --------------- */
int chidg_gpu_vector_create(chidg_gpu_matrix* A, chidg_gpu_vector** out);
int chidg_gpu_vector_destroy(chidg_gpu_vector* x);
int chidg_gpu_vector_upload(chidg_gpu_vector* x, const double* host);
/* host[0..count) into entries first..first+count-1 (no counterpart in the
 * reference; see chidg_gpu_matrix_upload_range). */
int chidg_gpu_vector_upload_range(chidg_gpu_vector* x, const double* host, int64_t first, int64_t count);
int chidg_gpu_vector_download(chidg_gpu_vector* x, double* host);
/* Attach/read device memory directly (n doubles on this GPU). */
int chidg_gpu_vector_upload_device(chidg_gpu_vector* x, const double* dev);
int chidg_gpu_vector_device_ptr(chidg_gpu_vector* x, double** dev);
int chidg_gpu_vector_clear(chidg_gpu_vector* x);                               /* %clear  */
int chidg_gpu_vector_copy(chidg_gpu_vector* dst, const chidg_gpu_vector* src); /* =       */
int chidg_gpu_vector_axpy(chidg_gpu_vector* y, double a, const chidg_gpu_vector* x); /* y += a x */
int chidg_gpu_vector_scale(chidg_gpu_vector* x, double a);                      /* x = a x */
/* pseudo_transient_scaling (type_newton.f90:394-441), the vector side of the
 * pseudo-transient term that residual smoothing applies: for every element e,
 * time level t and field f, y's segment = scale[e,f] * mass_e * x's segment
 * (mass and scale packed as chidg_gpu_matrix_scale_diagonal takes them: mass
 * nterms x nterms column-major per element, nvars(e) scales per element).
 * x and y are distinct vectors of one matrix. */
int chidg_gpu_vector_mass_scale(const chidg_gpu_vector* x, chidg_gpu_vector* y, const double* mass, const double* scale);
/* operator_chidg_dot.f90:30-97 (dot) and type_chidg_vector.f90:1237-1305 (norm) */
int chidg_gpu_vector_dot(const chidg_gpu_vector* x, const chidg_gpu_vector* y, double* out);
int chidg_gpu_vector_norm(const chidg_gpu_vector* x, double* out);
/* chidg_vector%norm_fields (:1319-1352, sumsqr_fields of type_densevector.f90:
 * 806-830): out[f] = sqrt(sum over elements, time levels and modes of field f
 * squared), f < nfields <= 32; every element must have nfields fields. */
int chidg_gpu_vector_norm_fields(const chidg_gpu_vector* x, double* out, int32_t nfields);

/* Dot product of two device arrays that allocates no device memory.  It has
 * no counterpart in the reference.  It is for callers that cannot call
 * cudaMalloc at the point where they need a reduction: frameworks that own
 * all device memory through their own pool, and loops that cannot afford the
 * device-wide synchronisation an allocation may bring.  x, y (n doubles) and result (one double)
 * are device pointers on `device`; the work is queued on `stream` (NULL = the
 * default stream) and result is written asynchronously.  Partial sums live in
 * a fixed 128 KiB array inside this library on every GPU that loads it, so
 * n <= 67 108 864 (larger n returns CHIDG_GPU_EINVAL).  The first call on a
 * device also looks up that array's device address (a synchronous query).
 * All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int chidg_gpu_dot_noalloc(int device, const double* x, const double* y, int64_t n, double* result, void* stream);

/* ---- chidg_mv (src/containers/operator_chidg_mv.f90:46-645) --------------- */
/* y = A x over lblks, chi_blks, bc_blks and hb_blks (hb at tparent). */
int chidg_gpu_matvec(chidg_gpu_matrix* A, const chidg_gpu_vector* x, chidg_gpu_vector* y);

/* ---- preconditioner_t (src/preconditioners/type_preconditioner.f90:21-121) */
/* create + init: precon_ILU0%init (precon_ILU0.f90:64-90),
 * precon_RASILU0%init (RASILU0/precon_RASILU0.f90:139-182), precon_jacobi%init. */
int chidg_gpu_precon_create(chidg_gpu_matrix* A, int32_t kind, chidg_gpu_precon** out);
int chidg_gpu_precon_destroy(chidg_gpu_precon* M);                  /* %tear_down */
/* %update(A,b): ILU0 factorisation (precon_ILU0.f90:111-265) or RAS
 * factorisation with overlap rows (precon_RASILU0.f90:205-415).  `precision`
 * selects the factor storage: CHIDG_GPU_FP64, _MIXED_FP32 or _MIXED_PRECON_FP32
 * (FP32 copies), or _MIXED_BF16 (BF16 copies); the factorisation itself is FP64. */
int chidg_gpu_precon_update(chidg_gpu_precon* M, chidg_gpu_matrix* A, int32_t precision);
/* %apply(A,v) -> z: precon_ILU0.f90:286-411 / precon_RASILU0.f90:454-625. */
int chidg_gpu_precon_apply(chidg_gpu_precon* M, chidg_gpu_matrix* A,
                           const chidg_gpu_vector* v, chidg_gpu_vector* z);
/* Schedule of the triangular sweeps of precon%apply:
 * CHIDG_SCHED_LEVELS   one kernel launch per dependency level (wavefront);
 * CHIDG_SCHED_DATAFLOW one launch per sweep, rows taken in topological order,
 *                      each waiting (bounded) only for its own parents;
 * CHIDG_SCHED_TASKS    one launch per sweep, one task per block product, the
 *                      last task of a row completes it;
 * CHIDG_SCHED_STREAM   the TASKS work list run by persistent CTAs whose
 *                      blocks are copied into shared memory ahead of the
 *                      dependency waits (the default; blocks of more than
 *                      1024 rows run the TASKS schedule).
 * LEVELS and DATAFLOW run identical per-row arithmetic; TASKS and STREAM sum
 * each block's product before adding the blocks (same values to rounding). */
#define CHIDG_SCHED_LEVELS   0
#define CHIDG_SCHED_DATAFLOW 1
#define CHIDG_SCHED_TASKS    2
#define CHIDG_SCHED_STREAM   3
int chidg_gpu_precon_set_schedule(chidg_gpu_precon* M, int32_t schedule);
/* Packed factor blocks (L blocks and inverted diagonals at the positions of
 * the matrix's LOCAL blocks, zero elsewhere), as precon_ILU0_t%LD holds them.
 * For a transposed matrix the positions are those of A^T's blocks (the same
 * as A's for a structurally symmetric pattern). */
int chidg_gpu_precon_download_LD(chidg_gpu_precon* M, double* host);
/* The FP32 factors of the last update in a mixed precision (MIXED_FP32 and
 * MIXED_BF16: computed in FP32 with TF32 tensor-core products; MIXED_PRECON_FP32:
 * the FP64 factors rounded), in the same positions; no counterpart in the
 * reference.  CHIDG_GPU_ESTATE after an FP64 update. */
int chidg_gpu_precon_download_LD32(chidg_gpu_precon* M, float* host);
int chidg_gpu_precon_stamp(chidg_gpu_precon* M, int64_t* stamp);

/* ---- fgmres_t%solve (src/linear_solvers/type_fgmres.f90:81-310) ----------- */
/* Solve A x = b.  x is zeroed on entry (:132-136).  M is refreshed as the
 * options say; opts == NULL uses the reference defaults of linear_solver_t. */
int chidg_gpu_fgmres_solve(chidg_gpu_matrix* A, chidg_gpu_precon* M,
                           const chidg_gpu_vector* b, chidg_gpu_vector* x,
                           const chidg_gpu_fgmres_opts* opts,
                           chidg_gpu_fgmres_result* result,
                           double* hist, int32_t hist_cap);
/* Many independent solves in one: the systems are packed block-diagonally in
 * A (system s owns elements [sys_elem[s], sys_elem[s+1]), sys_elem[0] = 0,
 * sys_elem[nsys] = nelem, no block couples two systems).  Every system runs
 * its own fgmres_t%solve Arnoldi process (dot products, re-orthogonalisation
 * test, Givens rotations, convergence, restarts) while each matvec, ILU sweep
 * and reduction is one launch for the whole batch.  results[s] and
 * hist[s * hist_cap ...] are per system.  FP64 Krylov vectors for the outer
 * solve in every precision: CHIDG_GPU_FP64; CHIDG_GPU_MIXED_PRECON_FP32
 * (FP32 preconditioner blocks); CHIDG_GPU_MIXED_FP32 / _BF16 (each outer
 * step preconditioned by a batched FP32 inner FGMRES with the mixed_inner_*
 * options, FP32 or BF16 factors and copy of A; results[s].inner_iters
 * counts system s's inner iterations).  No FP64 inner FGMRES
 * (opts.inner_fgmres). */
int chidg_gpu_fgmres_solve_batched(chidg_gpu_matrix* A, chidg_gpu_precon* M, int32_t nsys,
                                   const int32_t* sys_elem, const chidg_gpu_vector* b,
                                   chidg_gpu_vector* x, const chidg_gpu_fgmres_opts* opts,
                                   chidg_gpu_fgmres_result* results, double* hist, int32_t hist_cap);
/* Fill opts with the reference defaults (type_linear_solver.f90:23-40). */
int chidg_gpu_fgmres_default_opts(chidg_gpu_fgmres_opts* opts);

/* ---- serving (no counterpart in the reference) ----------------------------
 * A continuous-batching server: requests (pattern, packed block values,
 * right-hand side) are submitted at any time; a dispatcher batches waiting
 * requests first come first served (same number of time levels, up to
 * max_batch systems, admission by a device-memory budget estimate of
 * 16 nval + 8 n (2 nkrylov + 8) bytes per request) onto `slots` worker
 * threads, each with its own context and stream, and solves each batch with
 * chidg_gpu_fgmres_solve_batched (opts; precon_kind a CHIDG_PRECON_*).  A
 * request's answer does not depend on the other requests of its batch.
 * submit copies the pattern; values and rhs are read from the caller's
 * memory until wait returns for that ticket, so they must stay valid and
 * unchanged until then.  wait blocks until the request is solved, copies x
 * (the request's vector length) and its result, and timing[0..3] = arrival,
 * batch start, batch finish (seconds since the server's creation) and the
 * batch size; it returns the batch's status.  destroy solves everything
 * queued, then stops. */
/* Failure detection without a fault (no counterpart in the reference): the
 * bounded waits the streamed kernels use (on another CTA's flag, on an
 * mbarrier) are run on a flag that nothing sets and an mbarrier that nobody
 * arrives at, each with a limit of limit_cycles clock cycles (<= 4e9).
 * *bits: bit 0 set when the flag wait gave up, bit 1 when the mbarrier wait
 * did (3: both detected).  The context stays usable. */
int chidg_gpu_selftest_bounded_waits(chidg_gpu_ctx* ctx, int64_t limit_cycles, int32_t* bits);

/* ---- launch shapes of the streamed kernels and their autotuner ------------- */
/* No counterpart in the reference (its loops have no launch shapes).  The
 * streamed kernels (forward sweep, backward sweep, backward sweep with
 * FGMRES's following matvec rows, matvec) each run with a shape: consumer
 * warps (4, 8, 16), ring stages (2..8) and bytes per stage, kept per kernel
 * kind, block-size class (largest block <= 64, 160, 384, 1024 rows) and value
 * width (8, 4, 2 bytes).  chidg_gpu_autotune times every candidate shape of
 * the four kinds on M (updated for A in `precision`, streamed schedule) and A,
 * `reps` runs each, and keeps the fastest in the table for this process; the
 * get / set calls let a host layer persist the table.  Kinds: 0 forward
 * sweep, 1 backward sweep, 2 backward sweep with matvec rows, 3 matvec. */
int chidg_gpu_autotune(chidg_gpu_precon* M, chidg_gpu_matrix* A, int32_t precision, int32_t reps);
int chidg_gpu_stream_shape_get(int32_t kind, int32_t max_b, int32_t value_bytes, int32_t* warps, int32_t* stages,
                               int32_t* stage_bytes);
int chidg_gpu_stream_shape_set(int32_t kind, int32_t max_b, int32_t value_bytes, int32_t warps, int32_t stages,
                               int32_t stage_bytes);

typedef struct chidg_gpu_server chidg_gpu_server;
int chidg_gpu_serve_create(int device, int32_t slots, int64_t mem_budget, int32_t max_batch,
                           int32_t precon_kind, const chidg_gpu_fgmres_opts* opts, chidg_gpu_server** out);
int chidg_gpu_serve_submit(chidg_gpu_server* s, const chidg_gpu_pattern* pat, const double* values,
                           const double* rhs, int64_t* ticket);
int chidg_gpu_serve_wait(chidg_gpu_server* s, int64_t ticket, double* x, chidg_gpu_fgmres_result* result,
                         double* timing);
int chidg_gpu_serve_stats(chidg_gpu_server* s, int64_t* batches, int64_t* peak_mem_bytes);
int chidg_gpu_serve_destroy(chidg_gpu_server* s);
/* A request whose system is written on the device when its batch is formed,
 * so that its values never exist in host memory: the worker creates the
 * batch's matrix A and vectors b and work (all of the packed layout), then
 * calls fill(user, ctx, A, b, work, elem0) on the worker's context, which must
 * write the request's blocks of A (its elements are A's elements elem0 ..
 * elem0 + nelem - 1), its segment of b (the right-hand side) and may use its
 * segment of work as scratch; a nonzero return fails the batch with that
 * status.  `user` must stay valid until the request's wait returns.
 * chidg_gpu_euler_fill_system is such a function. */
typedef int (*chidg_gpu_fill_fn)(void* user, chidg_gpu_ctx* ctx, chidg_gpu_matrix* A, chidg_gpu_vector* b,
                                 chidg_gpu_vector* work, int32_t elem0);
int chidg_gpu_serve_submit_fill(chidg_gpu_server* s, const chidg_gpu_pattern* pat, chidg_gpu_fill_fn fill, void* user,
                                int64_t* ticket);
/* Record of the server's batch i (0-based, in the order batches were formed):
 * rec[0] formed, rec[1] taken by a worker, rec[2] its systems on the device
 * (uploaded or filled), rec[3] preconditioner set up, rec[4] solved, rec[5]
 * solution on the host (seconds since the server's creation); rec[6] the
 * solve's device time in ms (CUDA events on the worker's stream); rec[7]
 * systems; rec[8] worker slot.  CHIDG_GPU_EINVAL for a batch not formed or
 * not yet finished. */
int chidg_gpu_serve_batch_log(chidg_gpu_server* s, int64_t i, double* rec);

/* ---- Euler DG assembly on hex boxes (the caller side of the solves) ------- */
/* The residual and Jacobian of ChiDG's Euler discretisation
 * (src/spatial/mod_spatial.f90:40-197 over the operators of
 * src/equations/fluid/euler/: euler_volume_operator, euler_boundary_average_
 * operator, euler_roe_operator, euler_bc_operator; boundary states
 * bc_state_farfield.f90 and bc_state_fluid_extrapolate.f90) on an
 * nx x ny x nz box of affine hexes, elements i-fastest, assembled on the
 * device: rhs = R(q) as the reference stores it (volume integrals negated,
 * face integrals added, mod_integrate.f90:652-1022), and the Jacobian dR/dq
 * into the DIAG and interior-face blocks of a matrix holding exactly the box
 * pattern (one time level, 5 fields, (P+1)^3 modes).  Orders 0..3; modal
 * Legendre basis in the reference's mode order (mod_ordering.f90),
 * Gauss-Legendre quadrature with ceil(3 (P+1) / 2) nodes per direction
 * (gq_rule = 2).  Not in the reference's C-callable surface: its assembly is
 * Fortran on the CPU ranks (replaces the call of update_space,
 * mod_spatial.f90:40, for such boxes). */
#define CHIDG_EULER_FARFIELD    0   /* bc_state_farfield: Riemann invariants, inflow by normal momentum <= RKTOL */
#define CHIDG_EULER_EXTRAPOLATE 1   /* bc_state_fluid_extrapolate: exterior state = interior state               */
typedef struct chidg_gpu_euler_box {
    int32_t nx, ny, nz;        /* elements per direction                                          */
    int32_t order;             /* polynomial order P, 0..3                                        */
    double lo[3], hi[3];       /* box extent                                                      */
    int32_t bc[6];             /* CHIDG_EULER_* on faces XI_MIN, XI_MAX, ETA_MIN, ..., ZETA_MAX     */
    double rho_inf, p_inf;     /* farfield density and pressure                                   */
    double vel_inf[3];         /* farfield velocity                                               */
} chidg_gpu_euler_box;
typedef struct chidg_gpu_euler chidg_gpu_euler;
int chidg_gpu_euler_create(chidg_gpu_ctx* ctx, const chidg_gpu_euler_box* box, chidg_gpu_euler** out);
int chidg_gpu_euler_destroy(chidg_gpu_euler* E);
/* rhs = R(q); with A non-NULL also A's blocks = dR/dq (every block of A is
 * overwritten; bumps A's stamp).  q and rhs: vectors of the box's length, on
 * E's context; q is read only. */
int chidg_gpu_euler_assemble(chidg_gpu_euler* E, chidg_gpu_vector* q, chidg_gpu_vector* rhs, chidg_gpu_matrix* A);
/* dtau[e * 5 + f] = cfl[f] h / (mean |u| + mean c) over the element's volume
 * nodes, h = vol^(1/3) (src/equations/fluid/type_fluid_pseudo_timestep.f90);
 * cfl holds 5 values, dtau nelem * 5 (host). */
int chidg_gpu_euler_pseudo_timestep(chidg_gpu_euler* E, chidg_gpu_vector* q, const double* cfl, double* dtau);
/* The same two calls for a box placed inside a larger layout, such as the
 * block-diagonal arena of many systems that chidg_gpu_fgmres_solve_batched
 * solves: the box's elements are A's elements elem0 .. elem0 + nelem - 1 (each
 * with 5 fields and the box's modes, A's rows there holding the box pattern);
 * q and rhs are vectors of A, of which only the box's segment is read or
 * written; with `jacobian` nonzero the box's blocks of A are overwritten. */
int chidg_gpu_euler_assemble_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0, chidg_gpu_vector* q,
                                chidg_gpu_vector* rhs, int32_t jacobian);
int chidg_gpu_euler_pseudo_timestep_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0, chidg_gpu_vector* q,
                                       const double* cfl, double* dtau);
/* Harmonic balance (assemble_harmonic_balance_t%assemble,
 * type_harmonic_balance.f90:127-229) on the device.  A holds the box's
 * pattern with ntime levels and hb_blks (every element's level t coupled to
 * its levels t' != t); vectors are element-major, then level, field, mode.
 * chidg_gpu_euler_assemble_level: level itime's spatial residual into its
 * segments of rhs and, with `jacobian`, its Jacobian into the LOCAL blocks of
 * the rows (e, itime); E is the box of that level (its own farfield state).
 * chidg_gpu_euler_pseudo_timestep_level: that level's dtau (nelem x 5).
 * chidg_gpu_hb_coupling: rhs(e, t) += sum_t' D(t, t') M q(e, t') per field, and
 * with `jacobian` every hb block (e, t) -> (e, t') = D(t, t') M on each field's
 * diagonal (the t' = t term stays in the residual, as the reference stores
 * it); D is ntime x ntime column-major (the pseudo-spectral operator,
 * mod_HB_matrices.f90), mass nterms x nterms column-major (every element has
 * nterms modes). */
int chidg_gpu_euler_assemble_level(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t itime, chidg_gpu_vector* q,
                                   chidg_gpu_vector* rhs, int32_t jacobian);
int chidg_gpu_euler_pseudo_timestep_level(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t itime, chidg_gpu_vector* q,
                                          const double* cfl, double* dtau);
int chidg_gpu_hb_coupling(chidg_gpu_matrix* A, int32_t nterms, const double* D, const double* mass, chidg_gpu_vector* q,
                          chidg_gpu_vector* rhs, int32_t jacobian);
/* The same for a box (or its hb levels) at elements elem0 .. of a larger
 * layout: the level call writes level itime of the box's rows, the coupling
 * acts on elements elem0 .. elem0 + nelem - 1 only. */
int chidg_gpu_euler_assemble_level_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0, int32_t itime,
                                      chidg_gpu_vector* q, chidg_gpu_vector* rhs, int32_t jacobian);
int chidg_gpu_hb_coupling_at(chidg_gpu_matrix* A, int32_t elem0, int32_t nelem, int32_t nterms, const double* D,
                             const double* mass, chidg_gpu_vector* q, chidg_gpu_vector* rhs, int32_t jacobian);
/* The Newton step's pseudo-transient term and right-hand side on the device
 * (newton_t%solve, type_newton.f90:181-190, contribute_pseudo_temporal :320-352):
 * dtau of the box's elements from level 0 of q (as
 * chidg_gpu_euler_pseudo_timestep), then on every time level of each element
 * field f's diagonal sub-block of the DIAG block += mass / min over the fields
 * of dtau (what chidg_gpu_matrix_scale_diagonal adds with that scale), and,
 * with rhs non-NULL, rhs = -rhs on the box's segment (b = -R).  mass: nterms x
 * nterms column-major, the same for every element; cfl: 5 values.  No host
 * round trip: the result equals chidg_gpu_euler_pseudo_timestep_at +
 * chidg_gpu_matrix_scale_diagonal + chidg_gpu_vector_scale(rhs, -1) on the box. */
int chidg_gpu_euler_pseudo_transient_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0, chidg_gpu_vector* q,
                                        chidg_gpu_vector* rhs, const double* cfl, const double* mass);
/* A Newton system of an Euler box, described for chidg_gpu_euler_fill_system:
 * the box (with ntime > 1, level t's farfield velocity replaces vel_inf:
 * harmonic balance with the levels' own inflow), the state q0 (host: the
 * box's segment, element-major, then level, field, mode), the
 * pseudo-transient cfl of every field and the element mass matrix (nterms x
 * nterms column-major); with ntime > 1 also the pseudo-spectral operator D
 * (ntime x ntime column-major) and level_vel (ntime x 3). */
typedef struct chidg_gpu_euler_system {
    chidg_gpu_euler_box box;
    int32_t ntime;
    const double* level_vel;
    const double* D;
    const double* mass;
    const double* q0;
    double cfl;
} chidg_gpu_euler_system;
/* The first Newton step's system of `user` (a chidg_gpu_euler_system) at
 * elements elem0 .. of A: A's blocks of the box = dR/dq(q0) (every level,
 * with the hb blocks) + the pseudo-transient term, b's segment = -R(q0); the
 * box's segment of work is overwritten (it holds q0).  The signature is
 * chidg_gpu_fill_fn's.  Returns once the work is done on ctx's stream. */
int chidg_gpu_euler_fill_system(void* user, chidg_gpu_ctx* ctx, chidg_gpu_matrix* A, chidg_gpu_vector* b,
                                chidg_gpu_vector* work, int32_t elem0);

#ifdef __cplusplus
}
#endif
#endif /* CHIDG_GPU_H */
