// chidg_gpu_internal.cuh -- internal objects behind the C ABI handles.
#pragma once
#include "../../include/chidg_gpu.h"
#include "kernels.cuh"
#include "stream_sweep.cuh"
#include "inverse_tc.cuh"
#include "stream_matvec.cuh"
#include "umma_gemm.cuh"

#include <array>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

namespace chidg {

// Device memory from the stream-ordered pool of its device, allocated and
// freed on the stream of the context that owns it (the only stream that uses it).
struct Buffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
};

// device scalar slots (ctx->d_scal): results of reductions read by the host
constexpr int kScalSlots = 8192;
constexpr int kSlotTmp = 0;        // one-off dots / norms
constexpr int kSlotNormBefore = 1; // ||w||^2 before orthogonalisation
constexpr int kSlotWnorm = 2;      // ||w||^2 after orthogonalisation
constexpr int kSlotR0 = 3;         // ||r0||^2
constexpr int kSlotStatus = 4;     // int status word of the dataflow sweeps (nonzero = a wait ran out)
constexpr long long kSpinLimit = 2000000000LL;   // clock cycles a sweep waits for a parent (~1 s)
constexpr int kSlotH = 16;         // h(1:j, j) of the current pass (up to 4000 entries)
constexpr int kSlotY = 4096;       // y coefficients of the solution update (up to 4000 entries)
constexpr int kSlotFields = 8160;  // per-field norms (up to 32 fields)
constexpr int kMaxKrylov = 4000;   // restart length bound set by the slots above

template <typename T> struct AccOf { using type = double; };
template <> struct AccOf<float> { using type = float; };

struct IluEntry {
    int parent = -1;         // programme row of the coupled element
    int64_t a_off = 0;       // block in A (lower: A_lower; upper: U)
    int64_t t_off = 0;       // lower only: A(parent, itranspose)
    int64_t l_off = 0;       // lower only: L slot in LD
    int nc = 0;              // columns (= parent's block size)
    int32_t blk = -1;        // matrix block id (LD download), -1 for overlap copies
};

struct IluProgram {
    int nprow = 0;
    int nlocal_rows = 0;
    int64_t n_ext = 0;       // work vector length: n + overlap rows
    int64_t ld_size = 0;
    int max_lo_cols = 0, max_up_cols = 0, max_b = 0;
    int sweep_threads = 32;
    std::vector<int32_t> prow_b, prow_elem, diag_blk;
    std::vector<int64_t> v_off, z_off, diagA_off, dinv_off;
    std::vector<std::vector<IluEntry>> lo, up;
    std::vector<int32_t> fwd_rows, bwd_rows;
    std::vector<int> fwd_ptr, bwd_ptr;
    std::vector<int> ltask_ptr, stask_ptr, ltask_dmma, stask_dmma;
    std::vector<std::array<int, 3>> inv_seg;   // per level: (row_begin, count, register-tile class)
    // task-split sweeps: tasks in hand-out order, partial offsets per entry
    int ntask_f = 0, ntask_b = 0;
    int64_t part_f = 0, part_b = 0;            // scratch sizes (values)
    Buffer d_tf_row, d_tf_ent, d_tb_row, d_tb_ent, d_poff_f, d_poff_b;
    int ntask_sb = 0;                          // streamed backward sweep: U tasks + inv(D) tasks
    Buffer d_sb_row, d_sb_ent;
    std::vector<int> lb;                       // backward dependency level of every programme row
    // streamed backward sweep with the following matvec's rows (entry -3),
    // built for one matrix structure (bmv_uid) on first use
    int ntask_bmv = 0, bmv_lag = -1;
    int64_t bmv_uid = -1;
    bool bmv_reuse = false;                    // every U entry is a block of its matrix row (d_mv_skip)
    Buffer d_bmv_row, d_bmv_ent, d_col_prow, d_mv_skip;
    // rows whose D is assembled from several blocks of A (precon_HB) instead
    // of starting from one diagonal block: pieces per row, placed at (r0, c0)
    bool assembled = false;
    std::vector<int32_t> asm_ptr, asm_r0, asm_c0, asm_nr, asm_nc;
    std::vector<int64_t> asm_src;
    Buffer d_asm_ptr, d_asm_src, d_asm_r0, d_asm_c0, d_asm_nr, d_asm_nc;
    std::vector<int> inv_seg_ptr;
    Buffer d_prow_b, d_prow_elem, d_v_off, d_z_off, d_dinv_off, d_lo_ptr, d_lo_L, d_lo_par, d_lo_nc, d_up_ptr,
        d_up_U, d_up_par, d_up_nc, d_fwd_rows, d_bwd_rows, d_ltasks, d_lpairs, d_stasks, d_spairs;
    IluRows rows{};
};

}  // namespace chidg

namespace chidg {
// Launch shape of a streamed kernel: consumer warps, ring stages, bytes per
// stage.  One shape per kernel kind, block-size class and value width: the
// defaults below, or what the autotuner measured best (chidg_gpu_autotune).
struct StreamShape { int cw = 8, nstage = 2, stage_bytes = 24 * 1024; };
enum { kShapeForward = 0, kShapeBackward = 1, kShapeBackwardMv = 2, kShapeMatvec = 3, kShapeKinds = 4 };
constexpr int kShapeClasses = 4;                 // largest block: <= 64, <= 160, <= 384, <= 1024 rows
inline int shape_class(int max_b) { return max_b <= 64 ? 0 : max_b <= 160 ? 1 : max_b <= 384 ? 2 : 3; }
StreamShape stream_shape_for(int kind, int max_b, int esz);
void set_stream_shape(int kind, int max_b, int esz, const StreamShape& sh);
// resident CTAs per SM of `func` (cached per function, block size and shared memory)
int resident_ctas(const void* func, int threads, size_t smem);
}  // namespace chidg

namespace chidg {
// kernel classes timed with CUDA events when profiling is on
enum { kProfMatvec = 0, kProfIluForward = 1, kProfIluBackward = 2, kProfFactor = 3, kProfMatvec32 = 4, kProfIlu32 = 5,
       kProfFactorGemm = 6, kProfFactorInv = 7, kProfIluBackwardMv = 8, kProfClasses = 9 };
struct EvPair { cudaEvent_t a, b; int cls; };
}  // namespace chidg

namespace chidg {
// Krylov storage of one FGMRES instance; the context keeps one for the
// top-level FP64 solver and one for the FP32 inner solver so that repeated
// solves reuse their device memory
struct Workspace {
    Buffer V, Z, x0, zr, dz, tmp, rowsq;
};
// device buffers of the batched solver's per-system segments and Arnoldi
// state, kept by the context (they only grow) so that a batched solve
// allocates nothing once they have grown; a pinned counter and two events
// let the host read the active-system count without waiting
struct BatchBuffers {
    Buffer cstart, csys, sys_chunk, sys_row, row_sys, state, partial, rowsq, out;
    int32_t* h_count = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
};
}  // namespace chidg

struct BatchGraphs;   // captured launch sequences of the last batch structure (batch.cu)

struct chidg_gpu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nsm = 148;
    std::string err;
    int32_t err_elem = -1;
    int64_t launches = 0;
    int* d_status = nullptr;
    int* h_status = nullptr;
    double* d_scal = nullptr;
    double* h_scal = nullptr;
    chidg::Buffer partial, partial2;
    chidg::Workspace ws64, ws32;
    chidg::Buffer mix_v32, mix_z32;   // mixed precision: FP32 copies of the outer loop's v and z
    chidg::BatchBuffers batch;
    chidg::BatchBuffers batch_inner;  // the FP32 inner solves of a mixed-precision batched solve
    BatchGraphs* batch_graphs = nullptr;
    BatchGraphs* batch_graphs_inner = nullptr;
    // frozen systems' rows, skipped by the streamed kernels while a batched
    // solve's Arnoldi step runs (empty otherwise)
    chidg::RowMask row_mask;
    bool profiling = false;
    std::vector<chidg::EvPair> prof_pending;
    std::vector<cudaEvent_t> prof_pool;
    double prof_ms[chidg::kProfClasses] = {};
    int64_t prof_count[chidg::kProfClasses] = {};
};

struct chidg_gpu_matrix {
    chidg_gpu_ctx* ctx = nullptr;
    int64_t uid = 0;                         // unique over the process (caches keyed on a matrix use it, not the address)
    int nelem = 0, ntime = 0, nrow = 0;
    int64_t n = 0, nval = 0, nblk = 0;
    std::vector<int32_t> nvars, nterms, proc, re, rt, ce, ct, kind;
    std::vector<int64_t> eoff, voff;
    std::vector<std::vector<int32_t>> rowblk, lblk;
    std::vector<int32_t> diag;
    int max_row_cols = 0, max_b = 0, mv_threads = 32;
    bool rows_contiguous = true;             // each row's blocks follow one another in val (the streamed matvec's layout)
    chidg::Buffer val, val32, val16;
    int64_t val32_stamp = -1, val16_stamp = -1;
    chidg::Buffer d_row_ptr, d_blk_voff, d_blk_xoff, d_blk_nc, d_row_yoff, d_row_b, d_diag_voff, d_elem_nvars,
        d_elem_nterms, row_sq;
    int64_t stamp = 0;
    // chidg_matrix_t%transposed (type_chidg_matrix.f90:49): products, ILU0 and
    // Jacobi then act on A^T, kept as a second matrix T in block-row storage
    bool transposed = false;
    chidg_gpu_matrix* T = nullptr;
    int64_t T_src_stamp = -1;                // stamp of A that T's values were transposed from
    chidg::Buffer d_tr_src, d_tr_dst, d_tr_nr, d_tr_nc;   // per block of T: source / target offsets, T's block dims
    chidg::Buffer d_mass_off, d_scale_off;   // scale_diagonal: per-element offsets into mass and scale

    int bsize(int e) const { return nvars[e] * nterms[e]; }
    int64_t seg(int e, int t) const { return eoff[e] + (int64_t)t * bsize(e); }
    int row(int e, int t) const { return e * ntime + t; }
};

struct chidg_gpu_vector {
    chidg_gpu_matrix* A = nullptr;
    chidg_gpu_ctx* ctx = nullptr;
    int64_t n = 0;
    chidg::Buffer buf;
};

struct chidg_gpu_precon {
    chidg_gpu_ctx* ctx = nullptr;
    chidg_gpu_matrix* A = nullptr;
    int kind = 0;
    int precision = 0;
    int64_t stamp = 0;
    bool ld64_valid = false;               // LD holds the FP64 factors (false after an FP32 factorisation)
    bool built_transposed = false;         // the programme was built from A^T (A->transposed at build time)
    chidg::IluProgram P;
    chidg::Buffer LD, LD32, LD16, zx, zx32, piv_scratch;
    int schedule = CHIDG_SCHED_STREAM;     // sweep schedule (TASKS for blocks over 1024 rows)
    chidg::Buffer sync;                    // [2 counters][flags][forward row counts][backward row counts]
    chidg::Buffer part64, part32;          // task-split sweep partials (FP64 / low precision)
    unsigned epoch = 0;
    int sf_grid[3] = {0, 0, 0};            // resident CTAs of the dataflow sweep per vector type
    int tk_grid[4] = {0, 0, 0, 0};         // resident CTAs of the task-split sweep per variant
    // the sweeps are being captured into a CUDA graph: each sweep clears its
    // row flags and publishes with a fixed epoch, so that every replay starts
    // from cleared flags (a host epoch would be frozen into the graph)
    bool graph_safe = false;
};

namespace chidg {
int fail(chidg_gpu_ctx* ctx, int code, const std::string& msg);
int cuda_fail(chidg_gpu_ctx* ctx, cudaError_t e, const char* what);
int check_launch(chidg_gpu_ctx* ctx, const char* what);
int ensure(chidg_gpu_ctx* ctx, Buffer& buf, size_t bytes);
void release(Buffer& buf);
int grid_for(int64_t n, int threads, int cap);
int reduce_partials(chidg_gpu_ctx* ctx, const double* partial, int ncta, int nq, int slot, bool do_sqrt);
int fetch_scalars(chidg_gpu_ctx* ctx, int slot, int count, double* out);
int push_scalars(chidg_gpu_ctx* ctx, int slot, int count, const double* in);
template <typename T>
int mdot(chidg_gpu_ctx* ctx, int64_t n, const T* x, const T* y, int64_t ystride, int nq, int slot);
int matrix_lowp(chidg_gpu_matrix* A, int precision);
// The matrix the operators act on: A itself, or A^T (A->T, its values
// re-transposed when A's stamp changed) when A->transposed is set.
int matrix_op(chidg_gpu_matrix* A, chidg_gpu_matrix** out);
template <typename TA, typename TV>
int matvec_launch(chidg_gpu_matrix* A, const TA* val, const TV* x, TV* y, const TV* z, double alpha, double beta, double* row_sq);
int set_matvec_smem(chidg_gpu_matrix* A);
// Let `func` launch with `bytes` of dynamic shared memory on the current
// device.  The limit belongs to the kernel, not to one matrix or
// preconditioner, so it is only ever raised: a smaller value set for one
// object would make another object's launches fail.
int raise_smem_limit(const void* func, size_t bytes);
template <typename TV>
int precon_apply_impl(chidg_gpu_precon* M, const TV* v, TV* z, int precision);
// z = M v followed by w = Aop z (with w's row sums of squares) when both can
// run as one streamed backward sweep with the matvec rows in it: returns
// CHIDG_GPU_OK having done both, 1 (+ nothing done) when this M / Aop / type
// combination does not take the fused path, or an error code.
template <typename TV, typename TA>
int precon_apply_mv(chidg_gpu_precon* M, const TV* v, TV* z, int precision, chidg_gpu_matrix* Aop, const TA* val,
                    TV* w, double* row_sq);
int precon_set_smem(chidg_gpu_precon* M);
void release_program(IluProgram& P);
int status_word(chidg_gpu_ctx* ctx, double slot_value);
void release_batch_graphs(chidg_gpu_ctx* ctx);
int prof_begin(chidg_gpu_ctx* ctx, int cls);        // -1 when profiling is off
void prof_end(chidg_gpu_ctx* ctx, int handle);
void prof_resolve(chidg_gpu_ctx* ctx);              // after a stream sync
}  // namespace chidg
