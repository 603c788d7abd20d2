// ILU programme: streamed task sweeps (CHIDG_SCHED_STREAM).
//
// The work of one triangular sweep is the task list of the task-split sweep
// (one block product per task, handed out in topological order of the parent
// rows), executed by persistent CTAs (several per SM, so that several tasks
// are in flight on each SM) with a producer/consumer split:
//
//   producer (one lane of the last warp)  takes a ticket, and copies the task's
//       block column-chunk by column-chunk into a ring of shared-memory stages
//       with cp.async.bulk (completion counted on the stage's mbarrier).  The
//       copy does not depend on the sweep's values, so it runs ahead of the
//       dependency waits: the block is in shared memory when the parent row is
//       published.
//   consumers (the other warps)  wait (bounded) for the parent row, stage its
//       segment of z, multiply the chunks as they land, release each stage, and
//       at the last chunk publish the block's partial product.  The last task of
//       a row to finish completes it.
//
// Backward sweep: the product with inv(D_r) is a task of its own (entry -2),
// ordered after the row's U tasks and before its children's; it waits for
// the row's partials to be complete (the `ready` flag set by the last U task),
// adds them to z_r in entry order and multiplies by inv(D_r) streamed through
// the same ring, so inv(D_r) is prefetched like every other block.
//
// Deadlock freedom: a task waits only for tasks with smaller tickets.  Each
// CTA consumes its tasks in ticket order, and a producer posts a task's chunks
// as soon as stages free, so the unfinished task with the smallest ticket can
// always proceed.  Every wait (flags, mbarriers) is bounded; on a timeout the
// sweep records status 1 and finishes with wrong values instead of hanging.
//
// Bulk copies need 16-byte aligned source, destination and size: each chunk's
// source is rounded down to 16 bytes (the element offset inside the stage is
// carried with the chunk) and its length rounded up; device buffers carry 256
// bytes of slack past their end, so the rounded copies stay inside them.
#pragma once

#include "kernels.cuh"

namespace chidg {

constexpr int SS_MAX_B = 1024;                              // rows per block
constexpr int SS_MAX_STAGES = 8;
constexpr int SS_MAX_NC = 512;                              // consumer threads (16 warps)

struct StreamMeta {
    int task;      // ticket, -1 = end of the sweep for this CTA
    int pr, q;     // programme row, entry (-1 combine-only, -2 backward diagonal)
    int chunk, nchunk;
    int col0, ncols;
    int shift;     // element offset of the chunk inside the stage
    int skip;      // the row's system is frozen: nothing is read, computed or written
};

// Rows of frozen systems in a batched solve (a system whose Arnoldi process
// has converged while the others go on): row r belongs to system row_sys[r],
// frozen when active[row_sys[r]] == 0.  The streamed kernels skip such rows:
// no block is copied, no wait is taken, nothing is written, so a step costs
// what its active systems read.  The rows of a system depend only on rows of
// the same system, and a frozen system's vectors are not read again before
// its next restart, so skipping them changes no active system's values.
// Empty (active == nullptr): every row runs.
struct RowMask {
    const int32_t* row_sys = nullptr;
    const int32_t* active = nullptr;
    int nrow = 0;              // rows the map covers
};
__device__ __forceinline__ bool row_frozen(const RowMask& mk, int row) {
    return mk.active != nullptr && mk.active[mk.row_sys[row]] == 0;
}

struct StreamTasks {
    const int32_t* task_row;
    const int32_t* task_ent;
    const int64_t* part_off;    // per entry: offset of its partial in the scratch vector
    unsigned* row_count;        // per row: completed entry tasks, never reset (wraps by entry count)
    unsigned* ready;            // backward: per row, epoch once all U partials are written
};

// the row structure of a matrix whose rows' blocks are stored one after
// another (the streamed matvec's view)
struct MatvecRowsView {
    const int64_t* row_ptr;     // blocks of row i: row_ptr[i] .. row_ptr[i+1]-1
    const int64_t* blk_voff;
    const int64_t* blk_xoff;
    const int32_t* blk_nc;
    const int64_t* row_yoff;
    const int32_t* row_b;
};

// ring of `stages` stages of `stage_bytes` (a multiple of 16), the parent
// segment (xcap values: the largest block of the programme), the row-sum
// scratch (nc values, one per consumer thread), mbarriers and descriptors
__host__ __device__ constexpr size_t stream_xcap(int max_b) { return (size_t)((max_b + 31) / 32) * 32; }
// (max_b: the largest segment staged at once -- a block's columns, or with
// fused matvec rows also a matrix row's columns; a 32-double scratch follows
// the row sums for the fused rows' sums of squares)
__host__ __device__ constexpr size_t stream_smem_bytes(size_t acc_size, int stages, int stage_bytes, int max_b, int nc) {
    return (size_t)stages * stage_bytes + (stream_xcap(max_b) + nc) * acc_size + 32 * sizeof(double) +
           2 * SS_MAX_STAGES * sizeof(uint64_t) + SS_MAX_STAGES * sizeof(StreamMeta) + 64;
}

// The matvec that follows the backward sweep in FGMRES (w = A z_j,
// type_fgmres.f90:175-189), run inside the backward sweep's launch: one task
// per matrix row (entry -3), handed out after the sweep tasks that publish
// the rows its columns read, so the rows' values stream while the sweep's
// dependency chain waits.
//
// The sweep has already formed the products of row r's upper blocks with z
// (the U partials U_rj z_j, ILU0's U being A's upper blocks,
// precon_ILU0.f90:370-395), and z_j is final when they are formed.  With
// `skip` set (the sweep's U blocks are the matvec's values, same type), the
// matvec row streams only the blocks the sweep did not read -- the diagonal,
// the lower blocks and any others -- and adds the row's U partials, in entry
// order, to their product: y_r = (A_rr z_r + sum_lower A_rk z_k) + sum_U
// part.  That drops the U blocks' second read (3/7 of the matrix on a hex
// box).  Without `skip`, row r computes y_r exactly as k_matvec_stream does
// (same chunks, same per-thread order).
template <typename TA, typename TX>
struct FusedMv {
    MatvecRowsView rows;         // the matrix rows (contiguous values per row)
    const TA* val;
    TX* y;
    double* row_sumsq;
    const int32_t* col_prow;     // per block of the matrix: the programme row publishing its column segment
    const uint8_t* skip = nullptr;   // per block of the matrix: 1 = a U block of the sweep, its partial reused
};

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
// The waiting thread is suspended (up to the hint, 0.1 ms) until the phase
// completes, so waiting warps do not take issue slots from working ones.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(100000u)
        : "memory");
    return ok != 0;
}
// wait until the phase with the given parity has completed; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, long long limit) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
template <int NC>
__device__ __forceinline__ void consumers_sync() { asm volatile("bar.sync 1, %0;" ::"n"(NC) : "memory"); }
// counter increment that releases the writes ordered before it (this thread's
// and, through the preceding barrier, the other consumers') and acquires the
// writes the other CTAs released with their increments
__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// the sum over the consumer threads (result in consumer thread 0)
template <int NC>
__device__ __forceinline__ double consumers_sum(double v, double* scratch, int ctid) {
    v = warp_sum(v);
    if ((ctid & 31) == 0) scratch[ctid >> 5] = v;
    consumers_sync<NC>();
    double s = 0.0;
    if (ctid < 32) {
        s = (ctid < NC / 32) ? scratch[ctid] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

// acc[rr] += sum over the chunk's columns of block(r, c) * x(c); rows r of this
// thread as set up by the caller (b <= NC: one row, columns strided by the G
// groups; otherwise rows r + NC*rr, all columns)
template <int NC, int RPT, typename TB, typename ACC>
__device__ __forceinline__ void stream_chunk(const TB* __restrict__ d, const ACC* __restrict__ xs, int b, int ncols, int r,
                                             int g, int G, ACC (&acc)[RPT]) {
    if (b <= NC) {
        if (g >= G) return;
        const TB* col = d + r;
        ACC a0 = acc[0], a1 = 0;
        int c = g;
        for (; c + G < ncols; c += 2 * G) {
            a0 += cvt<ACC>(col[(int64_t)c * b]) * xs[c];
            a1 += cvt<ACC>(col[(int64_t)(c + G) * b]) * xs[c + G];
        }
        if (c < ncols) a0 += cvt<ACC>(col[(int64_t)c * b]) * xs[c];
        acc[0] = a0 + a1;
    } else {
        for (int c = 0; c < ncols; ++c) {
            const ACC x = xs[c];
            #pragma unroll
            for (int rr = 0; rr < RPT; ++rr) {
                const int row = r + NC * rr;
                if (row < b) acc[rr] += cvt<ACC>(d[(int64_t)c * b + row]) * x;
            }
        }
    }
}

// the row sums of this task's product for rows ctid (+ NC*rr), as seen by
// threads ctid < b (b <= NC) or all threads otherwise
template <int NC, int RPT, typename ACC>
__device__ __forceinline__ void stream_reduce(ACC* red, int b, int r, int g, int G, int ctid, ACC (&acc)[RPT]) {
    if (b <= NC) {
        if (g < G) red[g * b + r] = acc[0];
        consumers_sync<NC>();
        if (ctid < b) {
            ACC s = 0;
            for (int gg = 0; gg < G; ++gg) s += red[gg * b + ctid];
            acc[0] = s;
        }
    }
}

// CW consumer warps; `stages` stages of `stage_bytes` bytes each.  MV: the
// backward sweep also runs the matvec rows of F (tasks with entry -3).
template <typename TL, typename TU, typename TX, typename ACC, bool FORWARD, int CW, typename TA = double, bool MV = false>
__global__ void __launch_bounds__(32 * CW + 32)
    k_ilu_stream(IluRows R, const TL* __restrict__ LD, const TU* __restrict__ Aval, StreamTasks T, int ntasks,
                 const TX* __restrict__ v, TX* __restrict__ zx, ACC* __restrict__ part, SweepSync S, int nstage,
                 int stage_bytes, int max_b, FusedMv<TA, TX> F, RowMask mask) {
    constexpr int NC = 32 * CW;                  // consumer threads
    static_assert(NC <= SS_MAX_NC, "row-sum scratch");
    static_assert(!(MV && FORWARD), "matvec rows run in the backward sweep");
    constexpr int RPT = (SS_MAX_B + NC - 1) / NC;
    extern __shared__ __align__(128) unsigned char ss_smem[];
    unsigned char* stages = ss_smem;
    ACC* xs = reinterpret_cast<ACC*>(ss_smem + (size_t)nstage * stage_bytes);
    ACC* red = xs + stream_xcap(max_b);          // G*b <= NC row sums
    double* scratch = reinterpret_cast<double*>(red + NC);   // 32 doubles
    uint64_t* full = reinterpret_cast<uint64_t*>(scratch + 32);
    uint64_t* empty = full + SS_MAX_STAGES;
    StreamMeta* meta = reinterpret_cast<StreamMeta*>(empty + SS_MAX_STAGES);
    __shared__ int s_last;
    const int chunk_bytes = stage_bytes - 16;    // payload before rounding out to 16 bytes

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < nstage; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, CW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    if (warp == CW) {
        // ------------------------------------------------------------ producer
        if (lane != 0) return;
        int stage = 0;
        unsigned phase = 0;
        for (;;) {
            const unsigned t = atomicAdd(S.counter, 1u);
            if (t >= (unsigned)ntasks) {
                if (!mbar_wait(empty + stage, phase ^ 1u, S.spin_limit)) atomicExch(S.status, 1);
                meta[stage].task = -1;
                mbar_arrive(full + stage);
                return;
            }
            const int pr = T.task_row[t], q = T.task_ent[t];
            if (row_frozen(mask, pr)) {
                if (!mbar_wait(empty + stage, phase ^ 1u, S.spin_limit)) atomicExch(S.status, 1);
                StreamMeta m;
                m.task = (int)t; m.pr = pr; m.q = q; m.chunk = 0; m.nchunk = 1;
                m.col0 = 0; m.ncols = 0; m.shift = 0; m.skip = 1;
                meta[stage] = m;
                mbar_arrive(full + stage);
                if (++stage == nstage) { stage = 0; phase ^= 1u; }
                continue;
            }
            int b = R.prow_b[pr];
            const unsigned char* base = nullptr;
            int cols = 0, esz = 1;
            if (MV && q == -3) {
                // matvec row pr: the row's blocks, one b x cols strip; with
                // F.skip, only its runs of blocks the sweep did not read
                const int64_t k0 = F.rows.row_ptr[pr], k1 = F.rows.row_ptr[pr + 1];
                b = F.rows.row_b[pr];
                base = reinterpret_cast<const unsigned char*>(F.val + (k1 > k0 ? F.rows.blk_voff[k0] : 0));
                esz = sizeof(TA);
                if (F.skip != nullptr) {
                    const int kc = max(1, chunk_bytes / (b * esz));
                    // the chunks of every run of streamed blocks: counted, then posted
                    int nchunk = 0;
                    for (int pass = 0; pass < 2; ++pass) {
                        int col = 0, ch = 0;
                        for (int64_t k = k0; k <= k1; ++k) {
                            int run0 = col;
                            while (k < k1 && !F.skip[k]) { col += F.rows.blk_nc[k]; ++k; }
                            for (int c0 = run0; c0 < col; c0 += kc, ++ch) {
                                if (pass == 0) continue;
                                if (!mbar_wait(empty + stage, phase ^ 1u, S.spin_limit)) atomicExch(S.status, 1);
                                StreamMeta m;
                                m.task = (int)t; m.pr = pr; m.q = q; m.chunk = ch; m.nchunk = nchunk;
                                m.skip = 0;
                                m.col0 = c0;
                                m.ncols = min(kc, col - c0);
                                const uintptr_t src = reinterpret_cast<uintptr_t>(base + (size_t)c0 * b * esz);
                                const uintptr_t a0 = src & ~(uintptr_t)15;
                                const unsigned bytes = (unsigned)((size_t)m.ncols * b * esz);
                                const unsigned len = (unsigned)(((src - a0) + bytes + 15) & ~(uintptr_t)15);
                                m.shift = (int)((src - a0) / esz);
                                meta[stage] = m;
                                mbar_arrive_expect_tx(full + stage, len);
                                bulk_copy_g2s(stages + (size_t)stage * stage_bytes, reinterpret_cast<const void*>(a0), len,
                                              full + stage);
                                if (++stage == nstage) { stage = 0; phase ^= 1u; }
                            }
                            if (k < k1) col += F.rows.blk_nc[k];      // a skipped block
                        }
                        nchunk = ch;
                    }
                    if (nchunk > 0) continue;
                    cols = 0;                                        // nothing streamed: one empty chunk
                } else {
                    for (int64_t k = k0; k < k1; ++k) cols += F.rows.blk_nc[k];
                }
            } else if (q >= 0) {
                if (FORWARD) { base = reinterpret_cast<const unsigned char*>(LD + R.lo_L[q]); cols = R.lo_nc[q]; esz = sizeof(TL); }
                else { base = reinterpret_cast<const unsigned char*>(Aval + R.up_U[q]); cols = R.up_nc[q]; esz = sizeof(TU); }
            } else if (q == -2) {
                base = reinterpret_cast<const unsigned char*>(LD + R.dinv_off[pr]);
                cols = b;
                esz = sizeof(TL);
            }
            const int kc = cols > 0 ? max(1, min(cols, chunk_bytes / (b * esz))) : 1;
            const int nchunk = cols > 0 ? (cols + kc - 1) / kc : 1;
            for (int ch = 0; ch < nchunk; ++ch) {
                if (!mbar_wait(empty + stage, phase ^ 1u, S.spin_limit)) atomicExch(S.status, 1);
                StreamMeta m;
                m.task = (int)t; m.pr = pr; m.q = q; m.chunk = ch; m.nchunk = nchunk;
                m.skip = 0;
                m.col0 = ch * kc;
                m.ncols = cols > 0 ? min(kc, cols - ch * kc) : 0;
                m.shift = 0;
                if (cols > 0) {
                    const uintptr_t src = reinterpret_cast<uintptr_t>(base + (size_t)m.col0 * b * esz);
                    const uintptr_t a0 = src & ~(uintptr_t)15;
                    const unsigned bytes = (unsigned)((size_t)m.ncols * b * esz);
                    const unsigned len = (unsigned)(((src - a0) + bytes + 15) & ~(uintptr_t)15);
                    m.shift = (int)((src - a0) / esz);
                    meta[stage] = m;
                    mbar_arrive_expect_tx(full + stage, len);
                    bulk_copy_g2s(stages + (size_t)stage * stage_bytes, reinterpret_cast<const void*>(a0), len, full + stage);
                } else {
                    meta[stage] = m;
                    mbar_arrive(full + stage);
                }
                if (++stage == nstage) { stage = 0; phase ^= 1u; }
            }
        }
    }

    // ---------------------------------------------------------------- consumers
    const int ctid = tid;
    int stage = 0;
    unsigned phase = 0;
    int pr = 0, q = 0, b = 0, G = 1, r = 0, g = 0;
    ACC acc[RPT];
    for (;;) {
        if (!mbar_wait(full + stage, phase, S.spin_limit)) { if (ctid == 0) atomicExch(S.status, 1); }
        const StreamMeta m = meta[stage];
        if (m.task < 0) break;
        if (m.skip) {
            // a frozen system's row: release the stage, nothing else
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + stage);
            if (++stage == nstage) { stage = 0; phase ^= 1u; }
            continue;
        }
        if (m.chunk == 0) {
            pr = m.pr;
            q = m.q;
            b = (MV && q == -3) ? F.rows.row_b[pr] : R.prow_b[pr];
            if (b <= NC) { G = NC / b; r = ctid % b; g = ctid / b; }
            else { G = 1; r = ctid; g = 0; }
            #pragma unroll
            for (int rr = 0; rr < RPT; ++rr) acc[rr] = 0;
            if (MV && q == -3) {
                // every column segment of the row published by the sweep, then staged
                const int64_t k0 = F.rows.row_ptr[pr], k1 = F.rows.row_ptr[pr + 1];
                if (ctid == 0)
                    for (int64_t k = k0; k < k1; ++k)
                        if (!wait_flag(S.flags, F.col_prow[k], S.epoch, S.spin_limit)) atomicExch(S.status, 1);
                consumers_sync<NC>();
                int off = 0;
                for (int64_t k = k0; k < k1; ++k) {
                    const int nc = F.rows.blk_nc[k];
                    if (F.skip == nullptr || !F.skip[k]) {
                        const TX* xp = zx + F.rows.blk_xoff[k];
                        for (int c = ctid; c < nc; c += NC) xs[off + c] = cvt<ACC>(ld_cg(xp + c));
                    }
                    off += nc;
                }
                consumers_sync<NC>();
            } else if (q >= 0) {
                const int par = FORWARD ? R.lo_par[q] : R.up_par[q];
                const int nc = FORWARD ? R.lo_nc[q] : R.up_nc[q];
                if (ctid == 0 && !wait_flag(S.flags, par, S.epoch, S.spin_limit)) atomicExch(S.status, 1);
                consumers_sync<NC>();
                const TX* zp = zx + R.z_off[par];
                for (int c = ctid; c < nc; c += NC) xs[c] = cvt<ACC>(ld_cg(zp + c));
                consumers_sync<NC>();
            } else if (q == -2) {
                // t_r = z_r - sum of the row's U partials, in entry order
                const int q0 = R.up_ptr[pr], q1 = R.up_ptr[pr + 1];
                if (q1 > q0 && ctid == 0 && !wait_flag(T.ready, pr, S.epoch, S.spin_limit)) atomicExch(S.status, 1);
                consumers_sync<NC>();
                for (int i = ctid; i < b; i += NC) {
                    ACC s = 0;
                    for (int qq = q0; qq < q1; ++qq) s += ld_cg(part + T.part_off[qq] + i);
                    xs[i] = cvt<ACC>(from_d<TX>(to_d(ld_cg(zx + R.z_off[pr] + i)) - (double)s));
                }
                consumers_sync<NC>();
            } else {
                // forward row without lower entries: z_r = v_r
                for (int i = ctid; i < b; i += NC) zx[R.z_off[pr] + i] = v[R.v_off[pr] + i];
                consumers_sync<NC>();
                if (ctid == 0) st_release(S.flags + pr, S.epoch);
            }
        }
        if (m.ncols > 0) {
            const unsigned char* sb = stages + (size_t)stage * stage_bytes;
            if (MV && q == -3)
                stream_chunk<NC, RPT, TA, ACC>(reinterpret_cast<const TA*>(sb) + m.shift, xs + m.col0, b, m.ncols, r, g, G, acc);
            else if (FORWARD || q == -2)
                stream_chunk<NC, RPT, TL, ACC>(reinterpret_cast<const TL*>(sb) + m.shift, xs + m.col0, b, m.ncols, r, g, G, acc);
            else
                stream_chunk<NC, RPT, TU, ACC>(reinterpret_cast<const TU*>(sb) + m.shift, xs + m.col0, b, m.ncols, r, g, G, acc);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + stage);
        if (++stage == nstage) { stage = 0; phase ^= 1u; }
        if (m.chunk != m.nchunk - 1 || q == -1) continue;

        // ------------------------------------------------ the task's last chunk
        stream_reduce<NC, RPT>(red, b, r, g, G, ctid, acc);
        if (MV && q == -3) {
            // y_r = A_r z and its sum of squares, as the streamed matvec writes
            // them (with F.skip: plus the row's U partials, in entry order)
            double sq = 0.0;
            const int64_t yo = F.rows.row_yoff[pr];
            const int u0 = F.skip != nullptr ? R.up_ptr[pr] : 0, u1 = F.skip != nullptr ? R.up_ptr[pr + 1] : 0;
            #pragma unroll
            for (int rr = 0; rr < RPT; ++rr) {
                const int i = (b <= NC) ? (rr == 0 ? ctid : b) : ctid + NC * rr;
                if (i < b) {
                    if (u1 > u0) {
                        ACC s = 0;
                        for (int u = u0; u < u1; ++u) s += ld_cg(part + T.part_off[u] + i);
                        acc[rr] += s;
                    }
                    const TX o = from_d<TX>((double)acc[rr]);
                    F.y[yo + i] = o;
                    const double od = to_d(o);
                    sq += od * od;
                }
            }
            if (F.row_sumsq != nullptr) {
                const double s2 = consumers_sum<NC>(sq, scratch, ctid);
                if (ctid == 0) F.row_sumsq[pr] = s2;
            }
            consumers_sync<NC>();        // xs, red and scratch are reused by the next task
            continue;
        }
        if (q == -2) {
            // x_r = inv(D_r) t_r: the row is complete
            if (b <= NC) { if (ctid < b) zx[R.z_off[pr] + ctid] = from_d<TX>((double)acc[0]); }
            else {
                #pragma unroll
                for (int rr = 0; rr < RPT; ++rr)
                    if (ctid + NC * rr < b) zx[R.z_off[pr] + ctid + NC * rr] = from_d<TX>((double)acc[rr]);
            }
            consumers_sync<NC>();
            if (ctid == 0) st_release(S.flags + pr, S.epoch);
            continue;
        }
        if (b <= NC) { if (ctid < b) part[T.part_off[q] + ctid] = acc[0]; }
        else {
            #pragma unroll
            for (int rr = 0; rr < RPT; ++rr)
                if (ctid + NC * rr < b) part[T.part_off[q] + ctid + NC * rr] = acc[rr];
        }
        consumers_sync<NC>();
        const int q0 = FORWARD ? R.lo_ptr[pr] : R.up_ptr[pr];
        const int q1 = FORWARD ? R.lo_ptr[pr + 1] : R.up_ptr[pr + 1];
        if (ctid == 0) {
            const unsigned old = atom_add_acq_rel(T.row_count + pr, 1u);
            const bool last = ((old + 1u) % (unsigned)(q1 - q0)) == 0u;
            if (last && !FORWARD) st_release(T.ready + pr, S.epoch);
            s_last = last;
        }
        consumers_sync<NC>();
        if constexpr (FORWARD) {
            if (!s_last) continue;
            for (int i = ctid; i < b; i += NC) {
                ACC s = 0;
                for (int qq = q0; qq < q1; ++qq) s += ld_cg(part + T.part_off[qq] + i);
                zx[R.z_off[pr] + i] = from_d<TX>(to_d(v[R.v_off[pr] + i]) - (double)s);
            }
            consumers_sync<NC>();
            if (ctid == 0) st_release(S.flags + pr, S.epoch);
        }
    }
}

}  // namespace chidg
