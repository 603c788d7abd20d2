// chidg_mv as a streamed kernel (operator_chidg_mv.f90:117-410): y = alpha A x
// (+ beta z), optionally with the row's sum of squares of y.
//
// A row's blocks are stored one after another, all with the row's b rows, so
// the row is one column-major b x ncols matrix (ncols = sum of the blocks'
// columns) and its x segments, concatenated, are the vector it multiplies.
// Persistent CTAs: a producer lane takes rows blockIdx.x, blockIdx.x + gridDim.x,
// ... (rows are alike in size) and copies each row's
// values, in column chunks, into a ring of shared-memory stages with
// cp.async.bulk (source rounded to 16 bytes, as in the streamed sweeps); the
// consumer warps stage the row's x segments, multiply the chunks as they land
// and write the row.  The loads of the next rows are in flight while a row is
// finished, so no row waits on a chain of memory round trips; narrow types
// (FP32, BF16) move as many bytes per copy as FP64.
//
// Sums: thread (r, g) adds columns c = g, g+G, ... of each chunk in increasing
// order, G(b) = NC / b fixed by the block size, then the G partial sums in
// order: the same order on every call, independent of which CTA takes a row.
#pragma once

#include "stream_sweep.cuh"

namespace chidg {

using MatvecRows = MatvecRowsView;

__host__ __device__ constexpr size_t matvec_stream_smem(size_t acc_size, int stages, int stage_bytes, int max_cols,
                                                         int nc) {
    return (size_t)stages * stage_bytes + (stream_xcap(max_cols) + nc + 32) * acc_size + 32 * sizeof(double) +
           2 * SS_MAX_STAGES * sizeof(uint64_t) + SS_MAX_STAGES * sizeof(StreamMeta) + 64;
}

template <typename TA, typename TX, typename ACC, int CW>
__global__ void __launch_bounds__(32 * CW + 32)
    k_matvec_stream(MatvecRows R, int nrow, const TA* __restrict__ val, const TX* __restrict__ x, TX* __restrict__ y,
                    const TX* __restrict__ z, double alpha, double beta, double* __restrict__ row_sumsq,
                    int* __restrict__ status, long long spin_limit, int nstage,
                    int stage_bytes, int max_cols, RowMask mask) {
    constexpr int NC = 32 * CW;
    constexpr int RPT = (SS_MAX_B + NC - 1) / NC;
    extern __shared__ __align__(128) unsigned char ss_smem[];
    unsigned char* stages = ss_smem;
    ACC* xs = reinterpret_cast<ACC*>(ss_smem + (size_t)nstage * stage_bytes);
    ACC* red = xs + stream_xcap(max_cols);
    double* scratch = reinterpret_cast<double*>(red + NC + 32);
    uint64_t* full = reinterpret_cast<uint64_t*>(scratch + 32);
    uint64_t* empty = full + SS_MAX_STAGES;
    StreamMeta* meta = reinterpret_cast<StreamMeta*>(empty + SS_MAX_STAGES);
    const int chunk_bytes = stage_bytes - 16;

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
        for (int row = blockIdx.x;; row += gridDim.x) {
            if (row >= nrow) {
                if (!mbar_wait(empty + stage, phase ^ 1u, spin_limit)) atomicExch(status, 1);
                meta[stage].task = -1;
                mbar_arrive(full + stage);
                return;
            }
            if (row_frozen(mask, row)) {
                // a frozen system's row: one empty chunk, nothing read or written
                if (!mbar_wait(empty + stage, phase ^ 1u, spin_limit)) atomicExch(status, 1);
                StreamMeta m;
                m.task = row; m.pr = row; m.q = 0; m.chunk = 0; m.nchunk = 1;
                m.col0 = 0; m.ncols = 0; m.shift = 0; m.skip = 1;
                meta[stage] = m;
                mbar_arrive(full + stage);
                if (++stage == nstage) { stage = 0; phase ^= 1u; }
                continue;
            }
            const int64_t k0 = R.row_ptr[row], k1 = R.row_ptr[row + 1];
            const int b = R.row_b[row];
            int cols = 0;
            for (int64_t k = k0; k < k1; ++k) cols += R.blk_nc[k];
            const unsigned char* base = reinterpret_cast<const unsigned char*>(val + (k1 > k0 ? R.blk_voff[k0] : 0));
            const int esz = sizeof(TA);
            const int kc = cols > 0 ? max(1, min(cols, chunk_bytes / (b * esz))) : 1;
            const int nchunk = cols > 0 ? (cols + kc - 1) / kc : 1;
            for (int ch = 0; ch < nchunk; ++ch) {
                if (!mbar_wait(empty + stage, phase ^ 1u, spin_limit)) atomicExch(status, 1);
                StreamMeta m;
                m.task = row; m.pr = row; m.q = 0; m.chunk = ch; m.nchunk = nchunk;
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
    int row = 0, b = 0, G = 1, r = 0, g = 0;
    ACC acc[RPT];
    for (;;) {
        if (!mbar_wait(full + stage, phase, spin_limit)) { if (ctid == 0) atomicExch(status, 1); }
        const StreamMeta m = meta[stage];
        if (m.task < 0) break;
        if (m.skip) {
            __syncwarp();
            if (lane == 0) mbar_arrive(empty + stage);
            if (++stage == nstage) { stage = 0; phase ^= 1u; }
            continue;
        }
        if (m.chunk == 0) {
            row = m.pr;
            b = R.row_b[row];
            if (b <= NC) { G = NC / b; r = ctid % b; g = ctid / b; }
            else { G = 1; r = ctid; g = 0; }
            #pragma unroll
            for (int rr = 0; rr < RPT; ++rr) acc[rr] = 0;
            // the row's x segments, concatenated
            int off = 0;
            for (int64_t k = R.row_ptr[row]; k < R.row_ptr[row + 1]; ++k) {
                const int nc = R.blk_nc[k];
                const TX* xp = x + R.blk_xoff[k];
                for (int c = ctid; c < nc; c += NC) xs[off + c] = cvt<ACC>(xp[c]);
                off += nc;
            }
            consumers_sync<NC>();
        }
        if (m.ncols > 0)
            stream_chunk<NC, RPT, TA, ACC>(reinterpret_cast<const TA*>(stages + (size_t)stage * stage_bytes) + m.shift,
                                           xs + m.col0, b, m.ncols, r, g, G, acc);
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + stage);
        if (++stage == nstage) { stage = 0; phase ^= 1u; }
        if (m.chunk != m.nchunk - 1) continue;

        // ------------------------------------------------- the row's last chunk
        stream_reduce<NC, RPT>(red, b, r, g, G, ctid, acc);
        double sq = 0.0;
        const int64_t yo = R.row_yoff[row];
        #pragma unroll
        for (int rr = 0; rr < RPT; ++rr) {
            const int i = (b <= NC) ? (rr == 0 ? ctid : b) : ctid + NC * rr;
            if (i < b) {
                double out = alpha * (double)acc[rr];
                if (z != nullptr) out += beta * to_d(z[yo + i]);
                const TX o = from_d<TX>(out);
                y[yo + i] = o;
                const double od = to_d(o);
                sq += od * od;
            }
        }
        if (row_sumsq != nullptr) {
            const double s = consumers_sum<NC>(sq, scratch, ctid);
            if (ctid == 0) row_sumsq[row] = s;
        }
        consumers_sync<NC>();        // xs, red and scratch are reused by the next row
    }
}

}  // namespace chidg
