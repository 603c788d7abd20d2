// In-place inverse of one diagonal block (b <= 136) per CTA: blocked
// Gauss-Jordan with partial (row) pivoting, the trailing updates on the FP64
// tensor cores.
//
// The block, padded to 136 x 136 with an identity, lives in registers as the
// accumulator fragments of mma.f64 (17 x 17 tiles of 8 x 8): warp w owns tile
// columns w and w + 9; lane (g, t) = (lane / 4, lane % 4) holds rows 8*ti + g
// and columns 8c + 2t + {0,1} of its tile columns c.  Two consecutive row tiles
// form the 16 x 8 accumulator of mma.m16n8k8.  Columns are eliminated in
// panels of eight:
//
//   panel J  the owner warp of tile column J moves the 136 x 8 panel into a
//            row-per-lane register layout (rows lane + 32r) and runs the eight
//            Gauss-Jordan steps alone: warp-shuffle argmax for the pivot,
//            shuffle broadcast of the pivot row, register updates.  The pivot of
//            column k is the entry of largest magnitude among rows not yet
//            used as pivots (first such row on ties) -- the pivot DGETRF
//            selects.  Rows are not swapped; step k records its pivot row p_k.
//   update   every other column c changes by the panel's eight steps as
//            a_c <- a_c with rows {p_k} zeroed + P X_c, P the eliminated panel
//            (136 x 8) and X_c the old values of a_c in rows p_k: a rank-8
//            update, one m16n8k8 product per pair of row tiles.
//
// Look-ahead: panels are double-buffered in shared memory and handed over by
// mbarriers ("panel J ready", "buffer of panel J read by every warp"), not by
// CTA-wide barriers.  Consecutive panels belong to different warps; the owner
// of panel J+1 applies panel J to that one column, runs panel J+1, and only
// then applies panel J to its other column, while the other warps are still
// applying panel J: the critical path is the chain of panels and one column
// update per panel.
//
// After the last panel the stored matrix R satisfies R(p_k, j) = inv(A)(k, p_j);
// the write-back undoes the permutation.  The padding never changes (its rows
// and columns stay those of the identity) and is not eliminated.  A zero pivot
// records the element in *status (ESINGULAR) and leaves garbage; a NaN entry
// is taken as pivot so the NaN propagates.  The mbarrier waits are bounded; a
// wait that runs out is reported the same way.
#pragma once

#include "kernels.cuh"
#include "stream_sweep.cuh"

namespace chidg {

constexpr int TCI_MAX = 136;          // largest block
constexpr int TCI_TILES = 17;         // 8 x 8 tiles per side
constexpr int TCI_LD = 140;           // shared leading dimension (conflict-free fragment loads)
constexpr int TCI_WARPS = 9;          // tile columns w and w + 9
constexpr int TCI_THREADS = 32 * TCI_WARPS;
constexpr long long TCI_WAIT_LIMIT = 1ll << 31;   // clock cycles

struct TciShared {
    double Pn[2][8 * TCI_LD];         // panels J even / odd, column-major
    double Xs[TCI_TILES][64];         // per tile column: old values of the panel's pivot rows
    double park[2 * TCI_TILES * 32];  // the panel owner's other column, parked during the panel
    int pivrow[TCI_MAX];              // step -> row
    int stepof[TCI_MAX];              // row -> step, -1 while not a pivot
    uint64_t bar_ready[2], bar_read[2];
};

// One Gauss-Jordan step of a panel held row-per-lane (rows lane + 32r), the
// pivot column in slot 0.  The step leaves the panel rotated by one column
// (slot c receives column c+1, slot 7 the eliminated column), so that every
// step pivots on slot 0 and the loop over the eight steps stays compact: after
// eight steps (a short panel rotates on without eliminating) the columns are
// back in place.
//
// Pivot search on integer keys: the bit pattern of |v| is monotone in |v| for
// doubles (a NaN sorts above +inf, so it is taken as pivot and propagates);
// key + 1 marks a candidate row, 0 a row already used or past b.  The lane's
// best row (first on ties) comes from a tree over its five rows, the warp's
// from three redux operations: max of the high words, max of the low words
// among the lanes that hold it, min row index among the lanes holding both.
__device__ __forceinline__ void tci_step(double (&pr)[5][8], unsigned& used, int lane, int b, int k, TciShared& sh,
                                         bool& singular) {
    unsigned long long key[5];
    #pragma unroll
    for (int r = 0; r < 5; ++r) {
        const int i = lane + 32 * r;
        const unsigned long long kb = (unsigned long long)__double_as_longlong(fabs(pr[r][0]));
        key[r] = (i < b && !((used >> r) & 1u)) ? kb + 1ull : 0ull;
    }
    const unsigned long long k01 = key[1] > key[0] ? key[1] : key[0];
    const int r01 = key[1] > key[0] ? 1 : 0;
    const unsigned long long k23 = key[3] > key[2] ? key[3] : key[2];
    const int r23 = key[3] > key[2] ? 3 : 2;
    const unsigned long long k03 = k23 > k01 ? k23 : k01;
    const int r03 = k23 > k01 ? r23 : r01;
    const unsigned long long kl = key[4] > k03 ? key[4] : k03;
    const int rl = key[4] > k03 ? 4 : r03;
    const unsigned hi = (unsigned)(kl >> 32), lo = (unsigned)kl;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const unsigned cand = (hi == mhi && lo == mlo) ? (unsigned)(lane + 32 * rl) : 0xffffffffu;
    const int p = (int)__reduce_min_sync(0xffffffffu, cand);   // b - k >= 1 candidates: always a row
    const int pr_r = p >> 5, pr_l = p & 31;
    // the pivot row, from its lane (pr_r is the same in every lane)
    double prow[8];
#define CHIDG_TCI_BCAST(R)                                                                             \
    {                                                                                                  \
        _Pragma("unroll") for (int c = 0; c < 8; ++c) prow[c] = __shfl_sync(0xffffffffu, pr[R][c], pr_l); \
    }
    if (pr_r == 0) CHIDG_TCI_BCAST(0)
    else if (pr_r == 1) CHIDG_TCI_BCAST(1)
    else if (pr_r == 2) CHIDG_TCI_BCAST(2)
    else if (pr_r == 3) CHIDG_TCI_BCAST(3)
    else CHIDG_TCI_BCAST(4)
#undef CHIDG_TCI_BCAST
    double piv = prow[0];
    if (piv == 0.0) { singular = true; piv = 1.0; }
    const double rp = 1.0 / piv;
    double prw[8];
    prw[0] = rp;
    #pragma unroll
    for (int c = 1; c < 8; ++c) prw[c] = prow[c] * rp;
    // every row, rotated (rows past b hold zeros in the panel's columns and
    // stay as they are); the pivot row is overwritten afterwards
    #pragma unroll
    for (int r = 0; r < 5; ++r) {
        const double f = pr[r][0];
        #pragma unroll
        for (int c = 0; c < 7; ++c) pr[r][c] = pr[r][c + 1] - f * prw[c + 1];
        pr[r][7] = -f * rp;
    }
    if (lane == pr_l) {
        #pragma unroll
        for (int r = 0; r < 5; ++r)
            if (r == pr_r) {
                #pragma unroll
                for (int c = 0; c < 8; ++c) pr[r][c] = prw[(c + 1) & 7];
            }
        used |= 1u << pr_r;
    }
    if (lane == 0) { sh.pivrow[k] = p; sh.stepof[p] = k; }
}

// the rotation of a step without its elimination (steps past b)
__device__ __forceinline__ void tci_rotate(double (&pr)[5][8]) {
    #pragma unroll
    for (int r = 0; r < 5; ++r) {
        const double t = pr[r][0];
        #pragma unroll
        for (int c = 0; c < 7; ++c) pr[r][c] = pr[r][c + 1];
        pr[r][7] = t;
    }
}

// Panel J held in tile column CC of this warp: eliminate it, publish it.
template <int CC>
__device__ __forceinline__ void tci_panel(double (&acc)[2][TCI_TILES][2], TciShared& sh, int J, int T, int b, int lane,
                                          bool& singular) {
    const int g = lane >> 2, tq = lane & 3, s = J & 1;
    double* P = sh.Pn[s];
    if (J >= 2 && !mbar_wait(sh.bar_read + s, ((unsigned)(J >> 1) & 1u) ^ 1u, TCI_WAIT_LIMIT)) singular = true;
    // every tile, padding included, so that no accumulator stays live across the panel
    #pragma unroll
    for (int ti = 0; ti < TCI_TILES; ++ti) {
        P[(2 * tq) * TCI_LD + 8 * ti + g] = acc[CC][ti][0];
        P[(2 * tq + 1) * TCI_LD + 8 * ti + g] = acc[CC][ti][1];
        sh.park[(2 * ti) * 32 + lane] = acc[1 - CC][ti][0];
        sh.park[(2 * ti + 1) * 32 + lane] = acc[1 - CC][ti][1];
    }
    __syncwarp();
    double pr[5][8];
    unsigned used = 0;
    #pragma unroll
    for (int r = 0; r < 5; ++r) {
        const int i = lane + 32 * r;
        #pragma unroll
        for (int c = 0; c < 8; ++c) pr[r][c] = (i < 8 * T) ? P[c * TCI_LD + i] : 0.0;
        if (i < b && sh.stepof[i] >= 0) used |= 1u << r;
    }
    const int k0 = 8 * J;
    #pragma unroll 1
    for (int kk = 0; kk < 8; ++kk) {
        if (k0 + kk < b) tci_step(pr, used, lane, b, k0 + kk, sh, singular);
        else tci_rotate(pr);
    }
    #pragma unroll
    for (int r = 0; r < 5; ++r) {
        const int i = lane + 32 * r;
        if (i < 8 * T) {
            #pragma unroll
            for (int c = 0; c < 8; ++c) P[c * TCI_LD + i] = pr[r][c];
        }
    }
    __syncwarp();
    #pragma unroll
    for (int ti = 0; ti < TCI_TILES; ++ti) {
        acc[CC][ti][0] = P[(2 * tq) * TCI_LD + 8 * ti + g];
        acc[CC][ti][1] = P[(2 * tq + 1) * TCI_LD + 8 * ti + g];
        acc[1 - CC][ti][0] = sh.park[(2 * ti) * 32 + lane];
        acc[1 - CC][ti][1] = sh.park[(2 * ti + 1) * 32 + lane];
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(sh.bar_ready + s);
}

// Apply panel J to tile column c (held in CC): rank-8 update on the tensor cores.
template <int CC>
__device__ __forceinline__ void tci_update(double (&acc)[2][TCI_TILES][2], TciShared& sh, int J, int c, int T, int b,
                                           int lane) {
    const int g = lane >> 2, tq = lane & 3;
    const double* P = sh.Pn[J & 1];
    double* X = sh.Xs[c];
    X[lane] = 0.0;
    X[lane + 32] = 0.0;
    __syncwarp();
    #pragma unroll
    for (int ti = 0; ti < TCI_TILES; ++ti)
        if (ti < T) {
            const int i = 8 * ti + g;
            const int st = (i < b) ? sh.stepof[i] - 8 * J : -1;
            if (st >= 0 && st < 8) {
                X[st * 8 + 2 * tq] = acc[CC][ti][0];
                X[st * 8 + 2 * tq + 1] = acc[CC][ti][1];
                acc[CC][ti][0] = 0.0;
                acc[CC][ti][1] = 0.0;
            }
        }
    __syncwarp();
    const double b0 = X[tq * 8 + g];
    const double b1 = X[(4 + tq) * 8 + g];
    #pragma unroll
    for (int t2 = 0; t2 < 8; ++t2)
        if (2 * t2 < T) {
            const double* Pc = P + 16 * t2 + g;
            dmma_16x8x8(acc[CC][2 * t2][0], acc[CC][2 * t2][1], acc[CC][2 * t2 + 1][0], acc[CC][2 * t2 + 1][1],
                        Pc[tq * TCI_LD], Pc[tq * TCI_LD + 8], Pc[(4 + tq) * TCI_LD], Pc[(4 + tq) * TCI_LD + 8], b0, b1);
        }
    if (T > 16) {
        dmma_8x8x4(acc[CC][16][0], acc[CC][16][1], P[tq * TCI_LD + 128 + g], b0);
        dmma_8x8x4(acc[CC][16][0], acc[CC][16][1], P[(4 + tq) * TCI_LD + 128 + g], b1);
    }
    __syncwarp();
}

// Apply panel J to both tile columns of this warp: the pivot-row positions and
// the panel's A fragments are loaded once for the two columns.
__device__ __forceinline__ void tci_update2(double (&acc)[2][TCI_TILES][2], TciShared& sh, int J, int c0, int c1, int T,
                                            int b, int lane) {
    const int g = lane >> 2, tq = lane & 3;
    const double* P = sh.Pn[J & 1];
    double* X0 = sh.Xs[c0];
    double* X1 = sh.Xs[c1];
    X0[lane] = 0.0;
    X0[lane + 32] = 0.0;
    X1[lane] = 0.0;
    X1[lane + 32] = 0.0;
    __syncwarp();
    #pragma unroll
    for (int ti = 0; ti < TCI_TILES; ++ti)
        if (ti < T) {
            const int i = 8 * ti + g;
            const int st = (i < b) ? sh.stepof[i] - 8 * J : -1;
            if (st >= 0 && st < 8) {
                X0[st * 8 + 2 * tq] = acc[0][ti][0];
                X0[st * 8 + 2 * tq + 1] = acc[0][ti][1];
                X1[st * 8 + 2 * tq] = acc[1][ti][0];
                X1[st * 8 + 2 * tq + 1] = acc[1][ti][1];
                acc[0][ti][0] = 0.0;
                acc[0][ti][1] = 0.0;
                acc[1][ti][0] = 0.0;
                acc[1][ti][1] = 0.0;
            }
        }
    __syncwarp();
    const double b00 = X0[tq * 8 + g], b01 = X0[(4 + tq) * 8 + g];
    const double b10 = X1[tq * 8 + g], b11 = X1[(4 + tq) * 8 + g];
    #pragma unroll
    for (int t2 = 0; t2 < 8; ++t2)
        if (2 * t2 < T) {
            const double* Pc = P + 16 * t2 + g;
            const double a0 = Pc[tq * TCI_LD], a1 = Pc[tq * TCI_LD + 8];
            const double a2 = Pc[(4 + tq) * TCI_LD], a3 = Pc[(4 + tq) * TCI_LD + 8];
            dmma_16x8x8(acc[0][2 * t2][0], acc[0][2 * t2][1], acc[0][2 * t2 + 1][0], acc[0][2 * t2 + 1][1], a0, a1, a2, a3,
                        b00, b01);
            dmma_16x8x8(acc[1][2 * t2][0], acc[1][2 * t2][1], acc[1][2 * t2 + 1][0], acc[1][2 * t2 + 1][1], a0, a1, a2, a3,
                        b10, b11);
        }
    if (T > 16) {
        const double a0 = P[tq * TCI_LD + 128 + g], a1 = P[(4 + tq) * TCI_LD + 128 + g];
        dmma_8x8x4(acc[0][16][0], acc[0][16][1], a0, b00);
        dmma_8x8x4(acc[1][16][0], acc[1][16][1], a0, b10);
        dmma_8x8x4(acc[0][16][0], acc[0][16][1], a1, b01);
        dmma_8x8x4(acc[1][16][0], acc[1][16][1], a1, b11);
    }
    __syncwarp();
}

static __global__ void __launch_bounds__(TCI_THREADS, 1)
    k_block_inverse_tc(double* __restrict__ LD, const int64_t* __restrict__ dinv_off, const int32_t* __restrict__ prow_b,
                       const int32_t* __restrict__ prow_elem, const int32_t* __restrict__ rows, int row_begin,
                       int* __restrict__ status) {
    __shared__ TciShared sh;
    const int prow = rows[row_begin + blockIdx.x];
    const int b = prow_b[prow];
    double* D = LD + dinv_off[prow];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int g = lane >> 2, tq = lane & 3;
    const int T = (b + 7) >> 3;                  // tile columns holding data
    const int WT = T < TCI_WARPS ? T : TCI_WARPS;   // warps holding data
    const int c0 = w, c1 = w + TCI_WARPS;          // this warp's tile columns

    double acc[2][TCI_TILES][2];
    #pragma unroll
    for (int cc = 0; cc < 2; ++cc)
        #pragma unroll
        for (int ti = 0; ti < TCI_TILES; ++ti)
            #pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int i = 8 * ti + g, j = 8 * (w + TCI_WARPS * cc) + 2 * tq + e;
                acc[cc][ti][e] = (i < b && j < b) ? D[i + (int64_t)j * b] : (i == j ? 1.0 : 0.0);
            }
    for (int i = threadIdx.x; i < TCI_MAX; i += blockDim.x) sh.stepof[i] = -1;
    if (threadIdx.x == 0) {
        for (int s = 0; s < 2; ++s) {
            mbar_init(sh.bar_ready + s, 1);
            mbar_init(sh.bar_read + s, WT);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    bool singular = false;
    __syncthreads();

    if (w < WT) {
        if (c0 == 0) tci_panel<0>(acc, sh, 0, T, b, lane, singular);
        for (int J = 0; J < T; ++J) {
            if (!mbar_wait(sh.bar_ready + (J & 1), (unsigned)(J >> 1) & 1u, TCI_WAIT_LIMIT)) singular = true;
            if (J + 1 == c0) {
                // look-ahead: the next panel is this warp's first column
                tci_update<0>(acc, sh, J, c0, T, b, lane);
                tci_panel<0>(acc, sh, c0, T, b, lane, singular);
                if (c1 < T) tci_update<1>(acc, sh, J, c1, T, b, lane);
            } else if (J + 1 == c1) {
                // look-ahead: the next panel is this warp's second column
                tci_update<1>(acc, sh, J, c1, T, b, lane);
                tci_panel<1>(acc, sh, c1, T, b, lane, singular);
                if (c0 != J) tci_update<0>(acc, sh, J, c0, T, b, lane);
            } else if (c0 != J && c1 != J && c1 < T) {
                tci_update2(acc, sh, J, c0, c1, T, b, lane);
            } else {
                if (c0 != J) tci_update<0>(acc, sh, J, c0, T, b, lane);
                if (c1 != J && c1 < T) tci_update<1>(acc, sh, J, c1, T, b, lane);
            }
            if (lane == 0) mbar_arrive(sh.bar_read + (J & 1));
        }
    }
    __syncthreads();
    if (singular && lane == 0) atomicMin(status, prow_elem[prow]);
    // R(p_k, j) = inv(A)(k, p_j)
    #pragma unroll
    for (int cc = 0; cc < 2; ++cc)
        #pragma unroll
        for (int ti = 0; ti < TCI_TILES; ++ti)
            #pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int i = 8 * ti + g, j = 8 * (w + TCI_WARPS * cc) + 2 * tq + e;
                if (ti < T && i < b && j < b) D[sh.stepof[i] + (int64_t)sh.pivrow[j] * b] = acc[cc][ti][e];
            }
}

}  // namespace chidg
