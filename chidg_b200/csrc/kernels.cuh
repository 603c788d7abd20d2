// kernels.cuh -- sm_100a kernels of the ChiDG implicit linear-solve path.
//
// Data layout in HBM (see also the host builders in chidg_gpu.cu):
//  * A: every block of the pattern, packed in pattern order, each block
//    column-major nrows x ncols (the reference's densematrix_t%mat storage,
//    so a host upload is one contiguous copy).  FP64, plus an FP32 copy with
//    the same packing for the mixed-precision inner solves.
//  * vectors: element-major, then time, field, mode (densevector_t layout).
//  * ILU programme: one "programme row" per matrix row (ILU0/Jacobi) or per
//    subdomain row / overlap row (RAS).  LD holds, per programme row, the
//    inverted diagonal and one L block per lower entry.  U blocks are read
//    from A.  Rows are grouped into dependency levels for the factorisation
//    and the two triangular sweeps.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

namespace chidg {

// Column groups per row of b rows: G(b) = max(1, cap / b).  It depends on the
// row's own block size only, never on the launch (which is sized for the
// largest block present), so a row sums in the same order whatever it shares
// a matrix or a batch with.
constexpr int MV_GCAP = 512;     // matvec
constexpr int SW_GCAP = 1024;    // triangular sweeps, one CTA per row
constexpr int TK_GCAP = 512;     // task-split sweeps, one CTA per block product
__host__ __device__ __forceinline__ int stripe_groups(int cap, int b) { return b >= cap ? 1 : cap / b; }

// ---------------------------------------------------------------------------
// conversions
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ double to_d(T v);
template <> __device__ __forceinline__ double to_d<double>(double v) { return v; }
template <> __device__ __forceinline__ double to_d<float>(float v) { return (double)v; }
template <> __device__ __forceinline__ double to_d<__nv_bfloat16>(__nv_bfloat16 v) { return (double)__bfloat162float(v); }
template <typename T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<double>(double v) { return (float)v; }
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename ACC, typename T> __device__ __forceinline__ ACC cvt(T v);
template <> __device__ __forceinline__ double cvt<double, double>(double v) { return v; }
template <> __device__ __forceinline__ double cvt<double, float>(float v) { return (double)v; }
template <> __device__ __forceinline__ double cvt<double, __nv_bfloat16>(__nv_bfloat16 v) { return (double)__bfloat162float(v); }
template <> __device__ __forceinline__ float cvt<float, double>(double v) { return (float)v; }
template <> __device__ __forceinline__ float cvt<float, float>(float v) { return v; }
template <> __device__ __forceinline__ float cvt<float, __nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename T> __device__ __forceinline__ T from_d(double v);
template <> __device__ __forceinline__ double from_d<double>(double v) { return v; }
template <> __device__ __forceinline__ float from_d<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ __nv_bfloat16 from_d<__nv_bfloat16>(double v) { return __float2bfloat16_rn((float)v); }

// Streaming load of matrix data: each block is read once per sweep and the
// arrays are far larger than L2, so do not let them evict the vectors.
template <typename T> __device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }
template <> __device__ __forceinline__ __nv_bfloat16 ld_stream<__nv_bfloat16>(const __nv_bfloat16* p) {
    unsigned short u = __ldcs(reinterpret_cast<const unsigned short*>(p));
    return __ushort_as_bfloat16(u);
}

// acc + sum over the column stripe c = g, g+G, ... < nc of B[c*ld] * x[c],
// summed in increasing c (the same order in every kernel that uses it).  The
// loads go out in predicated batches of 16, so a thread never waits on more
// than ceil(stripe / 16) round trips to memory.
template <typename T, typename ACC>
__device__ __forceinline__ ACC stripe_dot(const T* __restrict__ B, int64_t ld, int nc, int g, int G,
                                          const ACC* __restrict__ x, ACC acc) {
    constexpr int U = 16;
    for (int c = g; c < nc; c += U * G) {
        T a[U];
        #pragma unroll
        for (int u = 0; u < U; ++u) {
            const int cc = c + u * G;
            a[u] = (cc < nc) ? ld_stream(B + (int64_t)cc * ld) : T(0);
        }
        #pragma unroll
        for (int u = 0; u < U; ++u) {
            const int cc = c + u * G;
            if (cc < nc) acc += cvt<ACC>(a[u]) * x[cc];
        }
    }
    return acc;
}

// ---------------------------------------------------------------------------
// block reductions (deterministic: fixed tree for a fixed blockDim)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// returns the block sum in thread 0 (other threads: garbage). scratch >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[w] = v;
    __syncthreads();
    double s = 0.0;
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = (lane < nw) ? scratch[lane] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

// ---------------------------------------------------------------------------
// chidg_mv: one CTA per matrix row (element, time level).
//   y_row = alpha * sum_k A_k x_{col(k)} + beta * z_row
// Thread t owns output entry r = t % b and the column stripe c = g, g+G, ...
// (g = t / b), so consecutive threads read consecutive addresses of every
// column-major block.  The x segments of the row's blocks are staged in
// shared memory once.  Optionally writes the row's sum of squares of y.
// ---------------------------------------------------------------------------
template <typename TA, typename TX, typename TY, typename ACC>
__global__ void __launch_bounds__(1024) k_matvec(const TA* __restrict__ val, const int64_t* __restrict__ row_ptr,
                         const int64_t* __restrict__ blk_voff, const int64_t* __restrict__ blk_xoff,
                         const int32_t* __restrict__ blk_nc, const int64_t* __restrict__ row_yoff,
                         const int32_t* __restrict__ row_b, const TX* __restrict__ x,
                         TY* __restrict__ y, const TY* __restrict__ z, double alpha, double beta,
                         double* __restrict__ row_sumsq) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ACC* xs = reinterpret_cast<ACC*>(smem_raw);
    const int row = blockIdx.x;
    const int b = row_b[row];
    const int64_t k0 = row_ptr[row], k1 = row_ptr[row + 1];
    const int tid = threadIdx.x;
    int off = 0;
    for (int64_t k = k0; k < k1; ++k) {
        const int nc = blk_nc[k];
        const TX* xp = x + blk_xoff[k];
        for (int c = tid; c < nc; c += blockDim.x) xs[off + c] = cvt<ACC>(xp[c]);
        off += nc;
    }
    const int ncols_total = off;
    __syncthreads();
    const int G = stripe_groups(MV_GCAP, b);
    const int r = tid % b, g = tid / b;
    ACC acc = 0;
    if (g < G) {
        off = 0;
        for (int64_t k = k0; k < k1; ++k) {
            const int nc = blk_nc[k];
            const TA* Ab = val + blk_voff[k] + r;
            const ACC* xb = xs + off;
            acc = stripe_dot(Ab, (int64_t)b, nc, g, G, xb, acc);
            off += nc;
        }
    }
    ACC* red = xs + ncols_total;
    if (g < G) red[g * b + r] = acc;
    __syncthreads();
    double sq = 0.0;
    if (tid < b) {
        ACC s = 0;
        for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
        double out = alpha * (double)s;
        const int64_t yo = row_yoff[row] + tid;
        if (z != nullptr) out += beta * to_d(z[yo]);
        const TY o = from_d<TY>(out);
        y[yo] = o;
        const double od = to_d(o);
        sq = od * od;
    }
    if (row_sumsq != nullptr) {
        __syncthreads();
        double* scratch = reinterpret_cast<double*>(smem_raw);
        const double s = block_sum(sq, scratch);
        if (tid == 0) row_sumsq[row] = s;
    }
}

// ---------------------------------------------------------------------------
// BLAS-1.  All reductions are two-pass: per-CTA partials in fixed order, then
// one CTA sums the partials in fixed order, so results are reproducible.
// ---------------------------------------------------------------------------
// partial[q * gridDim.x + blockIdx.x] = sum_i x[i] * y_q[i],  y_q = y + q * ystride
template <typename T>
__global__ void k_mdot_partial(int64_t n, const T* __restrict__ x, const T* __restrict__ y,
                               int64_t ystride, int nq, double* __restrict__ partial) {
    // eight vectors per pass over x: x[i] is read once for the eight, and the
    // eight loads of y are in flight together; each sum is formed in the
    // order of a pass per vector (thread's i in stride order, then the
    // block_sum tree), so the partials do not depend on the grouping
    constexpr int QG = 8;
    __shared__ double scratch[QG][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q0 = 0; q0 < nq; q0 += QG) {
        const int qn = min(QG, nq - q0);
        const T* yq = y + (int64_t)q0 * ystride;
        double s[QG];
        #pragma unroll
        for (int k = 0; k < QG; ++k) s[k] = 0.0;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            const double xi = to_d(x[i]);
            #pragma unroll
            for (int k = 0; k < QG; ++k)
                if (k < qn) s[k] += xi * to_d(yq[(int64_t)k * ystride + i]);
        }
        #pragma unroll
        for (int k = 0; k < QG; ++k) s[k] = warp_sum(s[k]);
        __syncthreads();
        if (lane == 0) {
            #pragma unroll
            for (int k = 0; k < QG; ++k) scratch[k][w] = s[k];
        }
        __syncthreads();
        if (w == 0) {
            const int nw = (blockDim.x + 31) >> 5;
            #pragma unroll
            for (int k = 0; k < QG; ++k) {
                double t = (lane < nw) ? scratch[k][lane] : 0.0;
                t = warp_sum(t);
                if (lane == 0 && k < qn) partial[(int64_t)(q0 + k) * gridDim.x + blockIdx.x] = t;
            }
        }
    }
}
// out[q] = sum_c partial[q * ncta + c]  (optionally sqrt)
static __global__ void k_reduce_partials(const double* __restrict__ partial, int ncta, int nq,
                                  double* __restrict__ out, int do_sqrt) {
    __shared__ double scratch[32];
    for (int q = 0; q < nq; ++q) {
        double s = 0.0;
        for (int c = threadIdx.x; c < ncta; c += blockDim.x) s += partial[(int64_t)q * ncta + c];
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) out[q] = do_sqrt ? sqrt(s) : s;
        __syncthreads();
    }
}
// sumsqr_fields (type_densevector.f90:806-830) summed over the elements
// (type_domain_vector.f90:495-511): CTA c adds, for every field, the squares
// of the modes of rows c, c + gridDim.x, ... (row = element and time level)
// and writes partial[f * gridDim.x + c]; every sum runs in a fixed order.
static __global__ void k_field_sumsq(const double* __restrict__ x, const int64_t* __restrict__ row_yoff,
                                     const int32_t* __restrict__ elem_nterms, int nrow, int ntime, int nfields,
                                     double* __restrict__ partial) {
    __shared__ double scratch[32];
    for (int f = 0; f < nfields; ++f) {
        double s = 0.0;
        for (int r = blockIdx.x; r < nrow; r += gridDim.x) {
            const int nt = elem_nterms[r / ntime];
            const double* seg = x + row_yoff[r] + (int64_t)f * nt;
            for (int m = threadIdx.x; m < nt; m += blockDim.x) s += seg[m] * seg[m];
        }
        s = block_sum(s, scratch);
        if (threadIdx.x == 0) partial[(int64_t)f * gridDim.x + blockIdx.x] = s;
        __syncthreads();
    }
}
// w[i] = w[i] - sum_q h[q] * v_q[i]  (CGS update, h on device), with sum of squares partials
template <typename T>
__global__ void k_maxpy_sub_norm(int64_t n, T* __restrict__ w, const T* __restrict__ v, int64_t vstride,
                                 int nq, const double* __restrict__ h, double* __restrict__ partial) {
    __shared__ double scratch[32];
    __shared__ double hs[128];
    double sq = 0.0;
    for (int q0 = 0; q0 < nq; q0 += 128) {
        const int qn = min(128, nq - q0);
        __syncthreads();
        for (int q = threadIdx.x; q < qn; q += blockDim.x) hs[q] = h[q0 + q];
        __syncthreads();
        const bool last = (q0 + 128 >= nq);
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            double acc = to_d(w[i]);
            for (int q = 0; q < qn; ++q) acc = acc - hs[q] * to_d(v[(int64_t)(q0 + q) * vstride + i]);
            const T o = from_d<T>(acc);
            w[i] = o;
            if (last) { const double od = to_d(o); sq += od * od; }
        }
    }
    if (partial != nullptr) {
        sq = block_sum(sq, scratch);
        if (threadIdx.x == 0) partial[blockIdx.x] = sq;
    }
}
// MGS single step: w -= h[0] * v (h on device), with sum-of-squares partials
// x = x0 + sum_q y[q] * z_q   (y on device)
template <typename T>
__global__ void k_lincomb(int64_t n, T* __restrict__ x, const T* __restrict__ x0, const T* __restrict__ z,
                          int64_t zstride, int nq, const double* __restrict__ y) {
    __shared__ double ys[128];
    for (int q0 = 0; q0 < nq || q0 == 0; q0 += 128) {
        const int qn = min(128, nq - q0);
        __syncthreads();
        for (int q = threadIdx.x; q < qn; q += blockDim.x) ys[q] = y[q0 + q];
        __syncthreads();
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
            double acc = (q0 == 0) ? (x0 ? to_d(x0[i]) : 0.0) : to_d(x[i]);
            for (int q = 0; q < qn; ++q) acc = acc + ys[q] * to_d(z[(int64_t)(q0 + q) * zstride + i]);
            x[i] = from_d<T>(acc);
        }
        if (nq == 0) break;
    }
}
// y = a * x + b * y, with the scalars either given or read from device memory
// (a = 1 / *adiv when adiv != nullptr).
template <typename TX, typename TY>
__global__ void k_axpby(int64_t n, double a, const double* adiv, const TX* x, double b, TY* y) {
    const double aa = adiv ? 1.0 / (*adiv) : a;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double yv = (b == 0.0) ? 0.0 : b * to_d(y[i]);
        y[i] = from_d<TY>(aa * to_d(x[i]) + yv);
    }
}
template <typename TS, typename TD>
__global__ void k_convert(int64_t n, const TS* __restrict__ s, TD* __restrict__ d) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        d[i] = from_d<TD>(to_d(s[i]));
}

// ---------------------------------------------------------------------------
// Pseudo-transient term: DIAG(e,t)[field block] += scale[e*nvars+f] * mass_e
// (chidg_matrix%scale_diagonal).  One CTA per (element, time).
// ---------------------------------------------------------------------------
static __global__ void k_scale_diagonal(double* __restrict__ val, const int64_t* __restrict__ diag_voff,
                                 const int32_t* __restrict__ elem_nvars, const int32_t* __restrict__ elem_nterms,
                                 const int64_t* __restrict__ mass_off, const double* __restrict__ mass,
                                 const double* __restrict__ scale, const int64_t* __restrict__ scale_off, int ntime) {
    const int row = blockIdx.x;
    const int e = row / ntime;
    const int nv = elem_nvars[e], nt = elem_nterms[e];
    const int b = nv * nt;
    double* D = val + diag_voff[row];
    const double* M = mass + mass_off[e];
    for (int idx = threadIdx.x; idx < nv * nt * nt; idx += blockDim.x) {
        const int f = idx / (nt * nt);
        const int rem = idx % (nt * nt);
        const int i = rem % nt, j = rem / nt;
        const double s = scale[scale_off[e] + f];
        D[(int64_t)(f * nt + i) + (int64_t)(f * nt + j) * b] += s * M[i + j * nt];
    }
}

// ---------------------------------------------------------------------------
// y(e, t, f) = scale[e*nvars+f] M_e x(e, t, f) per field segment
// (pseudo_transient_scaling): one CTA per (element, time), one thread per row
// (f, i), the sum over the element's modes j in increasing order.
// ---------------------------------------------------------------------------
static __global__ void k_mass_scale(const double* __restrict__ x, double* __restrict__ y,
                                    const int64_t* __restrict__ row_yoff, const int32_t* __restrict__ elem_nvars,
                                    const int32_t* __restrict__ elem_nterms, const int64_t* __restrict__ mass_off,
                                    const double* __restrict__ mass, const double* __restrict__ scale,
                                    const int64_t* __restrict__ scale_off, int ntime) {
    const int row = blockIdx.x;
    const int e = row / ntime;
    const int nv = elem_nvars[e], nt = elem_nterms[e];
    const int64_t o = row_yoff[row];
    const double* M = mass + mass_off[e];
    for (int r = threadIdx.x; r < nv * nt; r += blockDim.x) {
        const int f = r / nt, i = r - f * nt;
        const double s = scale[scale_off[e] + f];
        const double* xf = x + o + (int64_t)f * nt;
        double acc = 0.0;
        for (int j = 0; j < nt; ++j) acc += (s * M[i + j * nt]) * xf[j];
        y[o + r] = acc;
    }
}

// ---------------------------------------------------------------------------
// A^T in block-row storage: block k of A^T (nr x nc, column-major) is the
// transpose of its source block of A (nc x nr).  32 x 32 tiles pass through
// shared memory so that the reads and the writes are both coalesced; CTAs of
// 32 x 8 threads stride over the blocks.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(256)
    k_block_transpose(const double* __restrict__ src, double* __restrict__ dst, const int64_t* __restrict__ src_off,
                      const int64_t* __restrict__ dst_off, const int32_t* __restrict__ blk_nr,
                      const int32_t* __restrict__ blk_nc, int64_t nblk) {
    __shared__ double tile[32][33];
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int64_t k = blockIdx.x; k < nblk; k += gridDim.x) {
        const int nr = blk_nr[k], nc = blk_nc[k];
        const double* S = src + src_off[k];
        double* D = dst + dst_off[k];
        for (int i0 = 0; i0 < nr; i0 += 32)
            for (int j0 = 0; j0 < nc; j0 += 32) {
                for (int ii = ty; ii < 32; ii += 8) {        // tile[ii][tx] = S(j0+tx, i0+ii) = T(i0+ii, j0+tx)
                    const int i = i0 + ii, j = j0 + tx;
                    if (i < nr && j < nc) tile[ii][tx] = S[j + (int64_t)i * nc];
                }
                __syncthreads();
                for (int jj = ty; jj < 32; jj += 8) {        // T(i0+tx, j0+jj)
                    const int i = i0 + tx, j = j0 + jj;
                    if (i < nr && j < nc) D[i + (int64_t)j * nr] = tile[tx][jj];
                }
                __syncthreads();
            }
    }
}

// ---------------------------------------------------------------------------
// D blocks assembled from several blocks of A (precon_HB): one CTA per
// programme row zeroes its B x B slot in LD and copies each piece (a block of
// A, nr x nc, column-major) to rows r0.., columns c0.. of it.
// ---------------------------------------------------------------------------
static __global__ void __launch_bounds__(256)
    k_assemble_rows(double* __restrict__ LD, const int64_t* __restrict__ dinv_off, const int32_t* __restrict__ prow_b,
                    const double* __restrict__ Aval, const int32_t* __restrict__ piece_ptr,
                    const int64_t* __restrict__ piece_src, const int32_t* __restrict__ piece_r0,
                    const int32_t* __restrict__ piece_c0, const int32_t* __restrict__ piece_nr,
                    const int32_t* __restrict__ piece_nc) {
    const int pr = blockIdx.x;
    const int B = prow_b[pr];
    double* D = LD + dinv_off[pr];
    for (int64_t i = threadIdx.x; i < (int64_t)B * B; i += blockDim.x) D[i] = 0.0;
    __syncthreads();
    for (int q = piece_ptr[pr]; q < piece_ptr[pr + 1]; ++q) {
        const int nr = piece_nr[q], r0 = piece_r0[q], c0 = piece_c0[q];
        const int64_t cnt = (int64_t)nr * piece_nc[q];
        const double* S = Aval + piece_src[q];
        for (int64_t i = threadIdx.x; i < cnt; i += blockDim.x) {
            const int r = (int)(i % nr), c = (int)(i / nr);
            D[(int64_t)(r0 + r) + (int64_t)(c0 + c) * B] = S[i];
        }
    }
}

// ---------------------------------------------------------------------------
// ILU programme: factorisation
// ---------------------------------------------------------------------------
struct GemmTask {            // C(m x n) = [Cinit] + sgn * sum_q A_q(m x k_q) B_q(k_q x n)
    int64_t c_off;           // into the output arena
    int64_t cinit_off;       // into the Cinit arena, or -1 (start from zero)
    int32_t m, n;
    int32_t q_begin, q_end;  // pairs
    int32_t elem;            // element id for status reporting
    // k_task_gemm_dmma: the task may be the tile of rows r0.. and columns c0..
    // of an output block of ldm rows (the A operands have ldm rows too);
    // ldm = m, r0 = c0 = 0 for a whole block, which every other kernel takes
    int32_t ldm, r0, c0;
};
struct GemmPair {
    int64_t a_off, b_off;
    int32_t k;
    int32_t pad;
};

// Tiled SIMT GEMM over a list of tasks.  64x64 output tile per CTA, 256
// threads each accumulating a 4x4 register tile, K staged 16 at a time, in
// TS (FP64; FP32 for the FP32 factors of the mixed modes).  All operands
// column-major with leading dimension = their row count.
constexpr int GT_M = 64, GT_N = 64, GT_K = 16;
template <typename TA, typename TB, typename TC, typename TS = double>
__global__ void __launch_bounds__(256) k_task_gemm(const GemmTask* __restrict__ tasks, const GemmPair* __restrict__ pairs,
                                                   int tiles_m, int tiles_n,
                                                   const TA* Abase, const TB* Bbase,
                                                   const double* Cinit, TC* Cbase, double sgn) {
    __shared__ TS As[GT_K][GT_M + 1];
    __shared__ TS Bs[GT_K][GT_N + 1];
    const int tiles = tiles_m * tiles_n;
    const GemmTask t = tasks[blockIdx.x / tiles];
    const int tile = blockIdx.x % tiles;
    const int i0 = (tile % tiles_m) * GT_M, j0 = (tile / tiles_m) * GT_N;
    if (i0 >= t.m || j0 >= t.n) return;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    TS acc[4][4];
    #pragma unroll
    for (int a = 0; a < 4; ++a)
        #pragma unroll
        for (int c = 0; c < 4; ++c) acc[a][c] = TS(0);
    for (int q = t.q_begin; q < t.q_end; ++q) {
        const GemmPair pr = pairs[q];
        const TA* A = Abase + pr.a_off;   // m x k
        const TB* B = Bbase + pr.b_off;   // k x n
        for (int k0 = 0; k0 < pr.k; k0 += GT_K) {
            // A tile: 64 rows x 16 k  (column-major => consecutive threads walk rows)
            for (int idx = threadIdx.x; idx < GT_M * GT_K; idx += 256) {
                const int ii = idx % GT_M, kk = idx / GT_M;
                const int gi = i0 + ii, gk = k0 + kk;
                As[kk][ii] = (gi < t.m && gk < pr.k) ? cvt<TS>(A[gi + (int64_t)gk * t.m]) : TS(0);
            }
            // B tile: 16 k x 64 cols
            for (int idx = threadIdx.x; idx < GT_K * GT_N; idx += 256) {
                const int kk = idx % GT_K, jj = idx / GT_K;
                const int gk = k0 + kk, gj = j0 + jj;
                Bs[kk][jj] = (gk < pr.k && gj < t.n) ? cvt<TS>(B[gk + (int64_t)gj * pr.k]) : TS(0);
            }
            __syncthreads();
            #pragma unroll
            for (int kk = 0; kk < GT_K; ++kk) {
                TS av[4], bv[4];
                #pragma unroll
                for (int a = 0; a < 4; ++a) av[a] = As[kk][tx + 16 * a];
                #pragma unroll
                for (int c = 0; c < 4; ++c) bv[c] = Bs[kk][ty + 16 * c];
                #pragma unroll
                for (int a = 0; a < 4; ++a)
                    #pragma unroll
                    for (int c = 0; c < 4; ++c) acc[a][c] = fma(av[a], bv[c], acc[a][c]);
            }
            __syncthreads();
        }
    }
    #pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int gj = j0 + ty + 16 * c;
        if (gj >= t.n) continue;
        #pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int gi = i0 + tx + 16 * a;
            if (gi >= t.m) continue;
            const int64_t o = gi + (int64_t)gj * t.m;
            double v = sgn * (double)acc[a][c];
            if (t.cinit_off >= 0) v = Cinit[t.cinit_off + o] + v;
            Cbase[t.c_off + o] = from_d<TC>(v);
        }
    }
}

// FP64 tensor-core version of k_task_gemm for blocks up to 136 x 136: one CTA
// computes a whole output block on the FP64 tensor cores (DMMA).  8 warps on
// a 2 x 4 grid.  The 17 row tiles of 8 are taken in pairs (rows 16p ..
// 16p+15, p < 8) by mma.sync m16n8k8, warp row wm owning pairs wm + 2i
// (i < 4), and the last tile (rows 128..135) by m8n8k4 in warp row 0; warp
// column wn owns the column tiles wn + 4j (j < 5).  Per slice of K = 8 a
// warp loads its five B fragments once and each pair's A fragment once: 20
// m16n8k8 (and 10 m8n8k4 in warp row 0) per slice, a third of the
// instructions of the same work in m8n8k4.  K is staged 32 at a time through
// shared memory in the same k-major layout for both operands, leading
// dimension 140 (= 12 mod 16 doubles: the fragment loads of a half-warp hit
// 16 distinct bank pairs); past the operands' K the stage holds zeros.
constexpr int DM_MAX = 136, DM_LD = 140, DM_KC = 32, DM_WM = 2, DM_WN = 4, DM_TI = 9, DM_TJ = 5;
constexpr int DM_THREADS = 32 * DM_WM * DM_WN;
constexpr size_t DM_SMEM = 4 * sizeof(double) * DM_KC * DM_LD;   // two stages of (A, B) panels
// 8-byte asynchronous global->shared copy; src_ok == false writes zeros
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool src_ok) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = src_ok ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" :: "r"(s), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory"); }
// D(16x8) += A(16x8) B(8x8): lane (g, t) holds A(g, t), A(g+8, t), A(g, t+4),
// A(g+8, t+4); B(t, g), B(t+4, g); D(g, 2t), D(g, 2t+1), D(g+8, 2t), D(g+8, 2t+1)
__device__ __forceinline__ void dmma_16x8x8(double& d0, double& d1, double& d2, double& d3, double a0, double a1,
                                            double a2, double a3, double b0, double b1) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+d"(d0), "+d"(d1), "+d"(d2), "+d"(d3)
                 : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}
template <typename TA, typename TB, typename TC>
__global__ void __launch_bounds__(DM_THREADS, 1) k_task_gemm_dmma(const GemmTask* __restrict__ tasks, const GemmPair* __restrict__ pairs,
                                                               const TA* Abase, const TB* Bbase,
                                                               const double* Cinit, TC* Cbase, double sgn) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* As = reinterpret_cast<double*>(smem_raw);      // 2 stages x {A [DM_KC][DM_LD], B [DM_KC][DM_LD]}
    static_assert(sizeof(TA) == 8 && sizeof(TB) == 8, "FP64 operands");
    const GemmTask t = tasks[blockIdx.x];
    const int ldm = t.ldm;                        // rows of the whole output block and of A
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int wm = w % DM_WM, wn = w / DM_WM;
    const int g = lane >> 2, tq = lane & 3;
    double acc[DM_TI][DM_TJ][2];
    #pragma unroll
    for (int i = 0; i < DM_TI; ++i)
        #pragma unroll
        for (int j = 0; j < DM_TJ; ++j) { acc[i][j][0] = 0.0; acc[i][j][1] = 0.0; }
    const int tm = (t.m + 7) >> 3, tn = (t.n + 7) >> 3;
    // K is walked as one list of chunks over all pairs; chunk c+1 is copied
    // into the other shared-memory stage (cp.async, zero-filled outside the
    // operands) while chunk c feeds the tensor cores
    int nchunk = 0;
    for (int q = t.q_begin; q < t.q_end; ++q) nchunk += (pairs[q].k + DM_KC - 1) / DM_KC;
    int lq = t.q_begin, lk0 = 0;                  // next chunk to load
    auto issue = [&](int stage) {
        const GemmPair pr = pairs[lq];
        const TA* A = Abase + pr.a_off + t.r0;                  // the tile's rows of ldm x k, column-major
        const TB* B = Bbase + pr.b_off + (int64_t)t.c0 * pr.k;  // the tile's columns of k x N, column-major
        const int kc = min(DM_KC, pr.k - lk0);
        double* as = As + stage * 2 * DM_KC * DM_LD;
        double* bs = as + DM_KC * DM_LD;
        for (int idx = threadIdx.x; idx < DM_KC * DM_MAX; idx += blockDim.x) {
            const int i = idx % DM_MAX, kk = idx / DM_MAX;
            const bool ok = i < t.m && kk < kc;
            cp_async8(as + kk * DM_LD + i, ok ? (const void*)(A + i + (int64_t)(lk0 + kk) * ldm) : (const void*)A, ok);
        }
        for (int idx = threadIdx.x; idx < DM_KC * DM_MAX; idx += blockDim.x) {
            const int kk = idx % DM_KC, j = idx / DM_KC;
            const bool ok = j < t.n && kk < kc;
            cp_async8(bs + kk * DM_LD + j, ok ? (const void*)(B + (lk0 + kk) + (int64_t)j * pr.k) : (const void*)B, ok);
        }
        cp_async_commit();
        lk0 += DM_KC;
        if (lk0 >= pr.k) { ++lq; lk0 = 0; }
    };
    int cq = t.q_begin, ck0 = 0;                  // chunk being computed
    if (nchunk > 0) issue(0);
    for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) { issue((c + 1) & 1); cp_async_wait<1>(); }
        else cp_async_wait<0>();
        __syncthreads();
        const int kc = min(DM_KC, pairs[cq].k - ck0);
        const double* as = As + (c & 1) * 2 * DM_KC * DM_LD;
        const double* bs = as + DM_KC * DM_LD;
        for (int k8 = 0; k8 < kc; k8 += 8) {
            // slices past kc read the stage's zeros (rows kc..31)
            const double* a_lo = as + (k8 + tq) * DM_LD + g;       // A(., k8 + t)
            const double* a_hi = a_lo + 4 * DM_LD;                 // A(., k8 + t + 4)
            double b0[DM_TJ], b1[DM_TJ];
            #pragma unroll
            for (int j = 0; j < DM_TJ; ++j) {
                // column tiles past the 17th exist only in the warp grid: never read them
                const bool ok = wn + DM_WN * j < tn;
                const int col = (wn + DM_WN * j) * 8 + g;
                b0[j] = ok ? bs[(k8 + tq) * DM_LD + col] : 0.0;
                b1[j] = ok ? bs[(k8 + tq + 4) * DM_LD + col] : 0.0;
            }
            #pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int p = wm + DM_WM * i;                      // rows 16p .. 16p + 15
                if (2 * p >= tm) continue;
                const double a0 = a_lo[16 * p], a1 = a_lo[16 * p + 8], a2 = a_hi[16 * p], a3 = a_hi[16 * p + 8];
                #pragma unroll
                for (int j = 0; j < DM_TJ; ++j) {
                    if (wn + DM_WN * j >= tn) continue;
                    dmma_16x8x8(acc[2 * i][j][0], acc[2 * i][j][1], acc[2 * i + 1][j][0], acc[2 * i + 1][j][1], a0, a1,
                                a2, a3, b0[j], b1[j]);
                }
            }
            if (wm == 0 && tm > 16) {                               // rows 128 .. 135
                const double a0 = a_lo[128], a1 = a_hi[128];
                #pragma unroll
                for (int j = 0; j < DM_TJ; ++j) {
                    if (wn + DM_WN * j >= tn) continue;
                    dmma_8x8x4(acc[8][j][0], acc[8][j][1], a0, b0[j]);
                    dmma_8x8x4(acc[8][j][0], acc[8][j][1], a1, b1[j]);
                }
            }
        }
        ck0 += DM_KC;
        if (ck0 >= pairs[cq].k) { ++cq; ck0 = 0; }
        __syncthreads();                          // stage (c & 1) is refilled two chunks later
    }
    // acc[2i + h]: rows 16 (wm + 2i) + 8h + g; acc[8] (warp row 0): rows 128 + g
    #pragma unroll
    for (int i = 0; i < DM_TI; ++i) {
        const int row = (i < 8) ? 16 * (wm + DM_WM * (i >> 1)) + 8 * (i & 1) + g : (wm == 0 ? 128 + g : DM_MAX);
        if (row >= t.m) continue;
        #pragma unroll
        for (int j = 0; j < DM_TJ; ++j) {
            #pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int col = (wn + DM_WN * j) * 8 + 2 * tq + e;
                if (col >= t.n) continue;
                const int64_t o = (t.r0 + row) + (int64_t)(t.c0 + col) * ldm;
                double v = sgn * acc[i][j][e];
                if (t.cinit_off >= 0) v = Cinit[t.cinit_off + o] + v;
                Cbase[t.c_off + o] = from_d<TC>(v);
            }
        }
    }
}

// FP32 SIMT version of the factor products for blocks up to 144 x 144, used
// when the factors are only needed in FP32 (the mixed-precision inner solves):
// one CTA per output block, 256 threads on a 16 x 16 grid, thread (tx, ty)
// accumulating rows ty + 16i and columns tx + 16j (i, j < 9) in FP32.  K is
// staged 32 at a time (cp.async, zero-filled outside the operands, two
// stages).  A (m x k) and B (k x n) column-major FP32; the output is TC
// (FP32 L blocks, or FP64 D blocks for the FP64 diagonal inverse), with an
// optional FP64 Cinit.
constexpr int SF_MAX = 144, SF_KC = 32, SF_LDA = 144, SF_LDB = 145;
constexpr size_t SF_SMEM = 2 * sizeof(float) * SF_KC * (SF_LDA + SF_LDB);
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool src_ok) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = src_ok ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" :: "r"(s), "l"(gmem), "r"(n) : "memory");
}
template <typename TC>
__global__ void __launch_bounds__(256, 1) k_task_gemm_f32(const GemmTask* __restrict__ tasks, const GemmPair* __restrict__ pairs,
                                                          const float* Abase, const float* Bbase, const double* Cinit,
                                                          TC* Cbase, double sgn) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* As = reinterpret_cast<float*>(smem_raw);        // 2 stages x {A [SF_KC][SF_LDA], B [SF_KC][SF_LDB]}
    const GemmTask t = tasks[blockIdx.x];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float acc[9][9];
    #pragma unroll
    for (int i = 0; i < 9; ++i)
        #pragma unroll
        for (int j = 0; j < 9; ++j) acc[i][j] = 0.0f;
    int nchunk = 0;
    for (int q = t.q_begin; q < t.q_end; ++q) nchunk += (pairs[q].k + SF_KC - 1) / SF_KC;
    int lq = t.q_begin, lk0 = 0;
    auto issue = [&](int stage) {
        const GemmPair pr = pairs[lq];
        const float* A = Abase + pr.a_off;        // m x k
        const float* B = Bbase + pr.b_off;        // k x n
        const int kc = min(SF_KC, pr.k - lk0);
        float* as = As + stage * SF_KC * (SF_LDA + SF_LDB);
        float* bs = as + SF_KC * SF_LDA;
        for (int kk = warp; kk < SF_KC; kk += 8)              // A: coalesced along the rows
            for (int i = lane; i < SF_MAX; i += 32) {
                const bool ok = i < t.m && kk < kc;
                cp_async4(as + kk * SF_LDA + i, ok ? (const void*)(A + i + (int64_t)(lk0 + kk) * t.m) : (const void*)A, ok);
            }
        for (int j = warp; j < SF_MAX; j += 8) {               // B: coalesced along k
            const bool ok = j < t.n && lane < kc;
            cp_async4(bs + lane * SF_LDB + j, ok ? (const void*)(B + (lk0 + lane) + (int64_t)j * pr.k) : (const void*)B, ok);
        }
        cp_async_commit();
        lk0 += SF_KC;
        if (lk0 >= pr.k) { ++lq; lk0 = 0; }
    };
    if (nchunk > 0) issue(0);
    for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) { issue((c + 1) & 1); cp_async_wait<1>(); }
        else cp_async_wait<0>();
        __syncthreads();
        const float* as = As + (c & 1) * SF_KC * (SF_LDA + SF_LDB);
        const float* bs = as + SF_KC * SF_LDA;
        #pragma unroll 4
        for (int kk = 0; kk < SF_KC; ++kk) {          // a short last chunk is zero-filled
            float a[9], b[9];
            #pragma unroll
            for (int i = 0; i < 9; ++i) a[i] = as[kk * SF_LDA + ty + 16 * i];
            #pragma unroll
            for (int j = 0; j < 9; ++j) b[j] = bs[kk * SF_LDB + tx + 16 * j];
            #pragma unroll
            for (int i = 0; i < 9; ++i)
                #pragma unroll
                for (int j = 0; j < 9; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();                          // stage (c & 1) is refilled two chunks later
    }
    #pragma unroll
    for (int j = 0; j < 9; ++j) {
        const int col = tx + 16 * j;
        if (col >= t.n) continue;
        #pragma unroll
        for (int i = 0; i < 9; ++i) {
            const int row = ty + 16 * i;
            if (row >= t.m) continue;
            const int64_t o = row + (int64_t)col * t.m;
            double v = sgn * (double)acc[i][j];
            if (t.cinit_off >= 0) v = Cinit[t.cinit_off + o] + v;
            Cbase[t.c_off + o] = from_d<TC>(v);
        }
    }
}

// The same products on the tensor cores: mma.sync m16n8k8 with TF32 operands
// (rounded to nearest from the FP32 blocks) and FP32 accumulation.  One
// 144 x 144 output tile per CTA, 9 warps in a 3 x 3 grid of 48 x 48 regions
// (3 x 6 MMA tiles each).  K chunks of 32 in two cp.async stages: A stored
// [k][m] (leading dimension 152) and B stored [n][k] (leading dimension 36),
// so that the staging writes and the fragment reads are both free of bank
// conflicts.  Bounds: loads past m, n or k are zero-filled, stores are guarded.
constexpr int ST_LDA = 152, ST_LDB = 36, ST_THREADS = 288;
constexpr size_t ST_STAGE = (size_t)SF_KC * ST_LDA + (size_t)SF_MAX * ST_LDB;   // floats per stage
constexpr size_t ST_SMEM = 2 * sizeof(float) * ST_STAGE;
__device__ __forceinline__ unsigned to_tf32(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void mma_tf32_16x8x8(float (&d)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
template <typename TC>
__global__ void __launch_bounds__(ST_THREADS, 1) k_task_gemm_tf32(const GemmTask* __restrict__ tasks, const GemmPair* __restrict__ pairs,
                                                                  const float* Abase, const float* Bbase, const double* Cinit,
                                                                  TC* Cbase, double sgn) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* S = reinterpret_cast<float*>(smem_raw);          // 2 stages x {A [SF_KC][ST_LDA], B [SF_MAX][ST_LDB]}
    const GemmTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int wm = (warp / 3) * 48, wn = (warp % 3) * 48;    // this warp's region
    float acc[3][6][4];
    #pragma unroll
    for (int i = 0; i < 3; ++i)
        #pragma unroll
        for (int j = 0; j < 6; ++j)
            #pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0f;
    int nchunk = 0;
    for (int q = t.q_begin; q < t.q_end; ++q) nchunk += (pairs[q].k + SF_KC - 1) / SF_KC;
    int lq = t.q_begin, lk0 = 0;
    auto issue = [&](int stage) {
        const GemmPair pr = pairs[lq];
        const float* A = Abase + pr.a_off;        // m x k, column-major
        const float* B = Bbase + pr.b_off;        // k x n, column-major
        const int kc = min(SF_KC, pr.k - lk0);
        float* as = S + stage * ST_STAGE;
        float* bs = as + SF_KC * ST_LDA;
        for (int idx = tid; idx < SF_KC * SF_MAX; idx += ST_THREADS) {   // A: consecutive m, coalesced
            const int kk = idx / SF_MAX, i = idx % SF_MAX;
            const bool ok = i < t.m && kk < kc;
            cp_async4(as + kk * ST_LDA + i, ok ? (const void*)(A + i + (int64_t)(lk0 + kk) * t.m) : (const void*)A, ok);
        }
        for (int idx = tid; idx < SF_MAX * SF_KC; idx += ST_THREADS) {   // B: consecutive k, coalesced
            const int j = idx / SF_KC, kk = idx % SF_KC;
            const bool ok = j < t.n && kk < kc;
            cp_async4(bs + j * ST_LDB + kk, ok ? (const void*)(B + (lk0 + kk) + (int64_t)j * pr.k) : (const void*)B, ok);
        }
        cp_async_commit();
        lk0 += SF_KC;
        if (lk0 >= pr.k) { ++lq; lk0 = 0; }
    };
    if (nchunk > 0) issue(0);
    for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) { issue((c + 1) & 1); cp_async_wait<1>(); }
        else cp_async_wait<0>();
        __syncthreads();
        const float* as = S + (c & 1) * ST_STAGE;
        const float* bs = as + SF_KC * ST_LDA;
        #pragma unroll
        for (int k0 = 0; k0 < SF_KC; k0 += 8) {   // a short last chunk is zero-filled
            unsigned af[3][4], bf[6][2];
            #pragma unroll
            for (int i = 0; i < 3; ++i) {
                const float* ap = as + (k0 + tig) * ST_LDA + wm + 16 * i + g;
                af[i][0] = to_tf32(ap[0]);
                af[i][1] = to_tf32(ap[8]);
                af[i][2] = to_tf32(ap[4 * ST_LDA]);
                af[i][3] = to_tf32(ap[4 * ST_LDA + 8]);
            }
            #pragma unroll
            for (int j = 0; j < 6; ++j) {
                const float* bp = bs + (wn + 8 * j + g) * ST_LDB + k0 + tig;
                bf[j][0] = to_tf32(bp[0]);
                bf[j][1] = to_tf32(bp[4]);
            }
            #pragma unroll
            for (int i = 0; i < 3; ++i)
                #pragma unroll
                for (int j = 0; j < 6; ++j) mma_tf32_16x8x8(acc[i][j], af[i], bf[j]);
        }
        __syncthreads();                          // stage (c & 1) is refilled two chunks later
    }
    #pragma unroll
    for (int i = 0; i < 3; ++i)
        #pragma unroll
        for (int j = 0; j < 6; ++j)
            #pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int row = wm + 16 * i + g + ((r & 2) ? 8 : 0);
                const int col = wn + 8 * j + 2 * tig + (r & 1);
                if (row >= t.m || col >= t.n) continue;
                const int64_t o = row + (int64_t)col * t.m;
                double v = sgn * (double)acc[i][j][r];
                if (t.cinit_off >= 0) v = Cinit[t.cinit_off + o] + v;
                Cbase[t.c_off + o] = from_d<TC>(v);
            }
}

// FP32 copies of the inverted diagonal blocks of some programme rows (one CTA
// per row): the inverses of a wavefront, for the next wavefront's FP32 products
// and the FP32 sweeps
static __global__ void k_convert_dinv(const double* __restrict__ LD, float* __restrict__ LD32,
                                      const int64_t* __restrict__ dinv_off, const int32_t* __restrict__ prow_b,
                                      const int32_t* __restrict__ rows, int row_begin) {
    const int pr = rows[row_begin + blockIdx.x];
    const int64_t o = dinv_off[pr];
    const int n = prow_b[pr] * prow_b[pr];
    for (int i = threadIdx.x; i < n; i += blockDim.x) LD32[o + i] = (float)LD[o + i];
}

// In-place inverse of one diagonal block per CTA: Gauss-Jordan with partial
// (row) pivoting, restated from the textbook algorithm.  The pivot of column
// k is the entry of largest magnitude among rows not yet used as pivots
// (first such row on ties), which is the pivot DGETRF selects.  Rows are not
// swapped physically: each thread keeps a fixed RPL x CPW register tile
// (rows lane + 32*ri, columns warp + NW*cj) and the permutation is undone
// when the result is written.  A zero pivot records the element in *status
// (ESINGULAR) and leaves garbage, never traps.
template <int RPL, int CPW, int NW>
__global__ void __launch_bounds__(NW * 32) k_block_inverse(double* __restrict__ LD, const int64_t* __restrict__ dinv_off,
                                                           const int32_t* __restrict__ prow_b,
                                                           const int32_t* __restrict__ prow_elem,
                                                           const int32_t* __restrict__ rows, int row_begin,
                                                           int* __restrict__ status) {
    constexpr int RMAX = 32 * RPL, CMAX = NW * CPW;
    __shared__ double colbuf[2][RMAX];
    __shared__ double rowbuf[2][CMAX];
    __shared__ int used[RMAX];
    __shared__ int pivrow[CMAX > RMAX ? CMAX : RMAX];
    __shared__ int qinv[RMAX];
    __shared__ int s_p;
    __shared__ double s_piv;
    const int prow = rows[row_begin + blockIdx.x];
    const int b = prow_b[prow];
    double* D = LD + dinv_off[prow];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double a[RPL][CPW];
    #pragma unroll
    for (int ri = 0; ri < RPL; ++ri)
        #pragma unroll
        for (int cj = 0; cj < CPW; ++cj) {
            const int i = lane + 32 * ri, j = w + NW * cj;
            a[ri][cj] = (i < b && j < b) ? D[i + (int64_t)j * b] : 0.0;
        }
    for (int i = threadIdx.x; i < RMAX; i += blockDim.x) used[i] = 0;
    bool singular = false;
    __syncthreads();
    for (int k = 0; k < b; ++k) {
        const int wk = k % NW, ck = k / NW, buf = k & 1;
        if (w == wk) {
            double best = -1.0;
            int bi = 0x7fffffff;
            #pragma unroll
            for (int ri = 0; ri < RPL; ++ri) {
                const int i = lane + 32 * ri;
                double v = -1.0;
                #pragma unroll
                for (int cj = 0; cj < CPW; ++cj) if (cj == ck) v = fabs(a[ri][cj]);
                if (!(v == v)) v = INFINITY;   // a NaN entry is taken as pivot so the NaN propagates
                if (i < b && !used[i] && (v > best || (v == best && i < bi))) { best = v; bi = i; }
            }
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (lane == (bi & 31)) {
                const int rp = bi >> 5;
                double pv = 0.0;
                #pragma unroll
                for (int ri = 0; ri < RPL; ++ri)
                    #pragma unroll
                    for (int cj = 0; cj < CPW; ++cj) if (ri == rp && cj == ck) pv = a[ri][cj];
                s_p = bi;
                s_piv = pv;
                used[bi] = 1;
                pivrow[k] = bi;
            }
        }
        __syncthreads();
        const int p = s_p;
        double piv = s_piv;
        if (piv == 0.0) { singular = true; piv = 1.0; }
        const double rp = 1.0 / piv;
        if (lane == (p & 31)) {
            const int rip = p >> 5;
            #pragma unroll
            for (int cj = 0; cj < CPW; ++cj) {
                const int j = w + NW * cj;
                double v = 0.0;
                #pragma unroll
                for (int ri = 0; ri < RPL; ++ri) if (ri == rip) v = a[ri][cj];
                if (j == k) v = 1.0;
                if (j < CMAX) rowbuf[buf][j] = v * rp;
            }
        }
        if (w == wk) {
            #pragma unroll
            for (int ri = 0; ri < RPL; ++ri) {
                const int i = lane + 32 * ri;
                double v = 0.0;
                #pragma unroll
                for (int cj = 0; cj < CPW; ++cj) if (cj == ck) v = a[ri][cj];
                colbuf[buf][i] = (i == p) ? 0.0 : v;
            }
        }
        __syncthreads();
        #pragma unroll
        for (int ri = 0; ri < RPL; ++ri) {
            const int i = lane + 32 * ri;
            const double f = colbuf[buf][i];
            #pragma unroll
            for (int cj = 0; cj < CPW; ++cj) {
                const int j = w + NW * cj;
                const double rv = rowbuf[buf][j];
                if (i == p) a[ri][cj] = rv;
                else {
                    const double base = (j == k) ? 0.0 : a[ri][cj];
                    a[ri][cj] = fma(-f, rv, base);
                }
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < b; k += blockDim.x) qinv[pivrow[k]] = k;
    __syncthreads();
    #pragma unroll
    for (int ri = 0; ri < RPL; ++ri)
        #pragma unroll
        for (int cj = 0; cj < CPW; ++cj) {
            const int i = lane + 32 * ri, j = w + NW * cj;
            if (i < b && j < b) D[qinv[i] + (int64_t)pivrow[j] * b] = a[ri][cj];
        }
    if (singular && threadIdx.x == 0) atomicMin(status, prow_elem[prow]);
}

// In-place inverse, second layout: 16 warps, warp w owns rows w + 16*ri
// (ri < RW), lane l owns columns l + 32*cl (cl < CL), so b <= min(32*CL, 16*RW).  The
// pivot loop is split into a compile-time column slot ck and a runtime lane
// lk (k = 32*ck + lk): every access to the pivot column is then a static
// register index, and only the pivot row needs a runtime row select (done
// by its owning warp alone).  Same pivoting rule and result as
// k_block_inverse: Gauss-Jordan with implicit row pivoting, largest |a|
// among unused rows (first on ties), permutation undone on the store.
template <int CL, int RW>
__global__ void __launch_bounds__(512) k_block_inverse2(double* __restrict__ LD, const int64_t* __restrict__ dinv_off,
                                                       const int32_t* __restrict__ prow_b,
                                                       const int32_t* __restrict__ prow_elem,
                                                       const int32_t* __restrict__ rows, int row_begin,
                                                       int* __restrict__ status) {
    constexpr int NW = 16, NMAX = (32 * CL > NW * RW) ? 32 * CL : NW * RW;
    __shared__ double colbuf[NMAX];
    __shared__ double rowbuf[2][NMAX];
    __shared__ double cand_v[NW];
    __shared__ double cand_a[NW];
    __shared__ int cand_i[NW];
    __shared__ int pivrow[NMAX];
    __shared__ int qinv[NMAX];
    const int prow = rows[row_begin + blockIdx.x];
    const int b = prow_b[prow];
    double* D = LD + dinv_off[prow];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double a[RW][CL];
    #pragma unroll
    for (int ri = 0; ri < RW; ++ri)
        #pragma unroll
        for (int cl = 0; cl < CL; ++cl) {
            const int i = w + NW * ri, j = lane + 32 * cl;
            a[ri][cl] = (i < b && j < b) ? D[i + (int64_t)j * b] : 0.0;
        }
    unsigned used = 0;          // bit ri set: row w + NW*ri already used as a pivot
    bool singular = false;
    #pragma unroll
    for (int ck = 0; ck < CL; ++ck) {
        for (int lk = 0; lk < 32; ++lk) {
            const int k = 32 * ck + lk;
            if (k >= b) break;
            const int buf = k & 1;
            // (a) candidates of this warp's rows in column k; column k to colbuf
            if (lane == lk) {
                double best = -1.0, bestv = 0.0;
                int bi = 0x7fffffff;
                #pragma unroll
                for (int ri = 0; ri < RW; ++ri) {
                    const int i = w + NW * ri;
                    if (i < b) {
                        colbuf[i] = a[ri][ck];
                        double m = fabs(a[ri][ck]);
                        if (!(m == m)) m = INFINITY;   // a NaN pivot propagates
                        if (!((used >> ri) & 1u) && (m > best || (m == best && i < bi))) { best = m; bi = i; bestv = a[ri][ck]; }
                    }
                }
                cand_v[w] = best;
                cand_a[w] = bestv;
                cand_i[w] = bi;
            }
            __syncthreads();
            // (b) every thread picks the pivot from the 16 candidates
            double best = -1.0, piv = 0.0;
            int p = 0x7fffffff;
            #pragma unroll
            for (int q = 0; q < NW; ++q) {
                const double v = cand_v[q];
                const int iq = cand_i[q];
                if (v > best || (v == best && iq < p)) { best = v; p = iq; piv = cand_a[q]; }
            }
            if (piv == 0.0) { singular = true; piv = 1.0; }
            const double rp = 1.0 / piv;
            const int pw = p % NW, prr = p / NW;
            if (w == pw) {
                used |= 1u << prr;
                #pragma unroll
                for (int cl = 0; cl < CL; ++cl) {
                    double v = 0.0;
                    #pragma unroll
                    for (int ri = 0; ri < RW; ++ri) if (ri == prr) v = a[ri][cl];
                    if (cl == ck && lane == lk) v = 1.0;
                    rowbuf[buf][lane + 32 * cl] = v * rp;
                }
            }
            if (threadIdx.x == 0) pivrow[k] = p;
            __syncthreads();
            // (c) rank-1 update; row p becomes the scaled pivot row, column k
            // becomes -a(i,k)/piv
            double rv[CL];
            #pragma unroll
            for (int cl = 0; cl < CL; ++cl) rv[cl] = rowbuf[buf][lane + 32 * cl];
            #pragma unroll
            for (int ri = 0; ri < RW; ++ri) {
                const int i = w + NW * ri;
                if (i == p) {
                    #pragma unroll
                    for (int cl = 0; cl < CL; ++cl) a[ri][cl] = rv[cl];
                } else {
                    const double f = (i < b) ? colbuf[i] : 0.0;
                    #pragma unroll
                    for (int cl = 0; cl < CL; ++cl) a[ri][cl] = fma(-f, rv[cl], a[ri][cl]);
                    if (lane == lk) a[ri][ck] = -f * rp;
                }
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < b; k += blockDim.x) qinv[pivrow[k]] = k;
    __syncthreads();
    #pragma unroll
    for (int ri = 0; ri < RW; ++ri)
        #pragma unroll
        for (int cl = 0; cl < CL; ++cl) {
            const int i = w + NW * ri, j = lane + 32 * cl;
            if (i < b && j < b) D[qinv[i] + (int64_t)pivrow[j] * b] = a[ri][cl];
        }
    if (singular && threadIdx.x == 0) atomicMin(status, prow_elem[prow]);
}

// In-place inverse, third layout: the k_block_inverse2 tiles with one barrier
// per pivot step.  Before the barrier every warp proposes the best unused row
// of its own in column k, writes that candidate's value, reciprocal, index
// and whole row (scaled later) into a double-buffered shared slot, and lane
// lk writes the warp's part of column k.  After the barrier every warp picks
// the winner with a 16-lane shuffle reduction (largest |a|, lowest row on
// ties: the DGETRF choice) and reads the pivot row from the winner's slot, so
// no warp has to wait for the owner of the pivot row.
template <int CL, int RW>
__global__ void __launch_bounds__(512) k_block_inverse3(double* __restrict__ LD, const int64_t* __restrict__ dinv_off,
                                                       const int32_t* __restrict__ prow_b,
                                                       const int32_t* __restrict__ prow_elem,
                                                       const int32_t* __restrict__ rows, int row_begin,
                                                       int* __restrict__ status) {
    constexpr int NW = 16, NMAX = (32 * CL > NW * RW) ? 32 * CL : NW * RW;
    __shared__ double colbuf[2][NMAX];
    __shared__ double candrow[2][NW][32 * CL];
    __shared__ double cand_v[2][NW];
    __shared__ double cand_a[2][NW];
    __shared__ int cand_i[2][NW];
    __shared__ int pivrow[NMAX];
    __shared__ int qinv[NMAX];
    const int prow = rows[row_begin + blockIdx.x];
    const int b = prow_b[prow];
    double* D = LD + dinv_off[prow];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double a[RW][CL];
    #pragma unroll
    for (int ri = 0; ri < RW; ++ri)
        #pragma unroll
        for (int cl = 0; cl < CL; ++cl) {
            const int i = w + NW * ri, j = lane + 32 * cl;
            a[ri][cl] = (i < b && j < b) ? D[i + (int64_t)j * b] : 0.0;
        }
    unsigned used = 0;          // bit ri: row w + NW*ri already a pivot
    bool singular = false;
    #pragma unroll
    for (int ck = 0; ck < CL; ++ck) {
        for (int lk = 0; lk < 32; ++lk) {
            const int k = 32 * ck + lk;
            if (k >= b) break;
            const int buf = k & 1;
            // (a) this warp's candidate for column k
            double best = -1.0, bestv = 0.0;
            int bri = -1;
            if (lane == lk) {
                #pragma unroll
                for (int ri = 0; ri < RW; ++ri) {
                    const int i = w + NW * ri;
                    if (i < b) {
                        colbuf[buf][i] = a[ri][ck];
                        double m = fabs(a[ri][ck]);
                        if (!(m == m)) m = INFINITY;          // a NaN pivot propagates
                        if (!((used >> ri) & 1u) && m > best) { best = m; bri = ri; bestv = a[ri][ck]; }
                    }
                }
            }
            best = __shfl_sync(0xffffffffu, best, lk);
            bestv = __shfl_sync(0xffffffffu, bestv, lk);
            bri = __shfl_sync(0xffffffffu, bri, lk);
            if (bri >= 0) {
                #pragma unroll
                for (int cl = 0; cl < CL; ++cl) {
                    double vsel = 0.0;
                    #pragma unroll
                    for (int ri = 0; ri < RW; ++ri) if (ri == bri) vsel = a[ri][cl];
                    candrow[buf][w][lane + 32 * cl] = vsel;
                }
            }
            if (lane == 0) {
                cand_v[buf][w] = best;
                cand_a[buf][w] = (bestv == 0.0) ? 1.0 : 1.0 / bestv;
                cand_i[buf][w] = (bri >= 0) ? w + NW * bri : 0x7fffffff;
            }
            __syncthreads();
            // (b) winner by shuffle reduction over the 16 candidates
            double v = (lane < NW) ? cand_v[buf][lane] : -2.0;
            int ii = (lane < NW) ? cand_i[buf][lane] : 0x7fffffff;
            int src = lane;
            #pragma unroll
            for (int o = 8; o > 0; o >>= 1) {
                const double ov = __shfl_xor_sync(0xffffffffu, v, o);
                const int oi = __shfl_xor_sync(0xffffffffu, ii, o);
                const int os = __shfl_xor_sync(0xffffffffu, src, o);
                if (ov > v || (ov == v && oi < ii)) { v = ov; ii = oi; src = os; }
            }
            const int p = __shfl_sync(0xffffffffu, ii, 0);
            const int ws = __shfl_sync(0xffffffffu, src, 0);
            double rp = cand_a[buf][ws];
            if (v == 0.0) singular = true;        // every candidate zero
            if (w == (p % NW)) used |= 1u << (p / NW);
            if (threadIdx.x == 0) pivrow[k] = p;
            // (c) rank-1 update with the winner's row, scaled; row p becomes the
            // scaled pivot row, column k becomes -a(i,k)/piv
            double rv[CL];
            #pragma unroll
            for (int cl = 0; cl < CL; ++cl) {
                const int j = lane + 32 * cl;
                const double x = (cl == ck && lane == lk) ? 1.0 : candrow[buf][ws][j];
                rv[cl] = x * rp;
            }
            #pragma unroll
            for (int ri = 0; ri < RW; ++ri) {
                const int i = w + NW * ri;
                if (i == p) {
                    #pragma unroll
                    for (int cl = 0; cl < CL; ++cl) a[ri][cl] = rv[cl];
                } else {
                    const double f = (i < b) ? colbuf[buf][i] : 0.0;
                    #pragma unroll
                    for (int cl = 0; cl < CL; ++cl) a[ri][cl] = fma(-f, rv[cl], a[ri][cl]);
                    if (lane == lk) a[ri][ck] = -f * rp;
                }
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < b; k += blockDim.x) qinv[pivrow[k]] = k;
    __syncthreads();
    #pragma unroll
    for (int ri = 0; ri < RW; ++ri)
        #pragma unroll
        for (int cl = 0; cl < CL; ++cl) {
            const int i = w + NW * ri, j = lane + 32 * cl;
            if (i < b && j < b) D[qinv[i] + (int64_t)pivrow[j] * b] = a[ri][cl];
        }
    if (singular && threadIdx.x == 0) atomicMin(status, prow_elem[prow]);
}

// Same algorithm for blocks too large for the register tiles (b > 160):
// one CTA, matrix kept in global memory (L2 resident), explicit row swaps.
static __global__ void k_block_inverse_global(double* __restrict__ LD, const int64_t* __restrict__ dinv_off,
                                       const int32_t* __restrict__ prow_b, const int32_t* __restrict__ prow_elem,
                                       const int32_t* __restrict__ rows, int row_begin, int* __restrict__ status,
                                       int* __restrict__ piv_scratch) {
    __shared__ double sv[32];
    __shared__ int si[32];
    __shared__ int s_p;
    __shared__ double colk[1024];
    const int prow = rows[row_begin + blockIdx.x];
    const int b = prow_b[prow];
    double* D = LD + dinv_off[prow];
    int* piv = piv_scratch + (int64_t)blockIdx.x * 1024;
    bool singular = false;
    for (int k = 0; k < b; ++k) {
        double best = -1.0; int bi = 0x7fffffff;
        for (int i = k + threadIdx.x; i < b; i += blockDim.x) {
            double v = fabs(D[i + (int64_t)k * b]);
            if (!(v == v)) v = INFINITY;
            if (v > best || (v == best && i < bi)) { best = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if ((threadIdx.x & 31) == 0) { sv[threadIdx.x >> 5] = best; si[threadIdx.x >> 5] = bi; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double bb = -1.0; int ii = 0x7fffffff;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
                if (sv[q] > bb || (sv[q] == bb && si[q] < ii)) { bb = sv[q]; ii = si[q]; }
            s_p = ii;
            piv[k] = ii;
        }
        __syncthreads();
        const int p = s_p;
        if (p != k)
            for (int j = threadIdx.x; j < b; j += blockDim.x) {
                const double t = D[k + (int64_t)j * b];
                D[k + (int64_t)j * b] = D[p + (int64_t)j * b];
                D[p + (int64_t)j * b] = t;
            }
        __syncthreads();
        double pv = D[k + (int64_t)k * b];
        if (pv == 0.0) { singular = true; pv = 1.0; }
        const double rp = 1.0 / pv;
        __syncthreads();
        for (int i = threadIdx.x; i < b; i += blockDim.x) colk[i] = (i == k) ? 0.0 : D[i + (int64_t)k * b];
        __syncthreads();
        for (int j = threadIdx.x; j < b; j += blockDim.x) {
            const double v = (j == k) ? 1.0 : D[k + (int64_t)j * b];
            D[k + (int64_t)j * b] = v * rp;
        }
        __syncthreads();
        // row k is final for this step; every other row reads its multiplier
        // from the saved column, so column k can be overwritten in place
        for (int idx = threadIdx.x; idx < b * b; idx += blockDim.x) {
            const int i = idx % b, j = idx / b;
            if (i == k) continue;
            const double base = (j == k) ? 0.0 : D[i + (int64_t)j * b];
            D[i + (int64_t)j * b] = base - colk[i] * D[k + (int64_t)j * b];
        }
        __syncthreads();
    }
    // undo the row interchanges as column interchanges, last first
    for (int k = b - 1; k >= 0; --k) {
        const int p = piv[k];
        if (p != k)
            for (int i = threadIdx.x; i < b; i += blockDim.x) {
                const double t = D[i + (int64_t)k * b];
                D[i + (int64_t)k * b] = D[i + (int64_t)p * b];
                D[i + (int64_t)p * b] = t;
            }
        __syncthreads();
    }
    if (singular && threadIdx.x == 0) atomicMin(status, prow_elem[prow]);
}

// Blocks of 161..1024 rows: the same Gauss-Jordan with row interchanges,
// blocked by panels of NB columns.  A panel is factored in shared memory (its
// pivot searches, row interchanges, scaling and eliminations restricted to
// the panel's columns; the interchanges are applied to the rest of the rows in
// global memory at once).  Afterwards the panel holds G e_k for its pivot
// columns, G the product of the panel's elementary transformations, and every
// other column becomes D[:, j] + (G - I) D[k0:k0+nb, j]: a rank-nb update
// computed from the panel and the pivot rows staged in shared memory, 8 x 4
// outputs per thread.  Column interchanges undo the row interchanges at the
// end, as in k_block_inverse_global.  Dynamic shared memory:
// (2 NB + 1) b doubles.
template <int NB>
__global__ void __launch_bounds__(256) k_block_inverse_panels(double* __restrict__ LD, const int64_t* __restrict__ dinv_off,
                                                          const int32_t* __restrict__ prow_b,
                                                          const int32_t* __restrict__ prow_elem,
                                                          const int32_t* __restrict__ rows, int row_begin,
                                                          int* __restrict__ status, int* __restrict__ piv_scratch) {
    extern __shared__ double ip_smem[];
    __shared__ double sv[8];
    __shared__ int si[8];
    __shared__ int s_p;
    const int prow = rows[row_begin + blockIdx.x];
    const int b = prow_b[prow];
    double* D = LD + dinv_off[prow];
    int* piv = piv_scratch + (int64_t)blockIdx.x * 1024;
    double* Pn = ip_smem;                      // [nb][b]: panel column t at Pn[t * b]
    double* Rw = Pn + (size_t)NB * b;          // [b][NB]: pivot row t at column j in Rw[j * NB + t]
    double* colk = Rw + (size_t)NB * b;        // [b]: multipliers of one step
    const int tid = threadIdx.x, nthr = blockDim.x;
    bool singular = false;
    for (int k0 = 0; k0 < b; k0 += NB) {
        const int nb = min(NB, b - k0);
        for (int idx = tid; idx < nb * b; idx += nthr) {
            const int t = idx / b, i = idx - t * b;
            Pn[idx] = D[i + (int64_t)(k0 + t) * b];
        }
        __syncthreads();
        for (int t = 0; t < nb; ++t) {
            const int k = k0 + t;
            double best = -1.0;
            int bi = 0x7fffffff;
            for (int i = k + tid; i < b; i += nthr) {
                double v = fabs(Pn[t * b + i]);
                if (!(v == v)) v = INFINITY;
                if (v > best || (v == best && i < bi)) { best = v; bi = i; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if ((tid & 31) == 0) { sv[tid >> 5] = best; si[tid >> 5] = bi; }
            __syncthreads();
            if (tid == 0) {
                double bb = -1.0;
                int ii = 0x7fffffff;
                for (int q = 0; q < (nthr >> 5); ++q)
                    if (sv[q] > bb || (sv[q] == bb && si[q] < ii)) { bb = sv[q]; ii = si[q]; }
                s_p = ii;
                piv[k] = ii;
            }
            __syncthreads();
            const int p = s_p;
            if (p != k) {
                for (int tt = tid; tt < nb; tt += nthr) {
                    const double x = Pn[tt * b + k];
                    Pn[tt * b + k] = Pn[tt * b + p];
                    Pn[tt * b + p] = x;
                }
                for (int j = tid; j < b; j += nthr) {
                    if (j >= k0 && j < k0 + nb) continue;
                    const double x = D[k + (int64_t)j * b];
                    D[k + (int64_t)j * b] = D[p + (int64_t)j * b];
                    D[p + (int64_t)j * b] = x;
                }
            }
            __syncthreads();
            double pv = Pn[t * b + k];
            if (pv == 0.0) { singular = true; pv = 1.0; }
            const double rp = 1.0 / pv;
            for (int i = tid; i < b; i += nthr) colk[i] = (i == k) ? 0.0 : Pn[t * b + i];
            __syncthreads();
            for (int tt = tid; tt < nb; tt += nthr) Pn[tt * b + k] = ((tt == t) ? 1.0 : Pn[tt * b + k]) * rp;
            __syncthreads();
            for (int idx = tid; idx < nb * b; idx += nthr) {
                const int tt = idx / b, i = idx - tt * b;
                if (i == k) continue;
                const double base = (tt == t) ? 0.0 : Pn[idx];
                Pn[idx] = base - colk[i] * Pn[tt * b + k];
            }
            __syncthreads();
        }
        // the pivot rows outside the panel, then the panel back to memory
        const int nout = b - nb;
        for (int idx = tid; idx < nb * nout; idx += nthr) {
            const int t = idx % nb, jj = idx / nb;
            const int j = jj < k0 ? jj : jj + nb;
            Rw[j * NB + t] = D[(k0 + t) + (int64_t)j * b];
        }
        for (int idx = tid; idx < nb * b; idx += nthr) {
            const int t = idx / b, i = idx - t * b;
            D[i + (int64_t)(k0 + t) * b] = Pn[idx];
        }
        __syncthreads();
        // D[:, j] += (G - I)[:, panel] D[panel rows, j] for every j outside the panel
        const int ni = (b + 7) / 8, nj = (nout + 3) / 4;
        for (int w = tid; w < ni * nj; w += nthr) {
            const int i0 = (w % ni) * 8, jj0 = (w / ni) * 4;
            double acc[8][4];
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
            int jcol[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int jj = min(jj0 + c, nout - 1);
                jcol[c] = jj < k0 ? jj : jj + nb;
            }
            for (int t = 0; t < nb; ++t) {
                double pr[8], rw[4];
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const int i = min(i0 + r, b - 1);
                    pr[r] = Pn[t * b + i] - ((i == k0 + t) ? 1.0 : 0.0);
                }
#pragma unroll
                for (int c = 0; c < 4; ++c) rw[c] = Rw[jcol[c] * NB + t];
#pragma unroll
                for (int r = 0; r < 8; ++r)
#pragma unroll
                    for (int c = 0; c < 4; ++c) acc[r][c] += pr[r] * rw[c];
            }
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if (jj0 + c >= nout) continue;
                double* col = D + (int64_t)jcol[c] * b;
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const int i = i0 + r;
                    if (i < b) col[i] = col[i] + acc[r][c];
                }
            }
        }
        __syncthreads();
    }
    // undo the row interchanges as column interchanges, last first
    for (int k = b - 1; k >= 0; --k) {
        const int p = piv[k];
        if (p != k)
            for (int i = tid; i < b; i += nthr) {
                const double t = D[i + (int64_t)k * b];
                D[i + (int64_t)k * b] = D[i + (int64_t)p * b];
                D[i + (int64_t)p * b] = t;
            }
        __syncthreads();
    }
    if (singular && tid == 0) atomicMin(status, prow_elem[prow]);
}

// ---------------------------------------------------------------------------
// ILU programme: triangular sweeps, one CTA per programme row of a level.
//  forward:  z_r = v_r - sum_lower L z_parent                 (precon_ILU0.f90:336-359)
//  backward: z_r = Dinv_r (z_r - sum_upper U z_parent)         (precon_ILU0.f90:363-398)
// Thread layout as in k_matvec.  TL = factor storage, TU = A storage.
// ---------------------------------------------------------------------------
struct IluRows {
    const int32_t* prow_b;
    const int64_t* v_off;      // source of v (vector offset of the element row)
    const int64_t* z_off;      // work offset (extended vector)
    const int64_t* dinv_off;   // in LD
    const int32_t* lo_ptr;     // [nprow+1]
    const int64_t* lo_L;       // L block in LD
    const int32_t* lo_par;     // parent programme row
    const int32_t* lo_nc;
    const int32_t* up_ptr;
    const int64_t* up_U;       // U block in A
    const int32_t* up_par;
    const int32_t* up_nc;
};

template <typename TL, typename TX, typename ACC>
__global__ void __launch_bounds__(1024) k_ilu_forward(IluRows R, const TL* __restrict__ LD, const int32_t* __restrict__ rows, int row_begin,
                              const TX* __restrict__ v, TX* __restrict__ zx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ACC* xs = reinterpret_cast<ACC*>(smem_raw);
    const int pr = rows[row_begin + blockIdx.x];
    const int b = R.prow_b[pr];
    const int q0 = R.lo_ptr[pr], q1 = R.lo_ptr[pr + 1];
    const int tid = threadIdx.x;
    int off = 0;
    for (int q = q0; q < q1; ++q) {
        const int nc = R.lo_nc[q];
        const TX* zp = zx + R.z_off[R.lo_par[q]];
        for (int c = tid; c < nc; c += blockDim.x) xs[off + c] = cvt<ACC>(zp[c]);
        off += nc;
    }
    const int ncols_total = off;
    __syncthreads();
    const int G = stripe_groups(SW_GCAP, b);
    const int r = tid % b, g = tid / b;
    ACC acc = 0;
    if (g < G) {
        off = 0;
        for (int q = q0; q < q1; ++q) {
            const int nc = R.lo_nc[q];
            const TL* Lb = LD + R.lo_L[q] + r;
            const ACC* xb = xs + off;
            acc = stripe_dot(Lb, (int64_t)b, nc, g, G, xb, acc);
            off += nc;
        }
    }
    ACC* red = xs + ncols_total;
    if (g < G) red[g * b + r] = acc;
    __syncthreads();
    if (tid < b) {
        ACC s = 0;
        for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
        const double out = to_d(v[R.v_off[pr] + tid]) - (double)s;
        zx[R.z_off[pr] + tid] = from_d<TX>(out);
    }
}

template <typename TL, typename TU, typename TX, typename ACC>
__global__ void __launch_bounds__(1024) k_ilu_backward(IluRows R, const TL* __restrict__ LD, const TU* __restrict__ Aval,
                               const int32_t* __restrict__ rows, int row_begin, TX* __restrict__ zx) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ACC* xs = reinterpret_cast<ACC*>(smem_raw);
    const int pr = rows[row_begin + blockIdx.x];
    const int b = R.prow_b[pr];
    const int q0 = R.up_ptr[pr], q1 = R.up_ptr[pr + 1];
    const int tid = threadIdx.x;
    int off = 0;
    for (int q = q0; q < q1; ++q) {
        const int nc = R.up_nc[q];
        const TX* zp = zx + R.z_off[R.up_par[q]];
        for (int c = tid; c < nc; c += blockDim.x) xs[off + c] = cvt<ACC>(zp[c]);
        off += nc;
    }
    const int ncols_total = off;
    ACC* tvec = xs + ncols_total;          // b entries
    ACC* red = tvec + b;                   // G*b entries
    __syncthreads();
    const int G = stripe_groups(SW_GCAP, b);
    const int r = tid % b, g = tid / b;
    ACC acc = 0;
    if (g < G) {
        off = 0;
        for (int q = q0; q < q1; ++q) {
            const int nc = R.up_nc[q];
            const TU* Ub = Aval + R.up_U[q] + r;
            const ACC* xb = xs + off;
            acc = stripe_dot(Ub, (int64_t)b, nc, g, G, xb, acc);
            off += nc;
        }
        red[g * b + r] = acc;
    }
    __syncthreads();
    if (tid < b) {
        ACC s = 0;
        for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
        const double t = to_d(zx[R.z_off[pr] + tid]) - (double)s;
        tvec[tid] = cvt<ACC>(from_d<TX>(t));
    }
    __syncthreads();
    acc = 0;
    if (g < G) {
        const TL* Db = LD + R.dinv_off[pr] + r;
        acc = stripe_dot(Db, (int64_t)b, b, g, G, tvec, acc);
    }
    __syncthreads();
    if (g < G) red[g * b + r] = acc;
    __syncthreads();
    if (tid < b) {
        ACC s = 0;
        for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
        zx[R.z_off[pr] + tid] = from_d<TX>((double)s);
    }
}

// ---------------------------------------------------------------------------
// Segmented BLAS-1 for batches of independent systems packed one after the
// other in one vector.  The vector is cut into chunks that never straddle two
// systems; chunk c covers [cstart[c], cstart[c+1]) and belongs to csys[c].
// All sums run in a fixed order (chunk order, then a fixed tree), so results
// do not depend on the grid.
// ---------------------------------------------------------------------------
// partial[q * nchunk + c] = sum over chunk c of x * y_q
template <typename T>
__global__ void k_seg_mdot(const int64_t* __restrict__ cstart, int nchunk, const T* __restrict__ x,
                           const T* __restrict__ y, int64_t ystride, int nq, double* __restrict__ partial,
                           const int32_t* __restrict__ csys = nullptr, const int32_t* __restrict__ mask = nullptr) {
    // eight vectors per pass over the chunk of x, each sum formed in the
    // order of a pass per vector (as k_mdot_partial)
    constexpr int QG = 8;
    __shared__ double scratch[QG][32];
    const int c = blockIdx.x;
    if (mask != nullptr && !mask[csys[c]]) return;     // system not in this pass: its partials are not read
    const int64_t i0 = cstart[c], i1 = cstart[c + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int q0 = 0; q0 < nq; q0 += QG) {
        const int qn = min(QG, nq - q0);
        const T* yq = y + (int64_t)q0 * ystride;
        double s[QG];
        #pragma unroll
        for (int k = 0; k < QG; ++k) s[k] = 0.0;
        for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const double xi = to_d(x[i]);
            #pragma unroll
            for (int k = 0; k < QG; ++k)
                if (k < qn) s[k] += xi * to_d(yq[(int64_t)k * ystride + i]);
        }
        #pragma unroll
        for (int k = 0; k < QG; ++k) s[k] = warp_sum(s[k]);
        __syncthreads();
        if (lane == 0) {
            #pragma unroll
            for (int k = 0; k < QG; ++k) scratch[k][w] = s[k];
        }
        __syncthreads();
        if (w == 0) {
            const int nw = (blockDim.x + 31) >> 5;
            #pragma unroll
            for (int k = 0; k < QG; ++k) {
                double t = (lane < nw) ? scratch[k][lane] : 0.0;
                t = warp_sum(t);
                if (lane == 0 && k < qn) partial[(int64_t)(q0 + k) * nchunk + c] = t;
            }
        }
    }
}
// out[s * ostride + q] = sum over the chunks [sys_chunk[s], sys_chunk[s+1]) of partial[q * nchunk + c]
static __global__ void k_seg_reduce(const double* __restrict__ partial, int nchunk, const int32_t* __restrict__ sys_chunk,
                                    int nq, double* __restrict__ out, int ostride, const int32_t* __restrict__ mask = nullptr) {
    const int s = blockIdx.x;
    if (mask != nullptr && !mask[s]) return;
    const int c0 = sys_chunk[s], c1 = sys_chunk[s + 1];
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        double acc = 0.0;
        for (int c = c0; c < c1; ++c) acc += partial[(int64_t)q * nchunk + c];
        out[(int64_t)s * ostride + q] = acc;
    }
}
// w -= sum_q coef[sys * cstride + q] * v_q over each chunk; per-chunk sum of squares of w
template <typename T>
__global__ void k_seg_maxpy(const int64_t* __restrict__ cstart, const int32_t* __restrict__ csys, T* __restrict__ w,
                            const T* __restrict__ v, int64_t vstride, int nq, const double* __restrict__ coef,
                            int cstride, double* __restrict__ sumsq, const int32_t* __restrict__ mask = nullptr) {
    __shared__ double scratch[32];
    __shared__ double cs[256];
    const int c = blockIdx.x;
    if (mask != nullptr && !mask[csys[c]]) return;
    const int64_t i0 = cstart[c], i1 = cstart[c + 1];
    const double* cf = coef + (int64_t)csys[c] * cstride;
    double sq = 0.0;
    for (int q0 = 0; q0 < nq || q0 == 0; q0 += 256) {
        const int qn = min(256, nq - q0);
        __syncthreads();
        for (int q = threadIdx.x; q < qn; q += blockDim.x) cs[q] = cf[q0 + q];
        __syncthreads();
        const bool last = (q0 + 256 >= nq);
        for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            double acc = to_d(w[i]);
            for (int q = 0; q < qn; ++q) acc = acc - cs[q] * to_d(v[(int64_t)(q0 + q) * vstride + i]);
            const T o = from_d<T>(acc);
            w[i] = o;
            if (last) { const double od = to_d(o); sq += od * od; }
        }
        if (nq <= 0) break;
    }
    if (sumsq != nullptr) {
        sq = block_sum(sq, scratch);
        if (threadIdx.x == 0) sumsq[c] = sq;
    }
}
// x = x0 + sum_q coef[sys * cstride + q] * z_q   (x0 may be null)
template <typename T>
__global__ void k_seg_lincomb(const int64_t* __restrict__ cstart, const int32_t* __restrict__ csys, T* __restrict__ x,
                              const T* __restrict__ x0, const T* __restrict__ z, int64_t zstride, int nq,
                              const double* __restrict__ coef, int cstride, const int32_t* __restrict__ mask = nullptr) {
    const int c = blockIdx.x;
    if (mask != nullptr && !mask[csys[c]]) return;
    const int64_t i0 = cstart[c], i1 = cstart[c + 1];
    const double* cf = coef + (int64_t)csys[c] * cstride;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        double acc = x0 ? to_d(x0[i]) : 0.0;
        for (int q = 0; q < nq; ++q) acc = acc + cf[q] * to_d(z[(int64_t)q * zstride + i]);
        x[i] = from_d<T>(acc);
    }
}
// y = scale[sys] * x per chunk (in place allowed).  A scale of 0 (a system
// that is inactive) writes zeros whatever x holds: the rows of a frozen
// system are skipped by the streamed kernels, so its x may be stale, and its
// next basis vector must stay 0 (a zero right-hand side for an inner solve).
template <typename T>
__global__ void k_seg_scale(const int64_t* __restrict__ cstart, const int32_t* __restrict__ csys, const T* x, T* y,
                            const double* __restrict__ scale) {
    const int c = blockIdx.x;
    const int64_t i0 = cstart[c], i1 = cstart[c + 1];
    const double a = scale[csys[c]];
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) y[i] = from_d<T>(a == 0.0 ? 0.0 : a * to_d(x[i]));
}

// ---------------------------------------------------------------------------
// ILU programme: dependency-driven sweeps (one launch per sweep).
// CTAs take programme rows from an atomic ticket counter in a topological
// order (level-major).  A row waits, through per-row flags stamped with the
// sweep's epoch, only for its own parents, so no grid-wide barrier separates
// the levels.  Deadlock-free at any occupancy: a ticket holder only waits on
// rows with smaller tickets, whose holders are already running.  Every wait
// is bounded (about a second of clock cycles); when it runs out, status
// records ETIMEOUT and the sweep carries on with whatever it has, so the
// kernel always terminates.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
// wait (thread 0 only) until flags[row] == epoch; false on timeout
__device__ __forceinline__ bool wait_flag(const unsigned* flags, int row, unsigned epoch, long long limit) {
    if (ld_acquire(flags + row) == epoch) return true;
    const long long t0 = clock64();
    while (ld_acquire(flags + row) != epoch) {
        if (clock64() - t0 > limit) return false;
        __nanosleep(64);
    }
    return true;
}
template <typename T> __device__ __forceinline__ T ld_cg(const T* p) { return __ldcg(p); }

struct SweepSync {
    unsigned* counter;      // ticket counter, zero at launch
    unsigned* flags;        // per programme row
    unsigned epoch;
    int* status;            // set to CHIDG_GPU_ETIMEOUT-like code on a timeout
    long long spin_limit;   // clock cycles
};

template <typename TL, typename TU, typename TX, typename ACC, bool FORWARD>
__global__ void __launch_bounds__(1024) k_ilu_sweep_sf(IluRows R, const TL* __restrict__ LD, const TU* __restrict__ Aval,
                               const int32_t* __restrict__ order, int nrows, const TX* __restrict__ v,
                               TX* __restrict__ zx, SweepSync S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ACC* xs = reinterpret_cast<ACC*>(smem_raw);
    __shared__ int s_row;
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            const unsigned t = atomicAdd(S.counter, 1u);
            s_row = (t < (unsigned)nrows) ? order[t] : -1;
            s_ok = 1;
        }
        __syncthreads();
        const int pr = s_row;
        if (pr < 0) break;
        const int b = R.prow_b[pr];
        const int q0 = FORWARD ? R.lo_ptr[pr] : R.up_ptr[pr];
        const int q1 = FORWARD ? R.lo_ptr[pr + 1] : R.up_ptr[pr + 1];
        const int32_t* par = FORWARD ? R.lo_par : R.up_par;
        const int32_t* ncs = FORWARD ? R.lo_nc : R.up_nc;
        if (tid == 0)
            for (int q = q0; q < q1; ++q)
                if (!wait_flag(S.flags, par[q], S.epoch, S.spin_limit)) { s_ok = 0; atomicExch(S.status, 1); }
        __syncthreads();
        int off = 0;
        for (int q = q0; q < q1; ++q) {
            const int nc = ncs[q];
            const TX* zp = zx + R.z_off[par[q]];
            for (int c = tid; c < nc; c += blockDim.x) xs[off + c] = cvt<ACC>(ld_cg(zp + c));
            off += nc;
        }
        const int ncols_total = off;
        ACC* tvec = xs + ncols_total;
        ACC* red = tvec + b;
        __syncthreads();
        const int G = stripe_groups(SW_GCAP, b);
        const int r = tid % b, g = tid / b;
        ACC acc = 0;
        if (g < G) {
            off = 0;
            for (int q = q0; q < q1; ++q) {
                const int nc = ncs[q];
                const ACC* xb = xs + off;
                int c = g;
                if (FORWARD) {
                    const TL* Bb = LD + R.lo_L[q] + r;
                    acc = stripe_dot(Bb, (int64_t)b, nc, c, G, xb, acc);
                } else {
                    const TU* Bb = Aval + R.up_U[q] + r;
                    acc = stripe_dot(Bb, (int64_t)b, nc, c, G, xb, acc);
                }
                off += nc;
            }
            red[g * b + r] = acc;
        }
        __syncthreads();
        if (FORWARD) {
            if (tid < b) {
                ACC s = 0;
                for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
                zx[R.z_off[pr] + tid] = from_d<TX>(to_d(v[R.v_off[pr] + tid]) - (double)s);
            }
        } else {
            if (tid < b) {
                ACC s = 0;
                for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
                const double t = to_d(zx[R.z_off[pr] + tid]) - (double)s;
                tvec[tid] = cvt<ACC>(from_d<TX>(t));
            }
            __syncthreads();
            acc = 0;
            if (g < G) {
                const TL* Db = LD + R.dinv_off[pr] + r;
                acc = stripe_dot(Db, (int64_t)b, b, g, G, tvec, acc);
            }
            __syncthreads();
            if (g < G) red[g * b + r] = acc;
            __syncthreads();
            if (tid < b) {
                ACC s = 0;
                for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
                zx[R.z_off[pr] + tid] = from_d<TX>((double)s);
            }
        }
        // publish: every writer fences its stores, then one thread stamps the flag
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(S.flags + pr, S.epoch);
    }
}

// ---------------------------------------------------------------------------
// ILU programme: task-split sweeps.  A task is one block product of one row,
// partial = L_rq z_parent (forward) or U_rq z_parent (backward); the last task
// of a row to finish adds the row's partials in entry order, completes the row
// (z_r = v_r - sum, or z_r = inv(D_r) (z_r - sum)) and publishes it.  Rows
// without entries are single combine tasks.  Tasks are handed out in
// topological order of their parent rows, so a task only waits for rows whose
// tasks were all handed out earlier: deadlock-free at any occupancy, and every
// wait is bounded as in k_ilu_sweep_sf.
// ---------------------------------------------------------------------------
struct SweepTasks {
    const int32_t* task_row;    // programme row of each task
    const int32_t* task_ent;    // entry index (into lo_* / up_*) or -1 for a combine-only task
    const int64_t* part_off;    // per entry: offset of its partial in the scratch vector
    unsigned* row_count;        // per row: completed tasks, never reset (wraps by entry count)
};

template <typename TL, typename TU, typename TX, typename ACC, bool FORWARD>
__global__ void __launch_bounds__(1024) k_ilu_tasks(IluRows R, const TL* __restrict__ LD, const TU* __restrict__ Aval,
                                                    SweepTasks T, int ntasks, const TX* __restrict__ v,
                                                    TX* __restrict__ zx, ACC* __restrict__ part, SweepSync S, int gcap) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ACC* xs = reinterpret_cast<ACC*>(smem_raw);
    __shared__ int s_task, s_last;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) {
            const unsigned t = atomicAdd(S.counter, 1u);
            s_task = (t < (unsigned)ntasks) ? (int)t : -1;
        }
        __syncthreads();
        const int task = s_task;
        if (task < 0) break;
        const int pr = T.task_row[task];
        const int q = T.task_ent[task];
        const int b = R.prow_b[pr];
        const int q0 = FORWARD ? R.lo_ptr[pr] : R.up_ptr[pr];
        const int q1 = FORWARD ? R.lo_ptr[pr + 1] : R.up_ptr[pr + 1];
        const int G = stripe_groups(gcap, b);
        const int r = tid % b, g = tid / b;
        ACC* red = xs + 1024;        // after the staged parent segment (<= 1024 values)
        if (q >= 0) {
            const int par = FORWARD ? R.lo_par[q] : R.up_par[q];
            const int nc = FORWARD ? R.lo_nc[q] : R.up_nc[q];
            if (tid == 0 && !wait_flag(S.flags, par, S.epoch, S.spin_limit)) atomicExch(S.status, 1);
            __syncthreads();
            const TX* zp = zx + R.z_off[par];
            for (int c = tid; c < nc; c += blockDim.x) xs[c] = cvt<ACC>(ld_cg(zp + c));
            __syncthreads();
            ACC acc = 0;
            if (g < G) {
                if (FORWARD) acc = stripe_dot(LD + R.lo_L[q] + r, (int64_t)b, nc, g, G, xs, acc);
                else acc = stripe_dot(Aval + R.up_U[q] + r, (int64_t)b, nc, g, G, xs, acc);
                red[g * b + r] = acc;
            }
            __syncthreads();
            if (tid < b) {
                ACC s = 0;
                for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
                part[T.part_off[q] + tid] = s;
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) {
                const unsigned old = atomicAdd(T.row_count + pr, 1u);
                s_last = ((old + 1u) % (unsigned)(q1 - q0)) == 0u;
            }
            __syncthreads();
            if (!s_last) continue;
            __threadfence();
        }
        // combine: sum the row's partials in entry order
        ACC* tvec = xs + 1024 + 1024;
        if (tid < b) {
            ACC s = 0;
            for (int qq = q0; qq < q1; ++qq) s += ld_cg(part + T.part_off[qq] + tid);
            if (FORWARD) zx[R.z_off[pr] + tid] = from_d<TX>(to_d(v[R.v_off[pr] + tid]) - (double)s);
            else tvec[tid] = cvt<ACC>(from_d<TX>(to_d(zx[R.z_off[pr] + tid]) - (double)s));
        }
        if (!FORWARD) {
            __syncthreads();
            ACC acc = 0;
            if (g < G) acc = stripe_dot(LD + R.dinv_off[pr] + r, (int64_t)b, b, g, G, tvec, acc);
            if (g < G) red[g * b + r] = acc;
            __syncthreads();
            if (tid < b) {
                ACC s = 0;
                for (int gg = 0; gg < G; ++gg) s += red[gg * b + tid];
                zx[R.z_off[pr] + tid] = from_d<TX>((double)s);
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(S.flags + pr, S.epoch);
    }
}

}  // namespace chidg
