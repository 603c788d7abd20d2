// The mixed-precision factorisation's block products on the fifth-generation
// tensor cores: tcgen05.mma kind::tf32 with the accumulators in tensor memory.
//
// C(m x n) = [Cinit] + sgn * sum_q A_q(m x k_q) B_q(k_q x n) for m, n <= 144,
// one task per CTA, the task lists of k_task_gemm_tf32 (the L products
// L = A_lower inv(D_parent) and the S products D = A_diag - sum L U of
// precon_ILU0.f90:111-265).  All operands are column-major blocks in FP32,
// rounded to TF32 (nearest) when staged; accumulation is FP32.
//
// Shared memory: three stages of one K chunk of 32 for both operands, each
// in the tensor cores' K-major canonical layout without swizzle (core
// matrices of 8 rows x 16 bytes; A: rows 8r..8r+7 and k 4c..4c+3 at
// r * 1024 + c * 128 bytes; B the same with a K stride of 144 bytes so that
// the staging stores of consecutive k fall in distinct banks).  Every thread
// stages (plain loads, TF32 rounding, 16-byte shared stores), one thread
// issues the MMAs (M = 128, N = 144, K = 8) and commits them to the stage's
// mbarrier, which frees the stage three chunks later.  Rows 128..143 come from
// a second M = 128 tile that starts at row 16 (its accumulator 256 columns
// further on in the 512 allocated).  Read back with tcgen05.ld 32x32b: warp w
// reads the rows of lanes 32 (w & 3).. and half of the columns.
//
// 115 KB of shared memory keep one CTA per SM, so the 512 tensor-memory
// columns it allocates are never contended.  Every mbarrier wait is bounded;
// a wait that gives up records status 1, skips the read-back and still frees
// the tensor memory after a second bounded wait.
#pragma once

#include "kernels.cuh"
#include "stream_sweep.cuh"

namespace chidg {

constexpr int UM_THREADS = 256;
constexpr int UM_MAX = 144;                 // largest m, n
constexpr int UM_KC = 32;                   // K per stage: four MMAs of K = 8
constexpr int UM_STAGES = 3;
constexpr int UM_RG = UM_MAX / 8;           // 8-row groups
constexpr uint32_t UM_A_LBO = 128, UM_A_SBO = 1024;
constexpr uint32_t UM_B_LBO = 144, UM_B_SBO = 8 * 144;
constexpr int UM_A_BYTES = UM_RG * UM_A_SBO;
constexpr int UM_B_BYTES = UM_RG * UM_B_SBO;
constexpr int UM_STAGE_BYTES = UM_A_BYTES + UM_B_BYTES;
constexpr size_t UM_SMEM = (size_t)UM_STAGES * UM_STAGE_BYTES + 64;
constexpr uint32_t UM_TMEM_COLS = 512;
constexpr uint32_t UM_TILE1_COL = 256;      // accumulator column of the second M tile
constexpr int UM_TILE1_ROW = 16;            // its first row
// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12
// = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t UM_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(UM_MAX >> 3) << 17) | ((128u >> 4) << 24);
static_assert(UM_STAGE_BYTES % 16 == 0 && UM_A_BYTES % 16 == 0, "stages start on 16 bytes");
static_assert(UM_SMEM > 114 * 1024, "one CTA per SM: the tensor-memory allocation is not shared");

// shared-memory matrix descriptor, no swizzle: start, leading (K) and stride
// (8-row group) byte offsets in 16-byte units, version 1 at bit 46
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void tmem_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    #pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ float tf32_round(float x) {
    unsigned r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

template <typename TC>
__global__ void __launch_bounds__(UM_THREADS, 1)
    k_task_gemm_umma(const GemmTask* __restrict__ tasks, const GemmPair* __restrict__ pairs, const float* Abase,
                     const float* Bbase, const double* Cinit, TC* Cbase, double sgn, int* __restrict__ status,
                     long long spin_limit) {
    extern __shared__ __align__(128) unsigned char um_smem[];
    uint64_t* done = reinterpret_cast<uint64_t*>(um_smem + (size_t)UM_STAGES * UM_STAGE_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + UM_STAGES);
    const GemmTask t = tasks[blockIdx.x];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(UM_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < UM_STAGES; ++s) mbar_init(done + s, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tmem_fence_before();
    __syncthreads();
    tmem_fence_after();
    const uint32_t tmem = *tmem_slot;
    const bool two = t.m > 128;

    int nchunk = 0;
    for (int q = t.q_begin; q < t.q_end; ++q) nchunk += (pairs[q].k + UM_KC - 1) / UM_KC;
    int lq = t.q_begin, lk0 = 0, issued = 0;
    __shared__ int failed;
    if (tid == 0) failed = 0;
    __syncthreads();
    for (int c = 0; c < nchunk; ++c) {
        const int s = c % UM_STAGES;
        if (c >= UM_STAGES) {                         // the MMAs of chunk c - 3 read this stage
            if (tid == 0 && !mbar_wait(done + s, (unsigned)(((c - UM_STAGES) / UM_STAGES) & 1), spin_limit)) failed = 1;
            __syncthreads();
            if (failed) break;
        }
        const GemmPair pr = pairs[lq];
        const float* A = Abase + pr.a_off;            // m x k, column-major
        const float* B = Bbase + pr.b_off;            // k x n, column-major
        const int kc = min(UM_KC, pr.k - lk0);
        unsigned char* as = um_smem + (size_t)s * UM_STAGE_BYTES;
        unsigned char* bs = as + UM_A_BYTES;
        // A: item (row i, k group g), consecutive threads on consecutive rows
        for (int idx = tid; idx < UM_MAX * (UM_KC / 4); idx += UM_THREADS) {
            const int g = idx / UM_MAX, i = idx - g * UM_MAX;
            float v[4] = {0.f, 0.f, 0.f, 0.f};
            if (i < t.m) {
                #pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (4 * g + j < kc) v[j] = tf32_round(A[i + (int64_t)(lk0 + 4 * g + j) * t.m]);
            }
            *reinterpret_cast<float4*>(as + (i >> 3) * UM_A_SBO + g * UM_A_LBO + (i & 7) * 16) = make_float4(v[0], v[1], v[2], v[3]);
        }
        // B as n x k (K-major): item (column n, k group g), consecutive threads on consecutive k
        for (int idx = tid; idx < UM_MAX * (UM_KC / 4); idx += UM_THREADS) {
            const int n = idx / (UM_KC / 4), g = idx - n * (UM_KC / 4);
            float v[4] = {0.f, 0.f, 0.f, 0.f};
            if (n < t.n) {
                #pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (4 * g + j < kc) v[j] = tf32_round(B[(lk0 + 4 * g + j) + (int64_t)n * pr.k]);
            }
            *reinterpret_cast<float4*>(bs + (n >> 3) * UM_B_SBO + g * UM_B_LBO + (n & 7) * 16) = make_float4(v[0], v[1], v[2], v[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the stores, visible to the tensor cores
        __syncthreads();
        if (tid == 0) {
            tmem_fence_after();
            const uint32_t a0 = smem_addr(as), b0 = smem_addr(bs);
            #pragma unroll
            for (int ks = 0; ks < UM_KC / 8; ++ks) {  // a short chunk's missing k are zeros in both operands
                const uint32_t acc = (c > 0 || ks > 0) ? 1u : 0u;
                const uint64_t bd = umma_desc(b0 + ks * 2 * UM_B_LBO, UM_B_LBO, UM_B_SBO);
                umma_tf32(tmem, umma_desc(a0 + ks * 2 * UM_A_LBO, UM_A_LBO, UM_A_SBO), bd, UM_IDESC, acc);
                if (two)
                    umma_tf32(tmem + UM_TILE1_COL,
                              umma_desc(a0 + (UM_TILE1_ROW / 8) * UM_A_SBO + ks * 2 * UM_A_LBO, UM_A_LBO, UM_A_SBO), bd,
                              UM_IDESC, acc);
            }
            umma_commit(done + s);                    // arrives when these MMAs (and all before) are done
        }
        ++issued;
        lk0 += UM_KC;
        if (lk0 >= pr.k) { ++lq; lk0 = 0; }
    }
    // the last commit covers every MMA issued before it
    __shared__ int drained;
    if (tid == 0) {
        drained = 1;
        if (issued > 0) {
            const int last = issued - 1;
            bool ok = mbar_wait(done + last % UM_STAGES, (unsigned)((last / UM_STAGES) & 1), spin_limit);
            if (!ok) ok = mbar_wait(done + last % UM_STAGES, (unsigned)((last / UM_STAGES) & 1), spin_limit);
            if (!ok) drained = 0;
        }
        if (failed || !drained) atomicExch(status, 1);
    }
    __syncthreads();
    tmem_fence_after();
    if (!failed && drained) {
        const int quarter = warp & 3, half = warp >> 2;
        const int row = 32 * quarter + lane;
        const uint32_t lane_base = (uint32_t)(32 * quarter) << 16;
        for (int j0 = half * (UM_MAX / 2); j0 < (half + 1) * (UM_MAX / 2); j0 += 8) {
            float v[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (nchunk > 0) tmem_ld8(tmem + lane_base + (uint32_t)j0, v);
            #pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int col = j0 + j;
                if (row >= t.m || col >= t.n) continue;
                const int64_t o = row + (int64_t)col * t.m;
                double x = sgn * (double)v[j];
                if (t.cinit_off >= 0) x = Cinit[t.cinit_off + o] + x;
                Cbase[t.c_off + o] = from_d<TC>(x);
            }
        }
        if (two && quarter == 3) {                    // rows 128..143: lanes 112..127 of the second tile
            const int row1 = UM_TILE1_ROW + row;
            for (int j0 = half * (UM_MAX / 2); j0 < (half + 1) * (UM_MAX / 2); j0 += 8) {
                float v[8];
                tmem_ld8(tmem + UM_TILE1_COL + lane_base + (uint32_t)j0, v);
                #pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int col = j0 + j;
                    if (row1 < 128 || row1 >= t.m || col >= t.n) continue;
                    const int64_t o = row1 + (int64_t)col * t.m;
                    double x = sgn * (double)v[j];
                    if (t.cinit_off >= 0) x = Cinit[t.cinit_off + o] + x;
                    Cbase[t.c_off + o] = from_d<TC>(x);
                }
            }
        }
    }
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UM_TMEM_COLS) : "memory");
    }
}

}  // namespace chidg
