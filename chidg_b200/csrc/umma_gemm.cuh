// The mixed-precision factorisation's block products on the fifth-generation
// tensor cores: tcgen05.mma kind::tf32 with the accumulators in tensor memory.
//
// C(m x n) = [Cinit] + sgn * sum_q A_q(m x k_q) B_q(k_q x n) for m, n <= 144,
// over the task lists of k_task_gemm_tf32 (the L products
// L = A_lower inv(D_parent) and the S products D = A_diag - sum L U of
// precon_ILU0.f90:111-265).  All operands are column-major blocks in FP32,
// rounded to TF32 (nearest) in shared memory; accumulation is FP32.
//
// Work unit: half of a task's output columns (72; the MMA computes 80, N a
// multiple of 16), so two CTAs share a block and, with 256 tensor-memory
// columns and 88 KB of shared memory each, two CTAs share an SM.  CTAs are
// persistent over units.  Shared memory: three stages of one K chunk of 32,
// both operands in the tensor cores' K-major canonical layout without swizzle
// (core matrices of 8 rows x 16 bytes; A: rows 8r..8r+7 and k 4c..4c+3 at
// r * 1024 + c * 128 bytes; B the same with a K stride of 144 bytes so that
// the copies of consecutive k fall in distinct banks).  Every thread copies
// elements with cp.async (two chunks ahead of the tensor cores, across unit
// boundaries), rounds the ones it copied to TF32 in place, and one thread
// issues the MMAs (M = 128, N = 80, K = 8) and commits them to the stage's
// mbarrier; a stage is refilled once the MMAs of the chunk that used it have
// completed.  Rows 128..143 come from a second M = 128 tile that starts at
// row 16 (its accumulator 128 columns further on).  Read back with tcgen05.ld
// 32x32b: warp w reads the rows of lanes 32 (w & 3).. and part of the columns.
//
// Every mbarrier wait is bounded; a wait that gives up records status 1,
// skips the read-back and still frees the tensor memory after a second
// bounded wait for the MMAs in flight.
#pragma once

#include "kernels.cuh"
#include "stream_sweep.cuh"

namespace chidg {

constexpr int UM_THREADS = 256;
constexpr int UM_MAX = 144;                 // largest m, n
constexpr int UM_KC = 32;                   // K per stage: four MMAs of K = 8
constexpr int UM_STAGES = 3;                // two chunks in flight ahead of the tensor cores
constexpr int UM_RG = UM_MAX / 8;           // 8-row groups
constexpr int UM_NH = 72;                   // output columns a CTA owns: half of the block
constexpr int UM_N = 80;                    // columns it computes (N of the MMA: a multiple of 16)
constexpr uint32_t UM_A_LBO = 128, UM_A_SBO = 1024;
constexpr uint32_t UM_B_LBO = 144, UM_B_SBO = 8 * 144;
constexpr int UM_A_BYTES = UM_RG * UM_A_SBO;
constexpr int UM_B_BYTES = (UM_N / 8) * UM_B_SBO;
constexpr int UM_STAGE_BYTES = UM_A_BYTES + UM_B_BYTES;
constexpr size_t UM_SMEM = (size_t)UM_STAGES * UM_STAGE_BYTES + 64;
constexpr uint32_t UM_TMEM_COLS = 256;      // two CTAs per SM share the 512 columns
constexpr uint32_t UM_TILE1_COL = 128;      // accumulator column of the second M tile
constexpr int UM_TILE1_ROW = 16;            // its first row
// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12
// = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t UM_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(UM_N >> 3) << 17) | ((128u >> 4) << 24);
static_assert(UM_STAGE_BYTES % 16 == 0 && UM_A_BYTES % 16 == 0, "stages start on 16 bytes");
static_assert(UM_SMEM > 76 * 1024 && UM_SMEM <= 112 * 1024, "two CTAs per SM at most: 2 x 256 tensor-memory columns");

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

__device__ __forceinline__ void cp_async_wait_upto(int n) {   // at most n groups still in flight
    switch (n) {
        case 0: cp_async_wait<0>(); break;
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        case 3: cp_async_wait<3>(); break;
        default: cp_async_wait<4>(); break;
    }
}

// A walk over the K chunks of a CTA's units: unit u is columns
// [UM_NH (u & 1), + UM_NH) of task u >> 1; units blockIdx.x, + gridDim.x, ...
// A unit without products or without columns has no chunks.
struct UmmaWalk {
    int unit, q, k0;
    __device__ static bool empty(const GemmTask& t, int half) { return t.q_begin >= t.q_end || UM_NH * half >= t.n; }
    __device__ void start(const GemmTask* tasks, int nunit, const GemmPair* pairs) {
        unit = blockIdx.x;
        q = unit < nunit ? tasks[unit >> 1].q_begin : 0;
        k0 = 0;
        skip_empty(tasks, nunit);
    }
    __device__ void skip_empty(const GemmTask* tasks, int nunit) {
        while (unit < nunit && empty(tasks[unit >> 1], unit & 1)) {
            unit += gridDim.x;
            if (unit < nunit) q = tasks[unit >> 1].q_begin;
        }
    }
    __device__ void next(const GemmTask* tasks, int nunit, const GemmPair* pairs) {
        k0 += UM_KC;
        if (k0 >= pairs[q].k) {
            k0 = 0;
            if (++q >= tasks[unit >> 1].q_end) {
                unit += gridDim.x;
                if (unit < nunit) q = tasks[unit >> 1].q_begin;
                skip_empty(tasks, nunit);
            }
        }
    }
};

template <typename TC>
__device__ __forceinline__ void umma_store(const GemmTask& t, int row, int col, float v, const double* Cinit, TC* Cbase,
                                           double sgn) {
    if (row >= t.m || col >= t.n) return;
    const int64_t o = row + (int64_t)col * t.m;
    double x = sgn * (double)v;
    if (t.cinit_off >= 0) x = Cinit[t.cinit_off + o] + x;
    Cbase[t.c_off + o] = from_d<TC>(x);
}

// Persistent: CTA i takes units i, i + gridDim.x, ... (a unit: half of a
// task's output columns, so two CTAs share a block); its chunks form one
// stream that runs UM_STAGES - 1 chunks ahead of the tensor cores across unit
// boundaries, and a unit's accumulators are read back (and the tensor memory
// freed for the next unit's first MMA) while the next chunks are in flight.
template <typename TC>
__global__ void __launch_bounds__(UM_THREADS, 2)
    k_task_gemm_umma(const GemmTask* __restrict__ tasks, int nunit, const GemmPair* __restrict__ pairs,
                     const float* Abase, const float* Bbase, const double* Cinit, TC* Cbase, double sgn,
                     int* __restrict__ status, long long spin_limit) {
    extern __shared__ __align__(128) unsigned char um_smem[];
    uint64_t* done = reinterpret_cast<uint64_t*>(um_smem + (size_t)UM_STAGES * UM_STAGE_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + UM_STAGES);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int D = UM_STAGES - 1;                  // chunks in flight ahead of the one consumed

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

    // the number of chunks of this CTA's tasks; a task without products
    // (a row with no lower neighbours) is its start value alone
    int total = 0;
    for (int u = blockIdx.x; u < nunit; u += gridDim.x) {
        const GemmTask t = tasks[u >> 1];
        if (t.q_begin >= t.q_end && (u & 1) == 0)
            for (int o = tid; o < t.m * t.n; o += UM_THREADS) umma_store(t, o % t.m, o / t.m, 0.0f, Cinit, Cbase, sgn);
        if (UmmaWalk::empty(t, u & 1)) continue;
        for (int q = t.q_begin; q < t.q_end; ++q) total += (pairs[q].k + UM_KC - 1) / UM_KC;
    }

    UmmaWalk load, use;                               // the copies' walk and the tensor cores' walk
    load.start(tasks, nunit, pairs);
    use.start(tasks, nunit, pairs);
    // copy one chunk into a stage (cp.async, 4 bytes an element, zero-filled
    // outside the operands) and advance the copies' walk
    auto issue = [&](int stage) {
        const GemmTask t = tasks[load.unit >> 1];
        const int n0 = UM_NH * (load.unit & 1);       // the unit's first column
        const GemmPair pr = pairs[load.q];
        const float* A = Abase + pr.a_off;            // m x k, column-major
        const float* B = Bbase + pr.b_off;            // k x n, column-major
        const int kc = min(UM_KC, pr.k - load.k0), lk0 = load.k0;
        unsigned char* as = um_smem + (size_t)stage * UM_STAGE_BYTES;
        unsigned char* bs = as + UM_A_BYTES;
        // A: item (row i, k group g), consecutive threads on consecutive rows
        for (int idx = tid; idx < UM_MAX * (UM_KC / 4); idx += UM_THREADS) {
            const int g = idx / UM_MAX, i = idx - g * UM_MAX;
            unsigned char* d = as + (i >> 3) * UM_A_SBO + g * UM_A_LBO + (i & 7) * 16;
            #pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool ok = i < t.m && 4 * g + j < kc;
                cp_async4(d + 4 * j, ok ? (const void*)(A + i + (int64_t)(lk0 + 4 * g + j) * t.m) : (const void*)A, ok);
            }
        }
        // B as n x k (K-major), the unit's UM_N columns: item (column n0 + n, k
        // group g), consecutive threads on consecutive k
        for (int idx = tid; idx < UM_N * (UM_KC / 4); idx += UM_THREADS) {
            const int n = idx / (UM_KC / 4), g = idx - n * (UM_KC / 4);
            unsigned char* d = bs + (n >> 3) * UM_B_SBO + g * UM_B_LBO + (n & 7) * 16;
            #pragma unroll
            for (int j = 0; j < 4; ++j) {
                const bool ok = n0 + n < t.n && 4 * g + j < kc;
                cp_async4(d + 4 * j, ok ? (const void*)(B + (lk0 + 4 * g + j) + (int64_t)(n0 + n) * pr.k) : (const void*)B,
                          ok);
            }
        }
        cp_async_commit();
        load.next(tasks, nunit, pairs);
    };
    // this thread's elements of a stage, rounded to TF32 in place (its own
    // copies: complete once its cp.async group is)
    auto round_stage = [&](int stage) {
        unsigned char* as = um_smem + (size_t)stage * UM_STAGE_BYTES;
        unsigned char* bs = as + UM_A_BYTES;
        for (int idx = tid; idx < UM_MAX * (UM_KC / 4); idx += UM_THREADS) {
            const int g = idx / UM_MAX, i = idx - g * UM_MAX;
            float4* d = reinterpret_cast<float4*>(as + (i >> 3) * UM_A_SBO + g * UM_A_LBO + (i & 7) * 16);
            const float4 v = *d;
            *d = make_float4(tf32_round(v.x), tf32_round(v.y), tf32_round(v.z), tf32_round(v.w));
        }
        for (int idx = tid; idx < UM_N * (UM_KC / 4); idx += UM_THREADS) {
            const int n = idx / (UM_KC / 4), g = idx - n * (UM_KC / 4);
            float4* d = reinterpret_cast<float4*>(bs + (n >> 3) * UM_B_SBO + g * UM_B_LBO + (n & 7) * 16);
            const float4 v = *d;
            *d = make_float4(tf32_round(v.x), tf32_round(v.y), tf32_round(v.z), tf32_round(v.w));
        }
    };
    __shared__ int failed;
    if (tid == 0) failed = 0;
    __syncthreads();
    for (int g = 0; g < D && g < total; ++g) issue(g);
    int issued = 0;                                   // chunks whose MMAs were committed
    bool first = true;                                // the next chunk consumed starts its task
    for (int c = 0; c < total; ++c) {
        const int s = c % UM_STAGES;
        if (c + D < total) {
            if (c >= 1) {                             // chunk c+D goes where chunk c-1 was: its MMAs must be done
                const int p = c - 1;
                if (tid == 0 && !mbar_wait(done + p % UM_STAGES, (unsigned)((p / UM_STAGES) & 1), spin_limit)) failed = 1;
                __syncthreads();
                if (failed) break;
            }
            issue((c + D) % UM_STAGES);
            cp_async_wait<D>();
        } else {
            cp_async_wait_upto(total - 1 - c);
        }
        round_stage(s);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the stores, visible to the tensor cores
        __syncthreads();
        const GemmTask t = tasks[use.unit >> 1];
        const int n0 = UM_NH * (use.unit & 1);
        const bool two = t.m > 128;
        if (tid == 0) {
            tmem_fence_after();
            const uint32_t a0 = smem_addr(um_smem + (size_t)s * UM_STAGE_BYTES), b0 = a0 + UM_A_BYTES;
            #pragma unroll
            for (int ks = 0; ks < UM_KC / 8; ++ks) {  // a short chunk's missing k are zeros in both operands
                const uint32_t acc = (!first || ks > 0) ? 1u : 0u;
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
        const int unit_now = use.unit;
        use.next(tasks, nunit, pairs);
        first = use.unit != unit_now;
        if (!first) continue;
        // the task's last chunk: wait for its MMAs, read the accumulators back
        if (tid == 0) {
            bool ok = mbar_wait(done + s, (unsigned)((c / UM_STAGES) & 1), spin_limit);
            if (!ok) ok = mbar_wait(done + s, (unsigned)((c / UM_STAGES) & 1), spin_limit);
            if (!ok) failed = 1;
        }
        __syncthreads();
        if (failed) break;
        tmem_fence_after();
        const int quarter = warp & 3, half = warp >> 2;
        const int row = 32 * quarter + lane;
        const uint32_t lane_base = (uint32_t)(32 * quarter) << 16;
        // columns 8s .. 8s+7 of the unit, s < 9 (the unit owns UM_NH = 72): warps 0-3 take s = 0..4, warps 4-7 s = 5..8
        for (int s8 = half * 5; s8 < (half == 0 ? 5 : UM_NH / 8); ++s8) {
            float v[8];
            tmem_ld8(tmem + lane_base + (uint32_t)(8 * s8), v);
            #pragma unroll
            for (int j = 0; j < 8; ++j) umma_store(t, row, n0 + 8 * s8 + j, v[j], Cinit, Cbase, sgn);
        }
        if (two && quarter == 3) {                    // rows 128..143: lanes 112..127 of the second tile
            const int row1 = UM_TILE1_ROW + row;
            for (int s8 = half * 5; s8 < (half == 0 ? 5 : UM_NH / 8); ++s8) {
                float v[8];
                tmem_ld8(tmem + UM_TILE1_COL + lane_base + (uint32_t)(8 * s8), v);
                if (row1 >= 128) {
                    #pragma unroll
                    for (int j = 0; j < 8; ++j) umma_store(t, row1, n0 + 8 * s8 + j, v[j], Cinit, Cbase, sgn);
                }
            }
        }
        tmem_fence_before();
        __syncthreads();                              // the next task's MMAs overwrite the accumulators
    }
    cp_async_wait<0>();                               // nothing of this thread's copies is left in flight
    if (tid == 0 && failed) {
        // let the MMAs already issued finish before the tensor memory is freed
        if (issued > 0) {
            const int last = issued - 1;
            mbar_wait(done + last % UM_STAGES, (unsigned)((last / UM_STAGES) & 1), spin_limit);
        }
        atomicExch(status, 1);
    }
    tmem_fence_before();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(UM_TMEM_COLS) : "memory");
    }
}

}  // namespace chidg
