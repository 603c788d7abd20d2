// noalloc.cu -- a dot product that allocates no device memory.
//
// Some callers cannot call cudaMalloc when they need a reduction: host
// frameworks that own all device memory through their own pool and forbid
// allocations behind their back, and latency-bound loops that cannot afford
// the device-wide synchronisation cudaMalloc may bring.
// chidg_gpu_dot_noalloc serves them: the caller passes device pointers for
// the inputs and the output, and the per-chunk partial sums go to a
// fixed-size array in this library's own device memory.
//
// Scratch: one FP64 partial per 4096-element chunk, at most 16384 chunks
// (128 KiB on every GPU that loads this library, held until the process
// exits), so n is limited to 67 108 864 elements.  All calls share that
// array and it keeps the last call's contents: calls that overlap on the GPU
// (two streams, or two host threads) race on it and must be serialised by
// the caller.  Each call writes every partial it reads before reading it, so
// nothing needs clearing between calls.  The first call on a device looks up
// the array's device address (cudaGetSymbolAddress with that device
// current, a synchronous query).
#include "chidg_gpu_internal.cuh"

#include <mutex>

namespace {

constexpr int64_t kChunk = 4096;
constexpr int kMaxChunks = 16384;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_dot_partials[kMaxChunks];

// one CTA per chunk; fixed chunk boundaries make the sum order independent of
// the grid, so repeated calls give identical results
__global__ void k_dot_chunk(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                            double* __restrict__ partials) {
    __shared__ double scratch[32];
    const int64_t i0 = (int64_t)blockIdx.x * kChunk;
    const int64_t i1 = (i0 + kChunk < n) ? i0 + kChunk : n;
    double s = 0.0;
    for (int64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) s += x[i] * y[i];
    s = chidg::block_sum(s, scratch);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

__global__ void k_dot_finish(const double* __restrict__ partials, int nchunks, double* __restrict__ out) {
    __shared__ double scratch[32];
    double s = 0.0;
    for (int c = threadIdx.x; c < nchunks; c += blockDim.x) s += partials[c];
    s = chidg::block_sum(s, scratch);
    if (threadIdx.x == 0) *out = s;
}

std::mutex g_setup_mutex;
double* g_partials_addr[kMaxDevices] = {};

// Device address of g_dot_partials on `device`, looked up once per device with
// that device current.  The host-side symbol is only a stand-in; a kernel
// must be given this address.
int partials_address(int device, double** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_dot_partials);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return CHIDG_GPU_ECUDA;
        }
        g_partials_addr[device] = (double*)p;
    }
    *out = g_partials_addr[device];
    return CHIDG_GPU_OK;
}

}  // namespace

extern "C" int chidg_gpu_dot_noalloc(int device, const double* x, const double* y, int64_t n, double* result,
                                     void* stream) {
    if (device < 0 || device >= kMaxDevices || n < 0 || !result || (n > 0 && (!x || !y))) return CHIDG_GPU_EINVAL;
    if (n > kChunk * kMaxChunks) return CHIDG_GPU_EINVAL;   // beyond the static scratch
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) { cudaGetLastError(); return CHIDG_GPU_ECUDA; }
    if (prev != device && cudaSetDevice(device) != cudaSuccess) { cudaGetLastError(); return CHIDG_GPU_EINVAL; }
    double* partials = nullptr;
    int st = partials_address(device, &partials);
    if (st == CHIDG_GPU_OK) {
        const cudaStream_t s = (cudaStream_t)stream;
        const int nchunks = (int)((n + kChunk - 1) / kChunk);
        if (nchunks > 0) k_dot_chunk<<<nchunks, 256, 0, s>>>(x, y, n, partials);
        k_dot_finish<<<1, 1024, 0, s>>>(partials, nchunks, result);
        if (cudaGetLastError() != cudaSuccess) st = CHIDG_GPU_ECUDA;
    }
    if (prev != device) cudaSetDevice(prev);
    return st;
}
