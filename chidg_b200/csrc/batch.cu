// batch.cu -- many independent FGMRES solves sharing every GPU launch.
//
// The systems are packed block-diagonally into one chidg_gpu_matrix: system s
// owns elements [sys_elem[s], sys_elem[s+1]) and no block couples two systems.
// One matvec, one preconditioner sweep and one segmented reduction per Arnoldi
// step serve all systems at once, while every system keeps its own Arnoldi
// process exactly as fgmres_t%solve runs it (type_fgmres.f90:81-310): its own
// dot products, selective re-orthogonalisation, Givens rotations, convergence
// test and solution update.  Systems advance in lockstep through the Krylov
// index j; a converged system is frozen while the others continue, and all
// systems restart together at j = nkrylov.
//
// The Arnoldi bookkeeping runs on the device in FP64, one thread per system
// (k_bat_*): the re-orthogonalisation test (:203-223), the Givens rotations
// with hypot (:234-270), the convergence tests (:272-280) and the least
// squares y = inv(H) p (:287-288, mod_inv::inv semantics).  The second
// Gram-Schmidt pass is always launched and skips the systems that do not need
// it, so one Arnoldi step is a fixed sequence of launches with no host
// synchronisation; the host only reads the count of active systems, without
// waiting for it, to stop early, and synchronises once per restart cycle.
//
// A batch solved again with the same structure (the Newton steps of the same
// set of systems: new values, same pattern and buffers) replays each Arnoldi
// step and the cycle boundaries from CUDA graphs captured on the second call.
#include "chidg_gpu_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>

using namespace chidg;

namespace {

constexpr int64_t kChunk = 2048;
constexpr int kSysThreads = 64;

template <typename T>
int upload_vec(chidg_gpu_ctx* ctx, Buffer& b, const std::vector<T>& v) {
    int st = ensure(ctx, b, std::max<size_t>(sizeof(T) * v.size(), sizeof(T)));
    if (st) return st;
    if (!v.empty()) {
        const cudaError_t e = cudaMemcpyAsync(b.ptr, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batch set-up");
    }
    return CHIDG_GPU_OK;
}

// Per-system Arnoldi state in device memory (one array per field).
struct BatState {
    int32_t *active, *member, *reo, *fin, *niter, *nrestart, *nvecs, *nhist, *err;   // nsys each
    int32_t* inner;           // nsys: iterations of the inner solves (mixed precision)
    int32_t* count;           // [0] active systems, [1] error flag (1 + system of the first error)
    double *r0init, *res, *res_est, *nb, *wn, *wn2, *scale;                         // nsys each
    double *p, *c, *sn;       // nsys x (m + 1)
    double* H;                // nsys x (m + 1) x m, column-major per system
    double* work;             // nsys x m x m (least-squares inverse)
    int32_t* piv;             // nsys x 2m
    double* hist;             // nsys x hcap
    double* coef;             // nsys x hst: h of pass 1, then the solution coefficients y
    double* coef2;            // nsys x hst: h of pass 2
};

struct BatOpts {
    int m, hst, hcap, nmax;
    double tol, rtol;
};

// ---- device epilogue, one thread per system ------------------------------------
__global__ void k_bat_cycle_start(BatState S, BatOpts o, int nsys, const double* __restrict__ r0sq) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const int m = o.m;
    double* p = S.p + (size_t)s * (m + 1);      // p, c, sn and H were cleared by the caller
    S.scale[s] = 0.0;
    S.fin[s] = 0;
    S.member[s] = 0;
    if (!S.active[s]) return;
    const double r0n = sqrt(r0sq[s]);
    if (!isfinite(r0n)) {
        S.err[s] = CHIDG_GPU_ENONFINITE;
        atomicCAS(S.count + 1, 0, s + 1);
        S.active[s] = 0;
        return;
    }
    if (S.niter[s] == 0) S.r0init[s] = r0n;
    if (r0n == 0.0) {             // zero right-hand side: x = 0
        S.active[s] = 0;
        S.res_est[s] = 0.0;
        return;
    }
    p[0] = r0n;
    S.scale[s] = 1.0 / r0n;
    S.nvecs[s] = 0;
    S.member[s] = 1;
}

// selective re-orthogonalisation test (type_fgmres.f90:203-223): pass 1's h and
// ||A z|| decide whether the system takes a second Gram-Schmidt pass
__global__ void k_bat_reorth_test(BatState S, BatOpts o, int nsys, int j) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    S.reo[s] = 0;
    if (!S.active[s]) return;
    const double nb = sqrt(S.nb[s]);
    if (!isfinite(nb)) {
        S.err[s] = CHIDG_GPU_ENONFINITE;
        atomicCAS(S.count + 1, 0, s + 1);
        S.active[s] = 0;
        return;
    }
    const double* h1 = S.coef + (size_t)s * o.hst;
    double crit = 0.0;
    for (int i = 0; i < j; ++i) crit += fabs(h1[i]);
    crit /= nb;
    S.reo[s] = crit >= 1.0;
}

// y = inv(H(1:n,1:n)) p(1:n) into coef (type_fgmres.f90:287-288) for every
// system with fin set, n = nvecs: one warp per system.  Gauss-Jordan with
// partial pivoting on a copy of H (mod_inv::inv semantics, as the host
// solver's explicit inverse): row p is the pivot row of column k, the first
// unused row of largest magnitude; rows are never swapped and the permutation
// is undone when y is formed.  The lanes split the rows (or the columns) of
// each update; every entry is computed as the one-thread loop computes it.
__global__ void k_bat_lsq(BatState S, BatOpts o, int nsys) {
    const int s = blockIdx.x;
    if (s >= nsys || !S.fin[s]) return;
    const int lane = threadIdx.x;
    const int m = o.m, n = S.nvecs[s];
    const double* H = S.H + (size_t)s * (m + 1) * m;
    double* a = S.work + (size_t)s * m * m;
    int32_t* piv = S.piv + (size_t)s * 2 * m;
    int32_t* used = piv + m;
    for (int idx = lane; idx < n * n; idx += 32) {
        const int ii = idx % n, jj = idx / n;
        a[ii + jj * n] = H[ii + jj * (m + 1)];
    }
    for (int i = lane; i < n; i += 32) used[i] = 0;
    __syncwarp();
    for (int k = 0; k < n; ++k) {
        // pivot: largest |a(i,k)| over unused rows, NaN as infinity, first on ties
        double best = -1.0;
        int p = n;
        for (int i = lane; i < n; i += 32) {
            if (used[i]) continue;
            double v = fabs(a[i + k * n]);
            if (!(v == v)) v = INFINITY;
            if (v > best) { best = v; p = i; }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, off);
            const int op = __shfl_xor_sync(0xffffffffu, p, off);
            if (ob > best || (ob == best && op < p)) { best = ob; p = op; }
        }
        const double pv = a[p + k * n];
        __syncwarp();
        if (pv == 0.0) {
            if (lane == 0) {
                S.err[s] = CHIDG_GPU_ESINGULAR;
                atomicCAS(S.count + 1, 0, s + 1);
            }
            return;
        }
        const double rp = 1.0 / pv;
        // columns jj != k of the rows i != p, with the old column k and row p
        for (int i = lane; i < n; i += 32) {
            if (i == p) continue;
            const double aik = a[i + k * n];
            for (int jj = 0; jj < n; ++jj) {
                if (jj == k) continue;
                const double row = a[p + jj * n] * rp;
                a[i + jj * n] = a[i + jj * n] - aik * row;
            }
        }
        __syncwarp();
        for (int i = lane; i < n; i += 32)
            if (i != p) a[i + k * n] = 0.0 - a[i + k * n] * rp;
        __syncwarp();
        for (int jj = lane; jj < n; jj += 32) a[p + jj * n] = ((jj == k) ? 1.0 : a[p + jj * n]) * rp;
        if (lane == 0) { piv[k] = p; used[p] = 1; }
        __syncwarp();
    }
    // inverse(q[i], piv[jj]) = a(i, jj) with q = piv^-1: inverse row ii is a's
    // row piv[ii], inverse column col is a's column q[col]; y = inverse p,
    // summed over the columns in order
    int32_t* q = used;
    for (int k = lane; k < n; k += 32) q[piv[k]] = k;
    __syncwarp();
    const double* pp = S.p + (size_t)s * (m + 1);
    double* y = S.coef + (size_t)s * o.hst;
    for (int ii = lane; ii < n; ii += 32) {
        const int i = piv[ii];
        double acc = 0.0;
        for (int col = 0; col < n; ++col) acc += a[i + q[col] * n] * pp[col];
        y[ii] = acc;
    }
    for (int ii = n + lane; ii < o.hst; ii += 32) y[ii] = 0.0;
}

// h(:, j) from the passes, Givens rotations, the convergence tests and, for a
// system that converges now, its least squares (the step's x update)
__global__ void k_bat_givens(BatState S, BatOpts o, int nsys, int j) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    S.fin[s] = 0;
    if (!S.active[s]) { S.scale[s] = 0.0; return; }
    const int m = o.m;
    double* H = S.H + (size_t)s * (m + 1) * m;
    double* p = S.p + (size_t)s * (m + 1);
    double* c = S.c + (size_t)s * (m + 1);
    double* sn = S.sn + (size_t)s * (m + 1);
    auto h = [&](int i, int jj) -> double& { return H[(size_t)i + (size_t)jj * (m + 1)]; };
    const double* h1 = S.coef + (size_t)s * o.hst;
    const double* h2 = S.coef2 + (size_t)s * o.hst;
    const bool reo = S.reo[s] != 0;
    for (int i = 0; i < j; ++i) {
        double v = 0.0;
        v += h1[i];
        if (reo) v += h2[i];
        h(i, j - 1) = v;
    }
    h(j, j - 1) = sqrt(reo ? S.wn2[s] : S.wn[s]);
    const double inv_h = 1.0 / h(j, j - 1);
    for (int i = 0; i < j - 1; ++i) {
        const double hij = c[i] * h(i, j - 1) + sn[i] * h(i + 1, j - 1);
        const double hipj = -sn[i] * h(i, j - 1) + c[i] * h(i + 1, j - 1);
        h(i, j - 1) = hij;
        h(i + 1, j - 1) = hipj;
    }
    const double gam = hypot(h(j - 1, j - 1), h(j, j - 1));
    c[j - 1] = h(j - 1, j - 1) / gam;
    sn[j - 1] = h(j, j - 1) / gam;
    h(j - 1, j - 1) = gam;
    h(j, j - 1) = 0.0;
    const double pj = c[j - 1] * p[j - 1];
    const double pjp = -sn[j - 1] * p[j - 1];
    p[j - 1] = pj;
    p[j] = pjp;
    const int it = ++S.niter[s];
    S.nvecs[s] = j;
    const double res = fabs(p[j]);
    S.res[s] = res;
    if (it - 1 < o.hcap) S.hist[(size_t)s * o.hcap + it - 1] = res;
    S.nhist[s] = min(it, o.hcap);
    const bool cabs = res < o.tol;
    const bool crel = res / S.r0init[s] < o.rtol;
    const bool cmax = (it >= o.nmax) && (o.nmax > 0);
    S.scale[s] = inv_h;
    if (cabs || crel || cmax) {       // least squares in k_bat_lsq, x update in this step
        S.res_est[s] = res;
        S.active[s] = 0;
        S.fin[s] = 1;
        S.scale[s] = 0.0;
    }
}

// end of a full cycle: least squares of the systems still active (restart)
__global__ void k_bat_cycle_end(BatState S, BatOpts o, int nsys) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    S.fin[s] = 0;
    if (!S.active[s] || !S.member[s]) return;
    S.res_est[s] = S.res[s];
    S.nrestart[s]++;
    S.fin[s] = 1;                     // least squares in k_bat_lsq
}

// a new solve: every system active
__global__ void k_bat_reset(BatState S, int nsys) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nsys) S.active[s] = 1;
}

// inner[s] += iterations of system s's inner solve
__global__ void k_bat_add_inner(int32_t* __restrict__ inner, const int32_t* __restrict__ niter, int nsys) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nsys) inner[s] += niter[s];
}

// count[0] = number of active systems
__global__ void k_bat_count(BatState S, int nsys) {
    __shared__ int tot;
    if (threadIdx.x == 0) tot = 0;
    __syncthreads();
    int a = 0;
    for (int s = threadIdx.x; s < nsys; s += blockDim.x) a += S.active[s];
    atomicAdd(&tot, a);
    __syncthreads();
    if (threadIdx.x == 0) S.count[0] = tot;
}

// a graph of one piece of the batched solve, captured on the context's stream
struct GraphPiece {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    ~GraphPiece() {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
};

}  // namespace

// Captured graphs of a batch structure, kept by the context for the next call
// with the same key (matrix, preconditioner, systems, options and buffers).
struct BatchGraphs {
    std::vector<int64_t> key;
    int seen = 0;                                   // calls with this key so far
    std::unique_ptr<GraphPiece> start, end;         // cycle start (r0, scale), cycle end (restart update)
    std::vector<std::unique_ptr<GraphPiece>> step;  // Arnoldi step j = 1..m
};

void chidg::release_batch_graphs(chidg_gpu_ctx* ctx) {
    delete ctx->batch_graphs;
    ctx->batch_graphs = nullptr;
    delete ctx->batch_graphs_inner;
    ctx->batch_graphs_inner = nullptr;
}

namespace {

// CHIDG_BATCH_GRAPHS=0 keeps every batched solve on eager launches
bool graphs_enabled() {
    static const bool v = [] {
        const char* e = std::getenv("CHIDG_BATCH_GRAPHS");
        return !(e && e[0] == '0');
    }();
    return v;
}

int capture(chidg_gpu_ctx* ctx, GraphPiece& gp, const std::function<int()>& body) {
    cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph capture");
    const int st = body();
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(ctx->stream, &g);
    if (st) { if (g) cudaGraphDestroy(g); return st; }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph capture end");
    gp.g = g;
    e = cudaGraphInstantiate(&gp.x, g, 0);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph instantiate");
    return CHIDG_GPU_OK;
}

}  // namespace


namespace {

// CHIDG_BATCH_SKIP_FROZEN=0: the streamed kernels run the rows of converged
// (frozen) systems too (comparison runs)
bool skip_frozen_enabled() {
    static const bool v = [] {
        const char* e = std::getenv("CHIDG_BATCH_SKIP_FROZEN");
        return !(e && e[0] == '0');
    }();
    return v;
}

// sets the context's frozen-row mask for a scope, restores the previous one
struct MaskScope {
    chidg_gpu_ctx* ctx;
    RowMask saved;
    MaskScope(chidg_gpu_ctx* c, const RowMask& m) : ctx(c), saved(c->row_mask) { c->row_mask = m; }
    ~MaskScope() { ctx->row_mask = saved; }
};

// The chunks of the packed systems, shared by the instances of one call
struct Segs {
    const int64_t* CS = nullptr;
    const int32_t* CY = nullptr;
    const int32_t* SC = nullptr;
    const int32_t* SR = nullptr;
    const int32_t* row_sys = nullptr;      // system of each matrix row
    const int32_t* sys_elem = nullptr;     // host: first element of each system
    int nchunk = 0, nsys = 0;
};

// The restarted FGMRES of every system of the batch with vectors of type T:
// the FP64 solve of the call, and in the mixed modes also the FP32 inner
// solve that is the preconditioner of each of its Arnoldi steps (as the
// single-system solver nests them).  One instance owns its Arnoldi state,
// partial sums, Krylov basis and captured graphs.
template <typename T>
struct BatchEngine {
    chidg_gpu_ctx* ctx = nullptr;
    chidg_gpu_matrix* A = nullptr;           // the operator: A, or A^T
    chidg_gpu_precon* M = nullptr;           // set graph_safe while a sequence is captured
    Segs g;
    BatchBuffers* BB = nullptr;              // state, partials, row sums, pinned counter and events
    Workspace* ws = nullptr;                 // Krylov basis and work vectors
    BatchGraphs** graphs = nullptr;          // captured sequences, kept by the context
    bool capturable = false;                 // an Arnoldi step is a fixed launch sequence
    bool true_residual = true;               // ||b - A x|| per system after the solve (print_report)
    int m = 0;
    BatOpts bo{};
    BatState S{};
    size_t ibytes = 0;
    // z = M v and w = A z, with the row sums of squares of w
    std::function<int(const T*, T*, T*, double*)> step_mv;
    // y = alpha A x + beta z, with the row sums of squares of y
    std::function<int(const T*, T*, const T*, double, double, double*)> matvec;

    int prepare(int m_, double tol, double rtol, int nmax, int hist_cap);
    int run(const T* bb, T* xx, std::vector<int64_t> key);
};

template <typename T>
int BatchEngine<T>::prepare(int m_, double tol, double rtol, int nmax, int hist_cap) {
    const int nsys = g.nsys;
    m = m_;
    const int hst = m + 2;                 // per-system stride of the coefficient rows
    const int hcap = std::max(1, std::min(hist_cap > 0 ? hist_cap : 1, 8192));
    // device state: ints then doubles, in one buffer kept by the context
    const size_t ni = (size_t)nsys * 10 + 2 + (size_t)nsys * 2 * m;
    const size_t nd = (size_t)nsys * 7 + (size_t)nsys * (m + 1) * 3 + (size_t)nsys * (m + 1) * m + (size_t)nsys * m * m +
                      (size_t)nsys * hcap + (size_t)nsys * hst * 2;
    ibytes = ((sizeof(int32_t) * ni + 255) / 256) * 256;
    int st;
    if ((st = ensure(ctx, BB->state, ibytes + sizeof(double) * nd)) ||
        (st = ensure(ctx, BB->partial, sizeof(double) * (size_t)g.nchunk * std::max(m, 1))) ||
        (st = ensure(ctx, BB->rowsq, sizeof(double) * (size_t)A->nrow)) ||
        (st = ensure(ctx, BB->out, sizeof(double) * (size_t)nsys)))
        return st;
    if (!BB->h_count) {
        if (cudaHostAlloc((void**)&BB->h_count, 4 * sizeof(int32_t), cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            BB->h_count = nullptr;
            return fail(ctx, CHIDG_GPU_ENOMEM, "batched fgmres: pinned counter");
        }
        for (int i = 0; i < 2; ++i)
            if (cudaEventCreateWithFlags(&BB->ev[i], cudaEventDisableTiming) != cudaSuccess) {
                cudaGetLastError();
                return fail(ctx, CHIDG_GPU_ECUDA, "batched fgmres: events");
            }
    }
    int32_t* ip = (int32_t*)BB->state.ptr;
    S.active = ip; S.member = ip + nsys; S.reo = ip + 2 * nsys; S.fin = ip + 3 * nsys; S.niter = ip + 4 * nsys;
    S.nrestart = ip + 5 * nsys; S.nvecs = ip + 6 * nsys; S.nhist = ip + 7 * nsys; S.err = ip + 8 * nsys;
    S.inner = ip + 9 * nsys;
    S.count = ip + 10 * nsys;
    S.piv = ip + 10 * nsys + 2;
    double* dp = (double*)((unsigned char*)BB->state.ptr + ibytes);
    S.r0init = dp; S.res = dp + nsys; S.res_est = dp + 2 * nsys; S.nb = dp + 3 * nsys; S.wn = dp + 4 * nsys;
    S.wn2 = dp + 5 * nsys; S.scale = dp + 6 * nsys;
    dp += 7 * (size_t)nsys;
    S.p = dp; dp += (size_t)nsys * (m + 1);
    S.c = dp; dp += (size_t)nsys * (m + 1);
    S.sn = dp; dp += (size_t)nsys * (m + 1);
    S.H = dp; dp += (size_t)nsys * (m + 1) * m;
    S.work = dp; dp += (size_t)nsys * m * m;
    S.hist = dp; dp += (size_t)nsys * hcap;
    S.coef = dp; dp += (size_t)nsys * hst;
    S.coef2 = dp;
    bo = BatOpts{m, hst, hcap, nmax, tol, rtol};
    const int64_t n = A->n;
    if ((st = ensure(ctx, ws->V, sizeof(T) * (size_t)(m + 1) * n)) || (st = ensure(ctx, ws->Z, sizeof(T) * (size_t)(m + 1) * n)) ||
        (st = ensure(ctx, ws->x0, sizeof(T) * (size_t)n)) || (st = ensure(ctx, ws->tmp, sizeof(T) * (size_t)n)))
        return st;
    return CHIDG_GPU_OK;
}

// One batched solve of A x = bb from x = 0 (every system), to the options of
// prepare(); the per-system results stay in S (and, with true_residual,
// ||b - A x||^2 per system in BB->out).
template <typename T>
int BatchEngine<T>::run(const T* bb, T* xx, std::vector<int64_t> key) {
    const int nsys = g.nsys, nchunk = g.nchunk, hst = bo.hst;
    const int64_t n = A->n;
    T* Vb = (T*)ws->V.ptr;
    T* Zb = (T*)ws->Z.ptr;
    T* x0 = (T*)ws->x0.ptr;
    const int64_t* CS = g.CS;
    const int32_t* CY = g.CY;
    const int32_t* SC = g.SC;
    const int32_t* SR = g.SR;
    double* PART = (double*)BB->partial.ptr;
    double* ROWSQ = (double*)BB->rowsq.ptr;
    double* OUT = (double*)BB->out.ptr;
    const int TH = 256;
    const int sgrid = (nsys + kSysThreads - 1) / kSysThreads;
    auto check = [&](const char* what) { return check_launch(ctx, what); };
    // every row runs outside an Arnoldi step's z = M v, w = A z (the residuals
    // of a restart and the true residuals cover every system)
    MaskScope none(ctx, RowMask{});

    // ---- the launch sequences ---------------------------------------------------
    // cycle start: r0 = b - A x0 into V(1), per-system norms, v1 = r0 / ||r0||
    auto seq_start = [&]() -> int {
        int s2;
        if ((s2 = matvec(x0, Vb, bb, -1.0, 1.0, ROWSQ))) return s2;
        k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(ROWSQ, A->nrow, SR, 1, OUT, 1);
        if ((s2 = check("k_seg_reduce r0"))) return s2;
        // p, c, sn and H of every system, one contiguous range of the state
        const cudaError_t ce = cudaMemsetAsync(S.p, 0, sizeof(double) * (size_t)nsys * (m + 1) * (3 + m), ctx->stream);
        if (ce != cudaSuccess) return cuda_fail(ctx, ce, "batched fgmres state");
        k_bat_cycle_start<<<sgrid, kSysThreads, 0, ctx->stream>>>(S, bo, nsys, OUT);
        if ((s2 = check("k_bat_cycle_start"))) return s2;
        k_seg_scale<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, Vb, Vb, S.scale);
        return check("k_seg_scale v1");
    };
    // one Arnoldi step j: z_j = M v_j, w = A z_j, two CGS passes (the second
    // only for the systems the test selects), the epilogue, the solution of the
    // systems that converged now, v(j+1) = w / h(j+1,j), the active count
    auto seq_step = [&](int j) -> int {
        int s2;
        T* vj = Vb + (int64_t)(j - 1) * n;
        T* zj = Zb + (int64_t)(j - 1) * n;
        T* w = Vb + (int64_t)j * n;
        {
            // the rows of systems that have converged are skipped
            MaskScope on(ctx, skip_frozen_enabled() ? RowMask{g.row_sys, S.active, A->nrow} : RowMask{});
            if ((s2 = step_mv(vj, zj, w, ROWSQ))) return s2;
        }
        k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(ROWSQ, A->nrow, SR, 1, S.nb, 1);
        k_seg_mdot<T><<<nchunk, TH, 0, ctx->stream>>>(CS, nchunk, w, Vb, n, j, PART);
        k_seg_reduce<<<nsys, 128, 0, ctx->stream>>>(PART, nchunk, SC, j, S.coef, hst);
        k_seg_maxpy<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, w, Vb, n, j, S.coef, hst, PART);
        k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(PART, nchunk, SC, 1, S.wn, 1);
        k_bat_reorth_test<<<sgrid, kSysThreads, 0, ctx->stream>>>(S, bo, nsys, j);
        k_seg_mdot<T><<<nchunk, TH, 0, ctx->stream>>>(CS, nchunk, w, Vb, n, j, PART, CY, S.reo);
        k_seg_reduce<<<nsys, 128, 0, ctx->stream>>>(PART, nchunk, SC, j, S.coef2, hst, S.reo);
        k_seg_maxpy<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, w, Vb, n, j, S.coef2, hst, PART, S.reo);
        k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(PART, nchunk, SC, 1, S.wn2, 1, S.reo);
        k_bat_givens<<<sgrid, kSysThreads, 0, ctx->stream>>>(S, bo, nsys, j);
        k_bat_lsq<<<nsys, 32, 0, ctx->stream>>>(S, bo, nsys);
        // x = x0 + sum y_i z_i and x0 likewise for the systems that converged now
        k_seg_lincomb<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, xx, x0, Zb, n, j, S.coef, hst, S.fin);
        k_seg_lincomb<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, x0, x0, Zb, n, j, S.coef, hst, S.fin);
        k_seg_scale<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, w, w, S.scale);
        k_bat_count<<<1, 256, 0, ctx->stream>>>(S, nsys);
        return check("batched Arnoldi step");
    };
    // cycle end: the systems still active update x and x0 with their m vectors
    auto seq_end = [&]() -> int {
        k_bat_cycle_end<<<sgrid, kSysThreads, 0, ctx->stream>>>(S, bo, nsys);
        k_bat_lsq<<<nsys, 32, 0, ctx->stream>>>(S, bo, nsys);
        k_seg_lincomb<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, xx, x0, Zb, n, m, S.coef, hst, S.fin);
        k_seg_lincomb<T><<<nchunk, TH, 0, ctx->stream>>>(CS, CY, x0, x0, Zb, n, m, S.coef, hst, S.fin);
        k_bat_count<<<1, 256, 0, ctx->stream>>>(S, nsys);
        return check("batched cycle end");
    };

    // ---- graphs: captured on the second call with the same structure ------------
    for (const void* p : {(const void*)bb, (const void*)xx, (const void*)Vb, (const void*)Zb, (const void*)x0,
                          (const void*)BB->state.ptr, (const void*)BB->partial.ptr, (const void*)BB->rowsq.ptr})
        key.push_back((int64_t)(intptr_t)p);
    int64_t tolbits, rtolbits;
    std::memcpy(&tolbits, &bo.tol, 8);
    std::memcpy(&rtolbits, &bo.rtol, 8);
    key.insert(key.end(), {(int64_t)m, (int64_t)bo.nmax, (int64_t)bo.hcap, tolbits, rtolbits, (int64_t)sizeof(T)});
    if (!*graphs) *graphs = new BatchGraphs();
    BatchGraphs& GR = **graphs;
    if (GR.key != key) {
        GR.key = key;
        GR.seen = 0;
        GR.start.reset();
        GR.end.reset();
        GR.step.clear();
    }
    GR.seen++;
    // graphs need the streamed sweeps' flags reset inside each replay; the
    // preconditioner records that it runs in captured sequences
    const bool use = GR.seen >= 2 && !ctx->profiling && capturable && graphs_enabled();
    if (use && !GR.start) {
        M->graph_safe = true;
        GR.start.reset(new GraphPiece());
        GR.end.reset(new GraphPiece());
        int st;
        if ((st = capture(ctx, *GR.start, seq_start)) || (st = capture(ctx, *GR.end, seq_end))) {
            M->graph_safe = false;
            GR.start.reset();
            GR.end.reset();
            return st;
        }
        GR.step.resize(m);
        for (int j = 1; j <= m; ++j) {
            GR.step[j - 1].reset(new GraphPiece());
            if ((st = capture(ctx, *GR.step[j - 1], [&]() { return seq_step(j); }))) {
                M->graph_safe = false;
                GR.start.reset();
                GR.end.reset();
                GR.step.clear();
                return st;
            }
        }
        M->graph_safe = false;
    }
    auto exec = [&](GraphPiece* gp, const std::function<int()>& eager) -> int {
        if (gp) {
            const cudaError_t e = cudaGraphLaunch(gp->x, ctx->stream);
            return e == cudaSuccess ? CHIDG_GPU_OK : cuda_fail(ctx, e, "batch graph launch");
        }
        return eager();
    };
    const bool use_graphs = use && GR.start;

    // ---- solve --------------------------------------------------------------------
    int st;
    cudaMemsetAsync(x0, 0, sizeof(T) * n, ctx->stream);
    cudaMemsetAsync(xx, 0, sizeof(T) * n, ctx->stream);
    cudaMemsetAsync(BB->state.ptr, 0, ibytes, ctx->stream);       // every int field, the counters included
    k_bat_reset<<<sgrid, kSysThreads, 0, ctx->stream>>>(S, nsys);
    if ((st = check("k_bat_reset"))) return st;
    int32_t* hc = BB->h_count;
    for (;;) {
        if ((st = exec(use_graphs ? GR.start.get() : nullptr, seq_start))) return st;
        bool all_done = false;
        for (int j = 1; j <= m; ++j) {
            if ((st = exec(use_graphs ? GR.step[j - 1].get() : nullptr, [&]() { return seq_step(j); }))) return st;
            // the active count of this step lands in pinned memory; with step j
            // queued, the host waits for step j - 1's count, so the device is
            // never idle and at most one step runs after the last system converged
            const int slot = j & 1;
            cudaMemcpyAsync(hc + slot, S.count, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
            cudaEventRecord(BB->ev[slot], ctx->stream);
            if (j >= 2) {
                const cudaError_t e = cudaEventSynchronize(BB->ev[slot ^ 1]);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "batched fgmres");
                if (hc[slot ^ 1] == 0) { all_done = true; break; }
            }
        }
        if (!all_done) {
            if ((st = exec(use_graphs ? GR.end.get() : nullptr, seq_end))) return st;
        }
        int32_t cnt[2] = {0, 0};
        cudaError_t e = cudaMemcpyAsync(cnt, S.count, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "batched fgmres");
        if (cnt[1] != 0) {
            int32_t code = 0;
            cudaMemcpy(&code, S.err + (cnt[1] - 1), sizeof(int32_t), cudaMemcpyDeviceToHost);
            ctx->err_elem = g.sys_elem[cnt[1] - 1];
            return fail(ctx, code ? code : CHIDG_GPU_ENONFINITE,
                        code == CHIDG_GPU_ESINGULAR ? "batched fgmres: singular Hessenberg matrix"
                                                    : "batched fgmres: non-finite residual");
        }
        if (cnt[0] == 0) break;
    }
    if (!true_residual) return CHIDG_GPU_OK;
    // print_report: true residual per system
    if ((st = matvec(xx, (T*)ws->tmp.ptr, bb, -1.0, 1.0, ROWSQ))) return st;
    k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(ROWSQ, A->nrow, SR, 1, OUT, 1);
    return check("k_seg_reduce true residual");
}

}  // namespace

extern "C" int chidg_gpu_fgmres_solve_batched(chidg_gpu_matrix* A, chidg_gpu_precon* M, int32_t nsys,
                                              const int32_t* sys_elem, const chidg_gpu_vector* b,
                                              chidg_gpu_vector* x, const chidg_gpu_fgmres_opts* opts,
                                              chidg_gpu_fgmres_result* results, double* hist, int32_t hist_cap) {
    if (!A || !M || !b || !x || !sys_elem || nsys <= 0 || M->A != A || b->n != A->n || x->n != A->n || b == x)
        return CHIDG_GPU_EINVAL;
    chidg_gpu_ctx* ctx = A->ctx;
    cudaSetDevice(ctx->device);
    const auto t0 = std::chrono::steady_clock::now();
    chidg_gpu_fgmres_opts o;
    if (opts) o = *opts;
    else chidg_gpu_fgmres_default_opts(&o);
    if (o.inner_fgmres) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: inner FGMRES is not supported");
    // FP64 Krylov vectors for the outer solve in every mode; MIXED_PRECON_FP32
    // applies the preconditioner with FP32 copies of its blocks, MIXED_FP32 /
    // MIXED_BF16 precondition each outer step with an FP32 inner solve
    const int prec = o.precision;
    if (prec < CHIDG_GPU_FP64 || prec > CHIDG_GPU_MIXED_PRECON_FP32)
        return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: bad precision");
    const bool inner = prec == CHIDG_GPU_MIXED_FP32 || prec == CHIDG_GPU_MIXED_BF16;
    if (o.orthogonalization != CHIDG_ORTH_CGS) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: CGS only");
    const int m = o.nkrylov;
    if (m < 1 || m > 256) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: nkrylov outside [1, 256]");
    if (inner && (o.mixed_inner_nkrylov < 1 || o.mixed_inner_nkrylov > 256))
        return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: mixed_inner_nkrylov outside [1, 256]");
    // segments: systems must tile the elements and not couple to each other
    if (sys_elem[0] != 0 || sys_elem[nsys] != A->nelem) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: systems must cover all elements");
    std::vector<int> elem_sys(A->nelem);
    for (int s = 0; s < nsys; ++s) {
        if (sys_elem[s + 1] <= sys_elem[s]) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: empty or unordered system");
        for (int e = sys_elem[s]; e < sys_elem[s + 1]; ++e) elem_sys[e] = s;
    }
    for (int64_t k = 0; k < A->nblk; ++k)
        if (elem_sys[A->re[k]] != elem_sys[A->ce[k]]) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: a block couples two systems");
    BatchBuffers& BB = ctx->batch;
    std::vector<int64_t> cstart;
    std::vector<int32_t> csys, sys_chunk(nsys + 1), sys_row(nsys + 1);
    for (int s = 0; s < nsys; ++s) {
        sys_chunk[s] = (int32_t)csys.size();
        const int64_t v0 = A->eoff[sys_elem[s]];
        const int64_t v1 = (sys_elem[s + 1] < A->nelem) ? A->eoff[sys_elem[s + 1]] : A->n;
        for (int64_t c = v0; c < v1; c += kChunk) { cstart.push_back(c); csys.push_back(s); }
        sys_row[s] = sys_elem[s] * A->ntime;
    }
    sys_chunk[nsys] = (int32_t)csys.size();
    sys_row[nsys] = A->nrow;
    cstart.push_back(A->n);
    std::vector<int32_t> row_sys(A->nrow);
    for (int s = 0; s < nsys; ++s)
        for (int r = sys_row[s]; r < sys_row[s + 1]; ++r) row_sys[r] = s;
    int st;
    if ((st = upload_vec(ctx, BB.cstart, cstart)) || (st = upload_vec(ctx, BB.csys, csys)) ||
        (st = upload_vec(ctx, BB.sys_chunk, sys_chunk)) || (st = upload_vec(ctx, BB.sys_row, sys_row)) ||
        (st = upload_vec(ctx, BB.row_sys, row_sys)))
        return st;

    // M%update as the controller decides (type_fgmres.f90:118-122)
    if (!(o.use_controller && M->stamp == A->stamp && M->precision == prec))
        if ((st = chidg_gpu_precon_update(M, A, prec))) return st;
    // from here on A is the operator: A, or A^T when A->transposed (same rows and segments)
    if ((st = matrix_op(A, &A))) return st;
    // the FP32 / BF16 copy read by the inner solves' products
    if (inner && (st = matrix_lowp(A, prec))) return st;
    set_matvec_smem(A);
    if (M->kind != CHIDG_PRECON_IDENTITY) precon_set_smem(M);
    cudaMemsetAsync(ctx->d_scal + kSlotStatus, 0, sizeof(double), ctx->stream);

    const int64_t n = A->n;
    Segs g;
    g.CS = (const int64_t*)BB.cstart.ptr;
    g.CY = (const int32_t*)BB.csys.ptr;
    g.SC = (const int32_t*)BB.sys_chunk.ptr;
    g.SR = (const int32_t*)BB.sys_row.ptr;
    g.row_sys = (const int32_t*)BB.row_sys.ptr;
    g.sys_elem = sys_elem;
    g.nchunk = (int)csys.size();
    g.nsys = nsys;
    // only the streamed sweeps clear their flags inside a captured sequence
    const bool sweeps_ok = M->kind == CHIDG_PRECON_IDENTITY ||
                           (M->schedule == CHIDG_SCHED_STREAM && M->P.max_b <= SS_MAX_B);
    std::vector<int64_t> key = {A->uid, (int64_t)(intptr_t)M, (int64_t)M->kind, (int64_t)M->schedule, nsys, prec,
                                (int64_t)(intptr_t)BB.cstart.ptr, (int64_t)M->P.nprow, M->P.ntask_bmv};
    key.insert(key.end(), sys_elem, sys_elem + nsys + 1);

    BatchEngine<double> E;
    E.ctx = ctx; E.A = A; E.M = M; E.g = g; E.BB = &BB; E.ws = &ctx->ws64; E.graphs = &ctx->batch_graphs;
    E.matvec = [A](const double* xv, double* yv, const double* zv, double a, double bt, double* rs) {
        return matvec_launch<double, double>(A, (const double*)A->val.ptr, xv, yv, zv, a, bt, rs);
    };
    BatchEngine<float> In;
    if (!inner) {
        E.capturable = sweeps_ok;
        E.step_mv = [M, A, prec](const double* v, double* z, double* w, double* rs) -> int {
            int s2 = precon_apply_mv<double, double>(M, v, z, prec, A, (const double*)A->val.ptr, w, rs);
            if (s2 != 1) return s2;
            if ((s2 = precon_apply_impl<double>(M, v, z, prec))) return s2;
            return matvec_launch<double, double>(A, (const double*)A->val.ptr, z, w, nullptr, 1.0, 0.0, rs);
        };
    } else {
        // the inner solve: FP32 vectors, the FP32 (or BF16) copy of A and the
        // low-precision factors, tol 0, rtol / nmax / nkrylov of the mixed options
        const bool bf = prec == CHIDG_GPU_MIXED_BF16;
        In.ctx = ctx; In.A = A; In.M = M; In.g = g; In.BB = &ctx->batch_inner; In.ws = &ctx->ws32;
        In.graphs = &ctx->batch_graphs_inner;
        In.capturable = sweeps_ok;
        In.true_residual = false;
        In.matvec = [A, bf](const float* xv, float* yv, const float* zv, double a, double bt, double* rs) {
            return bf ? matvec_launch<__nv_bfloat16, float>(A, (const __nv_bfloat16*)A->val16.ptr, xv, yv, zv, a, bt, rs)
                      : matvec_launch<float, float>(A, (const float*)A->val32.ptr, xv, yv, zv, a, bt, rs);
        };
        In.step_mv = [M, A, prec, bf](const float* v, float* z, float* w, double* rs) -> int {
            int s2 = bf ? precon_apply_mv<float, __nv_bfloat16>(M, v, z, prec, A, (const __nv_bfloat16*)A->val16.ptr, w, rs)
                        : precon_apply_mv<float, float>(M, v, z, prec, A, (const float*)A->val32.ptr, w, rs);
            if (s2 != 1) return s2;
            if ((s2 = precon_apply_impl<float>(M, v, z, prec))) return s2;
            return bf ? matvec_launch<__nv_bfloat16, float>(A, (const __nv_bfloat16*)A->val16.ptr, z, w, nullptr, 1.0, 0.0, rs)
                      : matvec_launch<float, float>(A, (const float*)A->val32.ptr, z, w, nullptr, 1.0, 0.0, rs);
        };
        if ((st = In.prepare(o.mixed_inner_nkrylov, 0.0, o.mixed_inner_rtol, o.mixed_inner_nmax, 1))) return st;
        if ((st = ensure(ctx, ctx->mix_v32, sizeof(float) * (size_t)n)) || (st = ensure(ctx, ctx->mix_z32, sizeof(float) * (size_t)n)))
            return st;
        float* V32 = (float*)ctx->mix_v32.ptr;
        float* Z32 = (float*)ctx->mix_z32.ptr;
        // an outer step runs the inner solve's host loop: not captured
        E.capturable = false;
        E.step_mv = [ctx, A, &In, &E, V32, Z32, n, nsys, key](const double* v, double* z, double* w, double* rs) -> int {
            k_convert<double, float><<<grid_for(n, 256, ctx->nsm * 8), 256, 0, ctx->stream>>>(n, v, V32);
            int s2 = check_launch(ctx, "k_convert v");
            if (s2 || (s2 = In.run(V32, Z32, key))) return s2;
            k_bat_add_inner<<<(nsys + kSysThreads - 1) / kSysThreads, kSysThreads, 0, ctx->stream>>>(E.S.inner, In.S.niter, nsys);
            k_convert<float, double><<<grid_for(n, 256, ctx->nsm * 8), 256, 0, ctx->stream>>>(n, Z32, z);
            if ((s2 = check_launch(ctx, "k_convert z"))) return s2;
            return matvec_launch<double, double>(A, (const double*)A->val.ptr, z, w, nullptr, 1.0, 0.0, rs);
        };
    }
    if ((st = E.prepare(m, o.tol, o.rtol, o.nmax, hist_cap))) return st;
    double* xx = (double*)x->buf.ptr;
    const double* bb = (const double*)b->buf.ptr;
    if ((st = E.run(bb, xx, key))) return st;

    const BatState& S = E.S;
    const int hcap = E.bo.hcap;
    std::vector<double> tres(nsys), r0i(nsys), rest(nsys), hh((size_t)nsys * hcap);
    std::vector<int32_t> nit(nsys), nrs(nsys), nh(nsys), nin(nsys);
    double sw = 0.0;
    cudaError_t e = cudaMemcpyAsync(tres.data(), BB.out.ptr, sizeof(double) * nsys, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(r0i.data(), S.r0init, sizeof(double) * nsys, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(rest.data(), S.res_est, sizeof(double) * nsys, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nit.data(), S.niter, sizeof(int32_t) * nsys, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nrs.data(), S.nrestart, sizeof(int32_t) * nsys, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nh.data(), S.nhist, sizeof(int32_t) * nsys, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(nin.data(), S.inner, sizeof(int32_t) * nsys, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && hist) e = cudaMemcpyAsync(hh.data(), S.hist, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sw, ctx->d_scal + kSlotStatus, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batched fgmres results");
    if ((st = status_word(ctx, sw))) return st;
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int s = 0; s < nsys; ++s) {
        if (results) {
            chidg_gpu_fgmres_result& r = results[s];
            r.niter = nit[s];
            r.nrestart = nrs[s];
            r.inner_iters = nin[s];
            r.nhist = std::min(nh[s], std::max(hist_cap, 0));
            r.residual_norm = std::sqrt(tres[s]);
            r.res_estimate = rest[s];
            r.r0norm_initial = r0i[s];
            r.seconds = secs;
        }
        if (hist)
            for (int i = 0; i < nh[s] && i < hist_cap; ++i) hist[(size_t)s * hist_cap + i] = hh[(size_t)s * hcap + i];
    }
    return CHIDG_GPU_OK;
}
