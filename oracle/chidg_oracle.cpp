// chidg_oracle.cpp -- CPU FP64 restatement of ChiDG's implicit linear-solve path.
//
// TEST INFRASTRUCTURE ONLY (the parity oracle).  Never linked into or called by
// the CUDA product library.  Every routine cites the reference routine it
// restates; paths are relative to the ChiDG source tree.
//
// Reference behaviour restated here:
//   block layout / lower-upper / transpose  src/containers/type_domain_matrix.f90:102-632
//   chidg_mv                                src/containers/operator_chidg_mv.f90:117-645
//   dot / norm                              src/containers/operator_chidg_dot.f90:30-97,
//                                           src/containers/type_chidg_vector.f90:1237-1305
//   chidg_mv, transposed (A%transposed)     src/containers/operator_chidg_mv.f90:46-60,692-1049
//   inv (getrf + getri semantics)           src/numerical_methods/mod_inv.f90:97-150
//   precon_jacobi update/apply              src/preconditioners/precon_jacobi.f90:95-215
//   precon_ILU0 update/apply                src/preconditioners/precon_ILU0.f90:111-411
//   precon_RASILU0 update/apply             src/preconditioners/RASILU0/precon_RASILU0.f90:205-625
//   precon_HB update/apply                  src/preconditioners/precon_HB.f90:169-310
//     overlap set / ordering / transposes   .../RASILU0/type_RASILU0_send_comm.f90:66-275,
//                                           .../RASILU0/type_RASILU0_recv_dom_comm.f90:59-305
//   fgmres_t%solve, CGS, MGS                src/linear_solvers/type_fgmres.f90:81-442
//   solver_controller%update_preconditioner src/nonlinear_solvers/type_solver_controller.f90
#include "chidg_oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <immintrin.h>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace {

using std::vector;

// Host threads for the oracle's data-parallel loops.  A loop run through the
// pool hands each index to exactly one thread, and the work of an index is
// the serial loop's work for that index in the serial loop's order, so every
// result is bitwise the one-thread result whatever the thread count.  Loops
// whose serial order couples indices (a dot product's running sum, an ILU row
// that needs its parents) are either kept serial or split only where the
// serial order allows it (independent dots, rows of one dependency level).
// Calls made while the pool is busy on another caller's loop run serially.
class Pool {
  public:
    static Pool& get() {
        static Pool p;
        return p;
    }
    int threads() const { return nthreads_; }
    void set_threads(int n) {
        n = std::max(1, std::min(n, 1024));
        std::lock_guard<std::mutex> busy(run_mu_);
        stop_workers();
        nthreads_ = n;
        // workers start at the current generation: run() cannot advance it
        // while this call holds run_mu_
        for (int i = 1; i < n; ++i) workers_.emplace_back([this, g0 = gen_] { worker(g0); });
    }
    template <class F>
    void run(int64_t n, F&& f) {
        if (n <= 0) return;
        std::unique_lock<std::mutex> busy(run_mu_, std::try_to_lock);
        if (!busy.owns_lock() || nthreads_ == 1 || n == 1) {
            for (int64_t i = 0; i < n; ++i) f(i);
            return;
        }
        std::function<void(int64_t)> job = std::forward<F>(f);
        {
            std::lock_guard<std::mutex> g(mu_);
            job_ = &job;
            n_ = n;
            next_.store(0);
            pending_ = nthreads_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> g(mu_);
        done_.wait(g, [this] { return pending_ == 0; });
        job_ = nullptr;
    }
    // f(begin, end) over [0, n) in chunks of `grain`
    template <class F>
    void run_chunks(int64_t n, int64_t grain, F&& f) {
        const int64_t nc = (n + grain - 1) / grain;
        run(nc, [&](int64_t c) { f(c * grain, std::min(n, (c + 1) * grain)); });
    }
    ~Pool() {
        std::lock_guard<std::mutex> busy(run_mu_);
        stop_workers();
    }

  private:
    void work() {
        for (;;) {
            const int64_t i = next_.fetch_add(1);
            if (i >= n_) break;
            (*job_)(i);
        }
    }
    void worker(uint64_t seen) {
        for (;;) {
            {
                std::unique_lock<std::mutex> g(mu_);
                cv_.wait(g, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
            std::lock_guard<std::mutex> g(mu_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    void stop_workers() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
        workers_.clear();
        stop_ = false;
    }
    int nthreads_ = 1;
    std::vector<std::thread> workers_;
    std::mutex run_mu_, mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int64_t)>* job_ = nullptr;
    int64_t n_ = 0;
    std::atomic<int64_t> next_{0};
    int pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};
constexpr int64_t kGrain = 1 << 14;   // vector entries per chunk of an elementwise loop

// A large FP64 array filled on the pool (zeroed, or copied) instead of by one
// thread: at the workload sizes these arrays hold up to tens of GB.
struct DBuf {
    std::unique_ptr<double[]> p;
    int64_t n = 0;
    double* data() { return p.get(); }
    const double* data() const { return p.get(); }
    int64_t size() const { return n; }
    void resize(int64_t n_) {
        if (n_ != n) {
            p.reset(n_ > 0 ? new double[n_] : nullptr);
            n = n_;
        }
    }
    void zeros(int64_t n_) {
        resize(n_);
        double* d = p.get();
        Pool::get().run_chunks(n, 1 << 20, [d](int64_t a, int64_t b) { std::memset(d + a, 0, sizeof(double) * (b - a)); });
    }
    void copy_from(const double* src) {
        double* d = p.get();
        Pool::get().run_chunks(n, 1 << 20, [d, src](int64_t a, int64_t b) { std::memcpy(d + a, src + a, sizeof(double) * (b - a)); });
    }
    void copy_to(double* dst) const {
        const double* d = p.get();
        Pool::get().run_chunks(n, 1 << 20, [d, dst](int64_t a, int64_t b) { std::memcpy(dst + a, d + a, sizeof(double) * (b - a)); });
    }
};

struct Mat {
    int nelem = 0, ntime = 0;
    vector<int> nvars, nterms, proc;
    vector<int64_t> eoff;   // vector offset of each element
    int64_t n = 0;          // vector length
    int64_t nblk = 0;
    vector<int> re, rt, ce, ct, kind, nr, nc;
    vector<int64_t> voff;   // packed value offset of each block
    int64_t nval = 0;
    DBuf val;
    vector<vector<int>> rowblk;   // per row (e*ntime+t): all blocks, lblks first then chi/bc/hb
    vector<vector<int>> lblk;     // per row: LOCAL blocks in storage order
    vector<int> diag;             // per row: DIAG block id
    long stamp = 1;
    bool transposed = false;      // chidg_matrix_t%transposed (type_chidg_matrix.f90:49)

    int bsize(int e) const { return nvars[e] * nterms[e]; }
    int64_t seg(int e, int t) const { return eoff[e] + (int64_t)t * bsize(e); }
    int row(int e, int t) const { return e * ntime + t; }
    const double* blk(int k) const { return val.data() + voff[k]; }
    double* blk(int k) { return val.data() + voff[k]; }
};

// y(0:nr) += A(nr x nc, column-major) * x(0:nc)
inline void gemv_acc(int nr, int nc, const double* A, const double* x, double* y) {
    for (int c = 0; c < nc; ++c) {
        const double xc = x[c];
        const double* col = A + (int64_t)c * nr;
        for (int r = 0; r < nr; ++r) y[r] += col[r] * xc;
    }
}
// y(0:nr) -= A * x
inline void gemv_sub(int nr, int nc, const double* A, const double* x, double* y) {
    for (int c = 0; c < nc; ++c) {
        const double xc = x[c];
        const double* col = A + (int64_t)c * nr;
        for (int r = 0; r < nr; ++r) y[r] -= col[r] * xc;
    }
}
// y(0:nc) += A(nr x nc)^T * x(0:nr)
inline void gemv_t_acc(int nr, int nc, const double* A, const double* x, double* y) {
    for (int c = 0; c < nc; ++c) {
        const double* col = A + (int64_t)c * nr;
        double s = 0.0;
        for (int r = 0; r < nr; ++r) s += col[r] * x[r];
        y[c] += s;
    }
}
// y(0:nc) -= A(nr x nc)^T * x(0:nr)
inline void gemv_t_sub(int nr, int nc, const double* A, const double* x, double* y) {
    for (int c = 0; c < nc; ++c) {
        const double* col = A + (int64_t)c * nr;
        double s = 0.0;
        for (int r = 0; r < nr; ++r) s += col[r] * x[r];
        y[c] -= s;
    }
}
// C(m x n) = A(k x m)^T * B(k x n)
void gemm_tn(int m, int n, int k, const double* A, const double* B, double* C) {
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double s = 0.0;
            for (int p = 0; p < k; ++p) s += A[p + (int64_t)i * k] * B[p + (int64_t)j * k];
            C[i + (int64_t)j * m] = s;
        }
}
// C(m x n) -= A(m x k) * B(n x k)^T
void gemm_sub_nt(int m, int n, int k, const double* A, const double* B, double* C) {
    for (int j = 0; j < n; ++j)
        for (int p = 0; p < k; ++p) {
            const double b = B[j + (int64_t)p * n];
            const double* a = A + (int64_t)p * m;
            double* c = C + (int64_t)j * m;
            for (int i = 0; i < m; ++i) c[i] -= a[i] * b;
        }
}
// C(m x n) +=/-= A(m x k) * B(k x n), all column-major.  Every entry is
// updated as c = fma(+-a(i,p), b(p,j), c) for p = 0 .. k-1 in order (the
// fused multiply-add the compiler makes of `c += a * b`), so the register
// tiles below give the same bits as the plain triple loop: they only keep a
// tile of C in registers across p instead of reloading it.  An AVX-512 tile
// (up to 24 rows x 8 columns, the last row vector masked) is used where the
// host has AVX-512, an AVX2 tile (12 x 4) otherwise.
template <bool SUB, int NV, int NJ>
__attribute__((target("avx512f"))) void tile512(int m, int k, const double* A, const double* B, double* C, int i,
                                                int j, __mmask8 last) {
    __m512d c[NV][NJ];
    for (int jj = 0; jj < NJ; ++jj)
        for (int ii = 0; ii < NV; ++ii)
            c[ii][jj] = _mm512_maskz_loadu_pd(ii == NV - 1 ? last : (__mmask8)0xFF, C + i + 8 * ii + (int64_t)(j + jj) * m);
    for (int p = 0; p < k; ++p) {
        const double* ap = A + i + (int64_t)p * m;
        __m512d a[NV];
        for (int ii = 0; ii < NV; ++ii) a[ii] = _mm512_maskz_loadu_pd(ii == NV - 1 ? last : (__mmask8)0xFF, ap + 8 * ii);
        for (int jj = 0; jj < NJ; ++jj) {
            const __m512d b = _mm512_set1_pd(B[p + (int64_t)(j + jj) * k]);
            for (int ii = 0; ii < NV; ++ii)
                c[ii][jj] = SUB ? _mm512_fnmadd_pd(a[ii], b, c[ii][jj]) : _mm512_fmadd_pd(a[ii], b, c[ii][jj]);
        }
    }
    for (int jj = 0; jj < NJ; ++jj)
        for (int ii = 0; ii < NV; ++ii)
            _mm512_mask_storeu_pd(C + i + 8 * ii + (int64_t)(j + jj) * m, ii == NV - 1 ? last : (__mmask8)0xFF, c[ii][jj]);
}
template <bool SUB, int NV>
void tile512_nj(int nj, int m, int k, const double* A, const double* B, double* C, int i, int j, __mmask8 last) {
    switch (nj) {
        case 8: tile512<SUB, NV, 8>(m, k, A, B, C, i, j, last); break;
        case 7: tile512<SUB, NV, 7>(m, k, A, B, C, i, j, last); break;
        case 6: tile512<SUB, NV, 6>(m, k, A, B, C, i, j, last); break;
        case 5: tile512<SUB, NV, 5>(m, k, A, B, C, i, j, last); break;
        case 4: tile512<SUB, NV, 4>(m, k, A, B, C, i, j, last); break;
        case 3: tile512<SUB, NV, 3>(m, k, A, B, C, i, j, last); break;
        case 2: tile512<SUB, NV, 2>(m, k, A, B, C, i, j, last); break;
        default: tile512<SUB, NV, 1>(m, k, A, B, C, i, j, last); break;
    }
}
template <bool SUB>
void gemm_update_avx512(int m, int n, int k, const double* A, const double* B, double* C) {
    for (int j = 0; j < n; j += 8) {
        const int nj = std::min(8, n - j);
        for (int i = 0; i < m; i += 24) {
            const int rows = std::min(24, m - i);
            const int nv = (rows + 7) / 8;
            const __mmask8 last = (rows % 8) ? (__mmask8)((1u << (rows % 8)) - 1u) : (__mmask8)0xFF;
            if (nv == 3) tile512_nj<SUB, 3>(nj, m, k, A, B, C, i, j, last);
            else if (nv == 2) tile512_nj<SUB, 2>(nj, m, k, A, B, C, i, j, last);
            else tile512_nj<SUB, 1>(nj, m, k, A, B, C, i, j, last);
        }
    }
}
template <bool SUB>
void gemm_update_avx2(int m, int n, int k, const double* A, const double* B, double* C) {
    auto upd = [](double a, double b, double c) { return SUB ? std::fma(-a, b, c) : std::fma(a, b, c); };
    int j = 0;
    for (; j + 4 <= n; j += 4) {
        int i = 0;
        for (; i + 12 <= m; i += 12) {
            __m256d c[3][4];
            for (int jj = 0; jj < 4; ++jj)
                for (int ii = 0; ii < 3; ++ii) c[ii][jj] = _mm256_loadu_pd(C + i + 4 * ii + (int64_t)(j + jj) * m);
            for (int p = 0; p < k; ++p) {
                const double* ap = A + i + (int64_t)p * m;
                const __m256d a0 = _mm256_loadu_pd(ap), a1 = _mm256_loadu_pd(ap + 4), a2 = _mm256_loadu_pd(ap + 8);
                for (int jj = 0; jj < 4; ++jj) {
                    const __m256d b = _mm256_broadcast_sd(B + p + (int64_t)(j + jj) * k);
                    if (SUB) {
                        c[0][jj] = _mm256_fnmadd_pd(a0, b, c[0][jj]);
                        c[1][jj] = _mm256_fnmadd_pd(a1, b, c[1][jj]);
                        c[2][jj] = _mm256_fnmadd_pd(a2, b, c[2][jj]);
                    } else {
                        c[0][jj] = _mm256_fmadd_pd(a0, b, c[0][jj]);
                        c[1][jj] = _mm256_fmadd_pd(a1, b, c[1][jj]);
                        c[2][jj] = _mm256_fmadd_pd(a2, b, c[2][jj]);
                    }
                }
            }
            for (int jj = 0; jj < 4; ++jj)
                for (int ii = 0; ii < 3; ++ii) _mm256_storeu_pd(C + i + 4 * ii + (int64_t)(j + jj) * m, c[ii][jj]);
        }
        for (; i < m; ++i)
            for (int jj = 0; jj < 4; ++jj) {
                double c = C[i + (int64_t)(j + jj) * m];
                for (int p = 0; p < k; ++p) c = upd(A[i + (int64_t)p * m], B[p + (int64_t)(j + jj) * k], c);
                C[i + (int64_t)(j + jj) * m] = c;
            }
    }
    for (; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double c = C[i + (int64_t)j * m];
            for (int p = 0; p < k; ++p) c = upd(A[i + (int64_t)p * m], B[p + (int64_t)j * k], c);
            C[i + (int64_t)j * m] = c;
        }
}
const bool kHostAvx512 = __builtin_cpu_supports("avx512f");
template <bool SUB>
void gemm_update(int m, int n, int k, const double* A, const double* B, double* C) {
    if (kHostAvx512) gemm_update_avx512<SUB>(m, n, k, A, B, C);
    else gemm_update_avx2<SUB>(m, n, k, A, B, C);
}
// C(m x n) = A(m x k) * B(k x n), all column-major
void gemm(int m, int n, int k, const double* A, const double* B, double* C) {
    std::fill(C, C + (int64_t)m * n, 0.0);
    gemm_update<false>(m, n, k, A, B, C);
}
// C -= A * B
void gemm_sub(int m, int n, int k, const double* A, const double* B, double* C) {
    gemm_update<true>(m, n, k, A, B, C);
}

// Explicit inverse with partial pivoting, following the semantics of
// mod_inv::inv (src/numerical_methods/mod_inv.f90:97-150): DGETRF (LU with
// row interchanges, pivot = first entry of largest magnitude in the column,
// exact-zero pivot => singular) followed by DGETRI (inv(U), then solve
// inv(A)*L = inv(U), then undo the column interchanges).  Written from the
// textbook algorithm (Golub & Van Loan Alg. 3.4.1); returns 0 or the 1-based
// index of the first zero pivot.
int inv_inplace(int n, double* a) {
    vector<int> ipiv(n);
    int info = 0;
    // getrf (unblocked, right-looking)
    for (int k = 0; k < n; ++k) {
        int p = k;
        double amax = std::fabs(a[k + (int64_t)k * n]);
        for (int i = k + 1; i < n; ++i) {
            double v = std::fabs(a[i + (int64_t)k * n]);
            if (v > amax) { amax = v; p = i; }
        }
        ipiv[k] = p;
        if (a[p + (int64_t)k * n] != 0.0) {
            if (p != k)
                for (int j = 0; j < n; ++j) std::swap(a[k + (int64_t)j * n], a[p + (int64_t)j * n]);
            const double rp = 1.0 / a[k + (int64_t)k * n];
            for (int i = k + 1; i < n; ++i) a[i + (int64_t)k * n] *= rp;
        } else if (info == 0) {
            info = k + 1;
        }
        for (int j = k + 1; j < n; ++j) {
            const double akj = a[k + (int64_t)j * n];
            if (akj != 0.0)
                for (int i = k + 1; i < n; ++i) a[i + (int64_t)j * n] -= a[i + (int64_t)k * n] * akj;
        }
    }
    if (info) return info;
    // getri: inv(U) in place (trtri, upper, non-unit)
    for (int j = 0; j < n; ++j) {
        a[j + (int64_t)j * n] = 1.0 / a[j + (int64_t)j * n];
        const double ajj = -a[j + (int64_t)j * n];
        // x = inv(U(0:j,0:j)) * U(0:j,j) using the already-inverted leading block
        for (int i = 0; i < j; ++i) {
            double s = 0.0;
            for (int l = i; l < j; ++l) s += a[i + (int64_t)l * n] * a[l + (int64_t)j * n];
            // rows are visited top-down and row i only reads rows >= i of
            // column j, so the product can overwrite column j in place
            a[i + (int64_t)j * n] = s;
        }
        for (int i = 0; i < j; ++i) a[i + (int64_t)j * n] *= ajj;
    }
    // solve inv(A) * L = inv(U) for inv(A), columns right to left
    vector<double> work(n);
    for (int j = n - 2; j >= 0; --j) {
        for (int i = j + 1; i < n; ++i) {
            work[i] = a[i + (int64_t)j * n];
            a[i + (int64_t)j * n] = 0.0;
        }
        for (int l = j + 1; l < n; ++l) {
            const double w = work[l];
            if (w != 0.0)
                for (int i = 0; i < n; ++i) a[i + (int64_t)j * n] -= a[i + (int64_t)l * n] * w;
        }
    }
    // apply column interchanges in reverse order
    for (int j = n - 2; j >= 0; --j) {
        const int jp = ipiv[j];
        if (jp != j)
            for (int i = 0; i < n; ++i) std::swap(a[i + (int64_t)j * n], a[i + (int64_t)jp * n]);
    }
    return 0;
}

// ---------------------------------------------------------------------------
// Preconditioners
// ---------------------------------------------------------------------------
struct Precon {
    int kind = 0;
    long stamp = 0;          // preconditioner%stamp (0 = never updated)
    int err_elem = -1;
    virtual ~Precon() {}
    virtual int update(Mat& A) = 0;
    virtual int apply(Mat& A, const double* v, double* z) = 0;
};

struct PreconIdentity : Precon {
    int update(Mat& A) override { stamp = A.stamp; return ORC_OK; }
    int apply(Mat& A, const double* v, double* z) override {
        std::memcpy(z, v, sizeof(double) * A.n);
        return ORC_OK;
    }
};

// Block ILU0 over LOCAL blocks; with nolower/noupper it degenerates to block
// Jacobi (precon_jacobi.f90:95-215 stores inv(diag) and applies it).
struct PreconILU0 : Precon {
    bool jacobi = false;
    DBuf LD;                                 // same packing as A: L blocks and inv(D)
    vector<vector<int>> lower, upper;        // per row, block ids (local_lower/upper_blocks)
    vector<int> itrans;                      // per block: transposed block in parent row
    // Rows of one time level grouped by dependency level: a row's factor and
    // forward-sweep work needs its lower parents finished (flev), its
    // backward-sweep work its upper parents (blev).  Rows of a level are
    // independent, so they run on the pool; each row's own arithmetic is the
    // serial loop's.
    vector<vector<vector<int>>> flev, blev;  // [t][level] -> elements, increasing
    void build(Mat& A) {
        lower.assign((size_t)A.nelem * A.ntime, {});
        upper.assign((size_t)A.nelem * A.ntime, {});
        itrans.assign(A.nblk, -1);
        if (!jacobi) {
            // type_domain_matrix.f90:295-302 with a single rank: lower iff eparent < ielem
            for (int e = 0; e < A.nelem; ++e)
                for (int t = 0; t < A.ntime; ++t) {
                    const int r = A.row(e, t);
                    for (int k : A.lblk[r]) {
                        if (A.ce[k] < e) lower[r].push_back(k);
                        else if (A.ce[k] > e) upper[r].push_back(k);
                        // transposed block (type_domain_matrix.f90:592-627)
                        const int p = A.ce[k];
                        for (int kk : A.lblk[A.row(p, t)])
                            if (A.ce[kk] == e) { itrans[k] = kk; break; }
                    }
                }
        }
        flev.assign(A.ntime, {});
        blev.assign(A.ntime, {});
        vector<int> lv(A.nelem);
        for (int t = 0; t < A.ntime; ++t) {
            for (int e = 0; e < A.nelem; ++e) {
                int l = 0;
                for (int k : lower[A.row(e, t)]) l = std::max(l, lv[A.ce[k]] + 1);
                lv[e] = l;
                if ((int)flev[t].size() <= l) flev[t].resize(l + 1);
                flev[t][l].push_back(e);
            }
            for (int e = A.nelem - 1; e >= 0; --e) {
                int l = 0;
                for (int k : upper[A.row(e, t)]) l = std::max(l, lv[A.ce[k]] + 1);
                lv[e] = l;
                if ((int)blev[t].size() <= l) blev[t].resize(l + 1);
                blev[t][l].push_back(e);
            }
        }
    }
    // precon_ILU0.f90:111-265; with A%transposed (:148-207) the factors are
    // those of A^T: D = A(e,e)^T, L = A(parent, itranspose)^T inv(D_parent),
    // D -= L A_lower^T.  precon_jacobi.f90:121-125 likewise inverts A(e,e)^T.
    int update(Mat& A) override {
        LD.zeros(A.nval);
        err_elem = -1;
        Pool& pool = Pool::get();
        for (int t = 0; t < A.ntime; ++t) {
            pool.run(A.nelem, [&](int64_t e) {
                const int k = A.diag[A.row((int)e, t)];
                const int b = A.nr[k];
                double* D = LD.data() + A.voff[k];
                if (A.transposed) {
                    for (int j = 0; j < b; ++j)
                        for (int i = 0; i < b; ++i) D[i + (int64_t)j * b] = A.blk(k)[j + (int64_t)i * b];
                } else {
                    std::memcpy(D, A.blk(k), sizeof(double) * A.nr[k] * A.nc[k]);
                }
            });
            // The serial loop stops at the first singular element in natural
            // order.  Once a level finds a singular element e_bad, later levels
            // only factor rows below e_bad (their parents are below them, so
            // all factored): the element reported is the serial loop's.
            int e_bad = A.nelem;
            vector<char> bad(A.nelem, 0);
            for (const vector<int>& level : flev[t]) {
                pool.run((int64_t)level.size(), [&](int64_t i) {
                    const int e = level[i];
                    if (e >= e_bad) return;
                    const int r = A.row(e, t);
                    const int kd = A.diag[r];
                    const int b = A.nr[kd];
                    double* D = LD.data() + A.voff[kd];
                    for (int kl : lower[r]) {
                        const int p = A.ce[kl];
                        const int kpd = A.diag[A.row(p, t)];
                        double* L = LD.data() + A.voff[kl];
                        const int kt = itrans[kl];
                        if (A.transposed) {
                            // L = A(parent, itranspose)^T * inv(D_parent); D -= L * A_lower^T
                            gemm_tn(A.nr[kl], A.nc[kl], A.nr[kt], A.blk(kt), LD.data() + A.voff[kpd], L);
                            gemm_sub_nt(b, A.nc[kl], A.nc[kl], L, A.blk(kl), D);
                        } else {
                            // L = A_lower * inv(D_parent); D -= L * A(parent, itranspose)
                            gemm(A.nr[kl], A.nc[kl], A.nc[kl], A.blk(kl), LD.data() + A.voff[kpd], L);
                            gemm_sub(b, A.nc[kt], A.nc[kl], L, A.blk(kt), D);
                        }
                    }
                    if (inv_inplace(b, D) != 0) bad[e] = 1;
                });
                for (int e : level)
                    if (bad[e]) e_bad = std::min(e_bad, e);
            }
            if (e_bad < A.nelem) { err_elem = e_bad; return ORC_ESINGULAR; }
        }
        stamp = A.stamp;
        return ORC_OK;
    }
    // precon_ILU0.f90:286-411; with A%transposed the backward solve uses
    // A(parent, itranspose)^T in place of the upper block (:378-383)
    int apply(Mat& A, const double* v, double* z) override {
        Pool& pool = Pool::get();
        pool.run_chunks(A.n, kGrain, [&](int64_t q0, int64_t q1) {
            std::memcpy(z + q0, v + q0, sizeof(double) * (q1 - q0));
        });
        for (int t = 0; t < A.ntime; ++t) {
            for (const vector<int>& level : flev[t])
                pool.run((int64_t)level.size(), [&](int64_t i) {
                    const int e = level[i];
                    const int r = A.row(e, t);
                    double* ze = z + A.seg(e, t);
                    for (int kl : lower[r])
                        gemv_sub(A.nr[kl], A.nc[kl], LD.data() + A.voff[kl], z + A.seg(A.ce[kl], t), ze);
                });
            for (const vector<int>& level : blev[t])
                pool.run((int64_t)level.size(), [&](int64_t i) {
                    const int e = level[i];
                    const int r = A.row(e, t);
                    double* ze = z + A.seg(e, t);
                    for (int ku : upper[r]) {
                        if (A.transposed) {
                            const int kt = itrans[ku];
                            gemv_t_sub(A.nr[kt], A.nc[kt], A.blk(kt), z + A.seg(A.ce[ku], t), ze);
                        } else {
                            gemv_sub(A.nr[ku], A.nc[ku], A.blk(ku), z + A.seg(A.ce[ku], t), ze);
                        }
                    }
                    const int kd = A.diag[r];
                    const int b = A.nr[kd];
                    vector<double> tmp(b, 0.0);
                    gemv_acc(b, b, LD.data() + A.voff[kd], ze, tmp.data());
                    std::memcpy(ze, tmp.data(), sizeof(double) * b);
                });
        }
        return ORC_OK;
    }
};

// Restricted additive Schwarz with ILU0 subdomain solves and a one-element
// overlap.  Subdomain s plays MPI rank s (elem_proc), all in one process.
struct PreconRAS : Precon {
    struct OvBlk {
        int parent;          // global element the block couples to
        bool parent_local;   // parent owned by the receiving subdomain
        int src;             // block id in A (row = overlap element)
        int trans_elem;      // overlap index (parent on owner) or -1
        int trans_src;       // block id in A of the transposed block
        vector<double> mat;  // received copy, factored in place
    };
    struct OvElem {
        int elem;            // global element id
        int owner;           // owning subdomain
        vector<OvBlk> blks;
        int diag = -1;
        vector<int> lower, upper;  // indices into blks
        vector<double> z;
    };
    struct Sub {
        vector<int> elems;                 // local rows in local order
        vector<vector<int>> lower, upper;  // per local row: block ids used by the solves
        vector<vector<std::pair<int,int>>> comms; // not used directly
        vector<vector<OvElem>> ov;         // per comm
        vector<int> comm_proc;
    };
    vector<int> lidx;                      // element -> local index on its owner
    vector<Sub> subs;
    vector<int> itrans;
    DBuf LD;                               // local L blocks and inv(D), packed as A
    int nsub = 0;

    void build(Mat& A) {
        nsub = 0;
        for (int e = 0; e < A.nelem; ++e) nsub = std::max(nsub, A.proc[e] + 1);
        subs.assign(nsub, {});
        lidx.assign(A.nelem, -1);
        for (int e = 0; e < A.nelem; ++e) {
            Sub& S = subs[A.proc[e]];
            lidx[e] = (int)S.elems.size();
            S.elems.push_back(e);
        }
        itrans.assign(A.nblk, -1);
        for (int e = 0; e < A.nelem; ++e)
            for (int k : A.lblk[A.row(e, 0)]) {
                const int p = A.ce[k];
                if (A.proc[p] != A.proc[e]) continue;
                for (int kk : A.lblk[A.row(p, 0)])
                    if (A.ce[kk] == e) { itrans[k] = kk; break; }
            }
        for (int s = 0; s < nsub; ++s) {
            Sub& S = subs[s];
            const int nl = (int)S.elems.size();
            S.lower.assign(nl, {});
            S.upper.assign(nl, {});
            for (int i = 0; i < nl; ++i) {
                const int e = S.elems[i];
                for (int k : A.lblk[A.row(e, 0)]) {
                    const int p = A.ce[k];
                    if (p == e) continue;
                    const int pp = A.proc[p];
                    // type_domain_matrix.f90:295-302
                    const bool lo = (pp == s && lidx[p] < i) || (pp < s);
                    const bool up = (pp == s && lidx[p] > i) || (pp > s);
                    if (lo) S.lower[i].push_back(k);
                    else if (up) S.upper[i].push_back(k);
                }
            }
            // receive procs in order of first appearance (type_domain.f90 get_recv_procs_local)
            S.comm_proc.clear();
            for (int e : S.elems)
                for (int k : A.lblk[A.row(e, 0)]) {
                    const int pp = A.proc[A.ce[k]];
                    if (pp != s && std::find(S.comm_proc.begin(), S.comm_proc.end(), pp) == S.comm_proc.end())
                        S.comm_proc.push_back(pp);
                }
            S.ov.assign(S.comm_proc.size(), {});
            for (size_t ic = 0; ic < S.comm_proc.size(); ++ic) {
                const int q = S.comm_proc[ic];
                auto touches = [&](int f) {
                    for (int k : A.lblk[A.row(f, 0)])
                        if (A.ce[k] != f && A.proc[A.ce[k]] == s) return true;
                    return false;
                };
                vector<OvElem>& O = S.ov[ic];
                for (int f : subs[q].elems) {
                    if (!touches(f)) continue;
                    OvElem oe;
                    oe.elem = f;
                    oe.owner = q;
                    const auto& fb = A.lblk[A.row(f, 0)];
                    // (1) blocks coupling to the receiver (send_comm.f90:170-175)
                    for (int k : fb)
                        if (A.ce[k] != f && A.proc[A.ce[k]] == s) oe.blks.push_back({A.ce[k], true, k, -1, -1, {}});
                    // (2) blocks coupling to neighbours that are also sent (send_comm.f90:183-210)
                    for (int k : fb) {
                        const int nb = A.ce[k];
                        if (nb == f || A.proc[nb] != q) continue;
                        if (touches(nb)) oe.blks.push_back({nb, false, k, -1, -1, {}});
                    }
                    // (3) diagonal (send_comm.f90:216-218)
                    oe.diag = (int)oe.blks.size();
                    oe.blks.push_back({f, false, A.diag[A.row(f, 0)], -1, -1, {}});
                    O.push_back(std::move(oe));
                }
                // lower/upper and transposes (recv_dom_comm.f90:178-300)
                for (size_t ie = 0; ie < O.size(); ++ie) {
                    OvElem& oe = O[ie];
                    for (int ib = 0; ib < (int)oe.blks.size(); ++ib) {
                        OvBlk& bk = oe.blks[ib];
                        if (ib == oe.diag) { bk.trans_elem = (int)ie; bk.trans_src = bk.src; continue; }
                        if (!bk.parent_local) {
                            if (bk.parent < oe.elem) oe.lower.push_back(ib);
                            else if (bk.parent > oe.elem) oe.upper.push_back(ib);
                            for (size_t je = 0; je < O.size(); ++je)
                                if (O[je].elem == bk.parent) {
                                    for (auto& bb : O[je].blks)
                                        if (A.ce[bb.src] == oe.elem) { bk.trans_elem = (int)je; bk.trans_src = bb.src; break; }
                                    break;
                                }
                        } else {
                            oe.lower.push_back(ib);
                            for (int kk : A.lblk[A.row(bk.parent, 0)])
                                if (A.ce[kk] == oe.elem) { bk.trans_src = kk; break; }
                        }
                    }
                }
            }
        }
    }

    // precon_RASILU0.f90:205-415 (native branch)
    int update(Mat& A) override {
        if (A.ntime != 1) return ORC_EINVAL;   // single time level only (recv_dom_comm.f90:83)
        if (A.transposed) return ORC_EINVAL;   // "transpose not implemented for 'native' containers" (:254)
        err_elem = -1;
        LD.zeros(A.nval);
        // Subdomains share nothing they write (each plays its own rank), so
        // they factor on the pool; the failure reported is the one of the
        // first failing subdomain in order, as the serial loop reports it.
        vector<int> fail_elem(nsub, -1);
        Pool::get().run(nsub, [&](int64_t si) { fail_elem[si] = update_sub(A, (int)si); });
        for (int s = 0; s < nsub; ++s)
            if (fail_elem[s] >= 0) { err_elem = fail_elem[s]; return ORC_ESINGULAR; }
        stamp = A.stamp;
        return ORC_OK;
    }
    // one subdomain's factorisation; the element whose inverse failed, or -1
    int update_sub(Mat& A, int s) {
        {
            Sub& S = subs[s];
            for (int e : S.elems) {
                const int k = A.diag[A.row(e, 0)];
                std::memcpy(LD.data() + A.voff[k], A.blk(k), sizeof(double) * A.nr[k] * A.nc[k]);
            }
            for (size_t i = 0; i < S.elems.size(); ++i) {
                const int e = S.elems[i];
                const int kd = A.diag[A.row(e, 0)];
                double* D = LD.data() + A.voff[kd];
                const int b = A.nr[kd];
                if (i > 0)
                    for (int kl : S.lower[i]) {
                        const int p = A.ce[kl];
                        if (A.proc[p] != s) continue;   // parent_proc /= IRANK blocks are skipped
                        double* L = LD.data() + A.voff[kl];
                        gemm(A.nr[kl], A.nc[kl], A.nc[kl], A.blk(kl), LD.data() + A.voff[A.diag[A.row(p, 0)]], L);
                        const int kt = itrans[kl];
                        gemm_sub(b, A.nc[kt], A.nc[kl], L, A.blk(kt), D);
                    }
                if (inv_inplace(b, D) != 0) return e;
            }
            // overlap rows (received copies)
            for (auto& O : S.ov)
                for (auto& oe : O)
                    for (auto& bk : oe.blks)
                        bk.mat.assign(A.blk(bk.src), A.blk(bk.src) + (int64_t)A.nr[bk.src] * A.nc[bk.src]);
            for (auto& O : S.ov)
                for (size_t ie = 0; ie < O.size(); ++ie) {
                    OvElem& oe = O[ie];
                    OvBlk& dg = oe.blks[oe.diag];
                    const int b = A.nr[dg.src];
                    for (int ib : oe.lower) {
                        OvBlk& bk = oe.blks[ib];
                        const int m = A.nr[bk.src], nn = A.nc[bk.src];
                        vector<double> tmp((size_t)m * nn);
                        if (!bk.parent_local) {
                            OvElem& pe = O[bk.trans_elem];
                            gemm(m, nn, nn, bk.mat.data(), pe.blks[pe.diag].mat.data(), tmp.data());
                            bk.mat = tmp;
                            const OvBlk* tb = nullptr;
                            for (auto& bb : pe.blks) if (bb.src == bk.trans_src) { tb = &bb; break; }
                            gemm_sub(b, A.nc[bk.trans_src], nn, bk.mat.data(), tb->mat.data(), dg.mat.data());
                        } else {
                            const int kpd = A.diag[A.row(bk.parent, 0)];
                            gemm(m, nn, nn, bk.mat.data(), LD.data() + A.voff[kpd], tmp.data());
                            bk.mat = tmp;
                            gemm_sub(b, A.nc[bk.trans_src], nn, bk.mat.data(), A.blk(bk.trans_src), dg.mat.data());
                        }
                    }
                    if (inv_inplace(b, dg.mat.data()) != 0) return oe.elem;
                }
        }
        return -1;
    }

    // precon_RASILU0.f90:454-625 (native branch)
    int apply(Mat& A, const double* v, double* z) override {
        if (A.transposed) return ORC_EINVAL;   // "not implemented for transposed matrices" (:494)
        vector<double> zl(A.n);
        std::memcpy(zl.data(), v, sizeof(double) * A.n);  // each subdomain only touches its own rows
        // subdomains write disjoint rows of zl and their own overlap copies
        Pool::get().run(nsub, [&](int64_t si) {
            const int s = (int)si;
            vector<double> tmp;
            Sub& S = subs[s];
            // halo of v for the overlap elements (z%comm_send/recv)
            for (auto& O : S.ov)
                for (auto& oe : O) oe.z.assign(v + A.seg(oe.elem, 0), v + A.seg(oe.elem, 0) + A.bsize(oe.elem));
            auto ovz = [&](int ic, int elem) -> double* {
                for (auto& oe : S.ov[ic]) if (oe.elem == elem) return oe.z.data();
                return nullptr;
            };
            auto anyovz = [&](int elem) -> double* {
                for (size_t ic = 0; ic < S.ov.size(); ++ic) { double* p = ovz((int)ic, elem); if (p) return p; }
                return nullptr;
            };
            // forward, local rows
            for (size_t i = 0; i < S.elems.size(); ++i) {
                const int e = S.elems[i];
                for (int kl : S.lower[i]) {
                    const int p = A.ce[kl];
                    if (A.proc[p] != s) continue;
                    gemv_sub(A.nr[kl], A.nc[kl], LD.data() + A.voff[kl], zl.data() + A.seg(p, 0), zl.data() + A.seg(e, 0));
                }
            }
            // forward, overlap rows
            for (size_t ic = 0; ic < S.ov.size(); ++ic)
                for (auto& oe : S.ov[ic])
                    for (int ib : oe.lower) {
                        OvBlk& bk = oe.blks[ib];
                        const double* xp = bk.parent_local ? zl.data() + A.seg(bk.parent, 0) : ovz((int)ic, bk.parent);
                        gemv_sub(A.nr[bk.src], A.nc[bk.src], bk.mat.data(), xp, oe.z.data());
                    }
            // backward, overlap rows
            for (int ic = (int)S.ov.size() - 1; ic >= 0; --ic)
                for (int ie = (int)S.ov[ic].size() - 1; ie >= 0; --ie) {
                    OvElem& oe = S.ov[ic][ie];
                    for (int ib : oe.upper) {
                        OvBlk& bk = oe.blks[ib];
                        gemv_sub(A.nr[bk.src], A.nc[bk.src], bk.mat.data(), ovz(ic, bk.parent), oe.z.data());
                    }
                    const int b = (int)oe.z.size();
                    tmp.assign(b, 0.0);
                    gemv_acc(b, b, oe.blks[oe.diag].mat.data(), oe.z.data(), tmp.data());
                    oe.z = tmp;
                }
            // backward, local rows
            for (int i = (int)S.elems.size() - 1; i >= 0; --i) {
                const int e = S.elems[i];
                double* ze = zl.data() + A.seg(e, 0);
                for (int ku : S.upper[i]) {
                    const int p = A.ce[ku];
                    const double* xp = (A.proc[p] == s) ? zl.data() + A.seg(p, 0) : anyovz(p);
                    gemv_sub(A.nr[ku], A.nc[ku], A.blk(ku), xp, ze);
                }
                const int kd = A.diag[A.row(e, 0)];
                const int b = A.nr[kd];
                tmp.assign(b, 0.0);
                gemv_acc(b, b, LD.data() + A.voff[kd], ze, tmp.data());
                std::memcpy(ze, tmp.data(), sizeof(double) * b);
            }
        });
        std::memcpy(z, zl.data(), sizeof(double) * A.n);
        return ORC_OK;
    }
};

// precon_HB (precon_HB.f90:169-310): per element one matrix over all its time
// levels, the DIAG block of level t at (t, t) and D(ta,tb) mass per field at
// (ta, tb), inverted (inv) and applied to the element's whole segment.  The
// hb_blks block of row (e,ta) and column (e,tb) holds D(ta,tb) mass per field
// (type_harmonic_balance.f90:127-229), so it is the (ta, tb) entry here.  Like
// the reference, A's own blocks are used whether or not A is transposed.
struct PreconHB : Precon {
    vector<vector<double>> inv;        // per element, (nt*b)^2 column-major
    int update(Mat& A) override {
        err_elem = -1;
        inv.assign(A.nelem, {});
        for (int e = 0; e < A.nelem; ++e) {
            const int b = A.bsize(e), B = b * A.ntime;
            vector<double>& M = inv[e];
            M.assign((size_t)B * B, 0.0);
            auto put = [&](int k, int ta, int tb) {
                const double* src = A.blk(k);
                for (int j = 0; j < b; ++j)
                    for (int i = 0; i < b; ++i) M[(size_t)(ta * b + i) + (size_t)(tb * b + j) * B] = src[i + (size_t)j * b];
            };
            for (int ta = 0; ta < A.ntime; ++ta) {
                put(A.diag[A.row(e, ta)], ta, ta);
                for (int k : A.rowblk[A.row(e, ta)])
                    if (A.kind[k] == ORC_BLK_HB && A.ce[k] == e && A.ct[k] != ta) put(k, ta, A.ct[k]);
            }
            if (inv_inplace(B, M.data()) != 0) { err_elem = e; return ORC_ESINGULAR; }
        }
        stamp = A.stamp;
        return ORC_OK;
    }
    int apply(Mat& A, const double* v, double* z) override {
        for (int e = 0; e < A.nelem; ++e) {
            const int B = A.bsize(e) * A.ntime;
            const double* ve = v + A.eoff[e];
            double* ze = z + A.eoff[e];
            std::fill(ze, ze + B, 0.0);
            gemv_acc(B, B, inv[e].data(), ve, ze);
        }
        return ORC_OK;
    }
};

// ---------------------------------------------------------------------------
// Vector kernels
// ---------------------------------------------------------------------------
// transposed_matrix_vector_product, local part (operator_chidg_mv.f90:692-1049):
// per time level, each lblks / chi_blks / bc_blks block of row (e,t) adds its
// transpose times x(e,t) into its parent's segment; then the harmonic-balance
// term y(e,t) += D(t',t) mass^T x(e,t') for t' /= t.  The hb_blks block of row
// (e,t') and column (e,t) holds D(t',t) mass per field
// (type_harmonic_balance.f90:127-229), so that term is its transpose times x(e,t').
void mtv(const Mat& A, const double* x, double* y) {
    std::fill(y, y + A.n, 0.0);
    for (int t = 0; t < A.ntime; ++t) {
        for (int e = 0; e < A.nelem; ++e) {
            const double* xe = x + A.seg(e, t);
            for (int k : A.rowblk[A.row(e, t)])
                if (A.kind[k] != ORC_BLK_HB) gemv_t_acc(A.nr[k], A.nc[k], A.blk(k), xe, y + A.seg(A.ce[k], A.ct[k]));
        }
        for (int e = 0; e < A.nelem; ++e)
            for (int ti = 0; ti < A.ntime; ++ti) {
                if (ti == t) continue;
                for (int k : A.rowblk[A.row(e, ti)])
                    if (A.kind[k] == ORC_BLK_HB && A.ce[k] == e && A.ct[k] == t)
                        gemv_t_acc(A.nr[k], A.nc[k], A.blk(k), x + A.seg(e, ti), y + A.seg(e, t));
            }
    }
}

// chidg_mv (operator_chidg_mv.f90:46-60 selects the transposed product when
// A%transposed), non-transposed local part :117-410
void mv(const Mat& A, const double* x, double* y) {
    if (A.transposed) { mtv(A, x, y); return; }
    // rows are independent: each row's sum runs in the serial order on one thread
    Pool::get().run((int64_t)A.nelem * A.ntime, [&](int64_t r) {
        const int e = (int)(r / A.ntime), t = (int)(r % A.ntime);
        double* ye = y + A.seg(e, t);
        std::fill(ye, ye + A.bsize(e), 0.0);
        for (int k : A.rowblk[A.row(e, t)])
            gemv_acc(A.nr[k], A.nc[k], A.blk(k), x + A.seg(A.ce[k], A.ct[k]), ye);
    });
}
double dotv(int64_t n, const double* x, const double* y) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}

// ---------------------------------------------------------------------------
// FGMRES (type_fgmres.f90:81-310) with CGS/MGS (:331-442)
// ---------------------------------------------------------------------------
struct Controller {                  // type_solver_controller.f90
    long lhs_stamp = 0;
    bool force = false;
    bool update_preconditioner(const Mat& A, const Precon& M) {
        const bool u = (lhs_stamp != A.stamp) || force || (A.stamp != M.stamp);
        lhs_stamp = A.stamp;
        force = false;
        return u;
    }
};

struct Fgmres {
    double tol, rtol;
    int nmax, nkrylov, orth;
    bool inner;
    double inner_tol, inner_rtol;
    int inner_nmax, inner_nkrylov, inner_orth;
    int niter = 0, nrestart = 0;
    double residual_norm = 0.0, res_est = 0.0, r0norm_initial = 0.0;
    vector<double>* hist = nullptr;
    std::unique_ptr<Fgmres> child;

    void orthogonalize(const Mat& A, vector<double>& w, const vector<vector<double>>& v, int j,
                       vector<double>& hcol, vector<double>& htmp) {
        const int64_t n = A.n;
        Pool& pool = Pool::get();
        if (orth == 0) {            // CGS (:331-396)
            // the j dots are independent (each a serial sum); every entry of w
            // takes its j updates in order
            pool.run(j, [&](int64_t i) { htmp[i] = dotv(n, w.data(), v[i].data()); });
            pool.run_chunks(n, kGrain, [&](int64_t q0, int64_t q1) {
                for (int i = 0; i < j; ++i) {
                    const double hi = htmp[i];
                    const double* vi = v[i].data();
                    for (int64_t q = q0; q < q1; ++q) w[q] = w[q] - hi * vi[q];
                }
            });
        } else {                    // MGS (:417-442)
            for (int i = 0; i < j; ++i) {
                htmp[i] = dotv(n, w.data(), v[i].data());
                const double hi = htmp[i];
                const double* vi = v[i].data();
                pool.run_chunks(n, kGrain, [&](int64_t q0, int64_t q1) {
                    for (int64_t q = q0; q < q1; ++q) w[q] = w[q] - hi * vi[q];
                });
            }
        }
        for (int i = 0; i < j; ++i) hcol[i] += htmp[i];
    }

    int solve(Mat& A, vector<double>& x, const vector<double>& b, Precon& M, Controller* ctl) {
        const int64_t n = A.n;
        if (inner) {
            if (!child) child.reset(new Fgmres());
            child->nkrylov = inner_nkrylov; child->tol = inner_tol; child->rtol = inner_rtol;
            child->nmax = inner_nmax; child->orth = inner_orth; child->inner = false;
        }
        int st;
        if (ctl) { if (ctl->update_preconditioner(A, M)) { st = M.update(A); if (st) return st; } }
        else { st = M.update(A); if (st) return st; }

        const int m = nkrylov;
        vector<vector<double>> v(m + 1, vector<double>(n)), z(m + 1, vector<double>(n));
        vector<double> p(m + 1), y(m + 1), c(m + 1), s(m + 1), htmp(m + 1);
        vector<double> h((size_t)(m + 1) * m);   // column-major (m+1) x m
        auto H = [&](int i, int j) -> double& { return h[(size_t)i + (size_t)j * (m + 1)]; };
        vector<double> x0(n, 0.0), w(n), r0(n), zr(n), deltaz(n, 0.0);
        std::fill(x.begin(), x.end(), 0.0);

        niter = 0; nrestart = 0;
        double res = DBL_MAX;
        bool cabs = false, crel = false, cmax = false;
        while (res > tol) {
            for (auto& q : v) std::fill(q.begin(), q.end(), 0.0);
            for (auto& q : z) std::fill(q.begin(), q.end(), 0.0);
            std::fill(p.begin(), p.end(), 0.0); std::fill(y.begin(), y.end(), 0.0);
            std::fill(c.begin(), c.end(), 0.0); std::fill(s.begin(), s.end(), 0.0);
            std::fill(h.begin(), h.end(), 0.0); std::fill(htmp.begin(), htmp.end(), 0.0);

            mv(A, x0.data(), r0.data());
            for (int64_t q = 0; q < n; ++q) r0[q] = b[q] - r0[q];
            const double r0norm = std::sqrt(dotv(n, r0.data(), r0.data()));
            for (int64_t q = 0; q < n; ++q) v[0][q] = r0[q] / r0norm;
            p[0] = r0norm;
            if (niter == 0) r0norm_initial = r0norm;
            int nvecs = 0;
            for (int j = 1; j <= m; ++j) {
                nvecs++;
                st = M.apply(A, v[j - 1].data(), z[j - 1].data());
                if (st) return st;
                if (inner) {
                    mv(A, z[j - 1].data(), zr.data());
                    for (int64_t q = 0; q < n; ++q) zr[q] = v[j - 1][q] - zr[q];
                    st = child->solve(A, deltaz, zr, M, ctl);
                    if (st) return st;
                    for (int64_t q = 0; q < n; ++q) z[j - 1][q] = z[j - 1][q] + deltaz[q];
                }
                mv(A, z[j - 1].data(), w.data());
                const double norm_before = std::sqrt(dotv(n, w.data(), w.data()));
                vector<double> hcol(j, 0.0);
                orthogonalize(A, w, v, j, hcol, htmp);
                double crit = 0.0;
                for (int i = 0; i < j; ++i) crit += std::fabs(hcol[i]);
                crit /= norm_before;
                if (crit >= 1.0) orthogonalize(A, w, v, j, hcol, htmp);
                for (int i = 0; i < j; ++i) H(i, j - 1) = hcol[i];
                H(j, j - 1) = std::sqrt(dotv(n, w.data(), w.data()));
                for (int64_t q = 0; q < n; ++q) v[j][q] = w[q] / H(j, j - 1);
                for (int i = 0; i < j - 1; ++i) {
                    const double hij = c[i] * H(i, j - 1) + s[i] * H(i + 1, j - 1);
                    const double hipj = -s[i] * H(i, j - 1) + c[i] * H(i + 1, j - 1);
                    H(i, j - 1) = hij;
                    H(i + 1, j - 1) = hipj;
                }
                const double gam = std::hypot(H(j - 1, j - 1), H(j, j - 1));
                c[j - 1] = H(j - 1, j - 1) / gam;
                s[j - 1] = H(j, j - 1) / gam;
                H(j - 1, j - 1) = gam;
                H(j, j - 1) = 0.0;
                const double pj = c[j - 1] * p[j - 1];
                const double pjp = -s[j - 1] * p[j - 1];
                p[j - 1] = pj;
                p[j] = pjp;
                niter++;
                res = std::fabs(p[j]);
                if (hist) hist->push_back(res);
                cabs = (res < tol);
                crel = (res / r0norm_initial < rtol);
                cmax = (niter >= nmax) && (nmax > 0);
                if (cabs || crel || cmax) break;
            }
            // y = inv(H(1:n,1:n)) * p(1:n)   (:287-288)
            vector<double> Hn((size_t)nvecs * nvecs);
            for (int jj = 0; jj < nvecs; ++jj)
                for (int ii = 0; ii < nvecs; ++ii) Hn[ii + (size_t)jj * nvecs] = H(ii, jj);
            if (inv_inplace(nvecs, Hn.data()) != 0) {
                // singular Hessenberg: the reference stops with FATAL; report it
                return ORC_ESINGULAR;
            }
            for (int ii = 0; ii < nvecs; ++ii) {
                double sacc = 0.0;
                for (int jj = 0; jj < nvecs; ++jj) sacc += Hn[ii + (size_t)jj * nvecs] * p[jj];
                y[ii] = sacc;
            }
            x = x0;
            Pool::get().run_chunks(n, kGrain, [&](int64_t q0, int64_t q1) {
                for (int iv = 0; iv < nvecs; ++iv) {
                    const double yi = y[iv];
                    const double* zi = z[iv].data();
                    for (int64_t q = q0; q < q1; ++q) x[q] = x[q] + yi * zi[q];
                }
            });
            res_est = res;
            if (cabs || crel || cmax) break;
            x0 = x;
            nrestart++;
        }
        // print_report: true residual (:512-520)
        mv(A, x.data(), w.data());
        for (int64_t q = 0; q < n; ++q) w[q] = b[q] - w[q];
        residual_norm = std::sqrt(dotv(n, w.data(), w.data()));
        return ORC_OK;
    }
};

}  // namespace

struct orc_matrix { Mat m; };
struct orc_precon { std::unique_ptr<Precon> p; };

extern "C" {

orc_matrix* orc_matrix_create(int32_t nelem, int32_t ntime, const int32_t* elem_nvars,
                              const int32_t* elem_nterms, const int32_t* elem_proc, int64_t nblocks,
                              const int32_t* bre, const int32_t* brt, const int32_t* bce,
                              const int32_t* bct, const int32_t* bkind) {
    if (nelem <= 0 || ntime <= 0 || nblocks <= 0) return nullptr;
    auto* h = new orc_matrix();
    Mat& A = h->m;
    A.nelem = nelem; A.ntime = ntime;
    A.nvars.assign(elem_nvars, elem_nvars + nelem);
    A.nterms.assign(elem_nterms, elem_nterms + nelem);
    A.proc.assign(nelem, 0);
    if (elem_proc) A.proc.assign(elem_proc, elem_proc + nelem);
    A.eoff.resize(nelem);
    int64_t off = 0;
    for (int e = 0; e < nelem; ++e) { A.eoff[e] = off; off += (int64_t)ntime * A.bsize(e); }
    A.n = off;
    A.nblk = nblocks;
    A.re.assign(bre, bre + nblocks); A.rt.assign(brt, brt + nblocks);
    A.ce.assign(bce, bce + nblocks); A.ct.assign(bct, bct + nblocks);
    A.kind.assign(bkind, bkind + nblocks);
    A.nr.resize(nblocks); A.nc.resize(nblocks); A.voff.resize(nblocks);
    const int nrow = nelem * ntime;
    A.rowblk.assign(nrow, {});
    A.lblk.assign(nrow, {});
    A.diag.assign(nrow, -1);
    int64_t v = 0;
    for (int64_t k = 0; k < nblocks; ++k) {
        if (A.re[k] < 0 || A.re[k] >= nelem || A.ce[k] < 0 || A.ce[k] >= nelem ||
            A.rt[k] < 0 || A.rt[k] >= ntime || A.ct[k] < 0 || A.ct[k] >= ntime) { delete h; return nullptr; }
        A.nr[k] = A.bsize(A.re[k]);
        A.nc[k] = A.bsize(A.ce[k]);
        A.voff[k] = v;
        v += (int64_t)A.nr[k] * A.nc[k];
    }
    A.nval = v;
    A.val.zeros(v);
    for (int kind = 0; kind < 4; ++kind)
        for (int64_t k = 0; k < nblocks; ++k) {
            if (A.kind[k] != kind) continue;
            const int r = A.row(A.re[k], A.rt[k]);
            A.rowblk[r].push_back((int)k);
            if (kind == ORC_BLK_LOCAL) {
                if (A.ct[k] != A.rt[k]) { delete h; return nullptr; }
                A.lblk[r].push_back((int)k);
                if (A.ce[k] == A.re[k]) A.diag[r] = (int)k;
            }
        }
    for (int r = 0; r < nrow; ++r) if (A.diag[r] < 0) { delete h; return nullptr; }
    return h;
}
void orc_matrix_destroy(orc_matrix* h) { delete h; }
int64_t orc_matrix_nvalues(const orc_matrix* h) { return h->m.nval; }
int64_t orc_matrix_nvec(const orc_matrix* h) { return h->m.n; }
int orc_matrix_set_values(orc_matrix* h, const double* packed) {
    h->m.val.copy_from(packed);
    h->m.stamp++;
    return ORC_OK;
}
int orc_matrix_get_values(const orc_matrix* h, double* packed) {
    h->m.val.copy_to(packed);
    return ORC_OK;
}
int orc_matrix_block_offsets(const orc_matrix* h, int64_t* offsets) {
    for (int64_t k = 0; k < h->m.nblk; ++k) offsets[k] = h->m.voff[k];
    return ORC_OK;
}
void orc_matrix_touch(orc_matrix* h) { h->m.stamp++; }
int orc_matrix_set_transposed(orc_matrix* h, int32_t transposed) { h->m.transposed = transposed != 0; return ORC_OK; }
int orc_mv(orc_matrix* h, const double* x, double* y) { mv(h->m, x, y); return ORC_OK; }
double orc_dot(const orc_matrix* h, const double* x, const double* y) { return dotv(h->m.n, x, y); }
double orc_norm(const orc_matrix* h, const double* x) { return std::sqrt(dotv(h->m.n, x, x)); }
int orc_set_threads(int32_t n) {
    if (n < 1) return ORC_EINVAL;
    Pool::get().set_threads(n);
    return ORC_OK;
}
int32_t orc_get_threads(void) { return Pool::get().threads(); }
int orc_inv(int32_t n, const double* a, double* ainv) {
    std::memcpy(ainv, a, sizeof(double) * n * n);
    return inv_inplace(n, ainv) ? ORC_ESINGULAR : ORC_OK;
}

orc_precon* orc_precon_create(orc_matrix* h, int32_t kind) {
    auto* pc = new orc_precon();
    switch (kind) {
        case ORC_PRECON_IDENTITY: pc->p.reset(new PreconIdentity()); break;
        case ORC_PRECON_JACOBI: { auto* q = new PreconILU0(); q->jacobi = true; q->build(h->m); pc->p.reset(q); break; }
        case ORC_PRECON_ILU0: { auto* q = new PreconILU0(); q->build(h->m); pc->p.reset(q); break; }
        case ORC_PRECON_HB: pc->p.reset(new PreconHB()); break;
        case ORC_PRECON_RASILU0: {
            if (h->m.ntime != 1) { delete pc; return nullptr; }
            auto* q = new PreconRAS(); q->build(h->m); pc->p.reset(q); break;
        }
        default: delete pc; return nullptr;
    }
    pc->p->kind = kind;
    return pc;
}
void orc_precon_destroy(orc_precon* pc) { delete pc; }
int orc_precon_update(orc_precon* pc, orc_matrix* h) { return pc->p->update(h->m); }
int orc_precon_apply(orc_precon* pc, orc_matrix* h, const double* v, double* z) { return pc->p->apply(h->m, v, z); }
int orc_precon_error_elem(const orc_precon* pc) { return pc->p->err_elem; }
int orc_precon_get_LD(const orc_precon* pc, double* packed) {
    auto* q = dynamic_cast<PreconILU0*>(pc->p.get());
    if (q) { q->LD.copy_to(packed); return ORC_OK; }
    auto* r = dynamic_cast<PreconRAS*>(pc->p.get());
    if (r) { r->LD.copy_to(packed); return ORC_OK; }
    return ORC_EINVAL;
}

int orc_fgmres_solve(orc_matrix* h, orc_precon* pc, const double* b, double* x,
                     const orc_fgmres_opts* o, orc_fgmres_result* res, double* hist, int32_t hist_cap) {
    Fgmres f;
    f.tol = o->tol; f.rtol = o->rtol; f.nmax = o->nmax; f.nkrylov = o->nkrylov;
    f.orth = o->orthogonalization; f.inner = o->inner_fgmres != 0;
    f.inner_tol = o->inner_tol; f.inner_rtol = o->inner_rtol; f.inner_nmax = o->inner_nmax;
    f.inner_nkrylov = o->inner_nkrylov; f.inner_orth = o->inner_orthogonalization;
    vector<double> hv;
    f.hist = &hv;
    Controller ctl;
    vector<double> xb(h->m.n), bb(b, b + h->m.n);
    const int st = f.solve(h->m, xb, bb, *pc->p, o->use_controller ? &ctl : nullptr);
    std::memcpy(x, xb.data(), sizeof(double) * h->m.n);
    if (res) {
        res->niter = f.niter; res->nrestart = f.nrestart;
        res->residual_norm = f.residual_norm; res->res_estimate = f.res_est;
        res->r0norm_initial = f.r0norm_initial;
        res->nhist = (int32_t)std::min<size_t>(hv.size(), (size_t)std::max(hist_cap, 0));
    }
    if (hist) for (int i = 0; i < (int)hv.size() && i < hist_cap; ++i) hist[i] = hv[i];
    return st;
}

}  // extern "C"
