// batch.cu -- many independent FGMRES solves sharing every GPU launch.
//
// The systems are packed block-diagonally into one chidg_gpu_matrix: system s
// owns elements [sys_elem[s], sys_elem[s+1]) and no block couples two systems.
// One matvec, one preconditioner sweep and one segmented reduction per Arnoldi
// step serve all systems at once, while every system keeps its own Arnoldi
// process exactly as fgmres_t%solve runs it (type_fgmres.f90:81-310): its own
// dot products, selective re-orthogonalisation, Givens rotations, convergence
// test and solution update.  Systems advance in lockstep through the Krylov
// index j; a converged system is frozen (its coefficients become zero) while
// the others continue, and all systems restart together at j = nkrylov.
#include "chidg_gpu_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstring>

using namespace chidg;

namespace {

constexpr int64_t kChunk = 2048;

// the segment layout of one batched call; its device buffers belong to the
// context and are reused by the next call
struct Seg {
    int nsys = 0, nchunk = 0;
    Buffer &cstart, &csys, &sys_chunk, &sys_row, &d_out, &d_coef, &d_scale, &partial, &rowsq;
    std::vector<int32_t> h_sys_chunk;
    explicit Seg(BatchBuffers& b)
        : cstart(b.cstart), csys(b.csys), sys_chunk(b.sys_chunk), sys_row(b.sys_row), d_out(b.d_out), d_coef(b.d_coef),
          d_scale(b.d_scale), partial(b.partial), rowsq(b.rowsq) {}
};

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

// Explicit inverse with partial pivoting of a small dense matrix (the
// Hessenberg least squares, mod_inv::inv semantics).
int small_inverse(int n, std::vector<double>& a) {
    std::vector<int> piv(n), used(n, 0);
    for (int k = 0; k < n; ++k) {
        int p = -1;
        double best = -1.0;
        for (int i = 0; i < n; ++i) {
            if (used[i]) continue;
            double v = std::fabs(a[i + (size_t)k * n]);
            if (!(v == v)) v = INFINITY;
            if (v > best) { best = v; p = i; }
        }
        piv[k] = p;
        used[p] = 1;
        const double pv = a[p + (size_t)k * n];
        if (pv == 0.0) return k + 1;
        const double rp = 1.0 / pv;
        std::vector<double> row(n), col(n);
        for (int j = 0; j < n; ++j) row[j] = ((j == k) ? 1.0 : a[p + (size_t)j * n]) * rp;
        for (int i = 0; i < n; ++i) col[i] = (i == p) ? 0.0 : a[i + (size_t)k * n];
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                if (i == p) a[i + (size_t)j * n] = row[j];
                else {
                    const double base = (j == k) ? 0.0 : a[i + (size_t)j * n];
                    a[i + (size_t)j * n] = base - col[i] * row[j];
                }
            }
    }
    std::vector<int> q(n);
    for (int k = 0; k < n; ++k) q[piv[k]] = k;
    std::vector<double> out((size_t)n * n);
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) out[q[i] + (size_t)piv[j] * n] = a[i + (size_t)j * n];
    a.swap(out);
    return 0;
}

struct SysState {
    bool active = true;
    int niter = 0, nrestart = 0, nvecs = 0;
    double r0norm_initial = 0.0, res = DBL_MAX, res_est = 0.0, residual_norm = 0.0;
    std::vector<double> p, c, s, h;
    std::vector<double> hist;
};

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
    // FP64 Krylov vectors in every batched mode; MIXED_PRECON_FP32 applies the
    // preconditioner with FP32 copies of its blocks
    if (o.precision != CHIDG_GPU_FP64 && o.precision != CHIDG_GPU_MIXED_PRECON_FP32)
        return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: precision must be FP64 or MIXED_PRECON_FP32");
    const int prec = o.precision;
    const int m = o.nkrylov;
    if (m < 1 || m > kMaxKrylov) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: nkrylov outside [1, 4000]");
    // segments: systems must tile the elements and not couple to each other
    if (sys_elem[0] != 0 || sys_elem[nsys] != A->nelem) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: systems must cover all elements");
    std::vector<int> elem_sys(A->nelem);
    for (int s = 0; s < nsys; ++s) {
        if (sys_elem[s + 1] <= sys_elem[s]) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: empty or unordered system");
        for (int e = sys_elem[s]; e < sys_elem[s + 1]; ++e) elem_sys[e] = s;
    }
    for (int64_t k = 0; k < A->nblk; ++k)
        if (elem_sys[A->re[k]] != elem_sys[A->ce[k]]) return fail(ctx, CHIDG_GPU_EINVAL, "batched fgmres: a block couples two systems");
    Seg G(ctx->batch);
    G.nsys = nsys;
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
    G.nchunk = (int)csys.size();
    int st;
    if ((st = upload_vec(ctx, G.cstart, cstart)) || (st = upload_vec(ctx, G.csys, csys)) ||
        (st = upload_vec(ctx, G.sys_chunk, sys_chunk)) || (st = upload_vec(ctx, G.sys_row, sys_row)))
        return st;
    const int hst = m + 2;   // per-system stride of the device output / coefficient rows
    if ((st = ensure(ctx, G.d_out, sizeof(double) * (size_t)nsys * hst)) ||
        (st = ensure(ctx, G.d_coef, sizeof(double) * (size_t)nsys * hst)) ||
        (st = ensure(ctx, G.d_scale, sizeof(double) * (size_t)nsys)) ||
        (st = ensure(ctx, G.partial, sizeof(double) * (size_t)G.nchunk * std::max(m, 1))) ||
        (st = ensure(ctx, G.rowsq, sizeof(double) * (size_t)A->nrow)))
        return st;
    const int64_t* CS = (const int64_t*)G.cstart.ptr;
    const int32_t* CY = (const int32_t*)G.csys.ptr;
    const int32_t* SC = (const int32_t*)G.sys_chunk.ptr;
    const int32_t* SR = (const int32_t*)G.sys_row.ptr;
    double* OUT = (double*)G.d_out.ptr;
    double* COEF = (double*)G.d_coef.ptr;
    double* SCALE = (double*)G.d_scale.ptr;
    double* PART = (double*)G.partial.ptr;
    double* ROWSQ = (double*)G.rowsq.ptr;

    // M%update as the controller decides (type_fgmres.f90:118-122)
    if (!(o.use_controller && M->stamp == A->stamp && M->precision == prec))
        if ((st = chidg_gpu_precon_update(M, A, prec))) return st;
    // from here on A is the operator: A, or A^T when A->transposed (same rows and segments)
    if ((st = matrix_op(A, &A))) return st;
    set_matvec_smem(A);
    if (M->kind != CHIDG_PRECON_IDENTITY) precon_set_smem(M);
    cudaMemsetAsync(ctx->d_scal + kSlotStatus, 0, sizeof(double), ctx->stream);

    const int64_t n = A->n;
    // the Krylov basis and work vectors of the context's FP64 workspace (a
    // context runs one solve at a time)
    Buffer& V = ctx->ws64.V;
    Buffer& Z = ctx->ws64.Z;
    Buffer& X0 = ctx->ws64.x0;
    Buffer& TMP = ctx->ws64.tmp;
    auto cleanup = [&]() {};
    if ((st = ensure(ctx, V, sizeof(double) * (size_t)(m + 1) * n)) || (st = ensure(ctx, Z, sizeof(double) * (size_t)(m + 1) * n)) ||
        (st = ensure(ctx, X0, sizeof(double) * (size_t)n)) || (st = ensure(ctx, TMP, sizeof(double) * (size_t)n))) {
        cleanup();
        return st;
    }
    double* Vb = (double*)V.ptr;
    double* Zb = (double*)Z.ptr;
    double* x0 = (double*)X0.ptr;
    double* xx = (double*)x->buf.ptr;
    const double* bb = (const double*)b->buf.ptr;
    cudaMemsetAsync(x0, 0, sizeof(double) * n, ctx->stream);
    cudaMemsetAsync(xx, 0, sizeof(double) * n, ctx->stream);

    std::vector<SysState> S(nsys);
    for (auto& q : S) {
        q.p.assign(m + 1, 0.0); q.c.assign(m + 1, 0.0); q.s.assign(m + 1, 0.0);
        q.h.assign((size_t)(m + 1) * m, 0.0);
    }
    std::vector<double> hout((size_t)nsys * hst), coef((size_t)nsys * hst), scale(nsys);
    const int TH = 256;
    auto check = [&](const char* what) { return check_launch(ctx, what); };
    // per-system sums of squares of the rows just written by the matvec
    auto rows_to_sys = [&](double* dst) {
        k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(ROWSQ, A->nrow, SR, 1, dst, 1);
        return check("k_seg_reduce rows");
    };
    auto fetch = [&](const double* dsrc, size_t count, double* hdst) -> int {
        cudaError_t e = cudaMemcpyAsync(hdst, dsrc, sizeof(double) * count, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        return e == cudaSuccess ? CHIDG_GPU_OK : cuda_fail(ctx, e, "batched fgmres scalars");
    };
    auto push = [&](double* ddst, const double* hsrc, size_t count) -> int {
        const cudaError_t e = cudaMemcpyAsync(ddst, hsrc, sizeof(double) * count, cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) return cudaStreamSynchronize(ctx->stream) == cudaSuccess ? CHIDG_GPU_OK : CHIDG_GPU_ECUDA;
        return cuda_fail(ctx, e, "batched fgmres coefficients");
    };
    // x (and x0) += sum_q coef[s][q] z_q for the systems with nonzero rows of coef
    auto update_solution = [&](int nq) -> int {
        if ((st = push(COEF, coef.data(), coef.size()))) return st;
        k_seg_lincomb<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, CY, xx, x0, Zb, n, nq, COEF, hst);
        if ((st = check("k_seg_lincomb x"))) return st;
        k_seg_lincomb<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, CY, x0, x0, Zb, n, nq, COEF, hst);
        return check("k_seg_lincomb x0");
    };
    auto solve_ls = [&](SysState& q, int nv, double* y) -> int {
        std::vector<double> Hn((size_t)nv * nv);
        for (int jj = 0; jj < nv; ++jj)
            for (int ii = 0; ii < nv; ++ii) Hn[ii + (size_t)jj * nv] = q.h[ii + (size_t)jj * (m + 1)];
        if (small_inverse(nv, Hn) != 0) return fail(ctx, CHIDG_GPU_ESINGULAR, "batched fgmres: singular Hessenberg matrix");
        for (int ii = 0; ii < nv; ++ii) {
            double acc = 0.0;
            for (int jj = 0; jj < nv; ++jj) acc += Hn[ii + (size_t)jj * nv] * q.p[jj];
            y[ii] = acc;
        }
        return CHIDG_GPU_OK;
    };

    int nactive = nsys;
    while (nactive > 0) {
        // r0 = b - A x0 into V(1), per-system norms
        if ((st = matvec_launch<double, double>(A, (const double*)A->val.ptr, x0, Vb, bb, -1.0, 1.0, ROWSQ)) ||
            (st = rows_to_sys(OUT)) || (st = fetch(OUT, nsys, hout.data()))) { cleanup(); return st; }
        for (int s = 0; s < nsys; ++s) {
            SysState& q = S[s];
            std::fill(q.p.begin(), q.p.end(), 0.0); std::fill(q.c.begin(), q.c.end(), 0.0);
            std::fill(q.s.begin(), q.s.end(), 0.0); std::fill(q.h.begin(), q.h.end(), 0.0);
            scale[s] = 0.0;
            if (!q.active) continue;
            const double r0n = std::sqrt(hout[s]);
            if (!std::isfinite(r0n)) { cleanup(); ctx->err_elem = sys_elem[s]; return fail(ctx, CHIDG_GPU_ENONFINITE, "batched fgmres: non-finite initial residual"); }
            if (q.niter == 0) q.r0norm_initial = r0n;
            if (r0n == 0.0) { q.active = false; nactive--; q.res_est = 0.0; continue; }   // zero right-hand side: x = 0
            q.p[0] = r0n;
            scale[s] = 1.0 / r0n;
            q.nvecs = 0;
        }
        if (nactive == 0) break;
        if ((st = push(SCALE, scale.data(), nsys))) { cleanup(); return st; }
        k_seg_scale<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, CY, Vb, Vb, SCALE);
        if ((st = check("k_seg_scale v1"))) { cleanup(); return st; }
        std::vector<char> cycle_member(nsys);
        for (int s = 0; s < nsys; ++s) cycle_member[s] = S[s].active;
        for (int j = 1; j <= m; ++j) {
            double* vj = Vb + (int64_t)(j - 1) * n;
            double* zj = Zb + (int64_t)(j - 1) * n;
            double* w = Vb + (int64_t)j * n;
            if ((st = precon_apply_impl<double>(M, vj, zj, prec))) { cleanup(); return st; }
            if ((st = matvec_launch<double, double>(A, (const double*)A->val.ptr, zj, w, nullptr, 1.0, 0.0, ROWSQ)) ||
                (st = rows_to_sys(OUT + (size_t)nsys * 0))) { cleanup(); return st; }
            std::vector<double> norm_before(nsys);
            if ((st = fetch(OUT, nsys, norm_before.data()))) { cleanup(); return st; }
            // CGS pass 1 with the fresh dot products as coefficients
            k_seg_mdot<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, G.nchunk, w, Vb, n, j, PART);
            if ((st = check("k_seg_mdot"))) { cleanup(); return st; }
            k_seg_reduce<<<nsys, 128, 0, ctx->stream>>>(PART, G.nchunk, SC, j, COEF, hst);
            if ((st = check("k_seg_reduce h"))) { cleanup(); return st; }
            k_seg_maxpy<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, CY, w, Vb, n, j, COEF, hst, PART);
            if ((st = check("k_seg_maxpy"))) { cleanup(); return st; }
            k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(PART, G.nchunk, SC, 1, OUT, 1);
            if ((st = check("k_seg_reduce wn"))) { cleanup(); return st; }
            std::vector<double> h1((size_t)nsys * hst), wn(nsys);
            if ((st = fetch(COEF, h1.size(), h1.data())) || (st = fetch(OUT, nsys, wn.data()))) { cleanup(); return st; }
            // selective re-orthogonalisation, per system
            bool any_reorth = false;
            std::vector<char> reorth(nsys, 0);
            for (int s = 0; s < nsys; ++s) {
                if (!S[s].active) continue;
                const double nb = std::sqrt(norm_before[s]);
                if (!std::isfinite(nb)) { cleanup(); ctx->err_elem = sys_elem[s]; return fail(ctx, CHIDG_GPU_ENONFINITE, "batched fgmres: non-finite A*z"); }
                double crit = 0.0;
                for (int i = 0; i < j; ++i) crit += std::fabs(h1[(size_t)s * hst + i]);
                if (crit / nb >= 1.0) { reorth[s] = 1; any_reorth = true; }
            }
            std::vector<double> h2((size_t)nsys * hst, 0.0);
            if (any_reorth) {
                k_seg_mdot<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, G.nchunk, w, Vb, n, j, PART);
                if ((st = check("k_seg_mdot 2"))) { cleanup(); return st; }
                k_seg_reduce<<<nsys, 128, 0, ctx->stream>>>(PART, G.nchunk, SC, j, OUT, hst);
                if ((st = check("k_seg_reduce h2")) || (st = fetch(OUT, h2.size(), h2.data()))) { cleanup(); return st; }
                for (int s = 0; s < nsys; ++s)
                    if (!reorth[s]) std::fill(h2.begin() + (size_t)s * hst, h2.begin() + (size_t)(s + 1) * hst, 0.0);
                if ((st = push(COEF, h2.data(), h2.size()))) { cleanup(); return st; }
                k_seg_maxpy<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, CY, w, Vb, n, j, COEF, hst, PART);
                if ((st = check("k_seg_maxpy 2"))) { cleanup(); return st; }
                k_seg_reduce<<<nsys, 32, 0, ctx->stream>>>(PART, G.nchunk, SC, 1, OUT, 1);
                if ((st = check("k_seg_reduce wn2")) || (st = fetch(OUT, nsys, wn.data()))) { cleanup(); return st; }
            }
            // Givens and convergence, per system
            bool any_finish = false;
            std::fill(coef.begin(), coef.end(), 0.0);
            for (int s = 0; s < nsys; ++s) {
                SysState& q = S[s];
                scale[s] = 0.0;
                if (!q.active) continue;
                auto H = [&](int i, int jj) -> double& { return q.h[(size_t)i + (size_t)jj * (m + 1)]; };
                for (int i = 0; i < j; ++i) H(i, j - 1) = h1[(size_t)s * hst + i] + h2[(size_t)s * hst + i];
                H(j, j - 1) = std::sqrt(wn[s]);
                scale[s] = 1.0 / H(j, j - 1);
                for (int i = 0; i < j - 1; ++i) {
                    const double hij = q.c[i] * H(i, j - 1) + q.s[i] * H(i + 1, j - 1);
                    const double hipj = -q.s[i] * H(i, j - 1) + q.c[i] * H(i + 1, j - 1);
                    H(i, j - 1) = hij;
                    H(i + 1, j - 1) = hipj;
                }
                const double gam = std::hypot(H(j - 1, j - 1), H(j, j - 1));
                q.c[j - 1] = H(j - 1, j - 1) / gam;
                q.s[j - 1] = H(j, j - 1) / gam;
                H(j - 1, j - 1) = gam;
                H(j, j - 1) = 0.0;
                const double pj = q.c[j - 1] * q.p[j - 1];
                const double pjp = -q.s[j - 1] * q.p[j - 1];
                q.p[j - 1] = pj;
                q.p[j] = pjp;
                q.niter++;
                q.nvecs = j;
                q.res = std::fabs(q.p[j]);
                q.hist.push_back(q.res);
                const bool cabs = q.res < o.tol;
                const bool crel = q.res / q.r0norm_initial < o.rtol;
                const bool cmax = (q.niter >= o.nmax) && (o.nmax > 0);
                if (cabs || crel || cmax) {
                    // x = x0 + sum y_i z_i for this system, then freeze it
                    if ((st = solve_ls(q, j, coef.data() + (size_t)s * hst))) { cleanup(); return st; }
                    q.res_est = q.res;
                    q.active = false;
                    nactive--;
                    scale[s] = 0.0;
                    any_finish = true;
                }
            }
            if (any_finish && (st = update_solution(j))) { cleanup(); return st; }
            if ((st = push(SCALE, scale.data(), nsys))) { cleanup(); return st; }
            k_seg_scale<double><<<G.nchunk, TH, 0, ctx->stream>>>(CS, CY, w, w, SCALE);
            if ((st = check("k_seg_scale v"))) { cleanup(); return st; }
            if (nactive == 0) break;
        }
        // end of a full cycle: update and restart the systems still active
        if (nactive > 0) {
            std::fill(coef.begin(), coef.end(), 0.0);
            for (int s = 0; s < nsys; ++s) {
                SysState& q = S[s];
                if (!q.active || !cycle_member[s]) continue;
                if ((st = solve_ls(q, q.nvecs, coef.data() + (size_t)s * hst))) { cleanup(); return st; }
                q.res_est = q.res;
                q.nrestart++;
            }
            if ((st = update_solution(m))) { cleanup(); return st; }
        }
    }
    // print_report: true residual per system
    if ((st = matvec_launch<double, double>(A, (const double*)A->val.ptr, xx, (double*)TMP.ptr, bb, -1.0, 1.0, ROWSQ)) ||
        (st = rows_to_sys(OUT)) || (st = fetch(OUT, nsys, hout.data()))) { cleanup(); return st; }
    double sw = 0.0;
    if ((st = fetch(ctx->d_scal + kSlotStatus, 1, &sw)) || (st = status_word(ctx, sw))) { cleanup(); return st; }
    cleanup();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int s = 0; s < nsys; ++s) {
        S[s].residual_norm = std::sqrt(hout[s]);
        if (results) {
            chidg_gpu_fgmres_result& r = results[s];
            r.niter = S[s].niter;
            r.nrestart = S[s].nrestart;
            r.inner_iters = 0;
            r.nhist = (int32_t)std::min<size_t>(S[s].hist.size(), (size_t)std::max(hist_cap, 0));
            r.residual_norm = S[s].residual_norm;
            r.res_estimate = S[s].res_est;
            r.r0norm_initial = S[s].r0norm_initial;
            r.seconds = secs;
        }
        if (hist)
            for (int i = 0; i < (int)S[s].hist.size() && i < hist_cap; ++i) hist[(size_t)s * hist_cap + i] = S[s].hist[i];
    }
    return CHIDG_GPU_OK;
}
