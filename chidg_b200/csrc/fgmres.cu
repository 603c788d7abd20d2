// fgmres.cu -- fgmres_t%solve on the GPU (src/linear_solvers/type_fgmres.f90:81-310).
//
// The vectors, the matvec, the preconditioner sweeps and the Gram-Schmidt
// reductions run on the device; the scalar Arnoldi bookkeeping (selective
// re-orthogonalisation test, Givens rotations, the explicit inverse of the
// Hessenberg matrix) runs on the host in FP64 exactly as the reference does,
// after one small device->host copy per Arnoldi step.
//
// Mixed precision (CHIDG_GPU_MIXED_*): the outer FP64 FGMRES keeps the FP64
// matvec, Krylov basis and Hessenberg least squares, and uses as its flexible
// preconditioner an FP32 FGMRES on an FP32 copy of A with the ILU factors in
// FP32 or BF16.  The outer loop is the iterative refinement that recovers
// FP64 accuracy.
#include "chidg_gpu_internal.cuh"

#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cstring>
#include <functional>
#include <memory>

using namespace chidg;

namespace {

// Explicit inverse with partial pivoting of the small Hessenberg system
// (mod_inv::inv semantics: LU with row interchanges, then the inverse).
int host_inverse(int n, std::vector<double>& a) {
    std::vector<int> piv(n);
    std::vector<int> used(n, 0);
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

template <typename T>
struct Solver {
    chidg_gpu_ctx* ctx = nullptr;
    chidg_gpu_matrix* A = nullptr;
    // options (linear_solver_t)
    double tol = 1e-8, rtol = 1e-10;
    int nmax = -1, nkrylov = 2000, orth = CHIDG_ORTH_CGS;
    bool inner = false;
    double inner_tol = 0.1, inner_rtol = 0.1;
    int inner_nmax = 100, inner_nkrylov = 100, inner_orth = CHIDG_ORTH_CGS;
    bool true_residual = true;
    int precision = CHIDG_GPU_FP64;     // float solvers: which low-precision copy of A
    // state
    int niter = 0, nrestart = 0;
    int64_t inner_iters = 0;
    double residual_norm = 0.0, res_est = 0.0, r0norm_initial = 0.0;
    std::vector<double>* hist = nullptr;
    std::function<int(const T*, T*)> precon;        // z = M v
    // z = M v and w = A z with w's row sums of squares in one streamed pass;
    // returns 1 (nothing done) when the preconditioner cannot fuse them
    std::function<int(const T*, T*, T*, double*)> precon_mv;
    std::function<int()> precon_update;              // M%update, or empty
    std::unique_ptr<Solver<T>> child;
    Workspace own;
    Workspace* ws = &own;          // Krylov storage (the context's, for top-level solvers)

    ~Solver() { for (Buffer* b : {&own.V, &own.Z, &own.x0, &own.zr, &own.dz, &own.tmp, &own.rowsq}) release(*b); }

    int matvec(const T* x, T* y, const T* z, double alpha, double beta, bool want_norm, int slot) {
        double* rs = nullptr;
        if (want_norm) {
            int st = ensure(ctx, ws->rowsq, sizeof(double) * (size_t)A->nrow);
            if (st) return st;
            rs = (double*)ws->rowsq.ptr;
        }
        int st = launch_mv(x, y, z, alpha, beta, rs);
        if (st) return st;
        if (want_norm) return reduce_partials(ctx, rs, A->nrow, 1, slot, false);
        return CHIDG_GPU_OK;
    }
    int launch_mv(const T* x, T* y, const T* z, double alpha, double beta, double* rs);
    int axpby(double a, const T* x, double b, T* y) {
        const int64_t n = A->n;
        k_axpby<T, T><<<grid_for(n, 256, ctx->nsm * 8), 256, 0, ctx->stream>>>(n, a, nullptr, x, b, y);
        return check_launch(ctx, "k_axpby");
    }
    // one Gram-Schmidt pass; h(0:j) for this pass left in d_scal[kSlotH..], ||w||^2 in kSlotWnorm
    int gs_pass(T* w, const T* Vb, int j) {
        const int64_t n = A->n;
        int st;
        const int threads = 256;
        const int ncta = grid_for(n, threads, ctx->nsm * 4);
        if ((st = ensure(ctx, ctx->partial2, sizeof(double) * (size_t)ncta))) return st;
        if (orth == CHIDG_ORTH_CGS) {
            if ((st = mdot<T>(ctx, n, w, Vb, n, j, kSlotH))) return st;
            k_maxpy_sub_norm<T><<<ncta, threads, 0, ctx->stream>>>(n, w, Vb, n, j, ctx->d_scal + kSlotH, (double*)ctx->partial2.ptr);
            if ((st = check_launch(ctx, "k_maxpy_sub_norm"))) return st;
        } else {
            for (int i = 0; i < j; ++i) {
                if ((st = mdot<T>(ctx, n, w, Vb + (int64_t)i * n, n, 1, kSlotH + i))) return st;
                k_maxpy_sub_norm<T><<<ncta, threads, 0, ctx->stream>>>(n, w, Vb + (int64_t)i * n, n, 1, ctx->d_scal + kSlotH + i,
                                                                       (i == j - 1) ? (double*)ctx->partial2.ptr : nullptr);
                if ((st = check_launch(ctx, "k_maxpy_sub_norm"))) return st;
            }
        }
        return reduce_partials(ctx, (const double*)ctx->partial2.ptr, ncta, 1, kSlotWnorm, false);
    }

    int solve(const T* b, T* x) {
        const int64_t n = A->n;
        int st;
        if (inner) {
            if (!child) child.reset(new Solver<T>());
            Solver<T>& c = *child;
            c.ctx = ctx; c.A = A;
            c.nkrylov = inner_nkrylov; c.tol = inner_tol; c.rtol = inner_rtol; c.nmax = inner_nmax;
            c.orth = inner_orth; c.inner = false;
            c.precon = precon; c.precon_mv = precon_mv; c.precon_update = precon_update;
            c.true_residual = true_residual;
        }
        if (precon_update && (st = precon_update())) return st;

        const int m = nkrylov;
        if (m < 1 || m > kMaxKrylov) return fail(ctx, CHIDG_GPU_EINVAL, "fgmres: nkrylov outside [1, 4000]");
        if ((st = ensure(ctx, ws->V, sizeof(T) * (size_t)(m + 1) * n)) || (st = ensure(ctx, ws->Z, sizeof(T) * (size_t)(m + 1) * n)) ||
            (st = ensure(ctx, ws->x0, sizeof(T) * (size_t)n)) || (st = ensure(ctx, ws->tmp, sizeof(T) * (size_t)n)))
            return st;
        if (inner && ((st = ensure(ctx, ws->zr, sizeof(T) * (size_t)n)) || (st = ensure(ctx, ws->dz, sizeof(T) * (size_t)n)))) return st;
        T* Vb = (T*)ws->V.ptr;
        T* Zb = (T*)ws->Z.ptr;
        T* X0 = (T*)ws->x0.ptr;
        cudaMemsetAsync(X0, 0, sizeof(T) * (size_t)n, ctx->stream);
        cudaMemsetAsync(x, 0, sizeof(T) * (size_t)n, ctx->stream);

        std::vector<double> p(m + 1), c(m + 1), s(m + 1), y(m + 1);
        std::vector<double> h((size_t)(m + 1) * m);
        auto H = [&](int i, int jj) -> double& { return h[(size_t)i + (size_t)jj * (m + 1)]; };
        std::vector<double> sc(kSlotH + m + 2);

        niter = 0; nrestart = 0; inner_iters = 0;
        double res = DBL_MAX;
        bool cabs = false, crel = false, cmax = false;
        while (res > tol) {
            std::fill(p.begin(), p.end(), 0.0); std::fill(c.begin(), c.end(), 0.0);
            std::fill(s.begin(), s.end(), 0.0); std::fill(y.begin(), y.end(), 0.0);
            std::fill(h.begin(), h.end(), 0.0);
            // r0 = b - A x0 into V(1); v1 = r0 / ||r0||
            if ((st = matvec(X0, Vb, b, -1.0, 1.0, true, kSlotR0))) return st;
            if ((st = fetch_scalars(ctx, kSlotR0, 1, sc.data()))) return st;
            const double r0norm = std::sqrt(sc[0]);
            if (!std::isfinite(r0norm)) return fail(ctx, CHIDG_GPU_ENONFINITE, "fgmres: non-finite initial residual");
            if ((st = axpby(1.0 / r0norm, Vb, 0.0, Vb))) return st;
            p[0] = r0norm;
            if (niter == 0) r0norm_initial = r0norm;
            int nvecs = 0;
            for (int j = 1; j <= m; ++j) {
                nvecs++;
                T* vj = Vb + (int64_t)(j - 1) * n;
                T* zj = Zb + (int64_t)(j - 1) * n;
                T* w = Vb + (int64_t)j * n;
                // z_j = M v_j, then w = A z_j and ||w|| before orthogonalisation;
                // without an inner solve both can run as one streamed pass
                bool fused = false;
                if (precon_mv && !inner) {
                    if ((st = ensure(ctx, ws->rowsq, sizeof(double) * (size_t)A->nrow))) return st;
                    st = precon_mv(vj, zj, w, (double*)ws->rowsq.ptr);
                    if (st == CHIDG_GPU_OK) {
                        fused = true;
                        if ((st = reduce_partials(ctx, (const double*)ws->rowsq.ptr, A->nrow, 1, kSlotNormBefore, false)))
                            return st;
                    } else if (st != 1) {
                        return st;
                    }
                }
                if (!fused) {
                    if ((st = precon(vj, zj))) return st;
                    if (inner) {
                        T* ZR = (T*)ws->zr.ptr;
                        T* DZ = (T*)ws->dz.ptr;
                        if ((st = matvec(zj, ZR, vj, -1.0, 1.0, false, 0))) return st;   // zr = v - A z
                        if ((st = child->solve(ZR, DZ))) return st;
                        inner_iters += child->niter;
                        if ((st = axpby(1.0, DZ, 1.0, zj))) return st;                     // z = z + dz
                    }
                    if ((st = matvec(zj, w, nullptr, 1.0, 0.0, true, kSlotNormBefore))) return st;
                }
                if ((st = gs_pass(w, Vb, j))) return st;
                if ((st = fetch_scalars(ctx, 0, kSlotH + j, sc.data()))) return st;
                if ((st = status_word(ctx, sc[kSlotStatus]))) return st;
                const double norm_before = std::sqrt(sc[kSlotNormBefore]);
                if (!std::isfinite(norm_before)) return fail(ctx, CHIDG_GPU_ENONFINITE, "fgmres: non-finite A*z");
                std::vector<double> hcol(sc.begin() + kSlotH, sc.begin() + kSlotH + j);
                double wn2 = sc[kSlotWnorm];
                // selective re-orthogonalisation (:203-223)
                double crit = 0.0;
                for (int i = 0; i < j; ++i) crit += std::fabs(hcol[i]);
                crit /= norm_before;
                if (crit >= 1.0) {
                    if ((st = gs_pass(w, Vb, j))) return st;
                    if ((st = fetch_scalars(ctx, 0, kSlotH + j, sc.data()))) return st;
                    for (int i = 0; i < j; ++i) hcol[i] += sc[kSlotH + i];
                    wn2 = sc[kSlotWnorm];
                }
                for (int i = 0; i < j; ++i) H(i, j - 1) = hcol[i];
                H(j, j - 1) = std::sqrt(wn2);
                if ((st = axpby(1.0 / H(j, j - 1), w, 0.0, w))) return st;   // v(j+1) = w / h(j+1,j)
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
            // y = inv(H(1:n,1:n)) p(1:n); x = x0 + sum y_i z_i  (:287-295)
            std::vector<double> Hn((size_t)nvecs * nvecs);
            for (int jj = 0; jj < nvecs; ++jj)
                for (int ii = 0; ii < nvecs; ++ii) Hn[ii + (size_t)jj * nvecs] = H(ii, jj);
            if (host_inverse(nvecs, Hn) != 0) return fail(ctx, CHIDG_GPU_ESINGULAR, "fgmres: singular Hessenberg matrix");
            for (int ii = 0; ii < nvecs; ++ii) {
                double acc = 0.0;
                for (int jj = 0; jj < nvecs; ++jj) acc += Hn[ii + (size_t)jj * nvecs] * p[jj];
                y[ii] = acc;
            }
            if ((st = push_scalars(ctx, kSlotY, nvecs, y.data()))) return st;
            k_lincomb<T><<<grid_for(n, 256, ctx->nsm * 8), 256, 0, ctx->stream>>>(n, x, X0, Zb, n, nvecs, ctx->d_scal + kSlotY);
            if ((st = check_launch(ctx, "k_lincomb"))) return st;
            res_est = res;
            if (cabs || crel || cmax) break;
            cudaMemcpyAsync(X0, x, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream);
            nrestart++;
        }
        if (true_residual) {   // print_report: ||b - A x|| (:512-520)
            if ((st = matvec(x, (T*)ws->tmp.ptr, b, -1.0, 1.0, true, kSlotTmp))) return st;
            if ((st = fetch_scalars(ctx, kSlotTmp, 1, sc.data()))) return st;
            residual_norm = std::sqrt(sc[0]);
        } else {
            residual_norm = res_est;
        }
        return CHIDG_GPU_OK;
    }
};

template <>
int Solver<double>::launch_mv(const double* x, double* y, const double* z, double alpha, double beta, double* rs) {
    return matvec_launch<double, double>(A, (const double*)A->val.ptr, x, y, z, alpha, beta, rs);
}
template <>
int Solver<float>::launch_mv(const float* x, float* y, const float* z, double alpha, double beta, double* rs) {
    if (precision == CHIDG_GPU_MIXED_BF16)
        return matvec_launch<__nv_bfloat16, float>(A, (const __nv_bfloat16*)A->val16.ptr, x, y, z, alpha, beta, rs);
    return matvec_launch<float, float>(A, (const float*)A->val32.ptr, x, y, z, alpha, beta, rs);
}

}  // namespace

extern "C" int chidg_gpu_fgmres_default_opts(chidg_gpu_fgmres_opts* o) {
    if (!o) return CHIDG_GPU_EINVAL;
    std::memset(o, 0, sizeof(*o));
    o->tol = 1e-8;            // type_linear_solver.f90:23-40
    o->rtol = 1e-10;
    o->nmax = -1;
    o->nkrylov = 2000;
    o->orthogonalization = CHIDG_ORTH_CGS;
    o->inner_fgmres = 1;
    o->inner_tol = 1e-1;
    o->inner_rtol = 1e-1;
    o->inner_nmax = 100;
    o->inner_nkrylov = 100;
    o->inner_orthogonalization = CHIDG_ORTH_CGS;
    o->use_controller = 0;
    o->precision = CHIDG_GPU_FP64;
    o->mixed_inner_nkrylov = 30;
    o->mixed_inner_rtol = 1e-2;
    o->mixed_inner_nmax = 60;
    return CHIDG_GPU_OK;
}

extern "C" int chidg_gpu_fgmres_solve(chidg_gpu_matrix* A, chidg_gpu_precon* M, const chidg_gpu_vector* b,
                                      chidg_gpu_vector* x, const chidg_gpu_fgmres_opts* opts,
                                      chidg_gpu_fgmres_result* result, double* hist, int32_t hist_cap) {
    if (!A || !M || !b || !x || M->A != A || b->n != A->n || x->n != A->n || b == x) return CHIDG_GPU_EINVAL;
    chidg_gpu_ctx* ctx = A->ctx;
    cudaSetDevice(ctx->device);
    const auto t0 = std::chrono::steady_clock::now();
    chidg_gpu_fgmres_opts o;
    if (opts) o = *opts;
    else chidg_gpu_fgmres_default_opts(&o);
    if (o.precision < CHIDG_GPU_FP64 || o.precision > CHIDG_GPU_MIXED_PRECON_FP32) return fail(ctx, CHIDG_GPU_EINVAL, "fgmres: bad precision");
    int st;
    // the operator: A, or A^T when A->transposed (chidg_mv, operator_chidg_mv.f90:46-60)
    chidg_gpu_matrix* Aop;
    if ((st = matrix_op(A, &Aop))) return st;
    // the FP32 / BF16 copy read by the inner solves' products (M%update makes it
    // too, but not for the identity preconditioner)
    if ((o.precision == CHIDG_GPU_MIXED_FP32 || o.precision == CHIDG_GPU_MIXED_BF16) &&
        (st = matrix_lowp(Aop, o.precision)))
        return st;
    set_matvec_smem(Aop);
    if (M->kind != CHIDG_PRECON_IDENTITY) precon_set_smem(M);
    ctx->err_elem = -1;
    cudaMemsetAsync(ctx->d_scal + kSlotStatus, 0, sizeof(double), ctx->stream);

    const int prec = o.precision;
    // M%update as solver_controller%update_preconditioner decides, or on every
    // call without a controller (type_fgmres.f90:118-122)
    auto do_update = [A, M, prec, &o]() -> int {
        if (o.use_controller && M->stamp == A->stamp && M->precision == prec) return CHIDG_GPU_OK;
        return chidg_gpu_precon_update(M, A, prec);
    };
    std::vector<double> hv;
    Solver<double> S;
    S.ctx = ctx; S.A = Aop;
    S.ws = &ctx->ws64;
    S.tol = o.tol; S.rtol = o.rtol; S.nmax = o.nmax; S.nkrylov = o.nkrylov; S.orth = o.orthogonalization;
    S.inner = o.inner_fgmres != 0; S.inner_tol = o.inner_tol; S.inner_rtol = o.inner_rtol;
    S.inner_nmax = o.inner_nmax; S.inner_nkrylov = o.inner_nkrylov; S.inner_orth = o.inner_orthogonalization;
    S.hist = &hv;
    S.precon_update = do_update;
    std::unique_ptr<Solver<float>> lo;
    Buffer& v32 = ctx->mix_v32;       // kept by the context: no allocation per solve
    Buffer& z32 = ctx->mix_z32;
    int64_t lo_iters = 0;
    if (prec == CHIDG_GPU_FP64 || prec == CHIDG_GPU_MIXED_PRECON_FP32) {
        S.precon = [M, prec](const double* v, double* z) { return precon_apply_impl<double>(M, v, z, prec); };
        S.precon_mv = [M, prec, Aop](const double* v, double* z, double* w, double* rs) {
            return precon_apply_mv<double, double>(M, v, z, prec, Aop, (const double*)Aop->val.ptr, w, rs);
        };
    } else {
        // FP32 inner FGMRES as the flexible preconditioner of the FP64 outer loop
        S.inner = false;
        lo.reset(new Solver<float>());
        lo->ctx = ctx; lo->A = Aop;
        lo->ws = &ctx->ws32;
        lo->tol = 0.0; lo->rtol = o.mixed_inner_rtol; lo->nmax = o.mixed_inner_nmax;
        lo->nkrylov = o.mixed_inner_nkrylov; lo->orth = CHIDG_ORTH_CGS; lo->inner = false;
        lo->true_residual = false;
        lo->precision = prec;
        lo->precon = [M, prec](const float* v, float* z) { return precon_apply_impl<float>(M, v, z, prec); };
        if (prec == CHIDG_GPU_MIXED_BF16)
            lo->precon_mv = [M, prec, Aop](const float* v, float* z, float* w, double* rs) {
                return precon_apply_mv<float, __nv_bfloat16>(M, v, z, prec, Aop, (const __nv_bfloat16*)Aop->val16.ptr, w, rs);
            };
        else
            lo->precon_mv = [M, prec, Aop](const float* v, float* z, float* w, double* rs) {
                return precon_apply_mv<float, float>(M, v, z, prec, Aop, (const float*)Aop->val32.ptr, w, rs);
            };
        if ((st = ensure(ctx, v32, sizeof(float) * (size_t)A->n)) || (st = ensure(ctx, z32, sizeof(float) * (size_t)A->n))) return st;
        Solver<float>* lp = lo.get();
        float* V32 = (float*)v32.ptr;
        float* Z32 = (float*)z32.ptr;
        S.precon = [ctx, A, lp, V32, Z32, &lo_iters](const double* v, double* z) -> int {
            const int64_t n = A->n;
            k_convert<double, float><<<grid_for(n, 256, ctx->nsm * 8), 256, 0, ctx->stream>>>(n, v, V32);
            int s2 = check_launch(ctx, "k_convert v");
            if (s2) return s2;
            if ((s2 = lp->solve(V32, Z32))) return s2;
            lo_iters += lp->niter;
            k_convert<float, double><<<grid_for(n, 256, ctx->nsm * 8), 256, 0, ctx->stream>>>(n, Z32, z);
            return check_launch(ctx, "k_convert z");
        };
    }
    st = S.solve((const double*)b->buf.ptr, (double*)x->buf.ptr);
    if (st == CHIDG_GPU_OK) {
        const cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) st = cuda_fail(ctx, e, "fgmres");
    }
    if (result) {
        result->niter = S.niter;
        result->nrestart = S.nrestart;
        result->inner_iters = (int32_t)(S.inner_iters + lo_iters);
        result->residual_norm = S.residual_norm;
        result->res_estimate = S.res_est;
        result->r0norm_initial = S.r0norm_initial;
        result->nhist = (int32_t)std::min<size_t>(hv.size(), (size_t)std::max(hist_cap, 0));
        result->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    if (hist)
        for (int i = 0; i < (int)hv.size() && i < hist_cap; ++i) hist[i] = hv[i];
    return st;
}
