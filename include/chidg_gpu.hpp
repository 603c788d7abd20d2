/*
 * chidg_gpu.hpp -- C++17 host layer over the C ABI of chidg_gpu.h.
 *
 * The reference's linear-solve path is compiled Fortran; this header is its
 * host side for C++ callers and tests, with the reference's class and method
 * names, option names, defaults and error behaviour:
 *
 *   chidg_matrix_t   (src/containers/type_chidg_matrix.f90)     -> ChidgMatrix
 *   chidg_vector_t   (src/containers/type_chidg_vector.f90)     -> ChidgVector
 *   chidg_mv         (src/containers/operator_chidg_mv.f90)     -> chidg_mv
 *   preconditioner_t (src/preconditioners/type_preconditioner.f90,
 *                     factory mod_preconditioner.f90:49-108)    -> Preconditioner,
 *                                                                  create_preconditioner
 *   fgmres_t         (src/linear_solvers/type_fgmres.f90, options of
 *                     type_linear_solver.f90:21-131)            -> LinearSolver,
 *                                                                  create_linear_solver
 *
 * Where the reference calls chidg_signal(FATAL, ...) these classes throw
 * chidg_gpu::Error carrying the library's status code, message and, for
 * ESINGULAR / ENONFINITE, the element id.  Objects own their handles (RAII);
 * a context must outlive the matrices, vectors and preconditioners made on it.
 */
#ifndef CHIDG_GPU_HPP
#define CHIDG_GPU_HPP

#include "chidg_gpu.h"

#include <algorithm>
#include <array>
#include <cctype>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace chidg_gpu {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg, int32_t element = -1)
        : std::runtime_error(msg), code(code), element(element) {}
    int code;
    int32_t element;
};

namespace detail {
inline void check(chidg_gpu_ctx* ctx, int st, const char* what) {
    if (st == CHIDG_GPU_OK) return;
    std::string msg = what;
    int32_t elem = -1;
    if (ctx) {
        char buf[512] = {0};
        chidg_gpu_last_error(ctx, buf, (int32_t)sizeof(buf));
        chidg_gpu_error_element(ctx, &elem);
        msg += std::string(": ") + buf;
    }
    throw Error(st, msg, elem);
}
}  // namespace detail

// One device and one stream (optionally the caller's cudaStream_t).
class Context {
public:
    explicit Context(int device = 0, void* stream = nullptr) {
        detail::check(nullptr, chidg_gpu_ctx_create(device, stream, &h_), "context create");
    }
    ~Context() { if (h_) chidg_gpu_ctx_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    chidg_gpu_ctx* handle() const { return h_; }
    void sync() { detail::check(h_, chidg_gpu_ctx_sync(h_), "sync"); }
    int64_t launches() const { int64_t c = 0; chidg_gpu_launch_count(h_, &c); return c; }
private:
    chidg_gpu_ctx* h_ = nullptr;
};

// A block pattern (domain_matrix_t's lblks / chi_blks / bc_blks / hb_blks,
// type_domain_matrix.f90:102-632) with owned arrays.
struct Pattern {
    int32_t nelem = 0, ntime = 1;
    std::vector<int32_t> elem_nvars, elem_nterms, elem_proc;
    std::vector<int32_t> blk_row_elem, blk_row_time, blk_col_elem, blk_col_time, blk_kind;

    int64_t nblocks() const { return (int64_t)blk_row_elem.size(); }
    void add_block(int32_t re, int32_t rt, int32_t ce, int32_t ct, int32_t kind) {
        blk_row_elem.push_back(re); blk_row_time.push_back(rt);
        blk_col_elem.push_back(ce); blk_col_time.push_back(ct); blk_kind.push_back(kind);
    }
    chidg_gpu_pattern view() const {
        chidg_gpu_pattern p{};
        p.nelem = nelem; p.ntime = ntime; p.nblocks = nblocks();
        p.elem_nvars = elem_nvars.data(); p.elem_nterms = elem_nterms.data();
        p.elem_proc = elem_proc.empty() ? nullptr : elem_proc.data();
        p.blk_row_elem = blk_row_elem.data(); p.blk_row_time = blk_row_time.data();
        p.blk_col_elem = blk_col_elem.data(); p.blk_col_time = blk_col_time.data();
        p.blk_kind = blk_kind.data();
        return p;
    }
    // Patterns of independent systems packed block-diagonally (the layout of
    // chidg_gpu_fgmres_solve_batched); sys_elem[s] is system s's first element,
    // sys_elem[n] the total.  All systems must have the same time levels.
    static Pattern concat(const std::vector<const Pattern*>& parts, std::vector<int32_t>* sys_elem) {
        Pattern p;
        if (sys_elem) sys_elem->assign(1, 0);
        for (const Pattern* q : parts) {
            if (p.nelem == 0) p.ntime = q->ntime;
            else if (q->ntime != p.ntime) throw Error(CHIDG_GPU_EINVAL, "Pattern::concat: systems of different time levels");
            const int32_t e0 = p.nelem;
            p.elem_nvars.insert(p.elem_nvars.end(), q->elem_nvars.begin(), q->elem_nvars.end());
            p.elem_nterms.insert(p.elem_nterms.end(), q->elem_nterms.begin(), q->elem_nterms.end());
            p.elem_proc.insert(p.elem_proc.end(), q->elem_nvars.size(), 0);
            for (int64_t k = 0; k < q->nblocks(); ++k)
                p.add_block(q->blk_row_elem[k] + e0, q->blk_row_time[k], q->blk_col_elem[k] + e0, q->blk_col_time[k],
                            q->blk_kind[k]);
            p.nelem += q->nelem;
            if (sys_elem) sys_elem->push_back(p.nelem);
        }
        return p;
    }
    // The pattern of an nx x ny x nz hex box (elements i fastest), rows in the
    // reference's storage order: per (element, time) the interior faces in the
    // order XI_MIN, XI_MAX, ETA_MIN, ETA_MAX, ZETA_MIN, ZETA_MAX, then DIAG, then
    // with ntime > 1 the hb_blks coupling the element's other time levels.
    static Pattern box(int nx, int ny, int nz, int nvars, int nterms, int ntime = 1) {
        Pattern p;
        p.nelem = nx * ny * nz;
        p.ntime = ntime;
        p.elem_nvars.assign(p.nelem, nvars);
        p.elem_nterms.assign(p.nelem, nterms);
        p.elem_proc.assign(p.nelem, 0);
        for (int e = 0; e < p.nelem; ++e) {
            const int i = e % nx, j = (e / nx) % ny, k = e / (nx * ny);
            const std::array<int, 7> nbr = {i > 0 ? e - 1 : -1,           i < nx - 1 ? e + 1 : -1,
                                            j > 0 ? e - nx : -1,          j < ny - 1 ? e + nx : -1,
                                            k > 0 ? e - nx * ny : -1,     k < nz - 1 ? e + nx * ny : -1, e};
            for (int t = 0; t < ntime; ++t) {
                for (int f = 0; f < 7; ++f)
                    if (nbr[f] >= 0) p.add_block(e, t, nbr[f], t, CHIDG_BLK_LOCAL);
                for (int tt = 0; tt < ntime; ++tt)
                    if (tt != t) p.add_block(e, t, e, tt, CHIDG_BLK_HB);
            }
        }
        return p;
    }
};

class ChidgVector;

// chidg_matrix_t with backend 'cuda': the pattern's blocks in device memory,
// packed in pattern order, each column-major (densematrix_t%mat).
class ChidgMatrix {
public:
    ChidgMatrix() = default;
    ChidgMatrix(Context& ctx, const Pattern& pat) { init(ctx, pat); }
    ~ChidgMatrix() { release(); }
    ChidgMatrix(const ChidgMatrix&) = delete;
    ChidgMatrix& operator=(const ChidgMatrix&) = delete;

    // chidg_matrix%init (:221-248)
    void init(Context& ctx, const Pattern& pat) {
        release();
        ctx_ = &ctx;
        pat_ = pat;
        const chidg_gpu_pattern v = pat_.view();
        detail::check(ctx.handle(), chidg_gpu_matrix_create(ctx.handle(), &v, &h_), "chidg_matrix%init");
        chidg_gpu_matrix_nvalues(h_, &nvalues_);
        chidg_gpu_matrix_nvec(h_, &nvec_);
    }
    // the values chidg_matrix%store* writes (:575-747), all blocks at once
    void store(const std::vector<double>& packed) {
        if ((int64_t)packed.size() != nvalues_) throw Error(CHIDG_GPU_EINVAL, "chidg_matrix%store: value count");
        detail::check(c(), chidg_gpu_matrix_upload(h_, packed.data()), "chidg_matrix%store");
        ctx_->sync();
    }
    std::vector<double> values() const {
        std::vector<double> out((size_t)nvalues_);
        detail::check(c(), chidg_gpu_matrix_download(h_, out.data()), "chidg_matrix download");
        return out;
    }
    void clear() { detail::check(c(), chidg_gpu_matrix_clear(h_), "chidg_matrix%clear"); }
    // chidg_matrix%scale_diagonal (:769-792): mass per element, scale per (element, field)
    void scale_diagonal(const std::vector<double>& mass, const std::vector<double>& scale) {
        detail::check(c(), chidg_gpu_matrix_scale_diagonal(h_, mass.data(), scale.data()), "chidg_matrix%scale_diagonal");
    }
    int64_t stamp() const { int64_t s = 0; chidg_gpu_matrix_stamp(h_, &s); return s; }
    // chidg_matrix_t%transposed (:49)
    void set_transposed(bool t) { detail::check(c(), chidg_gpu_matrix_set_transposed(h_, t ? 1 : 0), "transposed"); }
    bool transposed() const { int32_t t = 0; chidg_gpu_matrix_get_transposed(h_, &t); return t != 0; }
    void to_file(const std::string& path) { detail::check(c(), chidg_gpu_matrix_to_file(h_, path.c_str()), "chidg_matrix%to_file"); }

    int64_t nvalues() const { return nvalues_; }
    int64_t nvec() const { return nvec_; }
    const Pattern& pattern() const { return pat_; }
    chidg_gpu_matrix* handle() const { return h_; }
    Context& context() const { return *ctx_; }
    void release() { if (h_) { chidg_gpu_matrix_destroy(h_); h_ = nullptr; } }

private:
    chidg_gpu_ctx* c() const { return ctx_ ? ctx_->handle() : nullptr; }
    Context* ctx_ = nullptr;
    Pattern pat_;
    chidg_gpu_matrix* h_ = nullptr;
    int64_t nvalues_ = 0, nvec_ = 0;
};

// chidg_vector_t with backend 'cuda': element-major, then time, field, mode.
class ChidgVector {
public:
    ChidgVector() = default;
    explicit ChidgVector(const ChidgMatrix& A) { init(A); }
    ChidgVector(const ChidgMatrix& A, const std::vector<double>& values) { init(A); set(values); }
    ~ChidgVector() { release(); }
    ChidgVector(const ChidgVector& o) { init(*o.A_); assign(o); }
    ChidgVector& operator=(const ChidgVector& o) { if (this != &o) { if (!h_) init(*o.A_); assign(o); } return *this; }
    ChidgVector(ChidgVector&& o) noexcept : A_(o.A_), h_(o.h_) { o.h_ = nullptr; }

    // chidg_vector%init
    void init(const ChidgMatrix& A) {
        release();
        A_ = &A;
        detail::check(c(), chidg_gpu_vector_create(A.handle(), &h_), "chidg_vector%init");
    }
    void set(const std::vector<double>& v) {
        if ((int64_t)v.size() != A_->nvec()) throw Error(CHIDG_GPU_EINVAL, "chidg_vector: size mismatch");
        detail::check(c(), chidg_gpu_vector_upload(h_, v.data()), "chidg_vector upload");
        A_->context().sync();
    }
    std::vector<double> get() const {
        std::vector<double> out((size_t)A_->nvec());
        detail::check(c(), chidg_gpu_vector_download(h_, out.data()), "chidg_vector download");
        return out;
    }
    void clear() { detail::check(c(), chidg_gpu_vector_clear(h_), "chidg_vector%clear"); }
    void assign(const ChidgVector& o) { detail::check(c(), chidg_gpu_vector_copy(h_, o.h_), "chidg_vector ="); }
    void axpy(double a, const ChidgVector& x) { detail::check(c(), chidg_gpu_vector_axpy(h_, a, x.h_), "axpy"); }
    void scale(double a) { detail::check(c(), chidg_gpu_vector_scale(h_, a), "scale"); }
    // chidg_vector%norm (:1237-1305), %norm_fields (:1319-1352)
    double norm() const { double r = 0; detail::check(c(), chidg_gpu_vector_norm(h_, &r), "chidg_vector%norm"); return r; }
    std::vector<double> norm_fields(int nfields) const {
        std::vector<double> r(nfields);
        detail::check(c(), chidg_gpu_vector_norm_fields(h_, r.data(), nfields), "chidg_vector%norm_fields");
        return r;
    }
    chidg_gpu_vector* handle() const { return h_; }
    const ChidgMatrix& matrix() const { return *A_; }
    void release() { if (h_) { chidg_gpu_vector_destroy(h_); h_ = nullptr; } }

private:
    chidg_gpu_ctx* c() const { return A_ ? A_->context().handle() : nullptr; }
    const ChidgMatrix* A_ = nullptr;
    chidg_gpu_vector* h_ = nullptr;
};

// dot (operator_chidg_dot.f90:30-97) and the overloaded operators of
// chidg_vector_t (type_chidg_vector.f90:1740-2084): each returns a new vector
inline double dot(const ChidgVector& x, const ChidgVector& y) {
    double r = 0;
    detail::check(x.matrix().context().handle(), chidg_gpu_vector_dot(x.handle(), y.handle(), &r), "dot");
    return r;
}
inline ChidgVector operator+(const ChidgVector& x, const ChidgVector& y) { ChidgVector r(x); r.axpy(1.0, y); return r; }
inline ChidgVector operator-(const ChidgVector& x, const ChidgVector& y) { ChidgVector r(x); r.axpy(-1.0, y); return r; }
inline ChidgVector operator*(double a, const ChidgVector& x) { ChidgVector r(x); r.scale(a); return r; }
inline ChidgVector operator*(const ChidgVector& x, double a) { return a * x; }
inline ChidgVector operator/(const ChidgVector& x, double a) { return (1.0 / a) * x; }

// chidg_mv (operator_chidg_mv.f90:46-60): A x, or A^T x for a transposed A
inline ChidgVector chidg_mv(const ChidgMatrix& A, const ChidgVector& x) {
    ChidgVector y(A);
    detail::check(A.context().handle(), chidg_gpu_matvec(A.handle(), x.handle(), y.handle()), "chidg_mv");
    return y;
}

// preconditioner_t: init / update / apply / tear_down, stamp
class Preconditioner {
public:
    explicit Preconditioner(int32_t kind) : kind_(kind) {}
    ~Preconditioner() { tear_down(); }
    Preconditioner(const Preconditioner&) = delete;
    Preconditioner& operator=(const Preconditioner&) = delete;

    void init(ChidgMatrix& A) {
        tear_down();
        A_ = &A;
        detail::check(A.context().handle(), chidg_gpu_precon_create(A.handle(), kind_, &h_), "preconditioner%init");
        if (schedule_ >= 0) chidg_gpu_precon_set_schedule(h_, schedule_);
    }
    // %update(A, b): b is unused by the native preconditioners, as in the reference
    void update(ChidgMatrix& A, const ChidgVector* b = nullptr, int32_t precision = CHIDG_GPU_FP64) {
        (void)b;
        if (!h_ || A_ != &A) init(A);
        detail::check(A.context().handle(), chidg_gpu_precon_update(h_, A.handle(), precision), "preconditioner%update");
    }
    ChidgVector apply(ChidgMatrix& A, const ChidgVector& v) {
        ChidgVector z(A);
        detail::check(A.context().handle(), chidg_gpu_precon_apply(h_, A.handle(), v.handle(), z.handle()),
                      "preconditioner%apply");
        return z;
    }
    // precon_ILU0_t%LD in the matrix's block layout (ILU0 / Jacobi)
    std::vector<double> LD() const {
        std::vector<double> out((size_t)A_->nvalues());
        detail::check(A_->context().handle(), chidg_gpu_precon_download_LD(h_, out.data()), "preconditioner%LD");
        return out;
    }
    int64_t stamp() const { int64_t s = 0; if (h_) chidg_gpu_precon_stamp(h_, &s); return s; }
    void set_schedule(int32_t schedule) { schedule_ = schedule; if (h_) chidg_gpu_precon_set_schedule(h_, schedule); }
    void tear_down() { if (h_) { chidg_gpu_precon_destroy(h_); h_ = nullptr; } }
    chidg_gpu_precon* handle() const { return h_; }
    int32_t kind() const { return kind_; }

private:
    int32_t kind_;
    int32_t schedule_ = -1;
    ChidgMatrix* A_ = nullptr;
    chidg_gpu_precon* h_ = nullptr;
};

// create_preconditioner (mod_preconditioner.f90:49-108): 'identity', 'jacobi',
// 'ilu0', 'rasilu0', 'HB' (case-insensitive)
inline std::unique_ptr<Preconditioner> create_preconditioner(std::string name) {
    std::transform(name.begin(), name.end(), name.begin(), [](unsigned char ch) { return (char)std::tolower(ch); });
    static const std::map<std::string, int32_t> kinds = {
        {"identity", CHIDG_PRECON_IDENTITY}, {"jacobi", CHIDG_PRECON_JACOBI}, {"ilu0", CHIDG_PRECON_ILU0},
        {"rasilu0", CHIDG_PRECON_RASILU0}, {"hb", CHIDG_PRECON_HB}};
    const auto it = kinds.find(name);
    if (it == kinds.end()) throw Error(CHIDG_GPU_EINVAL, "create_preconditioner: invalid preconditioner '" + name + "'");
    return std::make_unique<Preconditioner>(it->second);
}

// fgmres_t with the options of linear_solver_t (defaults :23-40)
class LinearSolver {
public:
    LinearSolver() { chidg_gpu_fgmres_default_opts(&opts_); }
    // linear_solver%set (:113-131): numeric options by name
    void set(const std::string& key, double value) {
        static const std::map<std::string, double chidg_gpu_fgmres_opts::*> reals = {
            {"tol", &chidg_gpu_fgmres_opts::tol}, {"rtol", &chidg_gpu_fgmres_opts::rtol},
            {"inner_tol", &chidg_gpu_fgmres_opts::inner_tol}, {"inner_rtol", &chidg_gpu_fgmres_opts::inner_rtol},
            {"mixed_inner_rtol", &chidg_gpu_fgmres_opts::mixed_inner_rtol}};
        static const std::map<std::string, int32_t chidg_gpu_fgmres_opts::*> ints = {
            {"nmax", &chidg_gpu_fgmres_opts::nmax}, {"nkrylov", &chidg_gpu_fgmres_opts::nkrylov},
            {"inner_fgmres", &chidg_gpu_fgmres_opts::inner_fgmres}, {"inner_nmax", &chidg_gpu_fgmres_opts::inner_nmax},
            {"inner_nkrylov", &chidg_gpu_fgmres_opts::inner_nkrylov},
            {"use_controller", &chidg_gpu_fgmres_opts::use_controller},
            {"mixed_inner_nkrylov", &chidg_gpu_fgmres_opts::mixed_inner_nkrylov},
            {"mixed_inner_nmax", &chidg_gpu_fgmres_opts::mixed_inner_nmax}};
        if (auto r = reals.find(key); r != reals.end()) { opts_.*(r->second) = value; return; }
        if (auto i = ints.find(key); i != ints.end()) { opts_.*(i->second) = (int32_t)value; return; }
        throw Error(CHIDG_GPU_EINVAL, "linear_solver%set: unknown option '" + key + "'");
    }
    // string options: orthogonalization / inner_orthogonalization ('CGS', 'MGS'),
    // precision ('fp64', 'mixed_fp32', 'mixed_bf16', 'mixed_precon_fp32')
    void set(const std::string& key, const std::string& value) {
        auto orth = [&](const std::string& v) {
            if (v == "CGS" || v == "cgs") return CHIDG_ORTH_CGS;
            if (v == "MGS" || v == "mgs") return CHIDG_ORTH_MGS;
            throw Error(CHIDG_GPU_EINVAL, "linear_solver%set: orthogonalization must be 'CGS' or 'MGS'");
        };
        if (key == "orthogonalization") { opts_.orthogonalization = orth(value); return; }
        if (key == "inner_orthogonalization") { opts_.inner_orthogonalization = orth(value); return; }
        if (key == "precision") {
            static const std::map<std::string, int32_t> p = {{"fp64", CHIDG_GPU_FP64}, {"mixed_fp32", CHIDG_GPU_MIXED_FP32},
                                                             {"mixed_bf16", CHIDG_GPU_MIXED_BF16},
                                                             {"mixed_precon_fp32", CHIDG_GPU_MIXED_PRECON_FP32}};
            const auto it = p.find(value);
            if (it == p.end()) throw Error(CHIDG_GPU_EINVAL, "linear_solver%set: unknown precision '" + value + "'");
            opts_.precision = it->second;
            return;
        }
        throw Error(CHIDG_GPU_EINVAL, "linear_solver%set: unknown option '" + key + "'");
    }
    // fgmres%solve(A, x, b, M): x is zeroed on entry; niter, residual_norm set
    void solve(ChidgMatrix& A, ChidgVector& x, const ChidgVector& b, Preconditioner& M) {
        if (!M.handle()) M.init(A);
        chidg_gpu_fgmres_result r{};
        hist_.assign(8192, 0.0);
        detail::check(A.context().handle(),
                      chidg_gpu_fgmres_solve(A.handle(), M.handle(), b.handle(), x.handle(), &opts_, &r, hist_.data(),
                                             (int32_t)hist_.size()),
                      "fgmres%solve");
        hist_.resize((size_t)r.nhist);
        niter = r.niter;
        nrestart = r.nrestart;
        inner_iters = r.inner_iters;
        residual_norm = r.residual_norm;
        res_estimate = r.res_estimate;
        r0norm_initial = r.r0norm_initial;
    }
    // Independent systems packed block-diagonally in A (system s owns elements
    // sys_elem[s] .. sys_elem[s+1]-1): one result per system
    // (chidg_gpu_fgmres_solve_batched; no counterpart in the reference)
    std::vector<chidg_gpu_fgmres_result> solve_batched(ChidgMatrix& A, ChidgVector& x, const ChidgVector& b,
                                                       Preconditioner& M, const std::vector<int32_t>& sys_elem) {
        if (!M.handle()) M.init(A);
        if (sys_elem.size() < 2) throw Error(CHIDG_GPU_EINVAL, "solve_batched: no systems");
        std::vector<chidg_gpu_fgmres_result> r(sys_elem.size() - 1);
        detail::check(A.context().handle(),
                      chidg_gpu_fgmres_solve_batched(A.handle(), M.handle(), (int32_t)r.size(), sys_elem.data(), b.handle(),
                                                     x.handle(), &opts_, r.data(), nullptr, 0),
                      "fgmres%solve (batched)");
        return r;
    }
    const std::vector<double>& hist() const { return hist_; }
    const chidg_gpu_fgmres_opts& options() const { return opts_; }

    int32_t niter = 0, nrestart = 0, inner_iters = 0;
    double residual_norm = 0, res_estimate = 0, r0norm_initial = 0;

private:
    chidg_gpu_fgmres_opts opts_{};
    std::vector<double> hist_;
};

// create_linear_solver (mod_linear_solver.f90:27): 'fgmres'
inline std::unique_ptr<LinearSolver> create_linear_solver(std::string name) {
    std::transform(name.begin(), name.end(), name.begin(), [](unsigned char ch) { return (char)std::tolower(ch); });
    if (name != "fgmres") throw Error(CHIDG_GPU_EINVAL, "create_linear_solver: invalid linear solver '" + name + "'");
    return std::make_unique<LinearSolver>();
}

// The Euler DG residual and Jacobian of a hex box on the device
// (chidg_gpu_euler_*; the reference's update_space for the Euler equation set,
// src/spatial/mod_spatial.f90:40-197).  The matrix must hold the box's
// pattern: Pattern::box(nx, ny, nz, 5, (order + 1)^3).
class EulerAssembly {
public:
    EulerAssembly(Context& ctx, const chidg_gpu_euler_box& box) : ctx_(&ctx) {
        detail::check(ctx.handle(), chidg_gpu_euler_create(ctx.handle(), &box, &h_), "euler_create");
    }
    ~EulerAssembly() { if (h_) chidg_gpu_euler_destroy(h_); }
    EulerAssembly(const EulerAssembly&) = delete;
    EulerAssembly& operator=(const EulerAssembly&) = delete;

    // rhs = R(q); with A also A = dR/dq (every block overwritten)
    void assemble(const ChidgVector& q, ChidgVector& rhs, ChidgMatrix* A = nullptr) {
        detail::check(ctx_->handle(), chidg_gpu_euler_assemble(h_, q.handle(), rhs.handle(), A ? A->handle() : nullptr),
                      "euler_assemble");
    }
    // dtau[e * 5 + f] (type_fluid_pseudo_timestep.f90)
    std::vector<double> pseudo_timestep(const ChidgVector& q, const std::array<double, 5>& cfl, int nelem) {
        std::vector<double> dtau((size_t)nelem * 5);
        detail::check(ctx_->handle(), chidg_gpu_euler_pseudo_timestep(h_, q.handle(), cfl.data(), dtau.data()),
                      "euler_pseudo_timestep");
        return dtau;
    }

private:
    Context* ctx_ = nullptr;
    chidg_gpu_euler* h_ = nullptr;
};

// The first Newton step's system of a described Euler box (or harmonic-balance
// box) written into elements elem0.. of A and its segment of b
// (chidg_gpu_euler_fill_system; work's segment is overwritten)
inline void fill_euler_system(const chidg_gpu_euler_system& sys, ChidgMatrix& A, ChidgVector& b, ChidgVector& work,
                              int32_t elem0) {
    detail::check(A.context().handle(),
                  chidg_gpu_euler_fill_system(const_cast<chidg_gpu_euler_system*>(&sys), A.context().handle(), A.handle(),
                                              b.handle(), work.handle(), elem0),
                  "euler_fill_system");
}

// The continuous-batching server of the C ABI (chidg_gpu_serve_*; no
// counterpart in the reference).  A request's arrays (submit) or description
// (submit_fill's user pointer) must stay valid until its wait returns.
class Server {
public:
    Server(int device, int32_t slots, int64_t mem_budget, int32_t max_batch, int32_t precon_kind,
           const LinearSolver& solver) {
        detail::check(nullptr,
                      chidg_gpu_serve_create(device, slots, mem_budget, max_batch, precon_kind, &solver.options(), &h_),
                      "serve_create");
    }
    ~Server() { if (h_) chidg_gpu_serve_destroy(h_); }
    Server(const Server&) = delete;
    Server& operator=(const Server&) = delete;

    int64_t submit(const Pattern& pat, const double* values, const double* rhs) {
        const chidg_gpu_pattern v = pat.view();
        int64_t t = -1;
        detail::check(nullptr, chidg_gpu_serve_submit(h_, &v, values, rhs, &t), "serve_submit");
        return t;
    }
    int64_t submit_fill(const Pattern& pat, chidg_gpu_fill_fn fill, void* user) {
        const chidg_gpu_pattern v = pat.view();
        int64_t t = -1;
        detail::check(nullptr, chidg_gpu_serve_submit_fill(h_, &v, fill, user, &t), "serve_submit_fill");
        return t;
    }
    // an Euler system written on the device when its batch is formed
    int64_t submit_euler(const Pattern& pat, const chidg_gpu_euler_system& sys) {
        return submit_fill(pat, chidg_gpu_euler_fill_system, const_cast<chidg_gpu_euler_system*>(&sys));
    }
    // the request's solution into x (its vector length); timing: arrival,
    // start, finish (seconds since the server's creation) and the batch size
    chidg_gpu_fgmres_result wait(int64_t ticket, double* x, std::array<double, 4>* timing = nullptr) {
        chidg_gpu_fgmres_result r{};
        std::array<double, 4> t{};
        detail::check(nullptr, chidg_gpu_serve_wait(h_, ticket, x, &r, t.data()), "serve_wait");
        if (timing) *timing = t;
        return r;
    }
    // batch i's record (chidg_gpu_serve_batch_log)
    std::array<double, 9> batch_log(int64_t i) {
        std::array<double, 9> rec{};
        detail::check(nullptr, chidg_gpu_serve_batch_log(h_, i, rec.data()), "serve_batch_log");
        return rec;
    }

private:
    chidg_gpu_server* h_ = nullptr;
};

}  // namespace chidg_gpu

#endif
