// matrix_io.cu -- matrices to and from files: chidg_matrix%to_file
// (src/containers/type_chidg_matrix.f90:1451-1507) as text, and a binary
// image of a matrix (pattern and packed FP64 values) that saves and loads
// without loss.  Host code: the values pass through host memory in chunks.
#include "chidg_gpu_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace chidg;

namespace {

// Fortran Fw.d / Ew.d edit descriptors for w = 24, d = 14 as gfortran writes
// them: right-justified, a leading "0." in E form, "E+dd" exponents up to 99
// and "+ddd" beyond, asterisks when the value does not fit.
std::string fit24(const std::string& s) {
    if (s.size() > 24) return std::string(24, '*');
    return std::string(24 - s.size(), ' ') + s;
}
std::string fmt_F24_14(double v) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%.14f", v);
    return fit24(buf);
}
std::string fmt_E24_14(double v) {
    if (std::isnan(v)) return fit24("NaN");
    if (std::isinf(v)) return fit24(v > 0 ? "Infinity" : "-Infinity");
    std::string digits(14, '0');
    int exp10 = 0;
    if (v != 0.0) {
        char buf[64];
        std::snprintf(buf, sizeof(buf), "%.13e", std::fabs(v));   // d.ddddddddddddde+XX: 14 significant digits
        digits = std::string(1, buf[0]) + std::string(buf + 2, 13);
        exp10 = std::atoi(std::strchr(buf, 'e') + 1) + 1;           // 0.d1d2... x 10^exp10
    }
    std::string s = (std::signbit(v) && v != 0.0 ? "-" : "") + std::string("0.") + digits;
    const int ae = std::abs(exp10);
    char eb[16];
    if (ae <= 99) std::snprintf(eb, sizeof(eb), "E%c%02d", exp10 < 0 ? '-' : '+', ae);
    else std::snprintf(eb, sizeof(eb), "%c%03d", exp10 < 0 ? '-' : '+', ae);
    return fit24(s + eb);
}
// add_to_line (src/tools/messenger.f90:505-640): a real(8) in E24.14 below 0.1
// in magnitude and from 1e9 up, in F24.14 strictly between; an integer in
// I10; then adjustl + trim, centred in a 25-column field by adding a blank on
// each side until it is at least 25 long, cut to 25.
std::string trim_both(const std::string& s) {
    const size_t a = s.find_first_not_of(' ');
    if (a == std::string::npos) return std::string();
    return s.substr(a, s.find_last_not_of(' ') - a + 1);
}
std::string column25(std::string s) {
    while (s.size() < 25) s = " " + s + " ";
    return s.substr(0, 25);
}
std::string field_real(double v) {
    const double a = std::fabs(v);
    std::string s;
    if (a < 0.1) s = fmt_E24_14(v);
    else if (a > 0.1 && a < 1.e9) s = fmt_F24_14(v);
    else s = fmt_E24_14(v);
    return column25(trim_both(s));
}
std::string field_int(int64_t i) {
    return column25(std::to_string(i));
}

// Binary image: a fixed header, the pattern arrays, the packed values.
constexpr char kMagic[8] = {'C', 'H', 'I', 'D', 'G', 'M', 'A', 'T'};
constexpr uint32_t kVersion = 1;
struct ImageHeader {
    char magic[8];
    uint32_t version;
    uint32_t flags;          // bit 0: transposed
    int32_t nelem, ntime;
    int64_t nblocks, nval;
};
static_assert(sizeof(ImageHeader) == 40, "image header layout");

constexpr size_t kChunk = (size_t)64 << 20;   // bytes of values per host transfer

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() { if (f) std::fclose(f); }
};

}  // namespace

// chidg_matrix%to_file: for every time level, element and LOCAL block of the
// row (storage order), the block's entries column by column as lines
// " irow, icol, nblk, value" (25-column fields, 1-based indices
// irow = b (ielem - 1) + i, icol = b (ielement_g - 1) + j with b the block's
// row count, nblk the row's LOCAL block count).  Like the reference it writes
// no time offset and assumes one block size for all elements.
extern "C" int chidg_gpu_matrix_to_file(chidg_gpu_matrix* A, const char* path) {
    if (!A || !path) return CHIDG_GPU_EINVAL;
    chidg_gpu_ctx* ctx = A->ctx;
    cudaSetDevice(ctx->device);
    std::vector<double> v((size_t)A->nval);
    cudaError_t e = cudaMemcpyAsync(v.data(), A->val.ptr, sizeof(double) * v.size(), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "to_file download");
    File out(path, "w");
    if (!out.f) return fail(ctx, CHIDG_GPU_EINVAL, std::string("to_file: cannot open ") + path);
    std::string line;
    for (int t = 0; t < A->ntime; ++t)
        for (int el = 0; el < A->nelem; ++el) {
            const auto& blks = A->lblk[A->row(el, t)];
            const std::string nblk = field_int((int64_t)blks.size());
            for (int32_t k : blks) {
                const int nr = A->bsize(A->re[k]), nc = A->bsize(A->ce[k]);
                const int64_t r0 = 1 + (int64_t)nr * el, c0 = 1 + (int64_t)nr * A->ce[k];
                const double* blk = v.data() + A->voff[k];
                for (int j = 0; j < nc; ++j)
                    for (int i = 0; i < nr; ++i) {
                        line.clear();
                        line += ' ';
                        line += field_int(r0 + i); line += ',';
                        line += field_int(c0 + j); line += ',';
                        line += nblk; line += ',';
                        line += field_real(blk[i + (size_t)j * nr]);
                        line += '\n';
                        if (std::fwrite(line.data(), 1, line.size(), out.f) != line.size())
                            return fail(ctx, CHIDG_GPU_EINVAL, "to_file: write failed");
                    }
            }
        }
    return CHIDG_GPU_OK;
}

extern "C" int chidg_gpu_matrix_get_pattern(chidg_gpu_matrix* A, int32_t* nelem, int32_t* ntime, int64_t* nblocks,
                                            int32_t* elem_nvars, int32_t* elem_nterms, int32_t* elem_proc,
                                            int32_t* blk_row_elem, int32_t* blk_row_time, int32_t* blk_col_elem,
                                            int32_t* blk_col_time, int32_t* blk_kind) {
    if (!A) return CHIDG_GPU_EINVAL;
    if (nelem) *nelem = A->nelem;
    if (ntime) *ntime = A->ntime;
    if (nblocks) *nblocks = A->nblk;
    auto copy = [](int32_t* dst, const std::vector<int32_t>& src) {
        if (dst) std::memcpy(dst, src.data(), sizeof(int32_t) * src.size());
    };
    copy(elem_nvars, A->nvars); copy(elem_nterms, A->nterms); copy(elem_proc, A->proc);
    copy(blk_row_elem, A->re); copy(blk_row_time, A->rt); copy(blk_col_elem, A->ce); copy(blk_col_time, A->ct);
    copy(blk_kind, A->kind);
    return CHIDG_GPU_OK;
}

extern "C" int chidg_gpu_matrix_save(chidg_gpu_matrix* A, const char* path) {
    if (!A || !path) return CHIDG_GPU_EINVAL;
    chidg_gpu_ctx* ctx = A->ctx;
    cudaSetDevice(ctx->device);
    File out(path, "wb");
    if (!out.f) return fail(ctx, CHIDG_GPU_EINVAL, std::string("save: cannot open ") + path);
    ImageHeader h{};
    std::memcpy(h.magic, kMagic, 8);
    h.version = kVersion;
    h.flags = A->transposed ? 1u : 0u;
    h.nelem = A->nelem; h.ntime = A->ntime; h.nblocks = A->nblk; h.nval = A->nval;
    bool ok = std::fwrite(&h, sizeof(h), 1, out.f) == 1;
    for (const std::vector<int32_t>* a : {&A->nvars, &A->nterms, &A->proc, &A->re, &A->rt, &A->ce, &A->ct, &A->kind})
        ok = ok && std::fwrite(a->data(), sizeof(int32_t), a->size(), out.f) == a->size();
    std::vector<double> buf(kChunk / sizeof(double));
    for (int64_t first = 0; ok && first < A->nval; first += (int64_t)buf.size()) {
        const size_t cnt = (size_t)std::min<int64_t>((int64_t)buf.size(), A->nval - first);
        cudaError_t e = cudaMemcpyAsync(buf.data(), (const double*)A->val.ptr + first, sizeof(double) * cnt,
                                        cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "save download");
        ok = std::fwrite(buf.data(), sizeof(double), cnt, out.f) == cnt;
    }
    return ok ? CHIDG_GPU_OK : fail(ctx, CHIDG_GPU_EINVAL, "save: write failed");
}

extern "C" int chidg_gpu_matrix_load(chidg_gpu_ctx* ctx, const char* path, chidg_gpu_matrix** out) {
    if (!ctx || !path || !out) return CHIDG_GPU_EINVAL;
    *out = nullptr;
    cudaSetDevice(ctx->device);
    File in(path, "rb");
    if (!in.f) return fail(ctx, CHIDG_GPU_EINVAL, std::string("load: cannot open ") + path);
    ImageHeader h{};
    if (std::fread(&h, sizeof(h), 1, in.f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 || h.version != kVersion)
        return fail(ctx, CHIDG_GPU_EINVAL, "load: not a matrix image of this version");
    if (h.nelem <= 0 || h.ntime <= 0 || h.nblocks <= 0 || h.nval <= 0 || h.nelem > (1 << 28) || h.nblocks > ((int64_t)1 << 40))
        return fail(ctx, CHIDG_GPU_EINVAL, "load: bad sizes in the header");
    std::vector<int32_t> nv(h.nelem), nt(h.nelem), pr(h.nelem), re(h.nblocks), rt(h.nblocks), ce(h.nblocks),
        ct(h.nblocks), kd(h.nblocks);
    bool ok = true;
    for (std::vector<int32_t>* a : {&nv, &nt, &pr, &re, &rt, &ce, &ct, &kd})
        ok = ok && std::fread(a->data(), sizeof(int32_t), a->size(), in.f) == a->size();
    if (!ok) return fail(ctx, CHIDG_GPU_EINVAL, "load: truncated pattern");
    chidg_gpu_pattern pt{};
    pt.nelem = h.nelem; pt.ntime = h.ntime; pt.nblocks = h.nblocks;
    pt.elem_nvars = nv.data(); pt.elem_nterms = nt.data(); pt.elem_proc = pr.data();
    pt.blk_row_elem = re.data(); pt.blk_row_time = rt.data(); pt.blk_col_elem = ce.data(); pt.blk_col_time = ct.data();
    pt.blk_kind = kd.data();
    chidg_gpu_matrix* A = nullptr;
    int st = chidg_gpu_matrix_create(ctx, &pt, &A);
    if (st) return st;
    if (A->nval != h.nval) { chidg_gpu_matrix_destroy(A); return fail(ctx, CHIDG_GPU_EINVAL, "load: value count does not match the pattern"); }
    std::vector<double> buf(kChunk / sizeof(double));
    for (int64_t first = 0; first < A->nval; first += (int64_t)buf.size()) {
        const size_t cnt = (size_t)std::min<int64_t>((int64_t)buf.size(), A->nval - first);
        if (std::fread(buf.data(), sizeof(double), cnt, in.f) != cnt) {
            chidg_gpu_matrix_destroy(A);
            return fail(ctx, CHIDG_GPU_EINVAL, "load: truncated values");
        }
        cudaError_t e = cudaMemcpyAsync((double*)A->val.ptr + first, buf.data(), sizeof(double) * cnt,
                                        cudaMemcpyHostToDevice, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) { chidg_gpu_matrix_destroy(A); return cuda_fail(ctx, e, "load upload"); }
    }
    A->stamp++;
    if ((h.flags & 1u) && (st = chidg_gpu_matrix_set_transposed(A, 1))) { chidg_gpu_matrix_destroy(A); return st; }
    *out = A;
    return CHIDG_GPU_OK;
}
