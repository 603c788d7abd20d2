// synth.cpp -- seeded synthetic block Jacobians with the ChiDG block layout.
//
// Host-only input generator for tests and benchmarks (the reference cannot
// assemble Jacobians in this environment).  Every value depends only on
// (seed, block id, entry index) through a counter-based hash, so the result
// is independent of the thread count and any block can be regenerated alone.
//
// Block value model (column-major entry idx = r + c * nrows):
//   DIAG block   : shift * delta(r,c) + diag_rand / sqrt(ncols) * u
//   face block f : face_scale[f] / sqrt(ncols) * u      (f = XI_MIN .. ZETA_MAX)
//   other block  : other_scale / sqrt(ncols) * u        (chimera / bc / hb)
// with u uniform in [-1, 1).  Face scales let the lower (upwind) neighbours
// dominate, as the upwinded DG fluxes of a flow along +xi do.
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

namespace {

inline uint64_t mix(uint64_t z) {
    z ^= z >> 30;
    z *= 0xbf58476d1ce4e5b9ULL;
    z ^= z >> 27;
    z *= 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return z;
}
inline double unit(uint64_t seed, uint64_t blk, uint64_t idx) {
    const uint64_t h = mix(seed * 0x9E3779B97F4A7C15ULL ^ mix(blk * 0xC2B2AE3D27D4EB4FULL + 0x632BE59BD9B4E019ULL) ^
                           idx * 0x165667B19E3779F9ULL);
    return (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
}

template <typename F>
void parallel_for(int64_t n, int nthreads, F f) {
    if (nthreads <= 1 || n < 2) { f(0, n); return; }
    std::vector<std::thread> th;
    const int64_t chunk = (n + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; ++t) {
        const int64_t a = t * chunk, b = std::min<int64_t>(n, a + chunk);
        if (a >= b) break;
        th.emplace_back([=]() { f(a, b); });
    }
    for (auto& x : th) x.join();
}

}  // namespace

extern "C" {

// btype: 0..5 = face XI_MIN..ZETA_MAX, 6 = DIAG, 7 = other.
// params: [shift, diag_rand, s_ximin, s_ximax, s_etamin, s_etamax, s_zetamin, s_zetamax, other]
int chidg_synth_blocks(int64_t nblocks, const int32_t* nr, const int32_t* nc, const int64_t* voff,
                       const int32_t* btype, uint64_t seed, const double* params, double* out, int nthreads) {
    parallel_for(nblocks, nthreads, [&](int64_t k0, int64_t k1) {
        for (int64_t k = k0; k < k1; ++k) {
            const int m = nr[k], n = nc[k], t = btype[k];
            double* A = out + voff[k];
            double scale;
            if (t == 6) scale = params[1];
            else if (t >= 0 && t < 6) scale = params[2 + t];
            else scale = params[8];
            scale /= std::sqrt((double)n);
            for (int64_t idx = 0; idx < (int64_t)m * n; ++idx) A[idx] = scale * unit(seed, (uint64_t)k, (uint64_t)idx);
            if (t == 6)
                for (int r = 0; r < m && r < n; ++r) A[r + (int64_t)r * m] += params[0];
        }
    });
    return 0;
}

int chidg_synth_vector(int64_t n, uint64_t seed, double* out, int nthreads) {
    parallel_for(n, nthreads, [&](int64_t a, int64_t b) {
        for (int64_t i = a; i < b; ++i) out[i] = unit(seed, 0xFFFFFFFFULL, (uint64_t)i);
    });
    return 0;
}

}  // extern "C"
