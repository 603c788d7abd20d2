// The device Euler assembly through the C++ host layer (include/chidg_gpu.hpp):
// a freestream state (each element's mean mode holds the conserved variables,
// every other mode 0) has a zero residual, its Jacobian fills every block of
// the box pattern with finite values, and dtau = cfl h / (|u| + c).
#include "chidg_gpu.hpp"

#include <cmath>
#include <cstdio>

int main() {
    using namespace chidg_gpu;
    const int nx = 3, ny = 2, nz = 2, order = 1, nt = 8;
    chidg_gpu_euler_box box{};
    box.nx = nx; box.ny = ny; box.nz = nz; box.order = order;
    for (int d = 0; d < 3; ++d) { box.lo[d] = 0.0; box.hi[d] = 1.0; }
    for (int f = 0; f < 6; ++f) box.bc[f] = CHIDG_EULER_FARFIELD;
    const double gam = 1.4, rho = 1.0, p = 1.0 / gam, u[3] = {0.3, 0.1, -0.05};
    box.rho_inf = rho; box.p_inf = p;
    for (int d = 0; d < 3; ++d) box.vel_inf[d] = u[d];
    try {
        Context ctx(0);
        ChidgMatrix A(ctx, Pattern::box(nx, ny, nz, 5, nt));
        const int nelem = nx * ny * nz;
        std::vector<double> q0((size_t)nelem * 5 * nt, 0.0);
        const double u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        const double cons[5] = {rho, rho * u[0], rho * u[1], rho * u[2], p / (gam - 1.0) + 0.5 * rho * u2};
        for (int e = 0; e < nelem; ++e)
            for (int f = 0; f < 5; ++f) q0[((size_t)e * 5 + f) * nt] = cons[f];
        ChidgVector q(A, q0), rhs(A);
        EulerAssembly asmb(ctx, box);
        asmb.assemble(q, rhs, &A);
        const double rn = rhs.norm();
        const std::vector<double> vals = A.values();
        const int b = 5 * nt;
        int bad = 0;
        for (size_t k = 0; k < vals.size() / ((size_t)b * b); ++k) {
            double mx = 0.0;
            for (int i = 0; i < b * b; ++i) {
                const double v = vals[k * b * b + i];
                if (!std::isfinite(v)) ++bad;
                mx = std::fmax(mx, std::fabs(v));
            }
            if (mx == 0.0) ++bad;
        }
        const std::vector<double> dtau = asmb.pseudo_timestep(q, {2.0, 2.0, 2.0, 2.0, 2.0}, nelem);
        const double h = std::cbrt((1.0 / nx) * (1.0 / ny) * (1.0 / nz));
        const double want = 2.0 * h / (std::sqrt(u2) + 1.0);
        double derr = 0.0;
        for (double d : dtau) derr = std::fmax(derr, std::fabs(d - want) / want);
        std::printf("|R| = %.3e, bad blocks = %d, dtau error = %.3e\n", rn, bad, derr);
        return (rn < 1e-13 && bad == 0 && derr < 1e-13) ? 0 : 1;
    } catch (const Error& e) {
        std::printf("error: %s\n", e.what());
        return 2;
    }
}
