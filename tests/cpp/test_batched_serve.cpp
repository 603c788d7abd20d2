// Many systems through the C++ host layer (include/chidg_gpu.hpp): two Euler
// boxes of different orders, each system written on the device into its slice
// of one packed layout (fill_euler_system), solved together
// (LinearSolver::solve_batched) and one at a time (LinearSolver::solve), and
// served (Server::submit_euler).  Every solve reaches rtol 1e-8 and the three
// answers of each system agree to 1e-12.
#include "chidg_gpu.hpp"

#include <cmath>
#include <cstdio>

using namespace chidg_gpu;

namespace {
struct BoxSystem {
    int nx, ny, nz, order, nt;
    std::vector<double> q0, mass;
    chidg_gpu_euler_system sys{};
    Pattern pat;

    BoxSystem(int nx_, int ny_, int nz_, int order_, double mach) : nx(nx_), ny(ny_), nz(nz_), order(order_) {
        nt = (order + 1) * (order + 1) * (order + 1);
        const int nelem = nx * ny * nz;
        pat = Pattern::box(nx, ny, nz, 5, nt);
        const double gam = 1.4, rho = 1.0, p = 1.0 / gam, u = mach;
        q0.assign((size_t)nelem * 5 * nt, 0.0);
        for (int e = 0; e < nelem; ++e) {
            const double r = rho * (1.0 + 0.01 * std::sin(0.7 * e + 0.3));   // a density perturbation
            const double cons[5] = {r, r * u, 0.0, 0.0, p / (gam - 1.0) + 0.5 * r * u * u};
            for (int f = 0; f < 5; ++f) q0[((size_t)e * 5 + f) * nt] = cons[f];
        }
        const double vol = (1.0 / nx) * (1.0 / ny) * (1.0 / nz);
        mass.assign((size_t)nt * nt, 0.0);
        for (int i = 0; i < nt; ++i) mass[(size_t)i * nt + i] = vol;             // an SPD stand-in for the mass matrix
        chidg_gpu_euler_box& b = sys.box;
        b.nx = nx; b.ny = ny; b.nz = nz; b.order = order;
        for (int d = 0; d < 3; ++d) { b.lo[d] = 0.0; b.hi[d] = 1.0; b.vel_inf[d] = 0.0; }
        b.vel_inf[0] = u;
        for (int f = 0; f < 6; ++f) b.bc[f] = CHIDG_EULER_FARFIELD;
        b.rho_inf = rho; b.p_inf = p;
        sys.ntime = 1;
        sys.mass = mass.data();
        sys.q0 = q0.data();
        sys.cfl = 10.0;
    }
};

double relerr(const std::vector<double>& a, const std::vector<double>& b, size_t a0, size_t n) {
    double d = 0.0, s = 0.0;
    for (size_t i = 0; i < n; ++i) {
        d += (a[a0 + i] - b[i]) * (a[a0 + i] - b[i]);
        s += b[i] * b[i];
    }
    return std::sqrt(d / std::fmax(s, 1e-300));
}
}  // namespace

int main() {
    try {
        Context ctx(0);
        BoxSystem s1(3, 2, 2, 1, 0.3), s2(2, 2, 2, 2, 0.45);
        std::vector<int32_t> sys_elem;
        const Pattern packed = Pattern::concat({&s1.pat, &s2.pat}, &sys_elem);
        ChidgMatrix A(ctx, packed);
        ChidgVector b(A), work(A), x(A);
        fill_euler_system(s1.sys, A, b, work, sys_elem[0]);
        fill_euler_system(s2.sys, A, b, work, sys_elem[1]);
        auto solver = create_linear_solver("fgmres");
        solver->set("rtol", 1e-8);
        solver->set("tol", 0.0);
        solver->set("nkrylov", 30.0);
        solver->set("inner_fgmres", 0.0);
        auto M = create_preconditioner("ilu0");
        const auto res = solver->solve_batched(A, x, b, *M, sys_elem);
        const std::vector<double> xb = x.get();
        int fails = 0;
        std::vector<size_t> offs = {0, (size_t)s1.q0.size()};
        BoxSystem* systems[2] = {&s1, &s2};
        for (int s = 0; s < 2; ++s) {
            if (!(res[s].residual_norm <= 1.0001e-8 * res[s].r0norm_initial)) ++fails;
            // the same system alone
            ChidgMatrix As(ctx, systems[s]->pat);
            ChidgVector bs(As), ws(As), xs(As);
            fill_euler_system(systems[s]->sys, As, bs, ws, 0);
            auto Ms = create_preconditioner("ilu0");
            solver->solve(As, xs, bs, *Ms);
            const std::vector<double> x1 = xs.get();
            const double e1 = relerr(xb, x1, offs[s], x1.size());
            // and served
            Server srv(0, 1, (int64_t)1 << 32, 4, CHIDG_PRECON_ILU0, *solver);
            const int64_t t = srv.submit_euler(systems[s]->pat, systems[s]->sys);
            std::vector<double> x2(x1.size());
            const chidg_gpu_fgmres_result r2 = srv.wait(t, x2.data());
            const double e2 = relerr(xb, x2, offs[s], x2.size());
            const std::array<double, 9> rec = srv.batch_log(0);
            std::printf("system %d: %d iterations batched, %d alone, %d served; x alone %.2e, served %.2e; batch %g systems\n",
                        s, res[s].niter, solver->niter, r2.niter, e1, e2, rec[7]);
            if (!(e1 < 1e-12 && e2 < 1e-12 && r2.residual_norm <= 1.0001e-8 * r2.r0norm_initial && rec[7] == 1)) ++fails;
        }
        std::printf("%d failures\n", fails);
        return fails ? 1 : 0;
    } catch (const Error& e) {
        std::printf("error: %s\n", e.what());
        return 2;
    }
}
