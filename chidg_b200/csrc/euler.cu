// euler.cu -- Euler DG residual and Jacobian on hex boxes, assembled on the
// device straight into the vector and the block matrix of the linear solves.
//
// The discretisation is ChiDG's (mod_spatial.f90:40-197 driving the Euler
// operators of src/equations/fluid/euler/): modal tensor Legendre basis in the
// reference's mode order (mod_legendre.f90, mod_ordering.f90), Gauss-Legendre
// quadrature with ceil(3 (P+1) / 2) nodes per direction (gq_rule = 2,
// mod_quadrature.f90:68-80), R = -int grad(phi).F dV (euler_volume_operator,
// stored negated by store_volume_integrals, mod_integrate.f90:652-779) +
// int phi Fhat.n dA with Fhat the central average plus Roe's upwind term with
// Harten's entropy fix (euler_boundary_average_operator, euler_roe_operator)
// on interior faces and F(Q_bc).n on boundary faces (euler_bc_operator) with
// the farfield (bc_state_farfield.f90) or extrapolation
// (bc_state_fluid_extrapolate.f90) state.  The Jacobian is exact: forward-mode
// dual numbers through the pointwise functions, as the reference's DNAD types
// (AD_D) carry derivatives, and the chain rule through the basis.
//
// One CTA per element.  Shared memory holds the modes of the element and of
// its face neighbours and the weighted pointwise data (flux and its 5x5
// derivatives at every volume node; face integrand and its derivatives with
// respect to both states at every face node).  The residual, the DIAG block and
// the face blocks are then contractions over the nodes, each output written by
// one thread: no atomics, one writer per value.  Each element integrates its
// own faces (the reference evaluates a shared face once and negates it for the
// neighbour, integrate_boundary_scalar_flux, mod_integrate.f90:219-346; the
// two agree to rounding since the numerical flux is antisymmetric).
#include "chidg_gpu_internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

using namespace chidg;

namespace {

constexpr double kGamma = 1.4;          // mod_fluid.f90:10
constexpr double kRgas = 287.15;        // mod_fluid.f90:9
constexpr double kRkTol = 20.0 * 2.220446049250313e-16;   // RKTOL, mod_constants.f90:241
constexpr double kFixEps = 0.01;        // entropy-fix width, euler_roe_operator.f90
constexpr int kMaxOrder = 3;
constexpr int kThreads = 256;

// Legendre degrees (xi, eta, zeta) of the first 64 modes in the reference's
// order (mod_ordering.f90, xi/eta/zeta_order_3d, 0-based); each prefix of
// (P+1)^3 modes is the full order-P set.
constexpr int kModes[64][3] = {
    {0, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {1, 1, 1}, {0, 2, 0},
    {0, 0, 2}, {2, 0, 0}, {0, 2, 1}, {0, 1, 2}, {1, 2, 0}, {1, 0, 2}, {2, 1, 0}, {2, 0, 1}, {0, 2, 2},
    {1, 2, 1}, {1, 1, 2}, {2, 2, 0}, {2, 0, 2}, {2, 1, 1}, {1, 2, 2}, {2, 2, 1}, {2, 1, 2}, {2, 2, 2},
    {3, 0, 0}, {0, 3, 0}, {0, 0, 3}, {3, 1, 0}, {3, 0, 1}, {1, 3, 0}, {1, 0, 3}, {0, 3, 1}, {0, 1, 3},
    {3, 2, 0}, {3, 0, 2}, {3, 1, 1}, {2, 3, 0}, {2, 0, 3}, {1, 3, 1}, {1, 1, 3}, {0, 3, 2}, {0, 2, 3},
    {3, 2, 1}, {3, 1, 2}, {3, 3, 0}, {3, 0, 3}, {2, 3, 1}, {2, 1, 3}, {1, 3, 2}, {1, 2, 3}, {0, 3, 3},
    {3, 2, 2}, {3, 3, 1}, {3, 1, 3}, {2, 3, 2}, {2, 2, 3}, {1, 3, 3}, {3, 3, 2}, {3, 2, 3}, {2, 3, 3},
    {3, 3, 3}};

// ---- forward-mode dual numbers ------------------------------------------------
template <int N>
struct Dual {
    double v;
    double d[N];
};
template <int N> __device__ __forceinline__ Dual<N> mk(double v) {
    Dual<N> r; r.v = v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = 0.0;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r; r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r; r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, double b) { Dual<N> r = a; r.v += b; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator+(double b, const Dual<N>& a) { return a + b; }
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, double b) { Dual<N> r = a; r.v -= b; return r; }
template <int N> __device__ __forceinline__ Dual<N> operator-(double b, const Dual<N>& a) { return (-a) + b; }
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, double b) {
    Dual<N> r; r.v = a.v * b;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(double b, const Dual<N>& a) { return a * b; }
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, double b) { return a * (1.0 / b); }
template <int N> __device__ __forceinline__ Dual<N> operator/(double a, const Dual<N>& b) { return mk<N>(a) / b; }
template <int N> __device__ __forceinline__ Dual<N> dsqrt(const Dual<N>& a) {
    Dual<N> r; r.v = sqrt(a.v);
    const double h = 0.5 / r.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * h;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> dpow(const Dual<N>& a, double e) {
    Dual<N> r; r.v = pow(a.v, e);
    const double s = e * pow(a.v, e - 1.0);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> dabs(const Dual<N>& a) { return a.v < 0.0 ? -a : a; }
// select by a condition evaluated on values (the branch the AD type takes)
template <int N> __device__ __forceinline__ Dual<N> dsel(bool c, const Dual<N>& a, const Dual<N>& b) { return c ? a : b; }

// ---- pointwise Euler functions --------------------------------------------------
template <int N> __device__ __forceinline__ Dual<N> pressure(const Dual<N>* Q) {
    return (kGamma - 1.0) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0]);
}

// F_d(Q): the physical flux in direction d (euler_volume_operator.f90:112-181)
template <int N> __device__ __forceinline__ void flux_dir(const Dual<N>* Q, int d, Dual<N>* F) {
    const Dual<N> inv = 1.0 / Q[0];
    const Dual<N> vel = Q[1 + d] * inv;
    const Dual<N> p = pressure(Q);
    const Dual<N> H = (Q[4] + p) * inv;
    F[0] = Q[0] * vel;
    F[1] = Q[1] * vel;
    F[2] = Q[2] * vel;
    F[3] = Q[3] * vel;
    F[1 + d] = F[1 + d] + p;
    F[4] = Q[0] * H * vel;
}

// Roe's upwind term per unit area with the entropy fix (euler_roe_operator.f90)
template <int N> __device__ void roe_upwind(const Dual<N>* Qm, const Dual<N>* Qp, const double* n, Dual<N>* up) {
    const Dual<N> inv_m = 1.0 / Qm[0], inv_p = 1.0 / Qp[0];
    const Dual<N> p_m = pressure(Qm), p_p = pressure(Qp);
    const Dual<N> H_m = (Qm[4] + p_m) * inv_m, H_p = (Qp[4] + p_p) * inv_p;
    const Dual<N> u_m = Qm[1] * inv_m, v_m = Qm[2] * inv_m, w_m = Qm[3] * inv_m;
    const Dual<N> u_p = Qp[1] * inv_p, v_p = Qp[2] * inv_p, w_p = Qp[3] * inv_p;
    const Dual<N> vmag_m = u_m * n[0] + v_m * n[1] + w_m * n[2];
    const Dual<N> vmag_p = u_p * n[0] + v_p * n[1] + w_p * n[2];
    const Dual<N> sm = dsqrt(Qm[0]), sp = dsqrt(Qp[0]);
    const Dual<N> ssum = sm + sp;
    const Dual<N> rtil = dsqrt(Qp[0] * Qm[0]);
    const Dual<N> util = (sm * u_m + sp * u_p) / ssum;
    const Dual<N> vtil = (sm * v_m + sp * v_p) / ssum;
    const Dual<N> wtil = (sm * w_m + sp * w_p) / ssum;
    const Dual<N> Htil = (sm * H_m + sp * H_p) / ssum;
    const Dual<N> vmagtil = util * n[0] + vtil * n[1] + wtil * n[2];
    const Dual<N> qtil2 = util * util + vtil * vtil + wtil * wtil;
    const Dual<N> ctil = dsqrt((kGamma - 1.0) * (Htil - 0.5 * qtil2));
    const Dual<N> ctil2 = ctil * ctil;
    const Dual<N> delr = Qm[0] - Qp[0];
    const Dual<N> delu = u_m - u_p, delv = v_m - v_p, delw = w_m - w_p;
    const Dual<N> delvmag = vmag_m - vmag_p;
    const Dual<N> delp = p_m - p_p;
    Dual<N> lam[3] = {dabs(vmagtil - ctil), dabs(vmagtil), dabs(vmagtil + ctil)};
    const Dual<N> ec = kFixEps * ctil;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const bool small = (-ec.v < lam[i].v) && (lam[i].v < ec.v);
        lam[i] = dsel(small, 0.5 * (ec + lam[i] * lam[i] / ec), dabs(lam[i]));
    }
    const Dual<N> C1 = dabs(lam[0]) * (delp - rtil * ctil * delvmag) / (2.0 * ctil2);
    const Dual<N> C2a = dabs(lam[1]) * (delr - delp / ctil2);
    const Dual<N> C2b = dabs(lam[1]) * rtil;
    const Dual<N> C3 = dabs(lam[2]) * (delp + rtil * ctil * delvmag) / (2.0 * ctil2);
    up[0] = 0.5 * (C1 + C2a + C3);
    up[1] = 0.5 * (C1 * (util - ctil * n[0]) + C2a * util + C2b * (delu - delvmag * n[0]) + C3 * (util + ctil * n[0]));
    up[2] = 0.5 * (C1 * (vtil - ctil * n[1]) + C2a * vtil + C2b * (delv - delvmag * n[1]) + C3 * (vtil + ctil * n[1]));
    up[3] = 0.5 * (C1 * (wtil - ctil * n[2]) + C2a * wtil + C2b * (delw - delvmag * n[2]) + C3 * (wtil + ctil * n[2]));
    up[4] = 0.5 * (C1 * (Htil - ctil * vmagtil) + C2a * (qtil2 / 2.0)
                   + C2b * (util * delu + vtil * delv + wtil * delw - vmagtil * delvmag) + C3 * (Htil + ctil * vmagtil));
}

struct Freestream {
    double rho, p, u[3];
};

// exterior state of the farfield condition (bc_state_farfield.f90, compute_bc_state)
template <int N> __device__ void farfield_state(const Dual<N>* Qm, const double* n, const Freestream& fs, Dual<N>* Qb) {
    const double T_in = fs.p / (fs.rho * kRgas);
    const double c_in = sqrt(kGamma * kRgas * T_in);
    const Dual<N> p_m = pressure(Qm);
    const Dual<N> T_m = p_m / (Qm[0] * kRgas);
    const Dual<N> c_m = dsqrt(kGamma * kRgas * T_m);
    const Dual<N> nmom = Qm[1] * n[0] + Qm[2] * n[1] + Qm[3] * n[2];
    const bool inflow = nmom.v <= kRkTol;
    const Dual<N> u_m = Qm[1] / Qm[0], v_m = Qm[2] / Qm[0], w_m = Qm[3] / Qm[0];
    const double un_in = fs.u[0] * n[0] + fs.u[1] * n[1] + fs.u[2] * n[2];
    const double R_inf = un_in - 2.0 * c_in / (kGamma - 1.0);
    const Dual<N> un_m = u_m * n[0] + v_m * n[1] + w_m * n[2];
    const Dual<N> R_ext = un_m + 2.0 * c_m / (kGamma - 1.0);
    const Dual<N> c_bc = ((kGamma - 1.0) / 4.0) * (R_ext - R_inf);
    const Dual<N> half = 0.5 * (R_ext + R_inf);
    Dual<N> ut, vt, wt, entropy;
    if (inflow) {
        ut = mk<N>(fs.u[0] - un_in * n[0]);
        vt = mk<N>(fs.u[1] - un_in * n[1]);
        wt = mk<N>(fs.u[2] - un_in * n[2]);
        entropy = mk<N>(fs.p / pow(fs.rho, kGamma));
    } else {
        ut = u_m - un_m * n[0];
        vt = v_m - un_m * n[1];
        wt = w_m - un_m * n[2];
        entropy = p_m / dpow(Qm[0], kGamma);
    }
    const Dual<N> rho_bc = dpow(c_bc * c_bc / (entropy * kGamma), 1.0 / (kGamma - 1.0));
    Qb[0] = rho_bc;
    Qb[1] = (half * n[0] + ut) * rho_bc;
    Qb[2] = (half * n[1] + vt) * rho_bc;
    Qb[3] = (half * n[2] + wt) * rho_bc;
    const Dual<N> p_bc = dpow(rho_bc, kGamma) * entropy;
    Qb[4] = p_bc / (kGamma - 1.0) + 0.5 * (Qb[1] * Qb[1] + Qb[2] * Qb[2] + Qb[3] * Qb[3]) / rho_bc;
}

// ---- kernel --------------------------------------------------------------------
struct BoxGeom {
    int nx, ny, nz;
    int nt, qv, qf;             // modes, volume nodes, face nodes
    double area[3];             // |scaled normal| on xi, eta, zeta faces
    int bc[6];
    Freestream fs;
};

struct Tables {
    const double* phi;          // [qv][nt]
    const double* grad;         // [3][qv][nt] physical gradients
    const double* wv;           // [qv] weights * jinv
    const double* phif;         // [6][qf][nt]
    const double* wf;           // [qf] face weights (reference)
};

__device__ __forceinline__ int neighbour(const BoxGeom& g, int e, int face) {
    const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
    switch (face) {
        case 0: return i > 0 ? e - 1 : -1;
        case 1: return i < g.nx - 1 ? e + 1 : -1;
        case 2: return j > 0 ? e - g.nx : -1;
        case 3: return j < g.ny - 1 ? e + g.nx : -1;
        case 4: return k > 0 ? e - g.nx * g.ny : -1;
        default: return k < g.nz - 1 ? e + g.nx * g.ny : -1;
    }
}

// Shared memory (doubles): U[7][5 nt] | WF[qv][3][5] | WdF[qv][3][5][5] |
// FI[6][qf][5] | Fs[6][qf][5][5] | Fn[6][qf][5][5].  At P3 the volume data
// and the face data do not fit together: the element runs a volume pass and
// then a face pass over the same space after U (two_pass below).
__host__ __device__ constexpr bool two_pass(int nt) { return nt > 27; }
__host__ __device__ inline size_t smem_doubles(int nt, int qv, int qf) {
    const size_t vol = (size_t)qv * 15 + (size_t)qv * 75, face = (size_t)6 * qf * 5 + (size_t)12 * qf * 25;
    return (size_t)7 * 5 * nt + (two_pass(nt) ? (vol > face ? vol : face) : vol + face);
}

// the pointwise data of volume node t (flux and its 5x5 derivatives, weighted)
template <int NT>
__device__ __forceinline__ void volume_node(const Tables& tb, const double* sU, int t, int nt, double* sWF, double* sWdF) {
    const int b = 5 * nt;
    Dual<5> Q[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        double s = 0.0;
        for (int m = 0; m < nt; ++m) s += tb.phi[t * nt + m] * sU[6 * b + f * nt + m];
        Q[f] = mk<5>(s);
        Q[f].d[f] = 1.0;
    }
    const double w = tb.wv[t];
    for (int d = 0; d < 3; ++d) {
        Dual<5> F[5];
        flux_dir(Q, d, F);
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            sWF[(t * 3 + d) * 5 + f] = w * F[f].v;
#pragma unroll
            for (int gg = 0; gg < 5; ++gg) sWdF[((t * 3 + d) * 5 + f) * 5 + gg] = w * F[f].d[gg];
        }
    }
}

// the pointwise data of face node qq of face `face` (integrand and its
// derivatives with respect to the own and the neighbour's state, weighted)
template <int NT>
__device__ __forceinline__ void face_node(const BoxGeom& g, const Tables& tb, const double* sU, const int* nbr, int face,
                                          int qq, int nt, double* sFI, double* sFs, double* sFn) {
    const int b = 5 * nt, qf = g.qf;
    const int d = face >> 1;
    const double s = (face & 1) ? 1.0 : -1.0;
    const double a = g.area[d];
    double n[3] = {0.0, 0.0, 0.0};
    n[d] = s;
    const double w = tb.wf[qq];
    const double* pm = tb.phif + ((size_t)face * qf + qq) * nt;
    double Qm0[5], Qp0[5];
#pragma unroll
    for (int f = 0; f < 5; ++f) {
        double sm_ = 0.0;
        for (int m = 0; m < nt; ++m) sm_ += pm[m] * sU[6 * b + f * nt + m];
        Qm0[f] = sm_;
    }
    double* FI = sFI + ((size_t)face * qf + qq) * 5;
    double* Fs = sFs + ((size_t)face * qf + qq) * 25;
    double* Fn = sFn + ((size_t)face * qf + qq) * 25;
    if (nbr[face] >= 0) {
        const double* pp = tb.phif + ((size_t)(face ^ 1) * qf + qq) * nt;
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            double sp_ = 0.0;
            for (int m = 0; m < nt; ++m) sp_ += pp[m] * sU[face * b + f * nt + m];
            Qp0[f] = sp_;
        }
        // two passes: derivatives with respect to the own state, then the neighbour's
        for (int side = 0; side < 2; ++side) {
            Dual<5> Qm[5], Qp[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                Qm[f] = mk<5>(Qm0[f]);
                Qp[f] = mk<5>(Qp0[f]);
                if (side == 0) Qm[f].d[f] = 1.0; else Qp[f].d[f] = 1.0;
            }
            Dual<5> Fm[5], Fp[5], up[5];
            flux_dir(Qm, d, Fm);
            flux_dir(Qp, d, Fp);
            roe_upwind(Qm, Qp, n, up);
            double* dst = side == 0 ? Fs : Fn;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const Dual<5> I = (0.5 * s * a) * (Fm[f] + Fp[f]) + a * up[f];
                if (side == 0) FI[f] = w * I.v;
#pragma unroll
                for (int gg = 0; gg < 5; ++gg) dst[f * 5 + gg] = w * I.d[gg];
            }
        }
    } else {
        Dual<5> Qm[5], Qb[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            Qm[f] = mk<5>(Qm0[f]);
            Qm[f].d[f] = 1.0;
        }
        if (g.bc[face] == CHIDG_EULER_FARFIELD) {
            farfield_state(Qm, n, g.fs, Qb);
        } else {
#pragma unroll
            for (int f = 0; f < 5; ++f) Qb[f] = Qm[f];
        }
        Dual<5> F[5];
        flux_dir(Qb, d, F);
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            FI[f] = w * s * a * F[f].v;
#pragma unroll
            for (int gg = 0; gg < 5; ++gg) {
                Fs[f * 5 + gg] = w * s * a * F[f].d[gg];
                Fn[f * 5 + gg] = 0.0;
            }
        }
    }
}

// q and rhs: an element's segment at e * vs (vs = b for one time level, the
// element's stride over all its levels under harmonic balance)
template <int NT>
__global__ void __launch_bounds__(kThreads) k_euler_assemble(BoxGeom g, Tables tb, const double* __restrict__ q,
                                                            double* __restrict__ rhs, double* __restrict__ val,
                                                            const int64_t* __restrict__ blk_off, int64_t vs) {
    extern __shared__ double sm[];
    const int e = blockIdx.x;
    const int nt = NT, b = 5 * NT, qv = g.qv, qf = g.qf;
    constexpr bool TWO = two_pass(NT);
    double* sU = sm;                            // [7][5 nt]: own (slot 6) and face neighbours (slots 0..5)
    double* sWF = sU + 7 * 5 * nt;              // [qv][3][5]
    double* sWdF = sWF + (size_t)qv * 15;       // [qv][3][5][5]
    // face data after the volume data, or over it in the two-pass form
    double* sFI = TWO ? sWF : sWdF + (size_t)qv * 75;   // [6][qf][5]
    double* sFs = sFI + (size_t)6 * qf * 5;     // [6][qf][5][5]  d integrand / d own state
    double* sFn = sFs + (size_t)6 * qf * 25;    // [6][qf][5][5]  d integrand / d neighbour state
    int nbr[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) nbr[f] = neighbour(g, e, f);

    // 1. modes of the element and its neighbours
    for (int t = threadIdx.x; t < 7 * b; t += blockDim.x) {
        const int slot = t / b, i = t - slot * b;
        const int src = slot == 6 ? e : nbr[slot];
        sU[t] = src >= 0 ? q[(int64_t)src * vs + i] : 0.0;
    }
    __syncthreads();

    if constexpr (!TWO) {
        // 2. pointwise data at volume nodes and face nodes
        for (int t = threadIdx.x; t < qv + 6 * qf; t += blockDim.x) {
            if (t < qv) volume_node<NT>(tb, sU, t, nt, sWF, sWdF);
            else {
                const int u = t - qv, face = u / qf, qq = u - face * qf;
                face_node<NT>(g, tb, sU, nbr, face, qq, nt, sFI, sFs, sFn);
            }
        }
        __syncthreads();

        // 3. residual: R[f, m] = -sum_q sum_d grad_d[q, m] WF[q, d, f] + sum_faces sum_q phif[q, m] FI[q, f]
        for (int t = threadIdx.x; t < b; t += blockDim.x) {
            const int f = t / nt, m = t - f * nt;
            double r = 0.0;
            for (int qq = 0; qq < qv; ++qq)
                r -= tb.grad[(0 * qv + qq) * nt + m] * sWF[(qq * 3 + 0) * 5 + f]
                   + tb.grad[(1 * qv + qq) * nt + m] * sWF[(qq * 3 + 1) * 5 + f]
                   + tb.grad[(2 * qv + qq) * nt + m] * sWF[(qq * 3 + 2) * 5 + f];
            for (int face = 0; face < 6; ++face)
                for (int qq = 0; qq < qf; ++qq)
                    r += tb.phif[((size_t)face * qf + qq) * nt + m] * sFI[((size_t)face * qf + qq) * 5 + f];
            rhs[(int64_t)e * vs + t] = r;
        }

        // 4. DIAG block and 5. face blocks (skipped for a residual-only call): one
        // thread per pair of (f, m, g) rows with the same f and g and modes m0,
        // m0 + 1, all nt columns n of both in registers, so each basis value
        // loaded feeds two FMAs; block entry (f nt + m, g nt + n) stored
        // column-major.  Lanes of a warp take consecutive mode pairs.
        if (val == nullptr) return;
        const int npair = (nt + 1) >> 1;
        for (int blk = 6; blk >= 0; --blk) {
            if (blk < 6 && nbr[blk] < 0) continue;
            double* out = val + blk_off[(int64_t)e * 7 + blk];
            for (int item = threadIdx.x; item < 25 * npair; item += blockDim.x) {
                const int mp = item % npair, fg = item / npair, f = fg % 5, gg = fg / 5;
                const int m0 = 2 * mp;
                const bool two = m0 + 1 < nt;
                const int m1 = two ? m0 + 1 : m0;
                double a0[NT], a1[NT];
#pragma unroll
                for (int n = 0; n < NT; ++n) { a0[n] = 0.0; a1[n] = 0.0; }
                if (blk == 6) {
                    for (int qq = 0; qq < qv; ++qq) {
                        const double w0 = sWdF[((qq * 3 + 0) * 5 + f) * 5 + gg];
                        const double w1 = sWdF[((qq * 3 + 1) * 5 + f) * 5 + gg];
                        const double w2 = sWdF[((qq * 3 + 2) * 5 + f) * 5 + gg];
                        const double* g0 = tb.grad + (size_t)(0 * qv + qq) * nt;
                        const double* g1 = tb.grad + (size_t)(1 * qv + qq) * nt;
                        const double* g2 = tb.grad + (size_t)(2 * qv + qq) * nt;
                        const double t0 = -(g0[m0] * w0 + g1[m0] * w1 + g2[m0] * w2);
                        const double t1 = -(g0[m1] * w0 + g1[m1] * w1 + g2[m1] * w2);
                        const double* ph = tb.phi + (size_t)qq * nt;
#pragma unroll
                        for (int n = 0; n < NT; ++n) {
                            const double p = ph[n];
                            a0[n] += t0 * p;
                            a1[n] += t1 * p;
                        }
                    }
                    for (int face = 0; face < 6; ++face) {
                        for (int qq = 0; qq < qf; ++qq) {
                            const double* pf = tb.phif + ((size_t)face * qf + qq) * nt;
                            const double w = sFs[((size_t)face * qf + qq) * 25 + f * 5 + gg];
                            const double t0 = pf[m0] * w, t1 = pf[m1] * w;
#pragma unroll
                            for (int n = 0; n < NT; ++n) {
                                const double p = pf[n];
                                a0[n] += t0 * p;
                                a1[n] += t1 * p;
                            }
                        }
                    }
                } else {
                    for (int qq = 0; qq < qf; ++qq) {
                        const double* pf = tb.phif + ((size_t)blk * qf + qq) * nt;
                        const double* pn = tb.phif + ((size_t)(blk ^ 1) * qf + qq) * nt;
                        const double w = sFn[((size_t)blk * qf + qq) * 25 + f * 5 + gg];
                        const double t0 = pf[m0] * w, t1 = pf[m1] * w;
#pragma unroll
                        for (int n = 0; n < NT; ++n) {
                            const double p = pn[n];
                            a0[n] += t0 * p;
                            a1[n] += t1 * p;
                        }
                    }
                }
                const int row = f * nt + m0;
#pragma unroll
                for (int n = 0; n < NT; ++n) {
                    double* col = out + (int64_t)(gg * nt + n) * b + row;
                    col[0] = a0[n];
                    if (two) col[1] = a1[n];
                }
            }
        }
    } else {
        // Two passes over the same shared memory.  Every value is accumulated in
        // the single-pass order: the volume pass leaves the residual's and the
        // DIAG block's volume sums in the outputs, and the face pass reloads and
        // continues them (each output value is read back by the thread that
        // wrote it).  Block rows: one (f, m, g) row and one half of its nt
        // columns per item, so the accumulators fit in registers.
        constexpr int NH = NT / 2;
        const int64_t* bo = blk_off + (int64_t)e * 7;
        // ---- volume pass
        for (int t = threadIdx.x; t < qv; t += blockDim.x) volume_node<NT>(tb, sU, t, nt, sWF, sWdF);
        __syncthreads();
        for (int t = threadIdx.x; t < b; t += blockDim.x) {
            const int f = t / nt, m = t - f * nt;
            double r = 0.0;
            for (int qq = 0; qq < qv; ++qq)
                r -= tb.grad[(0 * qv + qq) * nt + m] * sWF[(qq * 3 + 0) * 5 + f]
                   + tb.grad[(1 * qv + qq) * nt + m] * sWF[(qq * 3 + 1) * 5 + f]
                   + tb.grad[(2 * qv + qq) * nt + m] * sWF[(qq * 3 + 2) * 5 + f];
            rhs[(int64_t)e * vs + t] = r;
        }
        if (val != nullptr) {
            double* out = val + bo[6];
            for (int item = threadIdx.x; item < 25 * nt * 2; item += blockDim.x) {
                const int h = item & 1, m = (item >> 1) % nt, fg = (item >> 1) / nt, f = fg % 5, gg = fg / 5;
                double a0[NH];
#pragma unroll
                for (int n = 0; n < NH; ++n) a0[n] = 0.0;
                for (int qq = 0; qq < qv; ++qq) {
                    const double w0 = sWdF[((qq * 3 + 0) * 5 + f) * 5 + gg];
                    const double w1 = sWdF[((qq * 3 + 1) * 5 + f) * 5 + gg];
                    const double w2 = sWdF[((qq * 3 + 2) * 5 + f) * 5 + gg];
                    const double t0 = -(tb.grad[(size_t)(0 * qv + qq) * nt + m] * w0 +
                                        tb.grad[(size_t)(1 * qv + qq) * nt + m] * w1 +
                                        tb.grad[(size_t)(2 * qv + qq) * nt + m] * w2);
                    const double* ph = tb.phi + (size_t)qq * nt + h * NH;
#pragma unroll
                    for (int n = 0; n < NH; ++n) a0[n] += t0 * ph[n];
                }
#pragma unroll
                for (int n = 0; n < NH; ++n) out[(int64_t)(gg * nt + h * NH + n) * b + f * nt + m] = a0[n];
            }
        }
        __syncthreads();
        // ---- face pass
        for (int t = threadIdx.x; t < 6 * qf; t += blockDim.x) {
            const int face = t / qf, qq = t - face * qf;
            face_node<NT>(g, tb, sU, nbr, face, qq, nt, sFI, sFs, sFn);
        }
        __syncthreads();
        for (int t = threadIdx.x; t < b; t += blockDim.x) {
            const int f = t / nt, m = t - f * nt;
            double r = rhs[(int64_t)e * vs + t];
            for (int face = 0; face < 6; ++face)
                for (int qq = 0; qq < qf; ++qq)
                    r += tb.phif[((size_t)face * qf + qq) * nt + m] * sFI[((size_t)face * qf + qq) * 5 + f];
            rhs[(int64_t)e * vs + t] = r;
        }
        if (val == nullptr) return;
        for (int blk = 6; blk >= 0; --blk) {
            if (blk < 6 && nbr[blk] < 0) continue;
            double* out = val + bo[blk];
            for (int item = threadIdx.x; item < 25 * nt * 2; item += blockDim.x) {
                const int h = item & 1, m = (item >> 1) % nt, fg = (item >> 1) / nt, f = fg % 5, gg = fg / 5;
                double a0[NH];
                double* dst = out + (int64_t)(gg * nt + h * NH) * b + f * nt + m;
                if (blk == 6) {
#pragma unroll
                    for (int n = 0; n < NH; ++n) a0[n] = dst[(int64_t)n * b];
                    for (int face = 0; face < 6; ++face)
                        for (int qq = 0; qq < qf; ++qq) {
                            const double* pf = tb.phif + ((size_t)face * qf + qq) * nt;
                            const double t0 = pf[m] * sFs[((size_t)face * qf + qq) * 25 + f * 5 + gg];
#pragma unroll
                            for (int n = 0; n < NH; ++n) a0[n] += t0 * pf[h * NH + n];
                        }
                } else {
#pragma unroll
                    for (int n = 0; n < NH; ++n) a0[n] = 0.0;
                    for (int qq = 0; qq < qf; ++qq) {
                        const double* pf = tb.phif + ((size_t)blk * qf + qq) * nt;
                        const double* pn = tb.phif + ((size_t)(blk ^ 1) * qf + qq) * nt + h * NH;
                        const double t0 = pf[m] * sFn[((size_t)blk * qf + qq) * 25 + f * 5 + gg];
#pragma unroll
                        for (int n = 0; n < NH; ++n) a0[n] += t0 * pn[n];
                    }
                }
#pragma unroll
                for (int n = 0; n < NH; ++n) dst[(int64_t)n * b] = a0[n];
            }
        }
    }
}

// dtau[e, f] = cfl[f] h / (mean |u| + mean c) over the volume nodes
// (type_fluid_pseudo_timestep.f90, compute)
template <int NT>
__global__ void __launch_bounds__(kThreads) k_euler_dtau(BoxGeom g, Tables tb, const double* __restrict__ q, int64_t vs,
                                                        double h, double c0, double c1, double c2, double c3, double c4,
                                                        double* __restrict__ dtau) {
    __shared__ double red[2][kThreads / 32];
    const int e = blockIdx.x, nt = NT;
    double sv = 0.0, sc = 0.0;
    for (int qq = threadIdx.x; qq < g.qv; qq += blockDim.x) {
        double Q[5];
        for (int f = 0; f < 5; ++f) {
            double s = 0.0;
            for (int m = 0; m < nt; ++m) s += tb.phi[qq * nt + m] * q[(int64_t)e * vs + f * nt + m];
            Q[f] = s;
        }
        const double p = (kGamma - 1.0) * (Q[4] - 0.5 * (Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / Q[0]);
        sc += sqrt(kGamma * p / Q[0]);
        sv += sqrt((Q[1] * Q[1] + Q[2] * Q[2] + Q[3] * Q[3]) / (Q[0] * Q[0]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        sv += __shfl_down_sync(0xffffffffu, sv, o);
        sc += __shfl_down_sync(0xffffffffu, sc, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = sv; red[1][threadIdx.x >> 5] = sc; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, c = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += red[0][w]; c += red[1][w]; }
        const double lam = a / g.qv + c / g.qv;
        const double cfl[5] = {c0, c1, c2, c3, c4};
        for (int f = 0; f < 5; ++f) dtau[(int64_t)e * 5 + f] = cfl[f] * h / lam;
    }
}

// ---- host tables ----------------------------------------------------------------
void legendre(int order, double x, double* L, double* D) {
    L[0] = 1.0;
    D[0] = 0.0;
    if (order >= 1) { L[1] = x; D[1] = 1.0; }
    for (int n = 2; n <= order; ++n) {
        L[n] = ((2.0 * n - 1.0) * x * L[n - 1] - (n - 1.0) * L[n - 2]) / n;
        D[n] = D[n - 2] + (2.0 * n - 1.0) * L[n - 1];
    }
}

// Gauss-Legendre nodes and weights on [-1, 1] by Newton's iteration on P_n
// from the asymptotic guesses cos(pi (i + 3/4) / (n + 1/2)); w = 2 / ((1 - x^2) P_n'(x)^2).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    std::vector<double> L(n + 1), D(n + 1);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            legendre(n, z, L.data(), D.data());
            const double dz = L[n] / D[n];
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        legendre(n, z, L.data(), D.data());
        x[n - 1 - i] = z;
        w[n - 1 - i] = 2.0 / ((1.0 - z * z) * D[n] * D[n]);
    }
}

}  // namespace

struct chidg_gpu_euler {
    chidg_gpu_ctx* ctx = nullptr;
    chidg_gpu_euler_box box{};
    BoxGeom g{};
    int order = 0, nelem = 0;
    double h = 0.0;
    Buffer phi, grad, wv, phif, wf, dtau, mass;
    Buffer blk_off;
    int64_t off_uid = 0;                           // matrix (uid) the block-offset table was built for
    int32_t off_elem0 = -1;                        // and the element the box starts at in it
    int32_t off_itime = -1;                        // and the time level of the rows
};

extern "C" int chidg_gpu_euler_create(chidg_gpu_ctx* ctx, const chidg_gpu_euler_box* box, chidg_gpu_euler** out) {
    if (!ctx || !box || !out) return CHIDG_GPU_EINVAL;
    *out = nullptr;
    if (box->nx < 1 || box->ny < 1 || box->nz < 1 || box->order < 0 || box->order > kMaxOrder)
        return fail(ctx, CHIDG_GPU_EINVAL, "euler_create: box sizes must be >= 1 and order 0..3");
    for (int d = 0; d < 3; ++d)
        if (!(box->hi[d] > box->lo[d])) return fail(ctx, CHIDG_GPU_EINVAL, "euler_create: empty extent");
    for (int f = 0; f < 6; ++f)
        if (box->bc[f] != CHIDG_EULER_FARFIELD && box->bc[f] != CHIDG_EULER_EXTRAPOLATE)
            return fail(ctx, CHIDG_GPU_EINVAL, "euler_create: unknown boundary condition");
    if (!(box->rho_inf > 0.0) || !(box->p_inf > 0.0)) return fail(ctx, CHIDG_GPU_EINVAL, "euler_create: freestream");
    const int64_t nelem = (int64_t)box->nx * box->ny * box->nz;
    if (nelem > (int64_t)INT32_MAX) return fail(ctx, CHIDG_GPU_EINVAL, "euler_create: too many elements");
    auto* E = new chidg_gpu_euler;
    E->ctx = ctx;
    E->box = *box;
    E->order = box->order;
    E->nelem = (int)nelem;
    const int P = box->order, n1 = (3 * (P + 1) + 1) / 2, nt = (P + 1) * (P + 1) * (P + 1);
    const int qv = n1 * n1 * n1, qf = n1 * n1;
    double hx[3];
    const int ne[3] = {box->nx, box->ny, box->nz};
    for (int d = 0; d < 3; ++d) hx[d] = (box->hi[d] - box->lo[d]) / ne[d];
    const double jinv = hx[0] * hx[1] * hx[2] / 8.0;
    E->h = std::cbrt(hx[0] * hx[1] * hx[2]);
    BoxGeom& g = E->g;
    g.nx = box->nx; g.ny = box->ny; g.nz = box->nz;
    g.nt = nt; g.qv = qv; g.qf = qf;
    g.area[0] = hx[1] * hx[2] / 4.0; g.area[1] = hx[0] * hx[2] / 4.0; g.area[2] = hx[0] * hx[1] / 4.0;
    for (int f = 0; f < 6; ++f) g.bc[f] = box->bc[f];
    g.fs.rho = box->rho_inf; g.fs.p = box->p_inf;
    for (int d = 0; d < 3; ++d) g.fs.u[d] = box->vel_inf[d];

    std::vector<double> xg, wg;
    gauss_legendre(n1, xg, wg);
    std::vector<double> Lv((P + 1) * n1), Ld((P + 1) * n1), Lend_lo(P + 1), Lend_hi(P + 1), tmpL(P + 1), tmpD(P + 1);
    for (int i = 0; i < n1; ++i) {
        legendre(P, xg[i], tmpL.data(), tmpD.data());
        for (int n = 0; n <= P; ++n) { Lv[n * n1 + i] = tmpL[n]; Ld[n * n1 + i] = tmpD[n]; }
    }
    for (int n = 0; n <= P; ++n) { Lend_hi[n] = 1.0; Lend_lo[n] = (n % 2) ? -1.0 : 1.0; }
    std::vector<double> phi((size_t)qv * nt), grad((size_t)3 * qv * nt), wv(qv), phif((size_t)6 * qf * nt), wf(qf);
    for (int k = 0; k < n1; ++k)
        for (int j = 0; j < n1; ++j)
            for (int i = 0; i < n1; ++i) {
                const int qq = (k * n1 + j) * n1 + i;                       // xi fastest
                wv[qq] = wg[i] * wg[j] * wg[k] * jinv;
                for (int m = 0; m < nt; ++m) {
                    const int a = kModes[m][0], bb = kModes[m][1], c = kModes[m][2];
                    const double la = Lv[a * n1 + i], lb = Lv[bb * n1 + j], lc = Lv[c * n1 + k];
                    phi[(size_t)qq * nt + m] = la * lb * lc;
                    grad[((size_t)0 * qv + qq) * nt + m] = Ld[a * n1 + i] * lb * lc * (2.0 / hx[0]);
                    grad[((size_t)1 * qv + qq) * nt + m] = la * Ld[bb * n1 + j] * lc * (2.0 / hx[1]);
                    grad[((size_t)2 * qv + qq) * nt + m] = la * lb * Ld[c * n1 + k] * (2.0 / hx[2]);
                }
            }
    for (int t0 = 0; t0 < n1; ++t0)
        for (int t1 = 0; t1 < n1; ++t1) wf[t0 * n1 + t1] = wg[t0] * wg[t1];
    for (int face = 0; face < 6; ++face) {
        const int d = face >> 1;
        const int ta = d == 0 ? 1 : 0, tb_ = d == 2 ? 1 : 2;                // tangential directions, ta < tb_
        const std::vector<double>& Lend = (face & 1) ? Lend_hi : Lend_lo;
        for (int t0 = 0; t0 < n1; ++t0)
            for (int t1 = 0; t1 < n1; ++t1) {
                const int qq = t0 * n1 + t1;
                for (int m = 0; m < nt; ++m) {
                    double v = 1.0;
                    for (int dd = 0; dd < 3; ++dd) {
                        const int deg = kModes[m][dd];
                        if (dd == d) v *= Lend[deg];
                        else if (dd == ta) v *= Lv[deg * n1 + t0];
                        else v *= Lv[deg * n1 + t1];
                    }
                    phif[((size_t)face * qf + qq) * nt + m] = v;
                }
            }
        (void)tb_;
    }
    auto up = [&](Buffer& buf, const std::vector<double>& v) {
        int st = ensure(ctx, buf, v.size() * sizeof(double));
        if (st) return st;
        const cudaError_t ce = cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice,
                                               ctx->stream);
        return ce == cudaSuccess ? CHIDG_GPU_OK : cuda_fail(ctx, ce, "euler tables");
    };
    int st = up(E->phi, phi);
    if (!st) st = up(E->grad, grad);
    if (!st) st = up(E->wv, wv);
    if (!st) st = up(E->phif, phif);
    if (!st) st = up(E->wf, wf);
    if (!st) st = ensure(ctx, E->dtau, (size_t)nelem * 5 * sizeof(double));
    if (!st) {
        const cudaError_t ce = cudaStreamSynchronize(ctx->stream);     // the host tables go out of scope
        if (ce != cudaSuccess) st = cuda_fail(ctx, ce, "euler tables");
    }
    const size_t smem = smem_doubles(nt, qv, qf) * sizeof(double);
    if (!st) {
        const void* fn = P == 0 ? (const void*)k_euler_assemble<1> : P == 1 ? (const void*)k_euler_assemble<8>
                         : P == 2 ? (const void*)k_euler_assemble<27> : (const void*)k_euler_assemble<64>;
        st = raise_smem_limit(fn, smem);
    }
    if (st) {
        chidg_gpu_euler_destroy(E);
        return st;
    }
    *out = E;
    return CHIDG_GPU_OK;
}

extern "C" int chidg_gpu_euler_destroy(chidg_gpu_euler* E) {
    if (!E) return CHIDG_GPU_OK;
    for (Buffer* b : {&E->phi, &E->grad, &E->wv, &E->phif, &E->wf, &E->dtau, &E->mass, &E->blk_off}) release(*b);
    delete E;
    return CHIDG_GPU_OK;
}

namespace {
Tables tables_of(const chidg_gpu_euler* E) {
    return Tables{(const double*)E->phi.ptr, (const double*)E->grad.ptr, (const double*)E->wv.ptr,
                  (const double*)E->phif.ptr, (const double*)E->wf.ptr};
}

int check_vector(chidg_gpu_euler* E, const chidg_gpu_vector* v, const char* what) {
    if (!v || v->ctx != E->ctx) return fail(E->ctx, CHIDG_GPU_EINVAL, std::string("euler: ") + what + " of another context");
    if (v->n != (int64_t)E->nelem * 5 * E->g.nt)
        return fail(E->ctx, CHIDG_GPU_EINVAL, std::string("euler: ") + what + " length does not match the box");
    return CHIDG_GPU_OK;
}

// The box placed at elements elem0 .. elem0 + nelem - 1 of A's layout: its
// elements must have 5 fields and the box's modes on one time level; returns
// the vector offset of its first element.
int box_fits(chidg_gpu_euler* E, const chidg_gpu_matrix* A, int32_t elem0, int64_t* voff) {
    if (!A || A->ctx != E->ctx) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler: matrix of another context");
    if (elem0 < 0 || (int64_t)elem0 + E->nelem > A->nelem)
        return fail(E->ctx, CHIDG_GPU_EINVAL, "euler: the box does not fit the matrix's elements");
    for (int e = 0; e < E->nelem; ++e)
        if (A->nvars[elem0 + e] != 5 || A->nterms[elem0 + e] != E->g.nt)
            return fail(E->ctx, CHIDG_GPU_EINVAL, "euler: element fields or modes differ from the box");
    *voff = A->eoff[elem0];
    return CHIDG_GPU_OK;
}

int box_in_layout(chidg_gpu_euler* E, const chidg_gpu_matrix* A, int32_t elem0, int64_t* voff) {
    if (A && A->ntime != 1) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler: the matrix has several time levels");
    return box_fits(E, A, elem0, voff);
}

// Offsets of each element's blocks in A's values: [e][face 0..5, DIAG], -1 on
// boundary faces.  A must hold exactly the box pattern: one time level, 5
// fields and (P+1)^3 modes per element, and in every row the DIAG block and
// one block per interior face.
int block_offsets(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0, int32_t itime = 0) {
    if (E->off_uid == A->uid && E->off_elem0 == elem0 && E->off_itime == itime) return CHIDG_GPU_OK;
    const int nt = E->g.nt;
    if (elem0 < 0 || (int64_t)elem0 + E->nelem > A->nelem || itime < 0 || itime >= A->ntime)
        return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: matrix is not this box's (elements or time levels)");
    std::vector<int64_t> off((size_t)E->nelem * 7, -1);
    BoxGeom g = E->g;
    for (int e = 0; e < E->nelem; ++e) {
        const int ea = elem0 + e;                 // the element in A
        if (A->nvars[ea] != 5 || A->nterms[ea] != nt)
            return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: element fields or modes differ from the box");
        const int i = e % g.nx, j = (e / g.nx) % g.ny, k = e / (g.nx * g.ny);
        const int nb[6] = {i > 0 ? ea - 1 : -1, i < g.nx - 1 ? ea + 1 : -1, j > 0 ? ea - g.nx : -1,
                           j < g.ny - 1 ? ea + g.nx : -1, k > 0 ? ea - g.nx * g.ny : -1,
                           k < g.nz - 1 ? ea + g.nx * g.ny : -1};
        int expect = 1;
        for (int f = 0; f < 6; ++f) expect += nb[f] >= 0;
        // the row's LOCAL blocks are the box pattern; harmonic-balance blocks
        // (coupling the element's time levels) may follow
        const std::vector<int32_t>& row = A->rowblk[A->row(ea, itime)];
        int nlocal = 0;
        for (int32_t kb : row) {
            if (A->kind[kb] == CHIDG_BLK_LOCAL) ++nlocal;
            else if (A->kind[kb] != CHIDG_BLK_HB || A->ce[kb] != ea)
                return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: matrix has chimera or boundary blocks");
        }
        if (nlocal != expect)
            return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: matrix row is not the box pattern");
        for (int32_t kb : row) {
            if (A->kind[kb] != CHIDG_BLK_LOCAL) continue;
            int slot = -1;
            if (A->ce[kb] == ea) slot = 6;
            for (int f = 0; f < 6 && slot < 0; ++f)
                if (nb[f] == A->ce[kb]) slot = f;
            if (slot < 0 || off[(size_t)e * 7 + slot] >= 0)
                return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: matrix row is not the box pattern");
            off[(size_t)e * 7 + slot] = A->voff[kb];
        }
    }
    int st = ensure(E->ctx, E->blk_off, off.size() * sizeof(int64_t));
    if (st) return st;
    cudaError_t ce = cudaMemcpyAsync(E->blk_off.ptr, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                                     E->ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->ctx->stream);
    if (ce != cudaSuccess) return cuda_fail(E->ctx, ce, "euler block offsets");
    E->off_uid = A->uid;
    E->off_elem0 = elem0;
    E->off_itime = itime;
    return CHIDG_GPU_OK;
}

// rhs(box) = R(q(box)) and, with val, A's blocks of the box = dR/dq: q and rhs
// point at the box's first element
int assemble_ptrs(chidg_gpu_euler* E, const double* q, double* rhs, chidg_gpu_matrix* A, int32_t elem0,
                  int32_t itime = 0, int64_t vs = 0) {
    const bool jac = A != nullptr;
    if (vs == 0) vs = (int64_t)5 * E->g.nt;
    int st;
    if (jac && (st = block_offsets(E, A, elem0, itime))) return st;
    const int P = E->order, nt = E->g.nt;
    const size_t smem = smem_doubles(nt, E->g.qv, E->g.qf) * sizeof(double);
    const Tables tb = tables_of(E);
    double* val = jac ? (double*)A->val.ptr : nullptr;
    const int64_t* off = jac ? (const int64_t*)E->blk_off.ptr : nullptr;
    const dim3 grid(E->nelem), block(kThreads);
    if (P == 0) k_euler_assemble<1><<<grid, block, smem, E->ctx->stream>>>(E->g, tb, q, rhs, val, off, vs);
    else if (P == 1) k_euler_assemble<8><<<grid, block, smem, E->ctx->stream>>>(E->g, tb, q, rhs, val, off, vs);
    else if (P == 2) k_euler_assemble<27><<<grid, block, smem, E->ctx->stream>>>(E->g, tb, q, rhs, val, off, vs);
    else k_euler_assemble<64><<<grid, block, smem, E->ctx->stream>>>(E->g, tb, q, rhs, val, off, vs);
    st = check_launch(E->ctx, "k_euler_assemble");
    if (st) return st;
    if (jac) A->stamp++;
    return CHIDG_GPU_OK;
}

int dtau_ptrs(chidg_gpu_euler* E, const double* qp, const double* cfl, double* dtau, int64_t vs = 0) {
    if (vs == 0) vs = (int64_t)5 * E->g.nt;
    const dim3 grid(E->nelem), block(kThreads);
    const Tables tb = tables_of(E);
    double* out = (double*)E->dtau.ptr;
    if (E->order == 0) k_euler_dtau<1><<<grid, block, 0, E->ctx->stream>>>(E->g, tb, qp, vs, E->h, cfl[0], cfl[1], cfl[2], cfl[3], cfl[4], out);
    else if (E->order == 1) k_euler_dtau<8><<<grid, block, 0, E->ctx->stream>>>(E->g, tb, qp, vs, E->h, cfl[0], cfl[1], cfl[2], cfl[3], cfl[4], out);
    else if (E->order == 2) k_euler_dtau<27><<<grid, block, 0, E->ctx->stream>>>(E->g, tb, qp, vs, E->h, cfl[0], cfl[1], cfl[2], cfl[3], cfl[4], out);
    else k_euler_dtau<64><<<grid, block, 0, E->ctx->stream>>>(E->g, tb, qp, vs, E->h, cfl[0], cfl[1], cfl[2], cfl[3], cfl[4], out);
    int st = check_launch(E->ctx, "k_euler_dtau");
    if (st) return st;
    cudaError_t ce = cudaMemcpyAsync(dtau, out, (size_t)E->nelem * 5 * sizeof(double), cudaMemcpyDeviceToHost,
                                     E->ctx->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(E->ctx->stream);
    return ce == cudaSuccess ? CHIDG_GPU_OK : cuda_fail(E->ctx, ce, "euler_pseudo_timestep");
}
}  // namespace

extern "C" int chidg_gpu_euler_assemble(chidg_gpu_euler* E, chidg_gpu_vector* q, chidg_gpu_vector* rhs,
                                        chidg_gpu_matrix* A) {
    if (!E) return CHIDG_GPU_EINVAL;
    int st = check_vector(E, q, "q");
    if (!st) st = check_vector(E, rhs, "rhs");
    if (st) return st;
    if (q == rhs) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: q and rhs must differ");
    if (A && A->ctx != E->ctx) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: matrix of another context");
    if (A && (A->nelem != E->nelem || A->ntime != 1))
        return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble: matrix is not this box's (elements or time levels)");
    return assemble_ptrs(E, (const double*)q->buf.ptr, (double*)rhs->buf.ptr, A, 0);
}

extern "C" int chidg_gpu_euler_assemble_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0, chidg_gpu_vector* q,
                                           chidg_gpu_vector* rhs, int32_t jacobian) {
    if (!E || !A || !q || !rhs) return E ? fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_at: null argument") : CHIDG_GPU_EINVAL;
    if (q == rhs) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_at: q and rhs must differ");
    if (q->A != A || rhs->A != A) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_at: q and rhs must be vectors of A");
    int64_t voff = 0;
    int st = box_in_layout(E, A, elem0, &voff);
    if (st) return st;
    return assemble_ptrs(E, (const double*)q->buf.ptr + voff, (double*)rhs->buf.ptr + voff, jacobian ? A : nullptr, elem0);
}

extern "C" int chidg_gpu_euler_pseudo_timestep(chidg_gpu_euler* E, chidg_gpu_vector* q, const double* cfl,
                                               double* dtau) {
    if (!E || !cfl || !dtau) return E ? fail(E->ctx, CHIDG_GPU_EINVAL, "euler_pseudo_timestep: null argument")
                                      : CHIDG_GPU_EINVAL;
    int st = check_vector(E, q, "q");
    if (st) return st;
    return dtau_ptrs(E, (const double*)q->buf.ptr, cfl, dtau);
}

extern "C" int chidg_gpu_euler_pseudo_timestep_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0,
                                                  chidg_gpu_vector* q, const double* cfl, double* dtau) {
    if (!E || !A || !q || !cfl || !dtau)
        return E ? fail(E->ctx, CHIDG_GPU_EINVAL, "euler_pseudo_timestep_at: null argument") : CHIDG_GPU_EINVAL;
    if (q->A != A) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_pseudo_timestep_at: q must be a vector of A");
    int64_t voff = 0;
    int st = box_in_layout(E, A, elem0, &voff);
    if (st) return st;
    return dtau_ptrs(E, (const double*)q->buf.ptr + voff, cfl, dtau);
}

// ---- harmonic balance --------------------------------------------------------------
extern "C" int chidg_gpu_euler_assemble_level_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0, int32_t itime,
                                                 chidg_gpu_vector* q, chidg_gpu_vector* rhs, int32_t jacobian) {
    if (!E || !A || !q || !rhs)
        return E ? fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_level: null argument") : CHIDG_GPU_EINVAL;
    if (q == rhs) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_level: q and rhs must differ");
    if (q->A != A || rhs->A != A) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_level: q and rhs must be vectors of A");
    if (itime < 0 || itime >= A->ntime) return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_level: no such time level");
    int64_t voff = 0;
    int st = box_fits(E, A, elem0, &voff);
    if (st) return st;
    const int64_t b = (int64_t)5 * E->g.nt, vs = b * A->ntime;
    return assemble_ptrs(E, (const double*)q->buf.ptr + voff + itime * b, (double*)rhs->buf.ptr + voff + itime * b,
                         jacobian ? A : nullptr, elem0, itime, vs);
}

extern "C" int chidg_gpu_euler_assemble_level(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t itime, chidg_gpu_vector* q,
                                              chidg_gpu_vector* rhs, int32_t jacobian) {
    if (E && A && A->nelem != E->nelem)
        return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_assemble_level: matrix is not this box's");
    return chidg_gpu_euler_assemble_level_at(E, A, 0, itime, q, rhs, jacobian);
}

extern "C" int chidg_gpu_euler_pseudo_timestep_level(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t itime,
                                                     chidg_gpu_vector* q, const double* cfl, double* dtau) {
    if (!E || !A || !q || !cfl || !dtau)
        return E ? fail(E->ctx, CHIDG_GPU_EINVAL, "euler_pseudo_timestep_level: null argument") : CHIDG_GPU_EINVAL;
    if (q->A != A || A->nelem != E->nelem || itime < 0 || itime >= A->ntime)
        return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_pseudo_timestep_level: q of another layout or no such time level");
    const int64_t b = (int64_t)5 * E->g.nt;
    return dtau_ptrs(E, (const double*)q->buf.ptr + itime * b, cfl, dtau, b * A->ntime);
}

// ---- the pseudo-transient term and b = -R on the device -------------------------
namespace {
// rows (elem0 + e, t) of the box, one CTA each (t fastest): field f's diagonal
// sub-block of the DIAG block += M / min_f' dtau(e, f') (contribute_pseudo_temporal
// applies minval(elems(ielem)%dtau) to every field and time level)
__global__ void k_ptc_add(double* __restrict__ val, const int64_t* __restrict__ diag_voff, int row0, int ntime, int nt,
                          const double* __restrict__ dtau, const double* __restrict__ M) {
    const int r = blockIdx.x;
    const int e = r / ntime, b = 5 * nt;
    const double* d = dtau + (int64_t)e * 5;
    const double s = 1.0 / fmin(fmin(fmin(fmin(d[0], d[1]), d[2]), d[3]), d[4]);
    double* D = val + diag_voff[row0 + r];
    for (int idx = threadIdx.x; idx < 5 * nt * nt; idx += blockDim.x) {
        const int f = idx / (nt * nt), rem = idx - f * nt * nt, i = rem % nt, j = rem / nt;
        D[(int64_t)(f * nt + i) + (int64_t)(f * nt + j) * b] += s * M[i + j * nt];
    }
}

__global__ void k_negate(double* __restrict__ x, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) x[i] = -x[i];
}
}  // namespace

extern "C" int chidg_gpu_euler_pseudo_transient_at(chidg_gpu_euler* E, chidg_gpu_matrix* A, int32_t elem0,
                                                   chidg_gpu_vector* q, chidg_gpu_vector* rhs, const double* cfl,
                                                   const double* mass) {
    if (!E || !A || !q || !cfl || !mass)
        return E ? fail(E->ctx, CHIDG_GPU_EINVAL, "euler_pseudo_transient_at: null argument") : CHIDG_GPU_EINVAL;
    if (q->A != A || (rhs && (rhs->A != A || rhs == q)))
        return fail(E->ctx, CHIDG_GPU_EINVAL, "euler_pseudo_transient_at: q and rhs must be distinct vectors of A");
    int64_t voff = 0;
    int st = box_fits(E, A, elem0, &voff);
    if (st) return st;
    chidg_gpu_ctx* ctx = E->ctx;
    const int nt = E->g.nt, T = A->ntime;
    const int64_t b = (int64_t)5 * nt, vs = b * T;
    const double c[5] = {cfl[0], cfl[1], cfl[2], cfl[3], cfl[4]};
    const dim3 grid(E->nelem), block(kThreads);
    const Tables tb = tables_of(E);
    const double* qp = (const double*)q->buf.ptr + voff;
    double* dt = (double*)E->dtau.ptr;
    if (E->order == 0) k_euler_dtau<1><<<grid, block, 0, ctx->stream>>>(E->g, tb, qp, vs, E->h, c[0], c[1], c[2], c[3], c[4], dt);
    else if (E->order == 1) k_euler_dtau<8><<<grid, block, 0, ctx->stream>>>(E->g, tb, qp, vs, E->h, c[0], c[1], c[2], c[3], c[4], dt);
    else if (E->order == 2) k_euler_dtau<27><<<grid, block, 0, ctx->stream>>>(E->g, tb, qp, vs, E->h, c[0], c[1], c[2], c[3], c[4], dt);
    else k_euler_dtau<64><<<grid, block, 0, ctx->stream>>>(E->g, tb, qp, vs, E->h, c[0], c[1], c[2], c[3], c[4], dt);
    if ((st = check_launch(ctx, "k_euler_dtau"))) return st;
    if ((st = ensure(ctx, E->mass, (size_t)nt * nt * sizeof(double)))) return st;
    // from pageable memory the copy returns once the bytes are staged, so the caller's array may go
    cudaError_t ce = cudaMemcpyAsync(E->mass.ptr, mass, (size_t)nt * nt * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "euler_pseudo_transient_at: mass");
    k_ptc_add<<<E->nelem * T, 256, 0, ctx->stream>>>((double*)A->val.ptr, (const int64_t*)A->d_diag_voff.ptr, elem0 * T, T,
                                                    nt, dt, (const double*)E->mass.ptr);
    if ((st = check_launch(ctx, "k_ptc_add"))) return st;
    A->stamp++;
    if (rhs) {
        const int64_t n = (int64_t)E->nelem * vs;
        k_negate<<<(int)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, ctx->stream>>>((double*)rhs->buf.ptr + voff, n);
        if ((st = check_launch(ctx, "k_negate"))) return st;
    }
    return CHIDG_GPU_OK;
}

namespace {
template <typename T>
int upload_array(chidg_gpu_ctx* ctx, Buffer& buf, const std::vector<T>& v) {
    int st = ensure(ctx, buf, std::max<size_t>(v.size(), 1) * sizeof(T));
    if (st) return st;
    if (v.empty()) return CHIDG_GPU_OK;
    const cudaError_t e = cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    return e == cudaSuccess ? CHIDG_GPU_OK : cuda_fail(ctx, e, "hb tables");
}

// rhs(e, t) += sum_t' D(t, t') (I_fields x M) q(e, t'), one CTA per element
__global__ void k_hb_residual(const double* __restrict__ q, double* __restrict__ rhs, const int64_t* __restrict__ eoff,
                              const int32_t* __restrict__ nvars, int ntime, int nt, const double* __restrict__ D,
                              const double* __restrict__ M) {
    const int e = blockIdx.x;
    const int b = nvars[e] * nt;
    const double* qe = q + eoff[e];
    double* re = rhs + eoff[e];
    for (int r = threadIdx.x; r < ntime * b; r += blockDim.x) {
        const int t = r / b, fm = r - t * b, f = fm / nt, m = fm - f * nt;
        double acc = 0.0;
        for (int tp = 0; tp < ntime; ++tp) {
            const double* qf = qe + (int64_t)tp * b + f * nt;
            double mq = 0.0;
            for (int n = 0; n < nt; ++n) mq += M[m + n * nt] * qf[n];
            acc += D[t + tp * ntime] * mq;
        }
        re[r] += acc;
    }
}
// the hb block of row (e, t), column (e, t'): D(t, t') (I_fields x M), one CTA per block
__global__ void k_hb_blocks(double* __restrict__ val, const int64_t* __restrict__ voff, const int32_t* __restrict__ rt,
                            const int32_t* __restrict__ ct, const int32_t* __restrict__ bsz, int ntime, int nt,
                            const double* __restrict__ D, const double* __restrict__ M) {
    const int k = blockIdx.x;
    const int b = bsz[k];
    const double d = D[rt[k] + ct[k] * ntime];
    double* out = val + voff[k];
    for (int idx = threadIdx.x; idx < b * b; idx += blockDim.x) {
        const int r = idx % b, c = idx / b;
        const int fr = r / nt, fc = c / nt;
        out[idx] = (fr == fc) ? d * M[(r - fr * nt) + (c - fc * nt) * nt] : 0.0;
    }
}
}  // namespace

extern "C" int chidg_gpu_hb_coupling_at(chidg_gpu_matrix* A, int32_t elem0, int32_t nelem, int32_t nterms, const double* D,
                                        const double* mass, chidg_gpu_vector* q, chidg_gpu_vector* rhs, int32_t jacobian) {
    if (!A || !D || !mass || !q || !rhs || q == rhs || q->A != A || rhs->A != A || nterms < 1 || elem0 < 0 || nelem < 1 ||
        (int64_t)elem0 + nelem > A->nelem)
        return A ? fail(A->ctx, CHIDG_GPU_EINVAL, "hb_coupling: bad argument") : CHIDG_GPU_EINVAL;
    chidg_gpu_ctx* ctx = A->ctx;
    cudaSetDevice(ctx->device);
    const int T = A->ntime;
    const int e1 = elem0 + nelem;
    for (int e = elem0; e < e1; ++e)
        if (A->nterms[e] != nterms) return fail(ctx, CHIDG_GPU_EINVAL, "hb_coupling: elements of another mode count");
    std::vector<int32_t> hb_rt, hb_ct, hb_b;
    std::vector<int64_t> hb_off;
    if (jacobian)
        for (int64_t k = 0; k < A->nblk; ++k)
            if (A->kind[k] == CHIDG_BLK_HB && A->re[k] >= elem0 && A->re[k] < e1) {
                if (A->re[k] != A->ce[k]) return fail(ctx, CHIDG_GPU_EINVAL, "hb_coupling: an hb block couples two elements");
                hb_rt.push_back(A->rt[k]);
                hb_ct.push_back(A->ct[k]);
                hb_b.push_back(A->bsize(A->re[k]));
                hb_off.push_back(A->voff[k]);
            }
    Buffer dD, dM, dE, dV, bo, br, bc, bb;
    auto cleanup = [&]() { for (Buffer* x : {&dD, &dM, &dE, &dV, &bo, &br, &bc, &bb}) release(*x); };
    int st;
    std::vector<double> hD(D, D + (size_t)T * T), hM(mass, mass + (size_t)nterms * nterms);
    const std::vector<int64_t> eo(A->eoff.begin() + elem0, A->eoff.begin() + e1);
    const std::vector<int32_t> nv(A->nvars.begin() + elem0, A->nvars.begin() + e1);
    if ((st = upload_array(ctx, dD, hD)) || (st = upload_array(ctx, dM, hM)) || (st = upload_array(ctx, dE, eo)) ||
        (st = upload_array(ctx, dV, nv))) {
        cleanup();
        return st;
    }
    k_hb_residual<<<nelem, 256, 0, ctx->stream>>>((const double*)q->buf.ptr, (double*)rhs->buf.ptr, (const int64_t*)dE.ptr,
                                                     (const int32_t*)dV.ptr, T, nterms, (const double*)dD.ptr,
                                                     (const double*)dM.ptr);
    if ((st = check_launch(ctx, "k_hb_residual"))) { cleanup(); return st; }
    if (jacobian && !hb_off.empty()) {
        if ((st = upload_array(ctx, bo, hb_off)) || (st = upload_array(ctx, br, hb_rt)) || (st = upload_array(ctx, bc, hb_ct)) ||
            (st = upload_array(ctx, bb, hb_b))) {
            cleanup();
            return st;
        }
        k_hb_blocks<<<(int)hb_off.size(), 256, 0, ctx->stream>>>((double*)A->val.ptr, (const int64_t*)bo.ptr,
                                                                 (const int32_t*)br.ptr, (const int32_t*)bc.ptr,
                                                                 (const int32_t*)bb.ptr, T, nterms, (const double*)dD.ptr,
                                                                 (const double*)dM.ptr);
        if ((st = check_launch(ctx, "k_hb_blocks"))) { cleanup(); return st; }
        A->stamp++;
    }
    const cudaError_t ce = cudaStreamSynchronize(ctx->stream);     // the host copies and buffers go out of scope
    cleanup();
    return ce == cudaSuccess ? CHIDG_GPU_OK : cuda_fail(ctx, ce, "hb_coupling");
}

extern "C" int chidg_gpu_hb_coupling(chidg_gpu_matrix* A, int32_t nterms, const double* D, const double* mass,
                                     chidg_gpu_vector* q, chidg_gpu_vector* rhs, int32_t jacobian) {
    if (!A) return CHIDG_GPU_EINVAL;
    return chidg_gpu_hb_coupling_at(A, 0, A->nelem, nterms, D, mass, q, rhs, jacobian);
}

// ---- a Newton system written in place (the serving and batching callers) ---------
extern "C" int chidg_gpu_euler_fill_system(void* user, chidg_gpu_ctx* ctx, chidg_gpu_matrix* A, chidg_gpu_vector* b,
                                           chidg_gpu_vector* work, int32_t elem0) {
    const auto* S = static_cast<const chidg_gpu_euler_system*>(user);
    if (!S || !ctx || !A || !b || !work || A->ctx != ctx || b->A != A || work->A != A || b == work || !S->q0 || !S->mass)
        return ctx ? fail(ctx, CHIDG_GPU_EINVAL, "euler_fill_system: bad argument") : CHIDG_GPU_EINVAL;
    const int T = S->ntime;
    if (T < 1 || T != A->ntime || (T > 1 && (!S->level_vel || !S->D)))
        return fail(ctx, CHIDG_GPU_EINVAL, "euler_fill_system: time levels differ from the matrix's or no hb operator");
    std::vector<chidg_gpu_euler*> lv((size_t)T, nullptr);
    auto done = [&](int st) {
        for (chidg_gpu_euler* E : lv) chidg_gpu_euler_destroy(E);
        return st;
    };
    for (int t = 0; t < T; ++t) {
        chidg_gpu_euler_box box = S->box;
        if (T > 1)
            for (int d = 0; d < 3; ++d) box.vel_inf[d] = S->level_vel[3 * t + d];
        const int st = chidg_gpu_euler_create(ctx, &box, &lv[t]);
        if (st) return done(st);
    }
    int64_t voff = 0;
    int st = box_fits(lv[0], A, elem0, &voff);
    if (st) return done(st);
    const int nelem = lv[0]->nelem, nt = lv[0]->g.nt;
    if ((st = chidg_gpu_vector_upload_range(work, S->q0, voff, (int64_t)nelem * T * 5 * nt))) return done(st);
    for (int t = 0; t < T && !st; ++t) st = chidg_gpu_euler_assemble_level_at(lv[t], A, elem0, t, work, b, 1);
    if (!st && T > 1) st = chidg_gpu_hb_coupling_at(A, elem0, nelem, nt, S->D, S->mass, work, b, 1);
    const double cfl[5] = {S->cfl, S->cfl, S->cfl, S->cfl, S->cfl};
    if (!st) st = chidg_gpu_euler_pseudo_transient_at(lv[0], A, elem0, work, b, cfl, S->mass);
    if (!st) {
        // the caller's arrays (q0, mass) are not read after this returns
        const cudaError_t ce = cudaStreamSynchronize(ctx->stream);
        if (ce != cudaSuccess) st = cuda_fail(ctx, ce, "euler_fill_system");
    }
    return done(st);
}
