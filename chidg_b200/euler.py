"""Euler DG residual and Jacobian on hex boxes: the caller side of the linear
solves, restating ChiDG's spatial discretisation for the Euler equations on a
static, affine, conforming box mesh.

What is restated, and from where:
  * basis: modal tensor-product Legendre polynomials P_n on [-1,1]^3
    (src/polynomial/mod_legendre.f90:62-87, 182-204), modes in the reference's
    order (src/polynomial/mod_ordering.f90:8-..., `MODE_ORDER` below);
  * quadrature: Gauss-Legendre, ceil(3 (P+1) / 2) nodes per direction, the
    default gq_rule = 2 (src/quadrature/mod_quadrature.f90:32-95,
    src/io/mod_io.f90:31);
  * volume operator: -int grad(phi) . F(Q) dV (euler_volume_operator.f90:78-183;
    integrate_volume_vector_flux, src/polynomial/mod_integrate.f90:44-126, with
    the sign of store_volume_integrals, :652-779);
  * interior faces: int phi (F(Q-) + F(Q+))/2 . n dA (euler_boundary_average_
    operator.f90; type_chidg_worker.f90:1459-1522) plus the Roe upwind term with
    Harten's entropy fix eps = 0.01 times the face area (euler_roe_operator.f90;
    integrate_boundary_upwind, type_chidg_worker.f90), applied to the element
    and, negated, to its neighbour (integrate_boundary_scalar_flux,
    mod_integrate.f90:219-346);
  * boundary faces: int phi F(Q_bc) . n dA (euler_bc_operator.f90) with the
    states of bc_state_farfield.f90 (Riemann invariants, inflow/outflow by the
    sign of the normal momentum against RKTOL) and bc_state_fluid_extrapolate.f90;
  * storage: R = rhs of the reference (volume integrals negated, face integrals
    added), row index (field, mode) = ifield * nterms + iterm, the linearisation
    of a boundary state on the element's own DIAG block (store_bc with local
    coupling, src/containers/type_domain_matrix.f90:758-798);
  * pseudo time step: dtau = cfl h / (mean |u| + mean c) with h = vol^(1/3)
    (src/equations/fluid/type_fluid_pseudo_timestep.f90);
  * mass matrix: int phi_i phi_j dV per element.

The reference differentiates with forward-mode AD (DNAD).  Here the pointwise
flux functions are differentiated by the complex step (Squire and Trapp 1998:
f'(x) = Im f(x + i h) / h, no subtractive cancellation, exact to rounding for
the analytic operations used; the entropy fix and the inflow test branch on
real parts, as AD branches on values), and the chain rule through the basis is
taken exactly.  Assembly runs on the host in numpy, as the reference's runs on
its CPU ranks; it is sized for boxes of a few thousand elements at P1/P2.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib, api, mesh

GAMMA = 1.4                      # src/equations/fluid/mod_fluid.f90:10
RGAS = 287.15                    # src/equations/fluid/mod_fluid.f90:9
RKTOL = 20.0 * np.finfo(np.float64).eps     # src/constants/mod_constants.f90:241
ENTROPY_FIX_EPS = 0.01           # euler_roe_operator.f90 (eps of the wave-speed limiter)
NFIELDS = 5                      # Density, Momentum-1..3, Energy

# Legendre degrees (xi, eta, zeta) of each mode, in the reference's mode order,
# for P <= 3 (src/polynomial/mod_ordering.f90, xi/eta/zeta_order_3d, first 64
# entries, 0-based here).  Every prefix of (P+1)^3 modes is the full order-P set.
_MODE_DIGITS = ("000 010 001 100 110 101 011 111 020 002 200 021 012 120 102 210 201 022 121 112 220 202 211 "
                "122 221 212 222 300 030 003 310 301 130 103 031 013 320 302 311 230 203 131 113 032 023 321 "
                "312 330 303 231 213 132 123 033 322 331 313 232 223 133 332 323 233 333")
MODE_ORDER = np.array([[int(c) for c in t] for t in _MODE_DIGITS.split()], dtype=np.int64)
MAX_ORDER = 3

_CS_H = 1.0e-30                  # complex-step size


def nnodes_1d(order: int) -> int:
    """gq_rule = 2: ceil(3 nterms1d / 2) (mod_quadrature.f90:68-80)."""
    return int(math.ceil(3.0 * (order + 1) / 2.0))


def _legendre_tables(order: int, x: np.ndarray):
    """P_n(x) and P_n'(x) for n = 0..order, by the three-term recurrence
    (mod_legendre.f90:62-87) and P_n' = n (x P_n - P_{n-1}) / (x^2 - 1) taken
    through the recurrence of the derivatives, P_n' = P_{n-2}' + (2n-1) P_{n-1}."""
    L = np.zeros((order + 1, x.size))
    D = np.zeros((order + 1, x.size))
    L[0] = 1.0
    if order >= 1:
        L[1] = x
        D[1] = 1.0
    for n in range(2, order + 1):
        L[n] = ((2.0 * n - 1.0) * x * L[n - 1] - (n - 1.0) * L[n - 2]) / n
        D[n] = D[n - 2] + (2.0 * n - 1.0) * L[n - 1]
    return L, D


# ---- pointwise Euler physics (real or complex arrays, fields on the last axis) ----

def _abs(z):
    """|z| for the complex step: z sign(Re z) (the analytic continuation of abs
    away from 0)."""
    return z * np.sign(z.real) if np.iscomplexobj(z) else np.abs(z)


def _pressure(Q):
    rho, m1, m2, m3, E = (Q[..., i] for i in range(5))
    return (GAMMA - 1.0) * (E - 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / rho)


def euler_flux(Q):
    """Physical flux F[..., d, field] (euler_volume_operator.f90:112-181)."""
    rho, m1, m2, m3, E = (Q[..., i] for i in range(5))
    inv = 1.0 / rho
    u, v, w = m1 * inv, m2 * inv, m3 * inv
    p = _pressure(Q)
    H = (E + p) * inv
    vel = (u, v, w)
    F = np.empty(Q.shape[:-1] + (3, 5), dtype=Q.dtype)
    for d in range(3):
        F[..., d, 0] = rho * vel[d]
        F[..., d, 1] = m1 * vel[d]
        F[..., d, 2] = m2 * vel[d]
        F[..., d, 3] = m3 * vel[d]
        F[..., d, 1 + d] += p
        F[..., d, 4] = rho * H * vel[d]
    return F


def roe_upwind(Qm, Qp, n):
    """Roe dissipation per unit area, with Harten's entropy fix
    (euler_roe_operator.f90, compute): Qm interior, Qp exterior, n the unit
    normal of the interior element (3,)."""
    n1, n2, n3 = n
    rho_m, rho_p = Qm[..., 0], Qp[..., 0]
    inv_m, inv_p = 1.0 / rho_m, 1.0 / rho_p
    p_m, p_p = _pressure(Qm), _pressure(Qp)
    H_m, H_p = (Qm[..., 4] + p_m) * inv_m, (Qp[..., 4] + p_p) * inv_p
    u_m, v_m, w_m = Qm[..., 1] * inv_m, Qm[..., 2] * inv_m, Qm[..., 3] * inv_m
    u_p, v_p, w_p = Qp[..., 1] * inv_p, Qp[..., 2] * inv_p, Qp[..., 3] * inv_p
    vmag_m = u_m * n1 + v_m * n2 + w_m * n3
    vmag_p = u_p * n1 + v_p * n2 + w_p * n3
    sm, sp = np.sqrt(rho_m), np.sqrt(rho_p)
    ssum = sm + sp
    rtil = np.sqrt(rho_p * rho_m)
    util = (sm * u_m + sp * u_p) / ssum
    vtil = (sm * v_m + sp * v_p) / ssum
    wtil = (sm * w_m + sp * w_p) / ssum
    Htil = (sm * H_m + sp * H_p) / ssum
    vmagtil = util * n1 + vtil * n2 + wtil * n3
    qtil2 = util ** 2 + vtil ** 2 + wtil ** 2
    ctil = np.sqrt((GAMMA - 1.0) * (Htil - 0.5 * qtil2))
    ctil2 = ctil ** 2
    delr = rho_m - rho_p
    delu, delv, delw = u_m - u_p, v_m - v_p, w_m - w_p
    delvmag = vmag_m - vmag_p
    delp = p_m - p_p
    eps = ENTROPY_FIX_EPS

    def limit(lam):
        lam = _abs(lam)
        small = (-eps * ctil.real < lam.real) & (lam.real < eps * ctil.real)
        return np.where(small, 0.5 * (eps * ctil + lam * lam / (eps * ctil)), _abs(lam))

    lam1 = limit(vmagtil - ctil)
    lam2 = limit(vmagtil)
    lam3 = limit(vmagtil + ctil)
    C1 = _abs(lam1) * (delp - rtil * ctil * delvmag) / (2.0 * ctil2)
    C2a = _abs(lam2) * (delr - delp / ctil2)
    C2b = _abs(lam2) * rtil
    C3 = _abs(lam3) * (delp + rtil * ctil * delvmag) / (2.0 * ctil2)
    up = np.empty(Qm.shape, dtype=np.result_type(Qm, Qp))
    up[..., 0] = 0.5 * (C1 + C2a + C3)
    up[..., 1] = 0.5 * (C1 * (util - ctil * n1) + C2a * util + C2b * (delu - delvmag * n1) + C3 * (util + ctil * n1))
    up[..., 2] = 0.5 * (C1 * (vtil - ctil * n2) + C2a * vtil + C2b * (delv - delvmag * n2) + C3 * (vtil + ctil * n2))
    up[..., 3] = 0.5 * (C1 * (wtil - ctil * n3) + C2a * wtil + C2b * (delw - delvmag * n3) + C3 * (wtil + ctil * n3))
    up[..., 4] = 0.5 * (C1 * (Htil - ctil * vmagtil) + C2a * (qtil2 / 2.0)
                        + C2b * (util * delu + vtil * delv + wtil * delw - vmagtil * delvmag)
                        + C3 * (Htil + ctil * vmagtil))
    return up


def farfield_state(Qm, n, rho_in, p_in, vel_in):
    """Exterior state of bc_state_farfield.f90 (compute_bc_state)."""
    n1, n2, n3 = n
    u_in, v_in, w_in = vel_in
    rho_m, m1, m2, m3 = Qm[..., 0], Qm[..., 1], Qm[..., 2], Qm[..., 3]
    T_in = p_in / (rho_in * RGAS)
    c_in = math.sqrt(GAMMA * RGAS * T_in)
    p_m = _pressure(Qm)
    T_m = p_m / (rho_m * RGAS)
    c_m = np.sqrt(GAMMA * RGAS * T_m)
    normal_momentum = m1 * n1 + m2 * n2 + m3 * n3
    inflow = normal_momentum.real <= RKTOL
    u_m, v_m, w_m = m1 / rho_m, m2 / rho_m, m3 / rho_m
    R_inf = (u_in * n1 + v_in * n2 + w_in * n3) - 2.0 * c_in / (GAMMA - 1.0)
    R_ext = (u_m * n1 + v_m * n2 + w_m * n3) + 2.0 * c_m / (GAMMA - 1.0)
    c_bc = ((GAMMA - 1.0) / 4.0) * (R_ext - R_inf)
    half = 0.5 * (R_ext + R_inf)
    un_in = u_in * n1 + v_in * n2 + w_in * n3
    un_m = u_m * n1 + v_m * n2 + w_m * n3
    ut = np.where(inflow, u_in - un_in * n1, u_m - un_m * n1)
    vt = np.where(inflow, v_in - un_in * n2, v_m - un_m * n2)
    wt = np.where(inflow, w_in - un_in * n3, w_m - un_m * n3)
    entropy = np.where(inflow, p_in / rho_in ** GAMMA, p_m / rho_m ** GAMMA)
    rho_bc = (c_bc * c_bc / (entropy * GAMMA)) ** (1.0 / (GAMMA - 1.0))
    Qb = np.empty(Qm.shape, dtype=np.result_type(Qm, c_bc))
    Qb[..., 0] = rho_bc
    Qb[..., 1] = (half * n1 + ut) * rho_bc
    Qb[..., 2] = (half * n2 + vt) * rho_bc
    Qb[..., 3] = (half * n3 + wt) * rho_bc
    p_bc = rho_bc ** GAMMA * entropy
    Qb[..., 4] = p_bc / (GAMMA - 1.0) + 0.5 * (Qb[..., 1] ** 2 + Qb[..., 2] ** 2 + Qb[..., 3] ** 2) / rho_bc
    return Qb


def _complex_jacobian(fn, *args):
    """d fn / d args[i][..., j] for every input i and field j, by the complex
    step: returns the value and a list (one per input) of arrays
    [..., out_field, in_field]."""
    val = fn(*[a.astype(np.float64) for a in args])
    jacs = []
    for i, a in enumerate(args):
        J = np.empty(val.shape + (a.shape[-1],))
        for j in range(a.shape[-1]):
            pert = [b.astype(np.complex128) for b in args]
            pert[i][..., j] += 1j * _CS_H
            J[..., j] = fn(*pert).imag / _CS_H
        jacs.append(J)
    return val, jacs


class EulerBox:
    """Euler DG discretisation on an nx x ny x nz box of affine hexes, with the
    Jacobian in the block layout of mesh.box_pattern.

    bcs: one of 'farfield' or 'extrapolate' for each face XI_MIN..ZETA_MAX (or a
    single name for all).  The farfield state is (rho_inf, p_inf, vel_inf).
    subdomains: box subdomains of the pattern's elem_proc (the RAS "ranks")."""

    def __init__(self, nx: int, ny: int, nz: int, order: int, extent=((0.0, 1.0),) * 3, bcs="farfield",
                 rho_inf: float = 1.0, p_inf: float = 1.0 / GAMMA, vel_inf=(0.3, 0.0, 0.0), subdomains=(1, 1, 1)):
        if not 0 <= order <= MAX_ORDER:
            raise ValueError(f"EulerBox: order must be 0..{MAX_ORDER}")
        self.shape = (nx, ny, nz)
        self.order = order
        self.nterms = (order + 1) ** 3
        self.nelem = nx * ny * nz
        self.pattern = mesh.box_pattern(nx, ny, nz, NFIELDS, self.nterms, subdomains=tuple(subdomains))
        self.bcs = [bcs] * 6 if isinstance(bcs, str) else list(bcs)
        if len(self.bcs) != 6 or any(b not in ("farfield", "extrapolate") for b in self.bcs):
            raise ValueError("EulerBox: bcs must name 'farfield' or 'extrapolate' for each of the 6 faces")
        self.rho_inf, self.p_inf, self.vel_inf = float(rho_inf), float(p_inf), tuple(float(v) for v in vel_inf)
        self.lo = np.array([e[0] for e in extent], dtype=np.float64)
        L = np.array([e[1] - e[0] for e in extent], dtype=np.float64)
        self.h = L / np.array(self.shape, dtype=np.float64)
        hx, hy, hz = self.h
        self.jinv = hx * hy * hz / 8.0                          # det(dx/dxi) of an affine hex
        self.vol = hx * hy * hz
        self.area = (hy * hz / 4.0, hx * hz / 4.0, hx * hy / 4.0)    # |scaled normal| of xi, eta, zeta faces

        n1 = nnodes_1d(order)
        xg, wg = np.polynomial.legendre.leggauss(n1)
        Lv, Ld = _legendre_tables(order, xg)
        modes = MODE_ORDER[:self.nterms]
        a, b, c = modes[:, 0], modes[:, 1], modes[:, 2]
        # volume nodes (xi fastest): phi[q, m] and reference-space gradients
        X = Lv[a][:, :, None, None] * Lv[b][:, None, :, None] * Lv[c][:, None, None, :]     # (m, i, j, k)
        DX = Ld[a][:, :, None, None] * Lv[b][:, None, :, None] * Lv[c][:, None, None, :]
        DY = Lv[a][:, :, None, None] * Ld[b][:, None, :, None] * Lv[c][:, None, None, :]
        DZ = Lv[a][:, :, None, None] * Lv[b][:, None, :, None] * Ld[c][:, None, None, :]
        flat = lambda T: T.transpose(0, 3, 2, 1).reshape(self.nterms, -1).T                 # (q, m), xi fastest
        self.phi = flat(X)
        self.grad = np.stack([flat(DX) * (2.0 / hx), flat(DY) * (2.0 / hy), flat(DZ) * (2.0 / hz)])   # (3, q, m)
        self.w = (wg[None, None, :] * wg[None, :, None] * wg[:, None, None]).reshape(-1)
        Kz, Jy, Ix = np.meshgrid(xg, xg, xg, indexing="ij")                  # [k, j, i]
        self.xq = np.stack([Ix, Jy, Kz], axis=-1).reshape(-1, 3)             # reference coordinates, xi fastest
        # face nodes: the two tangential coordinates over the Gauss grid, the
        # normal one at -1 (MIN faces) or +1 (MAX faces)
        self.wf = (wg[:, None] * wg[None, :]).reshape(-1)
        self.phif = []
        for fid in range(6):
            d, side = fid // 2, (-1.0 if fid % 2 == 0 else 1.0)
            Lend = np.array([1.0 if n % 2 == 0 or side > 0 else -1.0 for n in range(order + 1)])    # P_n(+-1)
            per_dir = []
            for dd, deg in zip(range(3), (a, b, c)):
                per_dir.append(Lend[deg][:, None] if dd == d else Lv[deg])                      # (m, nq1)
            t = [dd for dd in range(3) if dd != d]
            A, B = per_dir[t[0]], per_dir[t[1]]
            self.phif.append((A[:, :, None] * B[:, None, :] * per_dir[d][:, :, None]).reshape(self.nterms, -1).T)
        # element index helpers
        e = np.arange(self.nelem)
        self.ijk = np.stack([e % nx, (e // nx) % ny, e // (nx * ny)], axis=1)
        self.stride = (1, nx, nx * ny)
        M = self.jinv * np.einsum("q,qm,qn->mn", self.w, self.phi, self.phi)
        self.mass_block = M
        self.mass = np.tile(M.ravel(order="F"), self.nelem)
        self._diag_k, self._face_k = self._block_index()

    # ---- layout helpers --------------------------------------------------------
    def _block_index(self):
        """Pattern block number of the DIAG block of each element and of the
        block of each (element, face) (-1 on boundary faces)."""
        p = self.pattern
        diag = np.full(self.nelem, -1, dtype=np.int64)
        face = np.full((self.nelem, 6), -1, dtype=np.int64)
        k = np.arange(p.nblocks, dtype=np.int64)
        f = np.asarray(p.blk_face)
        row = np.asarray(p.blk_row_elem)
        d = f == mesh.DIAG
        diag[row[d]] = k[d]
        o = f < 6
        face[row[o], f[o]] = k[o]
        return diag, face

    def modes(self, q: np.ndarray) -> np.ndarray:
        return np.asarray(q, dtype=np.float64).reshape(self.nelem, NFIELDS, self.nterms)

    def coords(self) -> np.ndarray:
        """Physical coordinates of the volume nodes of every element (E, q, 3)."""
        centre = self.lo + (self.ijk + 0.5) * self.h
        return centre[:, None, :] + 0.5 * self.h[None, None, :] * self.xq[None, :, :]

    def project(self, fn) -> np.ndarray:
        """L2 projection of fn(x) -> (..., 5) conserved variables onto the modes."""
        vals = fn(self.coords())                                           # (E, q, 5)
        rhs = self.jinv * np.tensordot(vals, self.w[:, None] * self.phi, axes=([1], [0]))   # (E, 5, m)
        Minv = np.linalg.inv(self.mass_block)
        return np.tensordot(rhs, Minv, axes=([2], [1])).reshape(-1)

    def freestream(self) -> np.ndarray:
        u = np.array(self.vel_inf)
        E = self.p_inf / (GAMMA - 1.0) + 0.5 * self.rho_inf * float(u @ u)
        cons = np.array([self.rho_inf, *(self.rho_inf * u), E])
        return self.project(lambda x: np.broadcast_to(cons, x.shape[:-1] + (5,)))

    def density_bump(self, amplitude: float = 1e-2, width: float = 0.1, centre=(0.5, 0.5, 0.5)) -> np.ndarray:
        """Freestream with a Gaussian density bump rho_inf (1 + a exp(-|x-c|^2 / w^2))
        at the freestream pressure and velocity."""
        u = np.array(self.vel_inf)
        c = np.asarray(centre, dtype=np.float64)

        def fn(x):
            rho = self.rho_inf * (1.0 + amplitude * np.exp(-np.sum((x - c) ** 2, axis=-1) / width ** 2))
            out = np.empty(x.shape[:-1] + (5,))
            out[..., 0] = rho
            out[..., 1:4] = rho[..., None] * u
            out[..., 4] = self.p_inf / (GAMMA - 1.0) + 0.5 * rho * float(u @ u)
            return out
        return self.project(fn)

    # ---- residual and Jacobian -----------------------------------------------------
    def _interior_pairs(self, d):
        n = self.shape[d]
        left = np.nonzero(self.ijk[:, d] < n - 1)[0]
        return left, left + self.stride[d]

    def _boundary_elems(self, fid):
        d = fid // 2
        return np.nonzero(self.ijk[:, d] == (0 if fid % 2 == 0 else self.shape[d] - 1))[0]

    def _bc_integrand(self, fid):
        d, s = fid // 2, (-1.0 if fid % 2 == 0 else 1.0)
        n = np.zeros(3)
        n[d] = s
        a = self.area[d]
        kind = self.bcs[fid]

        def fn(Qm):
            Qb = farfield_state(Qm, n, self.rho_inf, self.p_inf, self.vel_inf) if kind == "farfield" else Qm
            return euler_flux(Qb)[..., d, :] * (s * a)
        return fn

    def _face_integrand(self, d):
        n = np.zeros(3)
        n[d] = 1.0
        a = self.area[d]

        def fn(QL, QR):
            avg = 0.5 * (euler_flux(QL)[..., d, :] + euler_flux(QR)[..., d, :]) * a
            return avg + a * roe_upwind(QL, QR, n)
        return fn

    def residual(self, q: np.ndarray, jacobian: bool = False):
        """R(q) in the vector layout, and with jacobian=True also dR/dq as the
        packed block values of self.pattern."""
        U = self.modes(q)
        nt = self.nterms
        R = np.zeros((self.nelem, NFIELDS, nt))
        if jacobian:
            D = np.zeros((self.nelem, NFIELDS, nt, NFIELDS, nt))
            FB = np.zeros((self.nelem, 6, NFIELDS, nt, NFIELDS, nt))
        Qv = np.einsum("qm,efm->eqf", self.phi, U)
        if jacobian:
            F, (dF,) = _complex_jacobian(euler_flux, Qv)                   # (E,q,3,5), (E,q,3,5,5)
            D -= self.jinv * np.einsum("dqm,q,eqdfg,qn->efmgn", self.grad, self.w, dF, self.phi, optimize=True)
        else:
            F = euler_flux(Qv)
        R -= self.jinv * np.einsum("dqm,q,eqdf->efm", self.grad, self.w, F, optimize=True)
        for d in range(3):
            L, Rr = self._interior_pairs(d)
            if L.size == 0:
                continue
            pmax, pmin = self.phif[2 * d + 1], self.phif[2 * d]
            QL = np.einsum("qm,efm->eqf", pmax, U[L])
            QR = np.einsum("qm,efm->eqf", pmin, U[Rr])
            fn = self._face_integrand(d)
            if jacobian:
                I, (dL, dR) = _complex_jacobian(fn, QL, QR)
                D[L] += np.einsum("qm,q,pqfg,qn->pfmgn", pmax, self.wf, dL, pmax, optimize=True)
                FB[L, 2 * d + 1] += np.einsum("qm,q,pqfg,qn->pfmgn", pmax, self.wf, dR, pmin, optimize=True)
                FB[Rr, 2 * d] -= np.einsum("qm,q,pqfg,qn->pfmgn", pmin, self.wf, dL, pmax, optimize=True)
                D[Rr] -= np.einsum("qm,q,pqfg,qn->pfmgn", pmin, self.wf, dR, pmin, optimize=True)
            else:
                I = fn(QL, QR)
            R[L] += np.einsum("qm,q,pqf->pfm", pmax, self.wf, I)
            R[Rr] -= np.einsum("qm,q,pqf->pfm", pmin, self.wf, I)
        for fid in range(6):
            E = self._boundary_elems(fid)
            pf = self.phif[fid]
            Qm = np.einsum("qm,efm->eqf", pf, U[E])
            fn = self._bc_integrand(fid)
            if jacobian:
                I, (dI,) = _complex_jacobian(fn, Qm)
                D[E] += np.einsum("qm,q,pqfg,qn->pfmgn", pf, self.wf, dI, pf, optimize=True)
            else:
                I = fn(Qm)
            R[E] += np.einsum("qm,q,pqf->pfm", pf, self.wf, I)
        if not jacobian:
            return R.reshape(-1)
        b = NFIELDS * nt
        blocks = np.empty((self.pattern.nblocks, b, b))
        blocks[self._diag_k] = D.reshape(self.nelem, b, b)
        e_idx, f_idx = np.nonzero(self._face_k >= 0)
        blocks[self._face_k[e_idx, f_idx]] = FB[e_idx, f_idx].reshape(-1, b, b)
        return R.reshape(-1), blocks.transpose(0, 2, 1).reshape(-1)        # column-major blocks

    def pseudo_timestep(self, q: np.ndarray, cfl) -> np.ndarray:
        """dtau[e, field] = cfl[field] h / (mean |u| + mean c) over the volume
        nodes (type_fluid_pseudo_timestep.f90, compute)."""
        Qv = np.einsum("qm,efm->eqf", self.phi, self.modes(q))
        rho = Qv[..., 0]
        p = _pressure(Qv)
        c = np.sqrt(GAMMA * p / rho)
        vmag = np.sqrt((Qv[..., 1] ** 2 + Qv[..., 2] ** 2 + Qv[..., 3] ** 2) / (rho * rho))
        lam = vmag.mean(axis=1) + c.mean(axis=1)
        h = self.vol ** (1.0 / 3.0)
        cfl = np.broadcast_to(np.asarray(cfl, dtype=np.float64), (NFIELDS,))
        return cfl[None, :] * (h / lam)[:, None]


def hb_times(freqs) -> np.ndarray:
    """Harmonic-balance time levels t_i = (2 pi / min |omega|) i / ntime,
    i = 1..ntime, ntime = 2 nfreq + 1 (type_time_manager.f90:153-187)."""
    w = np.asarray(freqs, dtype=np.float64)
    ntime = 2 * w.size + 1
    return (2.0 * np.pi / np.min(np.abs(w))) * (np.arange(1, ntime + 1) / ntime)


def hb_operator(freqs, times) -> np.ndarray:
    """The pseudo-spectral time-derivative operator D = dE^-1 E with E^-1 the
    samples of (1, sin w_k t, cos w_k t) at the time levels and dE^-1 their time
    derivatives (mod_HB_matrices.f90: calc_inv_E, calc_diff_inv_E,
    calc_pseudo_spectral_operator)."""
    w = np.asarray(freqs, dtype=np.float64)
    t = np.asarray(times, dtype=np.float64)
    nf, nt = w.size, t.size
    invE = np.empty((nt, nt))
    dinvE = np.empty((nt, nt))
    invE[:, 0], dinvE[:, 0] = 1.0, 0.0
    for k in range(nf):
        invE[:, 1 + k] = np.sin(w[k] * t)
        dinvE[:, 1 + k] = w[k] * np.cos(w[k] * t)
        invE[:, 1 + nf + k] = np.cos(w[k] * t)
        dinvE[:, 1 + nf + k] = -w[k] * np.sin(w[k] * t)
    return dinvE @ np.linalg.inv(invE)


class EulerHB:
    """The Euler box under harmonic balance (assemble_harmonic_balance_t%assemble,
    type_harmonic_balance.f90:127-229): at every time level t the spatial
    residual and Jacobian of that level's state, with the farfield velocity
    vel_inf (1 + amplitude sin(w_1 t)) (a sinusoidal inflow), plus
    sum_t' D(t, t') M q_t' in the residual and D(t, t') M on each field's
    diagonal in the hb block coupling t to t' != t (the reference stores the
    t' = t term in the residual only).  The pattern is mesh.box_pattern with
    ntime levels; vectors are element-major, then time level, field, mode."""

    def __init__(self, nx, ny, nz, order, freqs, amplitude=1e-2, **box_args):
        self.freqs = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
        self.times = hb_times(self.freqs)
        self.D = hb_operator(self.freqs, self.times)
        self.ntime = self.times.size
        base = EulerBox(nx, ny, nz, order, **box_args)
        u0 = np.asarray(base.vel_inf)
        self.levels = []
        for t in self.times:
            args = dict(box_args)
            args["vel_inf"] = tuple(u0 * (1.0 + amplitude * np.sin(self.freqs[0] * t)))
            self.levels.append(EulerBox(nx, ny, nz, order, **args))
        self.base = base
        self.nelem, self.nterms = base.nelem, base.nterms
        self.mass = base.mass
        self.pattern = mesh.box_pattern(nx, ny, nz, NFIELDS, base.nterms, ntime=self.ntime)
        p = self.pattern
        local = np.asarray(p.blk_kind) == _lib.BLK_LOCAL
        e, f = np.asarray(p.blk_row_elem), np.asarray(p.blk_face)
        ks = np.where(f == mesh.DIAG, base._diag_k[e], base._face_k[e, np.minimum(f, 5)])
        self._local_k = np.nonzero(local)[0]                  # hb-pattern blocks from the spatial Jacobians
        self._local_src = ks[local]                           # their block in the level's pattern
        self._local_t = np.asarray(p.blk_row_time)[local]
        self._hb_k = np.nonzero(~local)[0]
        self._hb_to = np.asarray(p.blk_row_time)[~local]
        self._hb_from = np.asarray(p.blk_col_time)[~local]

    def freestream(self) -> np.ndarray:
        """Every level at its own farfield state."""
        return np.stack([lv.freestream().reshape(self.nelem, -1) for lv in self.levels], axis=1).reshape(-1)

    def density_bump(self, **kw) -> np.ndarray:
        return np.stack([lv.density_bump(**kw).reshape(self.nelem, -1) for lv in self.levels], axis=1).reshape(-1)

    def residual(self, q: np.ndarray, jacobian: bool = False):
        nt, b, T = self.nterms, NFIELDS * self.nterms, self.ntime
        U = np.asarray(q, dtype=np.float64).reshape(self.nelem, T, b)
        R = np.empty_like(U)
        if jacobian:
            vals = np.empty((self.pattern.nblocks, b, b))           # [block, column, row]
        for t, lv in enumerate(self.levels):
            if jacobian:
                Rt, vt = lv.residual(U[:, t].reshape(-1), jacobian=True)
                sel = self._local_t == t
                vals[self._local_k[sel]] = vt.reshape(-1, b, b)[self._local_src[sel]]
            else:
                Rt = lv.residual(U[:, t].reshape(-1))
            R[:, t] = Rt.reshape(self.nelem, b)
        Mq = np.einsum("mn,etfn->etfm", self.base.mass_block, U.reshape(self.nelem, T, NFIELDS, nt))
        R += np.einsum("ab,ebfm->eafm", self.D, Mq).reshape(self.nelem, T, b)
        if not jacobian:
            return R.reshape(-1)
        blk = np.kron(np.eye(NFIELDS), self.base.mass_block.T)
        vals[self._hb_k] = self.D[self._hb_to, self._hb_from][:, None, None] * blk[None]
        return R.reshape(-1), vals.reshape(-1)

    def pseudo_timestep(self, q: np.ndarray, cfl) -> np.ndarray:
        """The pseudo time steps of time level 1, as compute_pseudo_timestep
        takes them (type_newton.f90:294-306, itime = 1)."""
        U = np.asarray(q, dtype=np.float64).reshape(self.nelem, self.ntime, -1)
        return self.levels[0].pseudo_timestep(U[:, 0].reshape(-1), cfl)

    def add_pseudo_time(self, vals: np.ndarray, dtau: np.ndarray) -> np.ndarray:
        """vals + mass / dtau_e on every field's diagonal sub-block of the DIAG
        block of every time level, dtau_e the element's smallest pseudo time
        step over its fields (contribute_pseudo_temporal)."""
        nt, b = self.nterms, NFIELDS * self.nterms
        out = np.array(vals, dtype=np.float64, copy=True)
        blk = out.reshape(self.pattern.nblocks, b, b)                # [block, column, row]
        diag = np.nonzero(np.asarray(self.pattern.blk_face) == mesh.DIAG)[0]
        dmin = np.asarray(dtau, dtype=np.float64).reshape(self.nelem, -1).min(axis=1)
        scale = 1.0 / dmin[np.asarray(self.pattern.blk_row_elem)[diag]]
        Mt = self.base.mass_block.T
        for f in range(NFIELDS):
            s = slice(f * nt, (f + 1) * nt)
            blk[diag, s, s] += scale[:, None, None] * Mt[None]
        return out


def add_pseudo_time(box: EulerBox, vals: np.ndarray, dtau: np.ndarray) -> np.ndarray:
    """Host counterpart of chidg_gpu_matrix_scale_diagonal for a host-assembled
    Jacobian: vals + mass / dtau_e on every field's diagonal sub-block of the
    DIAG blocks, dtau_e the minimum of the element's pseudo time steps over its
    fields (contribute_pseudo_temporal, type_newton.f90:320-352)."""
    nb, b, nt = box.pattern.nblocks, NFIELDS * box.nterms, box.nterms
    out = np.array(vals, dtype=np.float64, copy=True)
    blk = out.reshape(nb, b, b)                            # [block, column, row]
    dtau = np.asarray(dtau, dtype=np.float64).reshape(box.nelem, -1).min(axis=1)
    dtau = np.broadcast_to(dtau[:, None], (box.nelem, NFIELDS))
    Mt = box.mass_block.T
    for f in range(NFIELDS):
        s = slice(f * nt, (f + 1) * nt)
        blk[box._diag_k, s, s] += Mt[None, :, :] / dtau[:, f, None, None]
    return out


class EulerSystem:
    """The Newton driver's `system` over an EulerBox: residual and Jacobian
    assembled on the host from the downloaded state, uploaded into the device
    matrix and vector."""

    def __init__(self, box: EulerBox):
        self.box = box
        self.pattern = box.pattern
        self.mass = box.mass
        self.assemble_seconds = 0.0
        self.nassemble = 0

    def assemble(self, q, A, rhs, differentiate):
        import time
        t0 = time.perf_counter()
        qh = q.download()
        if differentiate:
            R, vals = self.box.residual(qh, jacobian=True)
            A.upload(vals)
        else:
            R = self.box.residual(qh)
        rhs.upload(R)
        self.assemble_seconds += time.perf_counter() - t0
        self.nassemble += 1

    def pseudo_timestep(self, q, cfl):
        return self.box.pseudo_timestep(q.download(), cfl)


def box_desc(box: EulerBox):
    """The chidg_gpu_euler_box of an EulerBox."""
    from . import _lib
    d = _lib.EulerBoxDesc()
    d.nx, d.ny, d.nz = box.shape
    d.order = box.order
    for i in range(3):
        d.lo[i] = float(box.lo[i])
        d.hi[i] = float(box.lo[i] + box.h[i] * box.shape[i])
        d.vel_inf[i] = box.vel_inf[i]
    for f in range(6):
        d.bc[f] = _lib.EULER_FARFIELD if box.bcs[f] == "farfield" else _lib.EULER_EXTRAPOLATE
    d.rho_inf, d.p_inf = box.rho_inf, box.p_inf
    return d


class EulerDevice:
    """The same discretisation assembled on the GPU (chidg_gpu_euler_*): the
    residual into a device vector and the Jacobian straight into the device
    matrix's blocks, orders 0..3.  The extent, boundary conditions and
    freestream are the EulerBox's."""

    def __init__(self, box: EulerBox, ctx: api.Context | None = None):
        import ctypes as C

        from . import _lib
        if box.order > 3:
            raise ValueError("EulerDevice: orders 0..3")
        self.box = box
        self.ctx = ctx or api.default_context()
        d = box_desc(box)
        self._desc = d
        h = C.c_void_p()
        self.ctx.check(self.ctx.L.chidg_gpu_euler_create(self.ctx.h, C.byref(d), C.byref(h)), "euler_create")
        self.h = h

    def assemble(self, q: api.ChidgVector, rhs: api.ChidgVector, A: api.ChidgMatrix | None = None):
        """rhs = R(q); with A also A = dR/dq (every block of A overwritten)."""
        self.ctx.check(self.ctx.L.chidg_gpu_euler_assemble(self.h, q.h, rhs.h, A.h if A is not None else None),
                       "euler_assemble")

    def pseudo_timestep(self, q: api.ChidgVector, cfl) -> np.ndarray:
        cfl = np.ascontiguousarray(np.broadcast_to(np.asarray(cfl, dtype=np.float64), (NFIELDS,)))
        out = np.empty((self.box.nelem, NFIELDS))
        from . import _lib
        self.ctx.check(self.ctx.L.chidg_gpu_euler_pseudo_timestep(self.h, q.h, cfl.ctypes.data_as(_lib.DP),
                                                                  out.ctypes.data_as(_lib.DP)), "euler_pseudo_timestep")
        return out

    def assemble_at(self, A: api.ChidgMatrix, elem0: int, q: api.ChidgVector, rhs: api.ChidgVector,
                    jacobian: bool = True):
        """The box as elements elem0.. of a larger layout A (a batch arena):
        rhs's segment of the box = R(q), and with `jacobian` A's blocks of the box."""
        self.ctx.check(self.ctx.L.chidg_gpu_euler_assemble_at(self.h, A.h, int(elem0), q.h, rhs.h, int(bool(jacobian))),
                       "euler_assemble_at")

    def pseudo_timestep_at(self, A: api.ChidgMatrix, elem0: int, q: api.ChidgVector, cfl) -> np.ndarray:
        cfl = np.ascontiguousarray(np.broadcast_to(np.asarray(cfl, dtype=np.float64), (NFIELDS,)))
        out = np.empty((self.box.nelem, NFIELDS))
        from . import _lib
        self.ctx.check(self.ctx.L.chidg_gpu_euler_pseudo_timestep_at(self.h, A.h, int(elem0), q.h,
                                                                     cfl.ctypes.data_as(_lib.DP),
                                                                     out.ctypes.data_as(_lib.DP)),
                       "euler_pseudo_timestep_at")
        return out

    def release(self):
        if getattr(self, "h", None):
            self.ctx.L.chidg_gpu_euler_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class EulerHBDevice:
    """The harmonic-balance system of an EulerHB assembled on the GPU: every
    time level's spatial residual and Jacobian by the device kernel of that
    level's box (chidg_gpu_euler_assemble_level), then the time coupling
    sum_t' D(t, t') M q_t' and the hb blocks D(t, t') M (chidg_gpu_hb_coupling),
    into a matrix holding hb.pattern and vectors of it; the pseudo time steps
    are those of level 1 (chidg_gpu_euler_pseudo_timestep_level)."""

    def __init__(self, hb: "EulerHB", ctx: api.Context | None = None):
        self.hb = hb
        self.ctx = ctx or api.default_context()
        self.levels = [EulerDevice(lv, self.ctx) for lv in hb.levels]
        self._D = np.asfortranarray(hb.D, dtype=np.float64)
        self._M = np.asfortranarray(hb.base.mass_block, dtype=np.float64)

    def assemble(self, q: api.ChidgVector, rhs: api.ChidgVector, A: api.ChidgMatrix, jacobian: bool = True):
        from . import _lib
        L = self.ctx.L
        for t, dev in enumerate(self.levels):
            self.ctx.check(L.chidg_gpu_euler_assemble_level(dev.h, A.h, t, q.h, rhs.h, int(bool(jacobian))),
                           "euler_assemble_level")
        self.ctx.check(L.chidg_gpu_hb_coupling(A.h, int(self.hb.nterms), self._D.ctypes.data_as(_lib.DP),
                                               self._M.ctypes.data_as(_lib.DP), q.h, rhs.h, int(bool(jacobian))),
                       "hb_coupling")

    def pseudo_timestep(self, q: api.ChidgVector, A: api.ChidgMatrix, cfl) -> np.ndarray:
        from . import _lib
        cfl = np.ascontiguousarray(np.broadcast_to(np.asarray(cfl, dtype=np.float64), (NFIELDS,)))
        out = np.empty((self.hb.nelem, NFIELDS))
        self.ctx.check(self.ctx.L.chidg_gpu_euler_pseudo_timestep_level(self.levels[0].h, A.h, 0, q.h,
                                                                        cfl.ctypes.data_as(_lib.DP),
                                                                        out.ctypes.data_as(_lib.DP)),
                       "euler_pseudo_timestep_level")
        return out

    def release(self):
        for dev in self.levels:
            dev.release()


class NewtonSystem:
    """The first Newton step's system of an EulerBox or an EulerHB at the state
    q0, described for chidg_gpu_euler_fill_system: A = dR/dq(q0) (every level
    and the hb blocks) + mass / dtau (dtau of level 1 at `cfl`, its minimum over
    the fields), b = -R(q0), written on the device into elements elem0.. of a
    larger layout (a batch arena, or a served batch through
    chidg_gpu_serve_submit_fill).  Keeps the arrays the description points at."""

    def __init__(self, system, q0: np.ndarray, cfl: float):
        import ctypes as C

        from . import _lib
        hb = system if isinstance(system, EulerHB) else None
        box = hb.levels[0] if hb is not None else system
        if box.order > 3:
            raise ValueError("NewtonSystem: orders 0..3")
        self.pattern = system.pattern
        self.nelem = box.nelem
        self.ntime = hb.ntime if hb is not None else 1
        self.q0 = np.ascontiguousarray(q0, dtype=np.float64)
        if self.q0.size != self.pattern.vector_size():
            raise ValueError("NewtonSystem: q0 does not match the pattern")
        self.mass = np.asfortranarray(box.mass_block, dtype=np.float64)
        d = _lib.EulerSystemDesc()
        d.box = box_desc(box)
        d.ntime = self.ntime
        d.mass = self.mass.ctypes.data_as(_lib.DP)
        d.q0 = self.q0.ctypes.data_as(_lib.DP)
        d.cfl = float(cfl)
        if hb is not None:
            self.D = np.asfortranarray(hb.D, dtype=np.float64)
            self.level_vel = np.ascontiguousarray([lv.vel_inf for lv in hb.levels], dtype=np.float64)
            d.D = self.D.ctypes.data_as(_lib.DP)
            d.level_vel = self.level_vel.ctypes.data_as(_lib.DP)
        self.desc = d
        self.user = C.c_void_p(C.addressof(d))

    def fill(self, A: api.ChidgMatrix, b: api.ChidgVector, work: api.ChidgVector, elem0: int):
        """Write the system into elements elem0.. of A and its segment of b;
        work's segment is overwritten."""
        A.ctx.check(A.ctx.L.chidg_gpu_euler_fill_system(self.user, A.ctx.h, A.h, b.h, work.h, int(elem0)),
                    "euler_fill_system")


class EulerDeviceSystem:
    """The Newton driver's `system` with the assembly on the GPU: q, rhs and
    the Jacobian never leave the device; only the pseudo time steps (nelem x 5)
    come back to the host for chidg_gpu_matrix_scale_diagonal."""

    def __init__(self, box: EulerBox, ctx: api.Context | None = None):
        self.box = box
        self.pattern = box.pattern
        self.mass = box.mass
        self.device = EulerDevice(box, ctx)
        self.assemble_seconds = 0.0
        self.nassemble = 0

    def assemble(self, q, A, rhs, differentiate):
        import time
        t0 = time.perf_counter()
        self.device.assemble(q, rhs, A if differentiate else None)
        self.device.ctx.sync()
        self.assemble_seconds += time.perf_counter() - t0
        self.nassemble += 1

    def pseudo_timestep(self, q, cfl):
        return self.device.pseudo_timestep(q, cfl)
