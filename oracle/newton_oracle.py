"""Newton's method restated on the host over numpy arrays and the CPU oracle.

TEST INFRASTRUCTURE ONLY: the checker of the device Newton driver
(chidg_b200/newton.py).  Imported by tests/ only; the product never imports it.

newton_t%solve (src/nonlinear_solvers/type_newton.f90:64-266): the residual
and its Jacobian from the caller's host system, b = -R (:180), the
pseudo-transient term mass/dtau on the diagonal blocks with the element's
smallest pseudo time step over its fields (contribute_pseudo_temporal,
:320-352), the linear solve by the oracle's FGMRES and preconditioner
(type_fgmres.f90:81-310 and precon_ILU0.f90 restated in chidg_oracle.cpp),
the backtracking line search with its acceptance tests and the cfl update
(:466-549), and the stopping rules (:244-266).  Norms are the oracle's serial
FP64 norms (type_chidg_vector.f90:1237-1305).

Residual smoothing (:160-172 with apply_residual_smoother and
pseudo_transient_scaling, :360-441): the smoother (the oracle's block Jacobi,
or the linear solve's preconditioner kind) is built on the Jacobian before the
pseudo-transient term, and b = -R - smooth_relax * smoother(M / dtau R), every
field segment of R scaled by the element mass over the element's smallest
pseudo time step.  Without ptc the reference warns and leaves b unassigned;
this restatement then skips smoothing (b = -R), as the device driver does.

The host system provides
    residual(q, jacobian) -> R or (R, values)    packed block values of dR/dq
    pseudo_timestep(q, cfl) -> dtau              nelem x nfields
    add_pseudo_time(values, dtau) -> values      values + mass / dtau_e on the
                                                 diagonal blocks
    mass_block                                   the element mass matrix (nterms
                                                 x nterms; smoothing only)
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


def mass_scale(pattern, x, mass_block, dtau_min):
    """(M / dtau) x on every element, time level and field segment
    (pseudo_transient_scaling, type_newton.f90:394-441): y_i = sum_j
    (s M_ij) x_j with s = 1 / dtau_e, j in increasing order."""
    nt = mass_block.shape[0]
    ne, T = int(pattern.nelem), int(pattern.ntime)
    X = np.asarray(x, dtype=np.float64).reshape(ne, T, -1, nt)
    S = (1.0 / np.asarray(dtau_min, dtype=np.float64))[:, None, None] * mass_block[None, :, :]    # (e, i, j)
    Y = np.zeros_like(X)
    for j in range(nt):
        Y += S[:, None, None, :, j] * X[:, :, :, j:j + 1]
    return Y.reshape(-1)


def newton(system, pattern, q0, *, cfl0=1.0, cfl_up=1.5, cfl_down=0.1, cfl_max=-1.0, tol=1e-10, rtol=1e-10,
           nmax=-1, ptc=True, linear_opts=None, precon="ilu0", smooth=False, smoother="jacobi", smooth_relax=1.0):
    """Returns a dict: residual_norm (|R(q0)| then |R| after each step),
    alphas, linear_iterations, linear_rel_residual, q."""
    A = O.OracleMatrix(pattern)
    opts = O.default_opts(**(linear_opts or {}))
    q = np.array(q0, dtype=np.float64, copy=True)
    nfields = int(pattern.elem_nvars[0])
    cfl = np.full(nfields, float(cfl0))
    out = {"residual_norm": [], "alphas": [], "linear_iterations": [], "linear_rel_residual": [], "cfl": []}
    resid0 = None
    niter = 0
    while True:
        niter += 1
        qold = q.copy()
        R, vals = system.residual(q, jacobian=True)
        resid = A.norm(R)
        if niter == 1:
            resid0 = resid
            out["residual_norm"].append(resid)
        b = -R
        if smooth and ptc:
            A.set_values(vals)                               # the smoother sees the Jacobian before ptc
            Ms = O.OraclePrecon(A, "jacobi" if smoother == "jacobi" else precon)
            Ms.update()
            dmin = np.asarray(system.pseudo_timestep(q, cfl)).min(axis=1)
            f_smooth = smooth_relax * Ms.apply(mass_scale(pattern, R, system.mass_block, dmin))
            b = -R - f_smooth
            del Ms
        if ptc:
            vals = system.add_pseudo_time(vals, system.pseudo_timestep(q, cfl))
        if resid < tol:
            break
        if math.isnan(resid):
            raise ArithmeticError("newton: NaN residual norm")
        A.set_values(vals)
        dq, res = O.fgmres(A, O.OraclePrecon(A, precon), b, opts)
        out["linear_iterations"].append(res["niter"])
        out["linear_rel_residual"].append(res["residual_norm"] / max(res["r0norm_initial"], 1e-300))
        f0 = resid
        step = 0
        while True:
            alpha = 2.0 ** (-step)
            q = qold + alpha * dq
            fn = A.norm(system.residual(q))
            if math.isnan(fn):
                searching = True
            elif fn > 1.e-3 and fn > 2.0 * f0:
                searching = True
            elif fn < 1.e-3 and fn > f0:
                searching = True
            else:
                searching = False
            step += 1
            if not searching:
                break
            if step > 60:
                raise ArithmeticError("newton: backtracking found no acceptable step")
        if alpha > 0.75:
            cfl = cfl * cfl_up
        elif alpha < 0.2:
            cfl = cfl * cfl_down
        if cfl_max > 0.0:
            cfl = np.minimum(cfl, cfl_max)
        out["residual_norm"].append(fn)
        out["alphas"].append(alpha)
        out["cfl"].append(float(cfl[0]))
        if not (fn > tol and fn / resid0 > rtol and (niter < nmax or nmax <= 0)):
            break
    out["q"] = q
    return out
