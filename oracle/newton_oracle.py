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

The host system provides
    residual(q, jacobian) -> R or (R, values)    packed block values of dR/dq
    pseudo_timestep(q, cfl) -> dtau              nelem x nfields
    add_pseudo_time(values, dtau) -> values      values + mass / dtau_e on the
                                                 diagonal blocks
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O


def newton(system, pattern, q0, *, cfl0=1.0, cfl_up=1.5, cfl_down=0.1, cfl_max=-1.0, tol=1e-10, rtol=1e-10,
           nmax=-1, ptc=True, linear_opts=None, precon="ilu0"):
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
