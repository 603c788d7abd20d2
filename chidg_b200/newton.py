"""newton_t%solve (src/nonlinear_solvers/type_newton.f90:64-266) over the device
containers.

The state q, the update dq, the residual rhs and the Newton right-hand side
b = -rhs stay in GPU memory; the residual norms, b = -rhs, the pseudo-transient
term mass/dtau on the diagonal blocks (chidg_gpu_matrix_scale_diagonal), the
backtracking update q = q0 + alpha dq and the linear solve run on the device.
Assembly of the residual and its Jacobian stays with the caller, through a
`system` object:

    system.assemble(q, A, rhs, differentiate)   fill rhs = R(q), and A = dR/dq
                                                when differentiate is true
    system.pseudo_timestep(q, cfl) -> dtau      pseudo time steps, cfl per field:
                                                one per element, or one per element
                                                and field (nelem x nfields, as
                                                elems(:)%dtau(ieqn)), of which the
                                                element's minimum is applied to
                                                every field and time level
    system.mass -> packed per-element mass matrices (nterms x nterms,
                   column-major), as chidg_gpu_matrix_scale_diagonal takes them

Options are those of nonlinear_solver_t (src/nonlinear_solvers/
type_nonlinear_solver.f90:21-36), with the defaults of the input namelist
(src/io/mod_io.f90:58-77): residual smoothing off.  With `smooth` and `ptc`
the right-hand side is smoothed as type_newton.f90:160-172 does (Mavriplis
2018): the smoother (a block-Jacobi preconditioner, or the linear solver's own
preconditioner) is updated on the Jacobian before the pseudo-transient term is
added, then b = -R - smooth_relax * smoother(M / dtau R), where M / dtau scales
every field segment by the element mass over the element's smallest pseudo
time step (pseudo_transient_scaling, :394-441, on the device through
chidg_gpu_vector_mass_scale).  `nsmooth` is accepted and, as in the
reference's Newton loop, not used.  With `smooth` and not `ptc` the reference
prints a warning and leaves b unassigned; here smoothing is skipped with the
same warning and b = -R.
"""
from __future__ import annotations

import math
import sys
import time
from dataclasses import dataclass, field

import numpy as np

from . import api


@dataclass
class NewtonOptions:
    cfl0: float = 1.0
    cfl_max: float = -1.0        # negative: unlimited
    cfl_up: float = 1.5
    cfl_down: float = 0.1
    tol: float = 1e-10
    rtol: float = 1e-10
    nmax: int = -1               # <= 0: unlimited
    ptc: bool = True
    search: str = "backtrack"    # 'backtrack' or 'none'
    smooth: bool = False
    smoother: str = "jacobi"     # 'jacobi' or 'preconditioner'
    nsmooth: int = 3
    smooth_relax: float = 1.0


@dataclass
class NewtonResult:
    niter: int = 0
    residual_norm: list = field(default_factory=list)     # |R| after each step (the first entry: |R(q0)|)
    matrix_iterations: list = field(default_factory=list)
    linear_seconds: list = field(default_factory=list)
    linear_rel_residual: list = field(default_factory=list)    # true |b - A dq| / |b| of each linear solve
    alphas: list = field(default_factory=list)
    cfl: list = field(default_factory=list)
    seconds: float = 0.0
    phase_seconds: dict = field(default_factory=dict)    # wall time by phase: assembly, ptc, linear, search, other
    converged: bool = False


class Newton:
    """newton_t: Newton's method with pseudo-transient continuation and a
    backtracking line search."""

    def __init__(self, **options):
        self.options = NewtonOptions(**options)
        if self.options.smoother.lower() not in ("jacobi", "preconditioner"):
            raise ValueError("newton%solve: invalid smoother. 'default' or 'jacobi'.")
        if self.options.search.lower() not in ("backtrack", "none", ""):
            raise ValueError(f"Invalid nonlinear search algorithm in newton iteration routine: '{self.options.search}'")

    def solve(self, system, q: api.ChidgVector, A: api.ChidgMatrix, linear_solver, preconditioner) -> NewtonResult:
        o = self.options
        res = NewtonResult()
        t_start = time.perf_counter()
        ph = {"assembly": 0.0, "ptc": 0.0, "linear": 0.0, "search": 0.0}
        nfields = int(A.pattern.elem_nvars[0])
        rhs = api.ChidgVector(A)
        dq = api.ChidgVector(A)
        b = api.ChidgVector(A)
        qold = api.ChidgVector(A)
        qn = api.ChidgVector(A)
        qn.copy_from(q)
        resid, resid_prev, resid0 = 1.0, 1.0, 1.0
        cfln = np.full(nfields, o.cfl0)
        niter = 0
        smoother, fs, scaled = None, None, None
        if o.smooth:                                         # :101-110
            smoother = preconditioner if o.smoother.lower() == "preconditioner" else api.create_preconditioner("jacobi")
            fs, scaled = api.ChidgVector(A), api.ChidgVector(A)
            if not o.ptc:
                print("WARNING: residual smoothing expects pseudo-transient continuation, but pseudo-transient "
                      "continuation was found to be turned off. Residual smoothing is being turned off for "
                      "consistency.", file=sys.stderr)
        while True:
            niter += 1
            qold.copy_from(q)
            # residual and linearisation (:140-146)
            t0 = time.perf_counter()
            system.assemble(q, A, rhs, differentiate=True)
            ph["assembly"] += time.perf_counter() - t0
            if niter == 1:
                resid0 = rhs.norm()
                cfln = np.full(nfields, o.cfl0)
            resid_prev, resid = resid, rhs.norm()
            b.copy_from(rhs)                                 # b = -rhs (:180)
            b.scale(-1.0)
            if o.smooth and o.ptc:                           # residual smoothing (:160-172, :360-441)
                t0 = time.perf_counter()
                smoother.update(A)                           # before the pseudo-transient term
                scaled.assign_mass_scaled(rhs, system.mass, self._ptc_scale(system, q, cfln, A))
                smoother.apply(A, scaled, fs)
                b.axpy(-o.smooth_relax, fs)                  # b = -rhs - smooth_relax * f_smooth
                ph["ptc"] += time.perf_counter() - t0
            if o.ptc:                                        # contribute_pseudo_temporal (:320-352)
                t0 = time.perf_counter()
                A.scale_diagonal(system.mass, self._ptc_scale(system, q, cfln, A))
                ph["ptc"] += time.perf_counter() - t0
            if niter == 1:
                res.residual_norm.append(resid)
            if resid < o.tol:
                res.converged = True
                break
            if math.isnan(resid):
                raise ArithmeticError("newton%solve: NaN residual norm. Check initial solution and operator objects.")
            dq.clear()
            t0 = time.perf_counter()
            linear_solver.solve(A, dq, b, preconditioner)
            res.linear_seconds.append(time.perf_counter() - t0)
            ph["linear"] += res.linear_seconds[-1]
            t0 = time.perf_counter()
            res.linear_rel_residual.append(linear_solver.residual_norm / max(linear_solver.r0norm_initial, 1e-300))
            # line search (:219-240, backtracking :466-549)
            f0 = resid
            if o.search.lower() == "backtrack":
                step = 0
                while True:
                    alpha = 2.0 ** (-step)
                    qn.copy_from(qold)
                    qn.axpy(alpha, dq)
                    q.copy_from(qn)
                    system.assemble(q, A, rhs, differentiate=False)
                    fn = rhs.norm()
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
                if alpha > 0.75:                             # cfl update (:533-545)
                    cfln = cfln * o.cfl_up
                elif alpha < 0.2:
                    cfln = cfln * o.cfl_down
                if o.cfl_max > 0.0:
                    cfln = np.minimum(cfln, o.cfl_max)
            else:
                alpha = 1.0
                qn.copy_from(qold)
                qn.axpy(1.0, dq)
                q.copy_from(qn)
                system.assemble(q, A, rhs, differentiate=False)
                fn = rhs.norm()
            q.copy_from(qn)
            ph["search"] += time.perf_counter() - t0
            res.matrix_iterations.append(linear_solver.niter)
            res.residual_norm.append(fn)
            res.alphas.append(alpha)
            res.cfl.append(float(cfln[0]))
            if not (fn > o.tol and fn / resid0 > o.rtol and (niter < o.nmax or o.nmax <= 0)):
                res.converged = fn <= o.tol or fn / resid0 <= o.rtol
                break
        res.niter = niter
        res.seconds = time.perf_counter() - t_start
        ph["other"] = res.seconds - sum(ph.values())
        res.phase_seconds = ph
        for v in (rhs, dq, b, qold, qn) + ((fs, scaled) if fs is not None else ()):
            v.release()
        if smoother is not None and smoother is not preconditioner:
            smoother.tear_down()
        return res

    @staticmethod
    def _ptc_scale(system, q, cfln, A):
        """1 / dtau per element and field, dtau the element's smallest pseudo
        time step over its fields (minval(elems(ielem)%dtau), :336-342)."""
        dtau = np.asarray(system.pseudo_timestep(q, cfln), dtype=np.float64)
        if dtau.ndim == 2:
            dtau = dtau.min(axis=1)
        return np.repeat(1.0 / dtau, A.pattern.elem_nvars)


class SyntheticSystem:
    """A nonlinear system with the ChiDG block layout and a known root q*, to
    exercise the Newton driver without a flow solver:
        R(q) = A0 (q - q*) + c (q - q*)**2     (element-wise square)
        dR/dq = A0 + 2 c diag(q - q*)
    A0 is a seeded synthetic Jacobian (mesh.synth_values); the mass matrix of
    every element is the identity and the pseudo time step is dtau = cfl.
    Assembly runs on the host from the downloaded state (small systems)."""

    def __init__(self, pattern, seed: int = 0, c: float = 0.2, root_seed: int = 1, root_scale: float = 0.3):
        from . import mesh
        self.pattern = pattern
        self.values0 = mesh.synth_values(pattern, seed=seed)
        self.c = float(c)
        self.qstar = root_scale * mesh.synth_vector(pattern.vector_size(), seed=root_seed)
        voff, _ = pattern.value_offsets()
        nr, _ = pattern.block_dims()
        eo = pattern.elem_offsets()
        b = pattern.bsize()
        diag = np.nonzero((pattern.blk_row_elem == pattern.blk_col_elem) & (pattern.blk_row_time == pattern.blk_col_time)
                          & (pattern.blk_kind == 0))[0]
        pos, idx = [], []
        for k in diag:
            e, t, n = int(pattern.blk_row_elem[k]), int(pattern.blk_row_time[k]), int(nr[k])
            pos.append(voff[k] + np.arange(n) * (n + 1))       # diagonal entries of the block
            idx.append(eo[e] + t * int(b[e]) + np.arange(n))    # their vector entries
        self._diag_pos = np.concatenate(pos)
        self._diag_idx = np.concatenate(idx)
        nterms = pattern.elem_nterms
        self.mass = np.concatenate([np.eye(int(m)).ravel(order="F") for m in nterms])
        self._A0 = None

    def _a0(self, A):
        if self._A0 is None:
            self._A0 = api.ChidgMatrix(self.pattern, A.ctx)
            self._A0.upload(self.values0)
        return self._A0

    def residual(self, qh: np.ndarray, A0q: np.ndarray) -> np.ndarray:
        d = qh - self.qstar
        return A0q + self.c * d * d

    def assemble(self, q, A, rhs, differentiate):
        A0 = self._a0(A)
        qh = q.download()
        d = api.ChidgVector(A0, qh - self.qstar)
        A0d = api.chidg_mv(A0, d).download()
        rhs.upload(A0d + self.c * (qh - self.qstar) ** 2)
        d.release()
        if differentiate:
            v = self.values0.copy()
            v[self._diag_pos] += 2.0 * self.c * (qh - self.qstar)[self._diag_idx]
            A.upload(v)

    def pseudo_timestep(self, q, cfl):
        return np.full(self.pattern.nelem, float(np.mean(cfl)))
