"""Mixed-precision iterative refinement of pseudo-time steady states.

FP32 storage cannot represent a state whose pseudo-time residual
``||f^{n+1} - f^n|| / ||f^1 - f^0||`` is far below the FP32 rounding of the
populations: a plain FP32 solve stalls (1e-5 .. 1e-7 on the elasticity and
Darcy workloads) at a state that can be 1e-3 away from the FP64 solution.  The
refinement keeps an FP64 master state F and runs the bulk of the sweeps in
FP32 on the correction:

* defect, one FP64 sweep: ``D = F - S(F)``, with ``||D||`` the FP64 residual
  norm that decides convergence (the same quantity as the plain solve's
  ``||f^{n+1} - f^n||``);
* correction, FP32 sweeps: the steady state is ``F + e`` with ``e = A e - D``
  (``S(f) = A f + b``, A the homogeneous sweep: no force or source, boundary
  constants zero).  With ``u = e + D`` this is ``u = A (u - D)``, i.e. the
  fused sweep with its residual input set to D (``resid`` of
  ``xlbb_elast_sweep`` / ``xlbb_darcy_sweep``), iterated from u = 0 as a CUDA
  graph until its own pseudo-time residual has fallen as far as the
  remaining defect needs (the first correction: to its FP32 rounding floor,
  where it stalls);
* update in FP64: ``F <- F + u - D``.

Every outer step gains the accuracy an FP32 solve reaches on the correction,
so a few FP64 sweeps (one per outer step) and FP32 sweeps in the bulk reach
the FP64 tolerance.  The correction's convergence rate is the plain
iteration's: the sweep count is about that of the all-FP64 solve, at the FP32
sweep's cost.
"""
import numpy as np
import torch

from . import _lib
from ._common import iterate_to_tolerance, require_finite
from .bc_compile import CompiledRules


def homogeneous_rules(rules, ny, dtype, device):
    """The same rule cells and codes with every constant zero (the boundary
    data belong to the affine part b of the sweep, not to the correction)."""
    if rules.count == 0:
        return rules
    return CompiledRules(rules.q, ny, rules.cells, rules.code_np, np.zeros_like(rules.cst_np), dtype, device,
                         rules.nx, push=True, shape=rules.shape, cells_nd=rules.cells_nd)


def twin64(solver):
    """The same problem in FP64 (storage and arithmetic): the solver's class
    built again from its constructor keywords with an FP64 lattice."""
    kw = dict(solver._init_kwargs)
    kw["precision"] = "f64/f64"
    lat = kw.get("lattice")
    if lat is not None:
        kw["lattice"] = type(lat)("f64/f64")
    kw["print_info_rate"] = 0
    return type(solver)(**kw)


class CorrectionLoop:
    """FP32 sweeps of the correction equation ``u = A (u - r)`` captured once as
    a CUDA graph of ``n`` sweeps (n even); ``r`` is an owned FP32 buffer that
    the caller fills before every solve."""

    def __init__(self, solver, n, q, sweep):
        L = solver._L(0) if hasattr(solver, "_L") else solver._layout
        self.n = int(n) + (int(n) % 2)
        self.u, self.v, self.r = L.empty(q), L.empty(q), L.empty(q)
        self.sumsq = torch.zeros(1, dtype=torch.float64, device=L.device)
        self._sweep = sweep            # sweep(src, dst, sumsq, r) issuing one fused correction sweep
        self._reduce = solver._reduce_partials if hasattr(solver, "_reduce_partials") else solver.residual_sumsq
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self._body()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()

    def _body(self):
        a, b = self.u, self.v
        for k in range(self.n):
            self._sweep(a, b, k == self.n - 1, self.r)
            a, b = b, a
        self._reduce(self.sumsq)

    def solve(self, inner_tol, max_sweeps, stall_checks):
        """From u = 0 until ||u_{k+1} - u_k|| / ||u_1|| < inner_tol; returns
        (sweeps, relative residual, stalled); the correction is left in ``u``."""
        self.u.zero_()
        self._sweep(self.u, self.v, True, self.r)
        self._reduce(self.sumsq)
        first = float(self.sumsq[0]) ** 0.5
        require_finite(first, "first correction sweep's residual norm", 1)
        self.u.copy_(self.v)
        if first == 0.0:
            return 1, 0.0, False

        def replay():
            self.graph.replay()
            return self.n, (float(self.sumsq[0]) ** 0.5) / first
        it, rel, stalled = iterate_to_tolerance(replay, inner_tol, max_sweeps - 1, stall_checks,
                                                what="relative residual of the correction")
        return it + 1, rel, stalled


def refine(defect, loop, F, tol, inner_tol, max_sweeps, max_outer, stall_checks, relayout):
    """The outer loop.  ``defect(F)`` returns (D, ||D||) in FP64;
    ``relayout(x)`` puts an FP64 field into the kernels' layout.  Returns
    (F, statistics); F is the FP64 state after the last defect's sweep."""
    stats = {"outer": 0, "sweeps_f64": 0, "sweeps_f32": 0, "inner": []}
    F = relayout(F)
    d0 = None
    while True:
        D, dn = defect(F)
        stats["sweeps_f64"] += 1
        require_finite(dn, "FP64 defect norm", stats["sweeps_f64"])
        d0 = dn if d0 is None else d0
        rel = dn / d0 if d0 > 0 else 0.0
        stats["relative_residual"] = rel
        if rel < tol or stats["outer"] >= max_outer:
            return F - D, stats          # S(F): the sweep that measured the last defect
        loop.r.copy_(D)
        # the correction must take the defect below tol (with a factor 10 to
        # spare): the first outer step runs to the FP32 rounding floor, the
        # later ones only as far as the remaining defect needs
        target = min(0.5, 0.1 * tol * d0 / dn) if dn > 0 else 0.5
        if inner_tol is not None:
            target = max(target, inner_tol)
        n, irel, stalled = loop.solve(target, max_sweeps, stall_checks)
        stats["sweeps_f32"] += n
        stats["inner"].append({"sweeps": n, "relative_residual": irel, "stalled": stalled,
                               "defect_relative": rel})
        F = relayout(F + (loop.u.to(torch.float64) - D))
        stats["outer"] += 1
