"""D2Q9 advection-diffusion-reaction BGK (Darcy pressure) on B200.

Drop-in for ``src/darcy.py``: ``AdvectionDiffusionReactionBGK`` keeps the
reference's keywords, hooks (``get_source``, ``set_boundary_conditions``,
``initialize_macroscopic_fields``, ``output_data``) and methods; its sweep is the
fused CUDA kernel ``xlbb_darcy_sweep`` and its gradient the stencil kernel
``xlbb_darcy_gradient``, both applying the compiled ADR boundary rules.

Extension beyond the reference: ``omega_field`` (keyword or attribute), a
per-cell relaxation rate ``omega(x) = 1 / (3 K(x) + 1/2)`` for heterogeneous
permeability.  With a uniform field the sweep is the reference's.
"""
import time

import numpy as np
import torch

from . import _lib
from ._common import gathered, iterate_to_tolerance, require_finite
from .base import LBMBase
from .bc_compile import compile_rules
from .boundary_conditions import BoundaryCondition, BounceBackHalfway, _at_add, _at_set, _take

GRADIENT_BC_NAMES = ("ADR_Neumann_BounceBack", "ADR_AntiBounceBack")


class AdvectionDiffusionReactionBGK(LBMBase):
    """``src/darcy.py:22-296``."""

    def __init__(self, **kwargs):
        if kwargs.get("nz", 0):
            raise NotImplementedError("the Darcy (advection-diffusion) path is two-dimensional (nz = 0)")
        super().__init__(**kwargs)
        self.vel = kwargs.get("vel", None)
        if self.vel is None:
            print("The advection is set to zero.")
        else:
            raise NotImplementedError("advection velocity is not on the Biot path")
        src = self.get_source()
        self.source = self._layout.field(src, 1) if src is not None else None
        om = kwargs.get("omega_field", None)
        self.omega_field = self._layout.field(om, 1) if om is not None else None
        self._partials = torch.empty(0, dtype=torch.float64, device=self._layout.device)
        self._n_partials = 0
        self._grad_rules_by_shape = {}

    def _compile_rules(self):
        L = self._layout
        self._pc = compile_rules(self.BCs, L.nx, L.ny, 9, self._rule_dtype, L.device, step="PostCollision")
        self._ps = compile_rules(self.BCs, L.nx, L.ny, 9, self._rule_dtype, L.device, step="PostStreaming")
        self._grad_rules = compile_rules(self.BCs, L.nx, L.ny, 9, self._dtype, L.device, names=GRADIENT_BC_NAMES)

    def gradient_rules(self, nx, ny, dtype=None):
        """Gradient rules on an ``nx x ny`` grid in ``dtype`` (default: this
        solver's); a coarse multigrid level uses the fine-level index sets,
        clamped/dropped like JAX does."""
        dtype = self._dtype if dtype is None else dtype
        if (nx, ny) == (self.nx, self.ny) and dtype == self._dtype:
            return self._grad_rules
        key = (nx, ny, dtype)
        if key not in self._grad_rules_by_shape:
            L = self._layout
            if (nx, ny) == (self.nx, self.ny):
                r = compile_rules(self.BCs, L.nx, L.ny, 9, dtype, L.device, names=GRADIENT_BC_NAMES)
            else:
                r = self._grad_rules.restricted(nx, ny, dtype, L.device)
            self._grad_rules_by_shape[key] = r
        return self._grad_rules_by_shape[key]

    # ------------------------------------------------------------------ kernels
    def update_macroscopic(self, f, external_source=None, gradient=False):
        """``src/darcy.py:36-73`` (kernel ``xlbb_darcy_moments``)."""
        L = self._layout
        f = L.field(f, 9)
        rho = L.empty(1)
        grad = L.empty(2) if gradient else None
        ext = L.field(external_source, 1)       # keep alive across the asynchronous launch
        _lib.check(_lib.lib().xlbb_darcy_moments(
            self._dcode, L.grid(), _lib.ptr(f), float(self.omega), _lib.ptr(self.omega_field),
            _lib.ptr(self.source), _lib.ptr(ext), _lib.ptr(rho), _lib.ptr(grad),
            _lib.stream_ptr()), "xlbb_darcy_moments")
        return (rho, grad) if gradient else rho

    def gradient(self, q, scale=1.0, out=None, base=None, dtype=None):
        """``src/darcy.py:75-104`` (kernel ``xlbb_darcy_gradient``); works on any
        multigrid level's grid.  ``base`` (optional) is added to the result.
        ``dtype`` (default: this solver's precision) is the precision of the
        computation and of the result."""
        from .fields import Layout
        nx, ny = int(q.shape[0]), int(q.shape[1])
        dtype = self._dtype if dtype is None else dtype
        L = self._layout if (nx, ny, dtype) == (self.nx, self.ny, self._dtype) else Layout(nx, ny, dtype)
        qf = L.field(q, 1)
        base = L.field(base, 2)     # other precision / layout -> this grid (kept alive over the launch)
        out = L.empty(2) if out is None else out
        rules = self.gradient_rules(nx, ny, dtype)
        _lib.check(_lib.lib().xlbb_darcy_gradient(
            _lib.dtype_code(dtype), L.grid(), _lib.ptr(qf), float(scale), rules.struct(), _lib.ptr(base),
            _lib.ptr(out), _lib.stream_ptr()), "xlbb_darcy_gradient")
        return out

    def collision(self, f, external_source=None):
        """``src/darcy.py:106-129``: the collision alone (API compatibility; the
        time loop uses the fused sweep).  Device tensor algebra."""
        L = self._layout
        f = L.field(f, 9)
        rho = self.update_macroscopic(f, external_source)
        om = self.omega_field if self.omega_field is not None else self.omega
        w = torch.as_tensor(self.w, device=L.device, dtype=L.dtype)
        fout = f - om * (f - rho * w)
        S = None
        if self.source is not None and external_source is not None:
            S = self.source + L.field(external_source, 1)
        elif self.source is not None:
            S = self.source
        elif external_source is not None:
            S = L.field(external_source, 1)
        if S is not None:
            fout = fout + S * ((1 - 0.5 * om) * w)
        return L.field(fout, 9)

    def streaming(self, f):
        out = torch.empty_like(f)
        for i in range(self.q):
            out[..., i] = torch.roll(f[..., i], (int(self.c[0, i]), int(self.c[1, i])), dims=(0, 1))
        return out

    def apply_bc(self, fout, fin, timestep, implementation_step):
        from .bc_compile import apply_rules_device
        return apply_rules_device(self._pc if implementation_step == "PostCollision" else self._ps, fout, fin)

    def _sweep(self, f, external_source=None, out=None, sumsq=False, resid=None, homogeneous=False):
        L = self._layout
        out = L.empty(9) if out is None else out
        if sumsq:
            # a buffer for the largest launch shape; the reduction reads the
            # partials of the launch this sweep takes
            n_max = _lib.check(_lib.lib().xlbb_darcy_sweep_ctas(self._sweep_code, L.grid()), "xlbb_darcy_sweep_ctas")
            if self._partials.numel() < n_max:
                self._partials = torch.empty(n_max, dtype=torch.float64, device=L.device)
        s = self._sweep_args(f, out, external_source, sumsq, resid, homogeneous)
        if sumsq:
            self._n_partials = _lib.check(_lib.lib().xlbb_darcy_sweep_partials(self._sweep_code, L.grid(), s),
                                          "xlbb_darcy_sweep_partials")
        _lib.check(_lib.lib().xlbb_darcy_sweep(self._sweep_code, L.grid(), s, _lib.stream_ptr()), "xlbb_darcy_sweep")
        return out

    def _sweep_args(self, f, out, external_source=None, sumsq=False, resid=None, homogeneous=False):
        """Kernel arguments; ``homogeneous``: the linear part of the sweep (no
        sources, boundary constants zero), ``resid``: collide f - resid."""
        pc, ps = self._homogeneous_rules() if homogeneous else (self._pc, self._ps)
        source = None if homogeneous else self.source
        ext = None if homogeneous else external_source
        return _lib.DarcySweep(f.data_ptr(), out.data_ptr(), float(self.omega),
                               self.omega_field.data_ptr() if self.omega_field is not None else None,
                               source.data_ptr() if source is not None else None,
                               ext.data_ptr() if ext is not None else None,
                               pc.struct(), ps.struct(), self._partials.data_ptr() if sumsq else None,
                               resid.data_ptr() if resid is not None else None)

    def _homogeneous_rules(self):
        if "_hom_rules" not in self.__dict__:
            from .refine import homogeneous_rules
            L = self._layout
            self._hom_rules = (homogeneous_rules(self._pc, L.ny, self._rule_dtype, L.device),
                               homogeneous_rules(self._ps, L.ny, self._rule_dtype, L.device))
        return self._hom_rules

    def sweep_pipeline(self, f=None, out=None):
        """The launch pipeline a sweep of this solver runs now (3: collide and
        push; 4: the same with four cells per lane and 16-byte accesses; 0-2:
        row-marching kernels), as the library resolves it."""
        L = self._layout
        f = L.empty(9) if f is None else f
        out = L.empty(9) if out is None else out
        return _lib.check(_lib.lib().xlbb_darcy_sweep_pipeline(self._sweep_code, L.grid(), self._sweep_args(f, out)),
                          "xlbb_darcy_sweep_pipeline")

    def step(self, f_poststreaming, timestep, return_fpost=False, external_source=None):
        """``src/darcy.py:131-171``: one fused sweep."""
        L = self._layout
        f = L.field(f_poststreaming, 9)
        ext = L.field(external_source, 1)
        out = self._sweep(f, ext)
        if return_fpost:
            return out, self.apply_bc(self.collision(f, ext), f, timestep, "PostCollision")
        return out, None

    def sweep_graph(self, n_sweeps, external_source=None):
        """A CUDA graph of ``n_sweeps`` fused sweeps (ping-pong between two owned
        buffers) whose last sweep also reduces the FP64 residual
        sum((f_new - f_old)^2).  Returns a ``SweepLoop``."""
        return SweepLoop(self, n_sweeps, external_source)

    def solve(self, f=None, tol=1e-8, check_every=1000, max_sweeps=10 ** 8, external_source=None,
              stall_checks=20, r0=None):
        """Pseudo-time iteration of the Darcy step (``src/darcy.py:131-171``) to
        steady state: until the relative residual ``||f^{n+1} - f^n|| /
        ||f^1 - f^0||`` (FP64 norms, reduced on the device) is below ``tol``.
        Sweeps run as one CUDA-graph replay of ``check_every`` sweeps between
        host checks; a residual that stops falling for ``stall_checks`` checks
        (the rounding floor of the storage precision) ends the loop with
        ``self.stalled = True``; a NaN or Inf residual raises
        ``NonFiniteError``.  ``r0``: the reference norm of the relative
        residual when continuing an earlier solve (default: this solve's
        first sweep).  Returns ``(f, sweeps, relative_residual)``."""
        L = self._layout
        f = self.assign_fields_sharded() if f is None else L.field(f, 9)
        loop = self._sweep_loop(check_every, external_source)
        first = loop.first(f)
        require_finite(first, "first sweep's residual norm", 1)
        r0 = first if r0 is None else float(r0)

        def replay():
            loop.replay()
            return loop.n, ((float(loop.sumsq[0]) ** 0.5) / r0 if r0 > 0 else 0.0)
        it, rel, self.stalled = iterate_to_tolerance(replay, tol, max_sweeps - 1, stall_checks)
        return loop.result, it + 1, rel

    def solve_refined(self, f=None, tol=1e-8, inner_tol=None, check_every=1000, max_sweeps=10 ** 8, max_outer=30,
                      stall_checks=20):
        """Steady state to an FP64 relative residual ``tol`` with the bulk of the
        sweeps in FP32 (mixed-precision iterative refinement, ``refine.py``):
        FP64 master state and defect sweeps, FP32 correction sweeps.  The
        solver must be FP32 ('f32/f32') without post-collision rules; an FP64
        twin of it (same class and keywords) computes the defects.  Returns
        ``(F, sweeps, relative_residual)`` with F the FP64 populations;
        ``self.refine_stats`` holds the outer/inner breakdown."""
        from .refine import CorrectionLoop, refine, twin64
        L = self._layout
        if L.dtype != torch.float32:
            raise _lib.XlbbError("solve_refined runs its bulk sweeps in FP32: use precision 'f32/f32'")
        if self._pc.count:
            raise NotImplementedError("solve_refined: post-collision rules are not supported")
        if "_twin" not in self.__dict__:
            self._twin = twin64(self)
        twin = self._twin
        F = twin.assign_fields_sharded() if f is None else twin._layout.field(f, 9).clone()
        key = ("refine", int(check_every))
        cache = self.__dict__.setdefault("_loops", {})
        if key not in cache:
            cache[key] = CorrectionLoop(self, check_every, 9, lambda a, b, sq, r: self._sweep(
                a, out=b, sumsq=sq, resid=r, homogeneous=True))
        loop = cache[key]
        G = twin._layout.empty(9)
        sc = torch.zeros(1, dtype=torch.float64, device=L.device)

        def defect(F):
            twin._sweep(F, out=G, sumsq=True)
            twin.residual_sumsq(sc)
            return F - G, float(sc[0]) ** 0.5
        F, stats = refine(defect, loop, F, tol, inner_tol, max_sweeps, max_outer, stall_checks,
                          lambda x: twin._layout.field(x, 9))
        self.refine_stats = stats
        return F, stats["sweeps_f32"] + stats["sweeps_f64"], stats["relative_residual"]

    def _sweep_loop(self, n, external_source):
        """The ``SweepLoop`` of ``n`` sweeps (rounded up to even, so that its
        result lands in its input buffer); without an external source it is
        captured once per solver and reused."""
        n = int(n) + (int(n) % 2)
        if external_source is not None:
            return SweepLoop(self, n, external_source)
        cache = self.__dict__.setdefault("_loops", {})
        if n not in cache:
            cache[n] = SweepLoop(self, n)
        return cache[n]

    def residual_sumsq(self, out_scalar):
        """FP64 sum of (f_new - f_old)^2 of the last sweep run with ``sumsq=True``
        (deterministic two-pass reduction), written into a device scalar."""
        _lib.check(_lib.lib().xlbb_reduce_sum(self._partials.data_ptr(), self._n_partials,
                                              out_scalar.data_ptr(), _lib.stream_ptr()), "xlbb_reduce_sum")
        return out_scalar

    def run(self, t_max):
        """``src/darcy.py:173-252``: t_max steps, output at step 0 and I/O steps."""
        f = self.assign_fields_sharded()
        start_step = 0
        if self.restore_checkpoint:
            ck = self.load_latest_checkpoint()
            if ck is not None:
                start_step = int(ck["timestep"])
                f = self._layout.field(ck["f"], 9)
                print(f"Restored checkpoint at step {start_step}.")
        start = time.time()
        if self.ioRate > 0 and start_step % self.ioRate == 0:
            self.handle_io_timestep(start_step, f, None, gathered(self.update_macroscopic(f)), None)
        for timestep in range(start_step + 1, t_max + 1):
            io_flag = self.ioRate > 0 and (timestep % self.ioRate == 0 or timestep == t_max)
            print_iter_flag = self.printInfoRate > 0 and timestep % self.printInfoRate == 0
            checkpoint_flag = self.checkpointRate > 0 and timestep % self.checkpointRate == 0
            if io_flag:
                rho_prev = gathered(self.update_macroscopic(f))
            f, fstar = self.step(f, timestep, return_fpost=self.returnFpost)
            if print_iter_flag:
                print(f"Timestep {timestep} of {t_max} completed")
            if io_flag:
                self.handle_io_timestep(timestep, f, fstar, gathered(self.update_macroscopic(f)), rho_prev)
            if checkpoint_flag:
                self.save_checkpoint(timestep, f)
            if self.computeMLUPS and timestep == 1:
                torch.cuda.synchronize()
                start = time.time()
        if self.computeMLUPS:
            torch.cuda.synchronize()
            end = time.time()
            print(f"Domain: {self.nx} x {self.ny}")
            print(f"Number of voxels: {self.nx * self.ny}")
            print(f"MLUPS: {self.nx * self.ny * t_max / (end - start) / 1e6}")
        return f

    def handle_io_timestep(self, timestep, f, fstar, rho, rho_prev):
        self.output_data(timestep=timestep, rho=rho, rho_prev=rho_prev, f_poststreaming=f, f_postcollision=fstar)

    def get_source(self):
        pass


class ADR_AntiBounceBack(BoundaryCondition):
    """``src/darcy.py:298-392``: halfway anti-bounce-back (Dirichlet ``rho``)."""

    def __init__(self, indices, gridInfo, precision_policy, rho=None):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ADR_AntiBounceBack"
        self.implementationStep = "PostStreaming"
        self.needsExtraConfiguration = True
        self.isSolid = True
        self.rho = rho

    def configure(self, boundaryMask):
        nbd_orig = len(self.indices[0])
        first = self._halfway_index_shift(boundaryMask)
        nbd = len(self.indices[0])
        if nbd_orig != nbd and self.rho is not None:
            if isinstance(self.rho, float) or np.asarray(self.rho).size == 1:
                self.rho = np.full((nbd, 1), float(np.asarray(self.rho).reshape(-1)[0]))
            else:
                print("WARNING: Assuming a correct macroscopic (density) vector to impose at the BC cells!")
                self.rho = np.asarray(self.rho)[first]

    def impose_boundary_rho(self, fbd, bindex):
        tmp = np.broadcast_to(2 * self.lattice.w.astype(np.float64) * np.asarray(self.rho, dtype=np.float64),
                              (len(self.indices[0]), self.lattice.q))
        return _at_add(fbd, (bindex, self.imissing), tmp[bindex, self.iknown])

    def apply(self, fout, fin):
        nbd = len(self.indices[0])
        bindex = np.arange(nbd)[:, None]
        fbd = np.array(_take(fout, self.indices))
        _at_set(fbd, (bindex, self.imissing), -_take(fin, self.indices)[bindex, self.iknown])
        if self.rho is not None:
            fbd = self.impose_boundary_rho(fbd, bindex)
        return fbd


class ADR_Neumann_BounceBack(BounceBackHalfway):
    """``src/darcy.py:394-415``."""

    def __init__(self, indices, gridInfo, precision_policy):
        super().__init__(indices, gridInfo, precision_policy)
        self.name = "ADR_Neumann_BounceBack"


class ADR_EquilibriumBC(BoundaryCondition):
    """``src/darcy.py:417-466``."""

    def __init__(self, indices, gridInfo, precision_policy, rho, vel=None):
        super().__init__(indices, gridInfo, precision_policy)
        if vel is None:
            self.out = np.asarray(rho, dtype=np.float64) * self.lattice.w.astype(np.float64)
        else:
            self.out = self.equilibrium(rho, vel)
        self.name = "ADR_EquilibriumBC"
        self.implementationStep = "PostStreaming"

    def apply(self, fout, fin):
        return self.out


class SweepLoop:
    """``n`` Darcy sweeps captured once as a CUDA graph (the pseudo-time loop of
    ``run`` without host round trips).  ``state`` holds the input populations;
    ``replay()`` leaves the result in ``result`` and the FP64 residual
    sum((f_n - f_{n-1})^2) of the last sweep in ``sumsq`` (device scalar)."""

    def __init__(self, solver, n, external_source=None):
        L = solver._layout
        self.solver, self.n = solver, int(n)
        self.state = L.empty(9)
        self._other = L.empty(9)
        self.sumsq = torch.zeros(1, dtype=torch.float64, device=L.device)
        self.ext = L.field(external_source, 1)
        self.launches_per_replay = self.n + 1
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):           # warm-up outside capture (lazy module loading)
            self._body()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._body()
        self.result = self.state if self.n % 2 == 0 else self._other

    def _body(self):
        a, b = self.state, self._other
        for k in range(self.n):
            self.solver._sweep(a, self.ext, out=b, sumsq=(k == self.n - 1))
            a, b = b, a
        self.solver.residual_sumsq(self.sumsq)

    def first(self, f0):
        """One sweep from ``f0`` into ``state``; returns ||f^1 - f^0|| (FP64)."""
        self.solver._sweep(self.solver._layout.field(f0, 9), self.ext, out=self.state, sumsq=True)
        self.solver.residual_sumsq(self.sumsq)
        return float(self.sumsq[0]) ** 0.5

    def replay(self):
        self.graph.replay()
        return self.result
