"""Fluid collision models (``src/models.py``) on B200.

``BGKSim`` and ``KBCSim`` keep the reference's keywords, hooks
(``set_boundary_conditions``, ``initialize_macroscopic_fields``,
``output_data``) and ``run``/``step`` loop (``src/base.py:809-948``); their step
is one launch of a fused CUDA sweep (collision, compiled PostCollision rules,
periodic streaming, compiled PostStreaming rules): ``xlbb_fluid_sweep`` on
D2Q9 (BGK and KBC; the path of ``examples/performance/MLUPS2d.py``) and
``xlbb_fluid3_sweep`` on D3Q19 / D3Q27 (BGK, the path of ``MLUPS3d.py``;
KBC on D3Q27), both with the lid-driven cavity's ``BounceBack`` and
``EquilibriumBC``.

Scope: no body force (``get_force`` must return None).
"""
import time

import numpy as np
import torch

from . import _lib
from ._common import gathered
from .base import LBMBase
from .bc_compile import apply_rules_device, compile_rules

FLUID_BGK, FLUID_KBC = 0, 1


class _FluidSim(LBMBase):
    _model = FLUID_BGK

    def __init__(self, **kwargs):
        super().__init__(**kwargs)
        if self._acc64:
            raise NotImplementedError("the fluid models compute in their storage type: use 'f32/f32' or 'f64/f64'")
        if (self.lattice.d, self.lattice.q) not in ((2, 9), (3, 19), (3, 27)):
            raise NotImplementedError("the fluid models run on the D2Q9, D3Q19 and D3Q27 lattices")
        if self.force is not None:
            raise NotImplementedError("body forces (apply_force) are not implemented for the fluid models")
        self._partials = torch.empty(0, dtype=torch.float64, device=self._layout.device)
        self._n_partials = 0

    def _compile_rules(self):
        L = self._layout
        self._pc = compile_rules(self.BCs, L.nx, L.ny, self.q, self._dtype, L.device, step="PostCollision", nz=L.nz)
        self._ps = compile_rules(self.BCs, L.nx, L.ny, self.q, self._dtype, L.device, step="PostStreaming", nz=L.nz)
        if L.nz and self._ps.count and self._ps.push is None:
            raise NotImplementedError("the 3-D fluid sweep applies PostStreaming rules that rebuild populations "
                                      "from the cell's own post-collision values (no negated or shifted "
                                      "streamed values)")

    # ------------------------------------------------------------------ kernels
    def update_macroscopic(self, f):
        """``src/base.py:748-772``: rho = sum f, u = sum c f / rho (device
        tensor algebra)."""
        L = self._layout
        f = L.field(f, self.q)
        c = torch.as_tensor(self.c, device=L.device, dtype=L.dtype)
        rho = torch.sum(f, dim=-1, keepdim=True)
        return rho, (f @ c.T) / rho

    def streaming(self, f):
        out = torch.empty_like(f)
        for i in range(self.q):
            out[..., i] = torch.roll(f[..., i], tuple(int(self.c[k, i]) for k in range(self.dim)),
                                     dims=tuple(range(self.dim)))
        return out

    def apply_bc(self, fout, fin, timestep, implementation_step):
        return apply_rules_device(self._pc if implementation_step == "PostCollision" else self._ps, fout, fin)

    def _sweep(self, f, out=None, sumsq=False):
        L = self._layout
        out = L.empty(self.q) if out is None else out
        if L.nz:
            if sumsq:
                raise NotImplementedError("the 3-D fluid sweep has no fused residual sum")
            s = _lib.DarcySweep(f.data_ptr(), out.data_ptr(), float(self.omega), None, None, None,
                                self._pc.struct(), self._ps.struct(), None)
            _lib.check(_lib.lib().xlbb_fluid3_sweep(self._dcode, L.grid3(), s, self.q, self._model,
                                                    _lib.stream_ptr()),
                       "xlbb_fluid3_sweep")
            return out
        if sumsq:
            n_max = _lib.check(_lib.lib().xlbb_darcy_sweep_ctas(self._dcode, L.grid()), "xlbb_darcy_sweep_ctas")
            if self._partials.numel() < n_max:
                self._partials = torch.empty(n_max, dtype=torch.float64, device=L.device)
        s = _lib.DarcySweep(f.data_ptr(), out.data_ptr(), float(self.omega), None, None, None,
                            self._pc.struct(), self._ps.struct(), self._partials.data_ptr() if sumsq else None)
        if sumsq:
            self._n_partials = _lib.check(_lib.lib().xlbb_darcy_sweep_partials(self._dcode, L.grid(), s),
                                          "xlbb_darcy_sweep_partials")
        _lib.check(_lib.lib().xlbb_fluid_sweep(self._dcode, L.grid(), s, self._model, _lib.stream_ptr()),
                   "xlbb_fluid_sweep")
        return out

    def residual_sumsq(self, out_scalar):
        """FP64 sum of (f_new - f_old)^2 of the last sweep run with ``sumsq=True``."""
        _lib.check(_lib.lib().xlbb_reduce_sum(self._partials.data_ptr(), self._n_partials,
                                              out_scalar.data_ptr(), _lib.stream_ptr()), "xlbb_reduce_sum")
        return out_scalar

    def step(self, f_poststreaming, timestep, return_fpost=False):
        """``src/base.py:809-846``: one fused sweep; with ``return_fpost`` the
        post-collision populations (after the PostCollision rules) as well."""
        f = self._layout.field(f_poststreaming, self.q)
        out = self._sweep(f)
        if return_fpost:
            return out, self.apply_bc(self.collision(f), f, timestep, "PostCollision")
        return out, None

    def run(self, t_max):
        """``src/base.py:848-948``: t_max + 1 steps (0 .. t_max), I/O,
        checkpoints and the MLUPS report of the reference."""
        f = self.assign_fields_sharded()
        start_step = 0
        if self.restore_checkpoint:
            ck = self.load_latest_checkpoint()
            if ck is not None:
                latest = int(ck["timestep"])
                f = self._layout.field(ck["f"], self.q)
                print(f"Restored checkpoint at step {latest}.")
                start_step = latest + 1
                if not (t_max > start_step):
                    raise ValueError(f"Simulation already exceeded maximum allowable steps (t_max = {t_max}). "
                                     "Consider increasing t_max.")
        start = time.time()
        for timestep in range(start_step, t_max + 1):
            io_flag = self.ioRate > 0 and (timestep % self.ioRate == 0 or timestep == t_max)
            print_iter_flag = self.printInfoRate > 0 and timestep % self.printInfoRate == 0
            checkpoint_flag = self.checkpointRate > 0 and timestep % self.checkpointRate == 0
            if io_flag:
                rho_prev, u_prev = (gathered(x) for x in self.update_macroscopic(f))
            f, fstar = self.step(f, timestep, return_fpost=self.returnFpost)
            if print_iter_flag:
                print(f"Timestep {timestep} of {t_max} completed")
            if io_flag:
                rho, u = (gathered(x) for x in self.update_macroscopic(f))
                self.handle_io_timestep(timestep, f, fstar, rho, u, rho_prev, u_prev)
            if checkpoint_flag:
                self.save_checkpoint(timestep, f)
            if self.computeMLUPS and timestep == 1:
                torch.cuda.synchronize()
                start = time.time()
        if self.computeMLUPS:
            torch.cuda.synchronize()
            end = time.time()
            cells = self.nx * self.ny * (self.nz if self.dim == 3 else 1)
            print("Domain: " + " x ".join(str(n) for n in (self.nx, self.ny, self.nz)[:self.dim]))
            print(f"Number of voxels: {cells}")
            print(f"MLUPS: {cells * t_max / (end - start) / 1e6}")
        return f

    def handle_io_timestep(self, timestep, f, fstar, rho, u, rho_prev, u_prev):
        """``src/base.py:951-980``."""
        self.output_data(timestep=timestep, rho=rho, rho_prev=rho_prev, u=u, u_prev=u_prev,
                         f_poststreaming=f, f_postcollision=fstar)


class BGKSim(_FluidSim):
    """``src/models.py:9-34``: f* = f - omega (f - feq)."""
    _model = FLUID_BGK

    def collision(self, f):
        """The collision alone (API compatibility; the time loop uses the fused
        sweep).  Device tensor algebra."""
        L = self._layout
        f = L.field(f, self.q)
        rho, u = self.update_macroscopic(f)
        feq = self.equilibrium(rho, u, cast_output=False)
        return L.field(f - self.omega * (f - feq), self.q)


class KBCSim(_FluidSim):
    """``src/models.py:36-72``: the entropic KBC collision (shear
    decompositions ``fdecompose_shear_d2q9``, ``:127-154``, and
    ``fdecompose_shear_d3q27``, ``:156-214``)."""
    _model = FLUID_KBC

    def __init__(self, **kwargs):
        if kwargs.get('lattice').name != 'D3Q27' and (kwargs.get('nz') or 0) > 0:
            raise ValueError("KBC collision operator in 3D must only be used with D3Q27 lattice.")
        super().__init__(**kwargs)

    def fdecompose_shear_d2q9(self, fneq):
        c = torch.as_tensor(np.asarray(self.c, dtype=np.float64), device=fneq.device, dtype=fneq.dtype)
        cc = torch.stack([c[0] * c[0], c[0] * c[1], c[1] * c[1]], dim=1)
        Pi = fneq @ cc
        N = Pi[..., 0] - Pi[..., 2]
        s = torch.zeros_like(fneq)
        for i, v in ((6, N), (3, N), (2, -N), (1, -N), (8, Pi[..., 1]), (4, -Pi[..., 1]),
                     (5, -Pi[..., 1]), (7, Pi[..., 1])):
            s[..., i] = v
        return s

    def momentum_flux(self, fneq):
        """``src/base.py:727-746``: fneq . cc (cc: c_a c_b, a <= b)."""
        return fneq @ torch.as_tensor(np.asarray(self.lattice.cc, dtype=np.float64), device=fneq.device,
                                      dtype=fneq.dtype)

    def fdecompose_shear_d3q27(self, fneq):
        Pi = self.momentum_flux(fneq)
        nxz = Pi[..., 0] - Pi[..., 5]
        nyz = Pi[..., 3] - Pi[..., 5]
        s = torch.zeros_like(fneq)
        for i, v in ((9, (2.0 * nxz - nyz) / 6.0), (18, (2.0 * nxz - nyz) / 6.0),
                     (3, (-nxz + 2.0 * nyz) / 6.0), (6, (-nxz + 2.0 * nyz) / 6.0),
                     (1, (-nxz - nyz) / 6.0), (2, (-nxz - nyz) / 6.0)):
            s[..., i] = v
        for i, j, k in ((12, 24, 1), (10, 20, 2), (8, 4, 4)):
            s[..., i] = s[..., j] = Pi[..., k] / 4.0
        for i, j, k in ((21, 15, 1), (19, 11, 2), (7, 5, 4)):
            s[..., i] = s[..., j] = -Pi[..., k] / 4.0
        return s

    def collision(self, f):
        """The collision alone (API compatibility).  Device tensor algebra."""
        L = self._layout
        f = L.field(f, self.q)
        rho, u = self.update_macroscopic(f)
        feq = self.equilibrium(rho, u, cast_output=False)
        fneq = f - feq
        if self.dim == 2:
            dS = self.fdecompose_shear_d2q9(fneq) * rho / 4.0
        else:
            dS = self.fdecompose_shear_d3q27(fneq) * rho
        dH = fneq - dS
        beta = self.omega * 0.5
        ib = 1.0 / beta
        gamma = ib - (2.0 - ib) * torch.sum(dS * dH / feq, -1) / (1e-32 + torch.sum(dH * dH / feq, -1))
        return L.field(f - beta * (2.0 * dS + gamma[..., None] * dH), self.q)
