"""Gradients of a consolidation misfit with respect to per-cell material.

No counterpart in the reference (which has no adjoint).  ``BiotAdjointModel``
runs the Biot time loop of an ``LBMPoroelasticity`` (fixed V-cycle count per
step, no per-step host hooks) forward, keeps the state every
``checkpoint_every`` steps, and computes the discrete adjoint of

    J = 1/2 sum (eta_N - eta_obs)^2 + 1/2 sum (p_N - p_obs)^2

(displacement and pressure of the last step, over all cells) with respect to
the per-cell Lame fields of every multigrid level and the Darcy relaxation
field omega.  The backward pass recomputes each checkpoint segment with a tape
of every sweep's inputs and then runs the hand-written transposed kernels
(``xlb_biot_b200.adjoint``) in reverse order.  ``ConsolidationMisfit`` wraps
it as a ``torch.autograd.Function`` of the level-0 fields (lambda, mu, omega);
the coarse-level material is ``material_hierarchy`` of the level-0 fields, so
torch's autograd carries the per-level gradients back to level 0 and to any
parameterisation the caller builds (log-permeability, log-shear-modulus).

The initial state is taken as given (the consolidation workloads start from
zero populations, which do not depend on the material).
"""
import time

import torch

from .adjoint import (ElastGrads, add_, darcy_moments_adjoint, darcy_sweep_adjoint, divgrad_adjoint,
                      elast_moments_adjoint, elast_sweep_adjoint, f64_plane, gradient_adjoint)
from .elasticity import material_hierarchy


class BiotAdjointModel:
    """Forward / adjoint driver of ``steps`` coupled Biot steps of ``sim``."""

    def __init__(self, sim, steps, checkpoint_every=16, graphs=False):
        if sim.useDynamicForce or sim.useDynamicSource:
            raise ValueError("per-step force / source hooks are not supported by the adjoint")
        if sim.elasticityTol is not None or sim.alternative_gradient:
            raise ValueError("the adjoint needs a fixed V-cycle count and the default gradient form")
        self.sim, self.el, self.da = sim, sim.elasticity, sim.darcy
        if self.el._lam_fields is None:
            raise ValueError("the adjoint differentiates per-cell material: give lambda_field / mu_field")
        if self.da.omega_field is None:
            raise ValueError("the adjoint differentiates per-cell permeability: give omega_field")
        self.steps, self.every = int(steps), int(checkpoint_every)
        th, a = sim.couplingRatio, sim.alpha
        self.sN = 0.5 * th * a ** 2
        self.grads = ElastGrads(self.el)
        self.g_omega = f64_plane(self.da._layout)
        self.eta_obs = self.p_obs = None
        self.timing = {}
        # ``graphs``: the plain step, and per checkpoint slot the taping step and
        # its adjoint, run as CUDA graphs (captured on first use) over static
        # state buffers; results are identical to the eager path.
        self.graphs = bool(graphs)
        self._fwd_graph = None
        self._bwd_graphs = None

    # ------------------------------------------------------------------ parameters
    def set_parameters(self, lam0, mu0, omega):
        """Level-0 material (all (nx, ny)); coarse levels follow by coarsening."""
        self.el.set_material_fields(lam0, mu0)
        self.da.omega_field.copy_(torch.as_tensor(omega, device=self.da.omega_field.device).reshape(
            self.da.nx, self.da.ny, 1))

    def set_observations(self, eta_obs, p_obs):
        self.eta_obs = self.el._L().field(eta_obs, 2)
        self.p_obs = self.da._layout.field(p_obs, 1)

    # ------------------------------------------------------------------ forward
    def _N(self, f, level, fe):
        return self.el.coupling_force(f, level, self.da, self.sN, base=fe)

    def _vcycle(self, f, level, resid, fe, rec):
        """``LBMElasticity._mg_step`` with the coupling force N(f); appends the
        inputs of every sweep to ``rec`` (the prolongation goes into a copy so
        that the taped residual-sweep input stays intact)."""
        el, g = self.el, self.el.gamma
        for _ in range(el.k_smooth):
            ext = self._N(f, level, fe)
            out = el._sweep(f, level, 1.0 - g, g, resid=resid, fext=ext)
            rec.append(("s", level, f, resid, ext))
            f = out
        if level < el.levels - 1:
            ext = self._N(f, level, fe)
            res = el._sweep(f, level, 1.0, -1.0, resid=resid, fext=ext, acc64=(level == 0 and el._res64))
            rec.append(("r", level, f, resid, ext))
            rc = el._restrict_full(res, level)
            sub = []
            fc = self._vcycle(el._L(level + 1).zeros(8), level + 1, rc, None, sub)
            rec.append(("c", level, rc, sub))
            f = f.clone()
            el._prolong_add(fc, f, level)
        for _ in range(el.k_smooth):
            ext = self._N(f, level, fe)
            out = el._sweep(f, level, 1.0 - g, g, resid=resid, fext=ext)
            rec.append(("s", level, f, resid, ext))
            f = out
        return f

    def step(self, fe, fd, dtd, tape=None):
        """One coupled step (``LBMPoroelasticity.step``, ``src/poroelasticity.py:303-339``).
        Returns (fe, fd, dtd, eta, pressure); ``tape`` (a dict) receives the
        inputs the adjoint needs."""
        sim, el, da = self.sim, self.el, self.da
        th, a, eps = sim.couplingRatio, sim.alpha, sim.epsilon
        fe = el._f(fe)
        fd = da._layout.field(fd, 9)
        dtd = da._layout.field(dtd, 1)
        sb = da._layout.field(((1.0 - th) * -a / eps) * dtd, 1)
        _, pgb = da.update_macroscopic(fd, gradient=True)
        pgbase = da.gradient(sb, 0.5, base=pgb)
        force = el._L().field((-a * eps) * pgbase - da.gradient(el.update_divergence(fe), self.sN), 2)
        f, cycles = fe, []
        for _ in range(sim.elasticitySteps):
            rec = []
            f = self._vcycle(f, 0, None, force, rec)
            cycles.append(rec)
        eta, _ = el.update_macroscopic(f, self._N(f, 0, force))
        diff = el._f(f - fe)
        dtd_new = el.update_divergence(diff, 0)
        source = da._layout.field(sb - (th * a / eps) * dtd_new, 1)
        pressure = da.update_macroscopic(fd, source)
        fd_new = da._sweep(fd, source)
        if tape is not None:
            tape.update(fe=fe, fd=fd, force=force, cycles=cycles, f=f, diff=diff, source=source)
        return f, fd_new, dtd_new, eta, pressure

    # ------------------------------------------------------------------ CUDA graphs
    def _state_buffers(self):
        return self.el._L().empty(8), self.da._layout.empty(9), self.da._layout.empty(1)

    @staticmethod
    def _warm(fn):
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            fn()
        torch.cuda.current_stream().wait_stream(side)

    @staticmethod
    def _load(bufs, vals):
        for b, v in zip(bufs, vals):
            b.copy_(v)

    def _build_forward_graph(self):
        S = self._state_buffers()
        self._load(S, self.sim.init_state())
        self._warm(lambda: self.step(*S))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            out = self.step(*S)
            self._load(S, out[:3])
        self._fwd_graph = (g, S, out[3], out[4])

    def _build_backward_graphs(self):
        el, da = self.el, self.da
        n = min(self.every, self.steps)
        ins = [self._state_buffers() for _ in range(n + 1)]
        lam = (el._L().zeros(8), da._layout.zeros(9), da._layout.zeros(1))
        src = (el._L().zeros(2), da._layout.zeros(1))
        for b in ins:
            self._load(b, self.sim.init_state())

        def warm():
            tp = {}
            self.step(*ins[0], tape=tp)
            self.step_adjoint(tp, *lam, *src)
        self._warm(warm)
        self.grads.zero_()
        self.g_omega.zero_()
        tapes, steps_g, adj_g = [], [], []
        for j in range(n):
            g = torch.cuda.CUDAGraph()
            tp = {}
            with torch.cuda.graph(g):
                out = self.step(*ins[j], tape=tp)
                self._load(ins[j + 1], out[:3])
            tapes.append(tp)
            steps_g.append(g)
            a = torch.cuda.CUDAGraph()
            with torch.cuda.graph(a):
                out = self.step_adjoint(tp, *lam, *src)
                self._load(lam, out)
            adj_g.append(a)
        self._bwd_graphs = dict(ins=ins, lam=lam, src=src, tapes=tapes, steps=steps_g, adj=adj_g)

    def forward(self):
        """Runs the time loop from ``sim.init_state()``; keeps checkpoints;
        returns J (float) when observations are set, else None."""
        if self.graphs and self._fwd_graph is None:
            self._build_forward_graph()
        t0 = time.time()
        self.checkpoints = {}
        eta = p = None
        if self.graphs:
            g, S, eta_s, p_s = self._fwd_graph
            self._load(S, self.sim.init_state())
            for k in range(self.steps):
                if k % self.every == 0:
                    self.checkpoints[k] = tuple(t.clone() for t in S)
                g.replay()
            eta, p = eta_s, p_s
        else:
            fe, fd, dtd = self.sim.init_state()
            for k in range(self.steps):
                if k % self.every == 0:
                    self.checkpoints[k] = (fe.clone(), fd.clone(), dtd.clone())
                fe, fd, dtd, eta, p = self.step(fe, fd, dtd)
        self.eta, self.p = eta, p
        J = None
        if self.eta_obs is not None:
            de = (eta.double() - self.eta_obs.double())
            dp = (p.double() - self.p_obs.double())
            J = 0.5 * float((de * de).sum() + (dp * dp).sum())
        torch.cuda.synchronize()
        self.timing["forward_s"] = time.time() - t0
        return J

    # ------------------------------------------------------------------ adjoint
    def _N_adj(self, lam_ext, f, level, lam_f, lam_fe):
        """Transpose of ext = fe + G(div_level(f), sN): lam_fe += lam_ext (if
        given), lam_f += div^T G^T lam_ext, material gradient of div."""
        divgrad_adjoint(self.el, self.da, level, lam_ext, self.sN, lam_f, lam_fe=lam_fe, f=f, grads=self.grads)

    def _vcycle_adj(self, lam, rec, lam_resid, lam_fe):
        el, g = self.el, self.el.gamma
        lam_res = None
        for item in reversed(rec):
            if item[0] == "s":
                _, lv, f, r, ext = item
                lam_f, lam_ext = elast_sweep_adjoint(el, lv, lam, 1.0 - g, g, f_in=f, resid=r, fext=ext,
                                                     lam_resid=lam_resid, want_force=True, grads=self.grads)
                self._N_adj(lam_ext, f, lv, lam_f, lam_fe)
                lam = lam_f
            elif item[0] == "c":      # f_out = f + P(fc): lam_fc = P^T lam = block sums
                _, lv, rc, sub = item
                lam_fc = el._restrict_full(lam, lv)
                lam_rc = el._L(lv + 1).zeros(8)
                self._vcycle_adj(lam_fc, sub, lam_rc, None)
                lam_res = el._L(lv).zeros(8)          # rc = R(res): lam_res = R^T lam_rc = injection
                el._prolong_add(lam_rc, lam_res, lv)
            else:                     # residual sweep res = f - STEP(f - r)
                _, lv, f, r, ext = item
                lam_f, lam_ext = elast_sweep_adjoint(el, lv, lam_res, 1.0, -1.0, f_in=f, resid=r, fext=ext,
                                                     lam_resid=lam_resid, want_force=True, grads=self.grads)
                self._N_adj(lam_ext, f, lv, lam_f, lam_fe)
                lam = add_(lam_f, lam)
        return lam

    def step_adjoint(self, tp, lam_fe_new, lam_fd_new, lam_dtd_new, lam_eta=None, lam_p=None):
        """Transpose of ``step`` given the adjoints of its outputs; returns the
        adjoints of (fe, fd, dtd) and accumulates the material gradients."""
        sim, el, da = self.sim, self.el, self.da
        th, a, eps = sim.couplingRatio, sim.alpha, sim.epsilon
        Le, Ld = el._L(), da._layout
        lam_fd, lam_src = darcy_sweep_adjoint(da, lam_fd_new, f_in=tp["fd"], source=tp["source"],
                                              g_omega=self.g_omega, want_source=True)
        if lam_p is not None:              # pressure = sum fd + source / 2
            darcy_moments_adjoint(da, lam_fd, lam_rho=lam_p)
            lam_src = Ld.field(lam_src + 0.5 * lam_p, 1)
        # source = sb - (th a / eps) dtd_new;  dtd_new = div_0(f - fe)
        lam_div = Le.field(lam_dtd_new - (th * a / eps) * lam_src, 1)
        lam_f = Le.zeros(8)
        elast_moments_adjoint(el, 0, lam_f, lam_div=lam_div, f=tp["diff"], grads=self.grads)
        lam_fe = Le.field(-lam_f, 8)
        lam_f = Le.field(lam_f + lam_fe_new, 8)
        lam_force = Le.zeros(2)
        if lam_eta is not None:            # eta = sum c f + (force + N(f)) / 2
            elast_moments_adjoint(el, 0, lam_f, lam_eta=lam_eta)
            self._N_adj(Le.field(0.5 * lam_eta, 2), tp["f"], 0, lam_f, lam_force)
        for rec in reversed(tp["cycles"]):
            lam_f = self._vcycle_adj(lam_f, rec, None, lam_force)
        # force = (-a eps) pgbase - G(div_0(fe), sN), formed in the Darcy precision
        lam_force_d = Ld.field(lam_force, 2)
        lam_divp_d = Ld.zeros(1)
        gradient_adjoint(da, Ld.field(-lam_force_d, 2), self.sN, lam_divp_d)
        elast_moments_adjoint(el, 0, lam_fe, lam_div=Le.field(lam_divp_d, 1), f=tp["fe"], grads=self.grads)
        lam_pgbase = Ld.field((-a * eps) * lam_force_d, 2)
        # pgbase = G(sb, 1/2) + grad(fd);  sb = (1 - th)(-a / eps) dtd
        lam_sb = Ld.field(lam_src, 1).clone()
        gradient_adjoint(da, lam_pgbase, 0.5, lam_sb)
        darcy_moments_adjoint(da, lam_fd, lam_grad=lam_pgbase, f=tp["fd"], g_omega=self.g_omega)
        lam_dtd = Ld.field(((1.0 - th) * -a / eps) * lam_sb, 1)
        return Le.field(lam_fe + lam_f, 8), lam_fd, lam_dtd

    def backward(self):
        """Adjoint of the last ``forward``: returns (per-level d/d lambda,
        per-level d/d mu, d/d omega) as FP64 (nx_l, ny_l) tensors."""
        if self.graphs:
            if self._bwd_graphs is None:
                self._build_backward_graphs()
            return self._backward_graphs()
        t0 = time.time()
        el, da = self.el, self.da
        self.grads.zero_()
        self.g_omega.zero_()
        Le, Ld = el._L(), da._layout
        lam_fe, lam_fd, lam_dtd = Le.zeros(8), Ld.zeros(9), Ld.zeros(1)
        lam_eta = Le.field(self.eta.double() - self.eta_obs.double(), 2)
        lam_p = Ld.field(self.p.double() - self.p_obs.double(), 1)
        starts = sorted(self.checkpoints)
        for s in reversed(starts):
            end = min(s + self.every, self.steps)
            fe, fd, dtd = self.checkpoints[s]
            tapes = []
            for k in range(s, end):        # recompute the segment with tapes
                tp = {}
                fe, fd, dtd, _, _ = self.step(fe, fd, dtd, tape=tp)
                tapes.append(tp)
            for k in range(end - 1, s - 1, -1):
                last = k == self.steps - 1
                lam_fe, lam_fd, lam_dtd = self.step_adjoint(tapes[k - s], lam_fe, lam_fd, lam_dtd,
                                                            lam_eta if last else None, lam_p if last else None)
                tapes[k - s] = None
        torch.cuda.synchronize()
        self.timing["backward_s"] = time.time() - t0
        g_lam = [t[..., 0].clone() for t in self.grads.lam]
        g_mu = [t[..., 0].clone() for t in self.grads.mu]
        return g_lam, g_mu, self.g_omega[..., 0].clone()


    def _backward_graphs(self):
        t0 = time.time()
        B = self._bwd_graphs
        self.grads.zero_()
        self.g_omega.zero_()
        for t in B["lam"] + B["src"]:
            t.zero_()
        for s in reversed(sorted(self.checkpoints)):
            n = min(s + self.every, self.steps) - s
            self._load(B["ins"][0], self.checkpoints[s])
            for j in range(n):
                B["steps"][j].replay()
            for j in range(n - 1, -1, -1):
                last = s + j == self.steps - 1
                if last:
                    B["src"][0].copy_(self.eta.double() - self.eta_obs.double())
                    B["src"][1].copy_(self.p.double() - self.p_obs.double())
                B["adj"][j].replay()
                if last:
                    for t in B["src"]:
                        t.zero_()
        torch.cuda.synchronize()
        self.timing["backward_s"] = time.time() - t0
        g_lam = [t[..., 0].clone() for t in self.grads.lam]
        g_mu = [t[..., 0].clone() for t in self.grads.mu]
        return g_lam, g_mu, self.g_omega[..., 0].clone()


class ConsolidationMisfit(torch.autograd.Function):
    """J(lambda0, mu0, omega) of a ``BiotAdjointModel`` as a differentiable
    torch function of the level-0 material fields ((nx, ny) tensors)."""

    @staticmethod
    def forward(ctx, lam0, mu0, omega, model):
        model.set_parameters(lam0.detach(), mu0.detach(), omega.detach())
        J = model.forward()
        ctx.model = model
        ctx.save_for_backward(lam0, mu0, omega)
        return torch.tensor(J, dtype=torch.float64, device=lam0.device)

    @staticmethod
    def backward(ctx, gJ):
        lam0, mu0, omega = ctx.saved_tensors
        model = ctx.model
        g_lam, g_mu, g_om = model.backward()
        with torch.enable_grad():
            l0 = lam0.detach().double().requires_grad_()
            m0 = mu0.detach().double().requires_grad_()
            hier = material_hierarchy(l0, m0, model.el.mg_BCs, model.el.levels)
            s = sum((h[0] * g_lam[i]).sum() + (h[1] * g_mu[i]).sum() for i, h in enumerate(hier))
            dl, dm = torch.autograd.grad(s, (l0, m0))
        return (gJ * dl).to(lam0.dtype), (gJ * dm).to(mu0.dtype), (gJ * g_om).to(omega.dtype), None


def consolidation_parameters(log_mu, log_k, mu0=None, lam0=None, K0=None, nu=None):
    """Level-0 (lambda, mu, omega) of ``workloads.terzaghi_heterogeneous`` from
    the log-shear-modulus and log-permeability fields (torch, differentiable):
    mu = mu0 exp(log_mu), lambda = lam0 (or 2 mu nu / (1 - nu) if ``nu`` is
    given), omega = 1 / (3 K0 exp(log_k) + 1/2).  Defaults as the workload's."""
    from .workloads import TERZAGHI_K, TERZAGHI_LAM, TERZAGHI_MU
    mu0 = TERZAGHI_MU if mu0 is None else mu0
    lam0 = TERZAGHI_LAM if lam0 is None else lam0
    K0 = TERZAGHI_K if K0 is None else K0
    mu = mu0 * torch.exp(log_mu)
    lam = mu * (2.0 * nu / (1.0 - nu)) if nu is not None else torch.full_like(mu, lam0)
    omega = 1.0 / (3.0 * K0 * torch.exp(log_k) + 0.5)
    return lam, mu, omega
