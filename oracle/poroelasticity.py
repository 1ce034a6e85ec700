"""Biot poroelasticity coupling (oracle).  Restates ``src/poroelasticity.py``."""
import numpy as np


class LBMPoroelasticity:
    """``src/poroelasticity.py:23-455``."""

    def __init__(self, LBMElasticity, LBMDarcy, **kwargs):
        kw_el = kwargs.copy()
        kw_el["lattice"] = kwargs.pop("lattice_elasticity")
        kw_el["MG_levels"] = kwargs.pop("elasticity_MG_levels", 1)
        self.elasticity = LBMElasticity(**kw_el)
        kwargs["lattice"] = kwargs.pop("lattice_darcy")
        self.darcy = LBMDarcy(**kwargs)
        self.elasticitySteps = kwargs.get("elasticity_steps", 1)
        self.alpha = kwargs.get("alpha")
        self.epsilon = kwargs.get("epsilon", 1 / self.elasticity.nx)
        self.couplingMethod = kwargs.get("coupling_method", "centered")
        self.couplingRatio = {"explicit": 0.0, "implicit": 1.0, "centered": 0.5}[self.couplingMethod]
        self.alternative_gradient = kwargs.get("alternative_gradient", False)
        self.ioRate = kwargs.get("io_rate", 0)
        self.useDynamicForce = self.get_elastic_force(0) is not None
        self.useDynamicSource = self.get_darcy_source(0) is not None

    def get_elastic_force(self, timestep):
        return None

    def get_darcy_source(self, timestep):
        return None

    def initialize_macroscopic_fields(self):
        return None

    def output_data(self, **kwargs):
        pass

    def init_state(self):
        """Initial state of ``run`` (``:226-252``)."""
        start_step = 0
        dt_div_eta = self.initialize_macroscopic_fields()
        if dt_div_eta is None:
            dt_div_eta = np.zeros((self.darcy.nx, self.darcy.ny, 1), dtype=self.darcy.precisionPolicy.compute_dtype)
        f_darcy = self.darcy.assign_fields_sharded()
        source = (-self.alpha / self.epsilon) * dt_div_eta
        if self.useDynamicSource:
            source = source + self.get_darcy_source(start_step)
        f_darcy = f_darcy - 0.5 * source * self.darcy.w
        f_el = self.elasticity.assign_fields_sharded()
        if self.alternative_gradient:
            pressure = self.darcy.update_macroscopic(f_darcy, source)
            force = self.darcy.gradient(pressure, -self.alpha * self.epsilon)
        else:
            _, pressure_grad = self.darcy.update_macroscopic(f_darcy, gradient=True)
            pressure_grad = pressure_grad + self.darcy.gradient(source, 0.5)
            force = (-self.alpha * self.epsilon) * pressure_grad
        if self.useDynamicForce:
            force = force + self.get_elastic_force(start_step)
        eta, sigma = self.elasticity.initialize_macroscopic_fields()
        if eta is not None and sigma is not None:
            f_el = self.elasticity.equilibrium(eta, sigma, external_force=force)
        return f_el, f_darcy, dt_div_eta

    def run(self, t_max):
        """``:208-301`` (t_max + 1 coupled steps)."""
        f_el, f_darcy, dt_div_eta = self.init_state()
        for timestep in range(0, t_max + 1):
            io_flag = self.ioRate > 0 and (timestep % self.ioRate == 0 or timestep == t_max)
            f_el, f_darcy, eta, sigma, dt_div_eta, pressure, pressure_grad = \
                self.step(f_el, f_darcy, dt_div_eta, timestep)
            if io_flag:
                self.output_data(timestep=timestep, eta=eta[None], sigma=sigma[None],
                                 dt_div_eta=dt_div_eta[None], pressure=pressure[None],
                                 pressure_grad=pressure_grad[None],
                                 f_poststreaming_elasticity=f_el, f_poststreaming_darcy=f_darcy)
        return f_el, f_darcy

    def step(self, f_elasticity, f_darcy, dt_div_eta, timestep):
        """``:303-339``."""
        el, da = self.elasticity, self.darcy
        theta, a, eps = self.couplingRatio, self.alpha, self.epsilon
        fprev = f_elasticity.copy()
        source_base = ((1.0 - theta) * -a / eps) * dt_div_eta
        if self.useDynamicSource:
            source_base = source_base + self.get_darcy_source(timestep)
        if self.alternative_gradient:
            pressure_grad_base = da.gradient(da.update_macroscopic(f_darcy, source_base))
        else:
            _, pressure_grad_base = da.update_macroscopic(f_darcy, gradient=True)
            pressure_grad_base = pressure_grad_base + da.gradient(source_base, 0.5)
        force = (-a * eps) * pressure_grad_base - da.gradient(el.update_divergence(fprev), 0.5 * theta * a ** 2)
        if self.useDynamicForce:
            force = force + self.get_elastic_force(timestep)
        nonlinear_force = lambda f_el: da.gradient(el.update_divergence(f_el), 0.5 * theta * a ** 2)
        for _ in range(self.elasticitySteps):
            f_elasticity, *_ = el.step(f_elasticity, timestep, False, force, nonlinear_force=nonlinear_force)
        eta, sigma = el.update_macroscopic(f_elasticity, force + nonlinear_force(f_elasticity))
        dt_div_eta = el.update_divergence(f_elasticity - fprev)
        source = source_base - (theta * a / eps) * dt_div_eta
        pressure = da.update_macroscopic(f_darcy, source)
        if self.alternative_gradient:
            pressure_grad = da.gradient(pressure)
        else:
            pressure_grad = pressure_grad_base - da.gradient(dt_div_eta, 0.5 * theta * a / eps)
        f_darcy, *_ = da.step(f_darcy, timestep, False, source)
        return f_elasticity, f_darcy, eta, sigma, dt_div_eta, pressure, pressure_grad
