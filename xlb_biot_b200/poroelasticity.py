"""Biot poroelasticity coupling on B200 (drop-in for ``src/poroelasticity.py``).

``LBMPoroelasticity(ElasticityCls, DarcyCls, **kwargs)`` keeps the reference's
keywords, validation, hooks (``get_elastic_force``, ``get_darcy_source``,
``initialize_macroscopic_fields``, ``output_data``) and the 7-tuple ``step``.
The coupling's nonlinear force N(f) = gradient(divergence(f)) is passed to the
elasticity solver as a ``DivGradForce`` object, which the multigrid smoother
evaluates with the divergence and gradient kernels on every level instead of
calling back into Python per sweep.
"""
import time

import torch

from ._common import gathered, require_finite


class DivGradForce:
    """``lambda f_el: darcy.gradient(elasticity.update_divergence(f_el), scale)``
    of ``src/poroelasticity.py:324`` as an object the kernels can evaluate."""

    fusable = True          # the elasticity sweeps may compute it in-kernel (xlbb_elast_sweep_divgrad)

    def __init__(self, elasticity, darcy, scale):
        self.elasticity, self.darcy, self.scale = elasticity, darcy, scale

    def __call__(self, f_el):
        return self.darcy.gradient(self.elasticity.update_divergence(f_el), self.scale)

    def evaluate(self, el, f, level, external_force):
        """external_force + N(f) on multigrid level ``level``, computed in that
        level's precision (the precision of the sweep that consumes it), by the
        fused divergence-gradient kernel."""
        return el.coupling_force(f, level, self.darcy, self.scale, base=external_force)


class BiotStepGraph:
    """One coupled Biot step captured as a CUDA graph.

    The graph reads the state from three static buffers (elasticity and Darcy
    populations, dt_div_eta), runs ``LBMPoroelasticity.step`` (every kernel of
    the V-cycles, the coupling gradients and the Darcy sweep) and copies the new
    state back into the same buffers, so each ``replay`` advances one time step
    with one graph launch.  Valid while the step takes no host decisions: no
    dynamic force or source hooks and a fixed inner cycle count.  The other
    outputs (eta, sigma, pressure, pressure_grad) live in the graph's memory and
    are overwritten by the next replay."""

    def __init__(self, sim, f_el, f_darcy, dt_div_eta):
        el, da = sim.elasticity, sim.darcy
        self.f_el = el._L().empty(8)
        self.f_darcy = da._layout.empty(9)
        self.dt_div_eta = da._layout.empty(1)
        self.load(f_el, f_darcy, dt_div_eta)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            sim.step(self.f_el, self.f_darcy, self.dt_div_eta, 0)    # warm-up: scratch buffers, module loading
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            out = sim.step(self.f_el, self.f_darcy, self.dt_div_eta, 0)
            self.f_el.copy_(out[0])
            self.f_darcy.copy_(out[1])
            self.dt_div_eta.copy_(out[4])
        self.outputs = (self.f_el, self.f_darcy) + tuple(out[2:4]) + (self.dt_div_eta,) + tuple(out[5:7])

    def load(self, f_el, f_darcy, dt_div_eta):
        self.f_el.copy_(f_el)
        self.f_darcy.copy_(f_darcy)
        self.dt_div_eta.copy_(dt_div_eta)

    def replay(self):
        """One time step; returns the 7-tuple of ``step`` (static tensors)."""
        self.graph.replay()
        return self.outputs


class LBMPoroelasticity:
    """``src/poroelasticity.py:23-455``."""

    def __init__(self, LBMElasticity, LBMDarcy, **kwargs):
        kwargs_elasticity = kwargs.copy()
        kwargs_elasticity['lattice'] = kwargs.pop('lattice_elasticity')
        kwargs_elasticity['MG_levels'] = kwargs.pop('elasticity_MG_levels', 1)
        self.elasticity = LBMElasticity(**kwargs_elasticity)
        kwargs['lattice'] = kwargs.pop('lattice_darcy')
        # Extension: ``darcy_precision`` runs the pressure equation in another
        # precision than the elasticity solve (e.g. FP64 pressure, FP32 elasticity).
        kwargs_darcy = dict(kwargs)
        if kwargs.get('darcy_precision'):
            kwargs_darcy['precision'] = kwargs['darcy_precision']
        self.darcy = LBMDarcy(**kwargs_darcy)
        self.elasticitySteps = kwargs.get('elasticity_steps', 1)
        self.alpha = kwargs.get('alpha')
        self.epsilon = kwargs.get('epsilon', 1 / self.elasticity.nx)
        self.couplingMethod = kwargs.get('coupling_method', 'centered')
        self.alternative_gradient = kwargs.get('alternative_gradient', False)
        self.elasticityTol = kwargs.get('elasticity_tol', None)
        if self.elasticityTol is not None and self.elasticity.levels < 2:
            raise ValueError("elasticity_tol needs a multigrid elasticity solver (elasticity_MG_levels > 1)")
        self.downsamplingFactor = kwargs.get("downsampling_factor", 1)
        self.printInfoRate = kwargs.get("print_info_rate", 100)
        self.ioRate = kwargs.get("io_rate", 0)
        self.computeMLUPS = kwargs.get("compute_MLUPS", False)
        if self.computeMLUPS:
            self.ioRate = 0
            self.printInfoRate = 0
        self.useDynamicForce = self.get_elastic_force(0) is not None
        self.useDynamicSource = self.get_darcy_source(0) is not None
        # Extension: ``cuda_graph`` (default True) lets ``run`` replay the coupled
        # step as one CUDA graph when the step takes no host decisions.
        self.cudaGraph = kwargs.get("cuda_graph", True)
        self.show_simulation_parameters()

    # validation (src/poroelasticity.py:72-176)
    @property
    def elasticitySteps(self):
        return self._elasticitySteps

    @elasticitySteps.setter
    def elasticitySteps(self, value):
        if not isinstance(value, int) or value < 1:
            raise TypeError("elasticitySteps must be a positive integer.")
        self._elasticitySteps = value

    @property
    def alpha(self):
        return self._alpha

    @alpha.setter
    def alpha(self, value):
        if not isinstance(value, float) or value < 0 or value > 1:
            raise TypeError("alpha must be a float between 0 and 1.")
        self._alpha = value

    @property
    def epsilon(self):
        return self._epsilon

    @epsilon.setter
    def epsilon(self, value):
        if not isinstance(value, float) or value <= 0:
            raise TypeError("epsilon must be a positive float.")
        self._epsilon = value

    @property
    def alternative_gradient(self):
        return self._alternative_gradient

    @alternative_gradient.setter
    def alternative_gradient(self, value):
        if not isinstance(value, bool):
            raise TypeError("alternative_gradient must be a boolean.")
        self._alternative_gradient = value

    @property
    def couplingMethod(self):
        return self._couplingMethod

    @couplingMethod.setter
    def couplingMethod(self, value):
        if value == 'explicit':
            self.couplingRatio = 0.0
        elif value == 'implicit':
            self.couplingRatio = 1.0
        elif value == 'centered':
            self.couplingRatio = 0.5
        else:
            raise TypeError("couplingMethod must be 'explicit', 'implicit', 'centered', or 'alt_implicit', "
                            "'alt_centered'.")
        self._couplingMethod = value

    @property
    def couplingRatio(self):
        return self._couplingRatio

    @couplingRatio.setter
    def couplingRatio(self, value):
        if not isinstance(value, float) or value < 0.0 or value > 1.0:
            raise TypeError("couplingRatio must be a float beween 0 and 1")
        self._couplingRatio = value

    def _int_prop(name):
        def getter(self):
            return getattr(self, "_" + name)

        def setter(self, value):
            if not isinstance(value, int):
                raise TypeError(f"{name} must be an integer")
            setattr(self, "_" + name, value)
        return property(getter, setter)

    downsamplingFactor = _int_prop("downsamplingFactor")
    printInfoRate = _int_prop("printInfoRate")
    ioRate = _int_prop("ioRate")
    del _int_prop

    @property
    def computeMLUPS(self):
        return self._computeMLUPS

    @computeMLUPS.setter
    def computeMLUPS(self, value):
        if not isinstance(value, bool):
            raise TypeError("computeMLUPS must be a boolean")
        self._computeMLUPS = value

    def show_simulation_parameters(self):
        names = {'alpha': 'Biot-Willis Constant', 'couplingMethod': 'Coupling Method',
                 'elasticitySteps': 'Elasticity Steps', 'alternative_gradient': 'Alternative Gradient',
                 'downsamplingFactor': 'Downsampling Factor', 'printInfoRate': 'Print Info Rate',
                 'ioRate': 'I/O Rate', 'computeMLUPS': 'Compute MLUPS'}
        print(f"**** Simulation Parameters for {self.__class__.__name__} ****")
        for a, n in names.items():
            print(f"{n:>30} | {getattr(self, a, 'Attribute not set')}")

    # ------------------------------------------------------------------ driver
    def _dyn_force(self, t):
        return self.elasticity._L().field(self.get_elastic_force(t), 2)

    def _dyn_source(self, t):
        return self.darcy._layout.field(self.get_darcy_source(t), 1)

    def init_state(self):
        """Initial populations and coupling field of ``run`` (``:226-252``)."""
        el, da = self.elasticity, self.darcy
        start_step = 0
        dt_div_eta = self.initialize_macroscopic_fields()
        if dt_div_eta is None:
            dt_div_eta = da._layout.zeros(1)
        else:
            dt_div_eta = da._layout.field(dt_div_eta, 1)
        f_darcy = da.assign_fields_sharded()
        source = (-self.alpha / self.epsilon) * dt_div_eta
        if self.useDynamicSource:
            source = source + self._dyn_source(start_step)
        w = torch.as_tensor(da.w, device=f_darcy.device, dtype=f_darcy.dtype)
        f_darcy = da._layout.field(f_darcy - 0.5 * source * w, 9)
        pressure = da.update_macroscopic(f_darcy, source)
        f_el = el.assign_fields_sharded()
        if self.alternative_gradient:
            force = da.gradient(pressure, -self.alpha * self.epsilon)
        else:
            _, pressure_grad = da.update_macroscopic(f_darcy, gradient=True)
            pressure_grad = pressure_grad + da.gradient(source, 0.5)
            force = (-self.alpha * self.epsilon) * pressure_grad
        if self.useDynamicForce:
            force = force + self._dyn_force(start_step)
        eta, sigma = el.initialize_macroscopic_fields()
        if eta is not None and sigma is not None:
            f_el = el.equilibrium(eta, sigma, external_force=force)
        return f_el, f_darcy, dt_div_eta

    def graph_capturable(self):
        """True when one coupled step takes no host decisions (no dynamic force or
        source hooks, a fixed inner cycle count), so it can be a CUDA graph."""
        return not (self.useDynamicForce or self.useDynamicSource) and self.elasticityTol is None

    def capture_step(self, f_el, f_darcy, dt_div_eta):
        """A ``BiotStepGraph`` starting from the given state."""
        if not self.graph_capturable():
            raise ValueError("the coupled step takes host decisions (dynamic hooks or elasticity_tol)")
        return BiotStepGraph(self, f_el, f_darcy, dt_div_eta)

    def run(self, t_max):
        """``:208-301`` (t_max + 1 coupled steps; one CUDA graph replay per step
        when ``graph_capturable``)."""
        f_el, f_darcy, dt_div_eta = self.init_state()
        graph = self.capture_step(f_el, f_darcy, dt_div_eta) if self.cudaGraph and self.graph_capturable() else None
        start = time.time()
        for timestep in range(0, t_max + 1):
            io_flag = self.ioRate > 0 and (timestep % self.ioRate == 0 or timestep == t_max)
            print_iter_flag = self.printInfoRate > 0 and timestep % self.printInfoRate == 0
            if graph is not None:
                f_el, f_darcy, eta, sigma, dt_div_eta, pressure, pressure_grad = graph.replay()
            else:
                f_el, f_darcy, eta, sigma, dt_div_eta, pressure, pressure_grad = \
                    self.step(f_el, f_darcy, dt_div_eta, timestep)
            if print_iter_flag:
                print(f"Timestep {timestep} of {t_max} completed")
            if io_flag:
                self.handle_io_timestep(timestep, f_el, f_darcy, gathered(eta), gathered(sigma), gathered(pressure),
                                        gathered(pressure_grad), gathered(dt_div_eta))
            if self.computeMLUPS and timestep == 1:
                torch.cuda.synchronize()
                start = time.time()
        if self.computeMLUPS:
            torch.cuda.synchronize()
            end = time.time()
            nx, ny = self.elasticity.nx, self.elasticity.ny
            print(f"Domain: {nx} x {ny}")
            print(f"Number of voxels: {nx * ny}")
            print(f"MLUPS: {nx * ny * t_max / (end - start) / 1e6}")
        return f_el, f_darcy

    def step(self, f_elasticity, f_darcy, dt_div_eta, timestep):
        """``:303-339``: one coupled Biot step."""
        el, da = self.elasticity, self.darcy
        th, a, eps = self.couplingRatio, self.alpha, self.epsilon
        f_elasticity = el._f(f_elasticity)
        f_darcy = da._layout.field(f_darcy, 9)
        dt_div_eta = da._layout.field(dt_div_eta, 1)
        fprev = f_elasticity.clone()
        source_base = ((1.0 - th) * -a / eps) * dt_div_eta
        if self.useDynamicSource:
            source_base = source_base + self._dyn_source(timestep)
        source_base = da._layout.field(source_base, 1)
        if self.alternative_gradient:
            pressure_grad_base = da.gradient(da.update_macroscopic(f_darcy, source_base))
        else:
            _, pgb = da.update_macroscopic(f_darcy, gradient=True)
            pressure_grad_base = da.gradient(source_base, 0.5, base=pgb)
        force = (-a * eps) * pressure_grad_base - da.gradient(el.update_divergence(fprev), 0.5 * th * a ** 2)
        if self.useDynamicForce:
            force = force + self._dyn_force(timestep)
        force = el._L().field(force, 2)
        nonlinear_force = DivGradForce(el, da, 0.5 * th * a ** 2)
        if self.elasticityTol is None:
            for _ in range(self.elasticitySteps):
                f_elasticity, *_ = el.step(f_elasticity, timestep, False, force, nonlinear_force=nonlinear_force)
        else:
            # Extension: V-cycles until the level-0 residual norm fell by elasticity_tol
            # (FP64 norm on the device, read once per cycle); elasticity_steps caps the cycles.
            r0 = None
            self.last_inner_cycles = 0
            for k in range(self.elasticitySteps):
                f_elasticity, r = el.step(f_elasticity, timestep, False, force, nonlinear_force=nonlinear_force)
                self.last_inner_cycles = k + 1
                r = float(r)
                require_finite(r, "level-0 residual norm of the inner elasticity solve", k + 1)
                r0 = r if r0 is None else r0
                self.last_inner_rel = r / r0 if r0 > 0 else 0.0
                if r0 == 0.0 or r / r0 < self.elasticityTol:
                    break
        eta, sigma = el.update_macroscopic(f_elasticity, nonlinear_force.evaluate(el, f_elasticity, 0, force))
        dt_div_eta = el.update_divergence(f_elasticity - fprev)
        source = da._layout.field(source_base - (th * a / eps) * dt_div_eta, 1)
        pressure = da.update_macroscopic(f_darcy, source)
        if self.alternative_gradient:
            pressure_grad = da.gradient(pressure)
        else:
            pressure_grad = pressure_grad_base - da.gradient(dt_div_eta, 0.5 * th * a / eps)
        f_darcy, *_ = da.step(f_darcy, timestep, False, source)
        return f_elasticity, f_darcy, eta, sigma, dt_div_eta, pressure, pressure_grad

    def handle_io_timestep(self, timestep, f_elasticity, f_darcy, eta, sigma, pressure, pressure_grad, dt_div_eta):
        self.output_data(timestep=timestep, eta=eta, sigma=sigma, dt_div_eta=dt_div_eta, pressure=pressure,
                         pressure_grad=pressure_grad, f_poststreaming_elasticity=f_elasticity,
                         f_poststreaming_darcy=f_darcy)

    def output_data(self, **kwargs):
        pass

    def get_elastic_force(self, timestep):
        pass

    def get_darcy_source(self, timestep):
        pass

    def initialize_macroscopic_fields(self):
        print("WARNING: Default initial conditions assumed: dt_div_eta = 0")
        print("         To set explicit initial dt_div_eta, use self.initialize_macroscopic_fields.")
        return None
