"""``LBMBase`` pieces used by the Darcy solver (mirror of ``src/base.py``).

Only the parts of the reference base class that the Darcy / Biot path uses are
kept: keyword validation, the one-device grid set-up, BC preprocessing,
``distributed_array_init``, ``assign_fields_sharded`` and ``equilibrium``.
Checkpointing keywords are accepted; ``checkpoint_rate > 0`` saves the
populations with ``torch.save`` (the reference uses orbax, ``:82-87,869-928``).
"""
import os
import time

import numpy as np
import torch

from . import _lib
from ._common import make_policy, print_parameters, set_precisions, storage_and_sweep_dtypes
from .boundary_conditions import grid_mask, solid_halo_voxels
from .fields import Layout, torch_dtype


class LBMBase:
    """``src/base.py:30-146``."""

    def __init__(self, **kwargs):
        self._init_kwargs = dict(kwargs)       # an FP64 twin is built from them (refine.py)
        self.omega = kwargs.get("omega")
        self.nx = kwargs.get("nx")
        self.ny = kwargs.get("ny")
        self.nz = kwargs.get("nz")
        self.precision = kwargs.get("precision")
        self.precisionPolicy = make_policy(self.precision)
        self.lattice = kwargs.get("lattice")
        self.checkpointRate = kwargs.get("checkpoint_rate", 0)
        self.checkpointDir = kwargs.get("checkpoint_dir", './checkpoints')
        self.downsamplingFactor = kwargs.get("downsampling_factor", 1)
        self.printInfoRate = kwargs.get("print_info_rate", 100)
        self.ioRate = kwargs.get("io_rate", 0)
        self.returnFpost = kwargs.get("return_fpost", False)
        self.computeMLUPS = kwargs.get("compute_MLUPS", False)
        self.restore_checkpoint = kwargs.get("restore_checkpoint", False)
        self.nDevices = 1
        self.backend = "cuda"
        if self.computeMLUPS:
            self.restore_checkpoint = False
            self.ioRate = 0
            self.checkpointRate = 0
            self.printInfoRate = 0
        _lib.require_cuda()
        _lib.lib()
        self.c, self.q, self.w, self.dim = self.lattice.c, self.lattice.q, self.lattice.w, self.lattice.d
        self.show_simulation_parameters()
        self.gridInfo = {"nx": self.nx, "ny": self.ny, "nz": self.nz, "dim": self.lattice.d, "lattice": self.lattice}
        self.sharding = None
        # storage type of the fields; 'f64/f32' sweeps compute in FP64 on them
        self._dtype, self._acc64 = storage_and_sweep_dtypes(self.precisionPolicy)
        self._dcode = _lib.dtype_code(self._dtype)
        self._sweep_code = _lib.XLBB_F32_ACC64 if self._acc64 else self._dcode
        self._rule_dtype = torch.float64 if self._acc64 else self._dtype
        self._layout = Layout(self.nx, self.ny, self._dtype, nz=self.nz)
        self.boundingBoxIndices = self.bounding_box_indices()
        self._create_boundary_data()
        self.force = self.get_force()

    # validation (src/base.py:148-349)
    @property
    def lattice(self):
        return self._lattice

    @lattice.setter
    def lattice(self, value):
        if value is None:
            raise ValueError("Lattice type must be provided.")
        if self.nz == 0 and value.name not in ['D2Q9']:
            raise ValueError("For 2D simulations, lattice type must be LatticeD2Q9.")
        if self.nz != 0 and value.name not in ['D3Q19', 'D3Q27']:
            raise ValueError("For 3D simulations, lattice type must be LatticeD3Q19, or LatticeD3Q27.")
        self._lattice = value

    @property
    def omega(self):
        return self._omega

    @omega.setter
    def omega(self, value):
        if value is None:
            raise ValueError("omega must be provided")
        if not isinstance(value, float):
            raise TypeError("omega must be a float")
        self._omega = value

    def _int_prop(name, label, required=False):
        def getter(self):
            return getattr(self, "_" + name)

        def setter(self, value):
            if value is None and required:
                raise ValueError(f"{label} must be provided")
            if not isinstance(value, int) or isinstance(value, bool):
                raise TypeError(f"{label} must be an integer")
            setattr(self, "_" + name, value)
        return property(getter, setter)

    nx = _int_prop("nx", "nx", True)
    ny = _int_prop("ny", "ny", True)
    nz = _int_prop("nz", "nz", True)
    checkpointRate = _int_prop("checkpointRate", "checkpointRate")
    downsamplingFactor = _int_prop("downsamplingFactor", "downsamplingFactor")
    printInfoRate = _int_prop("printInfoRate", "printInfoRate")
    ioRate = _int_prop("ioRate", "ioRate")
    nDevices = _int_prop("nDevices", "nDevices")

    def _bool_prop(name, label):
        def getter(self):
            return getattr(self, "_" + name)

        def setter(self, value):
            if not isinstance(value, bool):
                raise TypeError(f"{label} must be a boolean")
            setattr(self, "_" + name, value)
        return property(getter, setter)

    returnFpost = _bool_prop("returnFpost", "returnFpost")
    computeMLUPS = _bool_prop("computeMLUPS", "computeMLUPS")
    restore_checkpoint = _bool_prop("restore_checkpoint", "restore_checkpoint")
    del _int_prop, _bool_prop

    @property
    def checkpointDir(self):
        return self._checkpointDir

    @checkpointDir.setter
    def checkpointDir(self, value):
        if not isinstance(value, str):
            raise TypeError("checkpointDir must be a string")
        self._checkpointDir = value

    @property
    def precision(self):
        return self._precision

    @precision.setter
    def precision(self, value):
        if not isinstance(value, str):
            raise TypeError("precision must be a string")
        self._precision = value

    def show_simulation_parameters(self):
        attrs = ['omega', 'nx', 'ny', 'nz', 'dim', 'precision', 'lattice', 'checkpointRate', 'checkpointDir',
                 'downsamplingFactor', 'printInfoRate', 'ioRate', 'computeMLUPS', 'restore_checkpoint',
                 'backend', 'nDevices']
        names = {'omega': 'Omega', 'nx': 'Grid Points in X', 'ny': 'Grid Points in Y', 'nz': 'Grid Points in Z',
                 'dim': 'Dimensionality', 'precision': 'Precision Policy', 'lattice': 'Lattice Type',
                 'checkpointRate': 'Checkpoint Rate', 'checkpointDir': 'Checkpoint Directory',
                 'downsamplingFactor': 'Downsampling Factor', 'printInfoRate': 'Print Info Rate',
                 'ioRate': 'I/O Rate', 'computeMLUPS': 'Compute MLUPS',
                 'restore_checkpoint': 'Restore Checkpoint', 'backend': 'Backend', 'nDevices': 'Number of Devices'}
        print_parameters(self, attrs, names)

    def set_precisions(self, precision):
        return set_precisions(precision)

    def bounding_box_indices(self):
        """``src/base.py:451-484``: edges (2D) or faces (3D) of the grid."""
        nx, ny, nz = self.nx, self.ny, self.nz
        if self.dim == 2:
            return {"bottom": np.array([[i, 0] for i in range(nx)], dtype=int),
                    "top": np.array([[i, ny - 1] for i in range(nx)], dtype=int),
                    "left": np.array([[0, i] for i in range(ny)], dtype=int),
                    "right": np.array([[nx - 1, i] for i in range(ny)], dtype=int)}
        return {"bottom": np.array([[i, j, 0] for i in range(nx) for j in range(ny)], dtype=int),
                "top": np.array([[i, j, nz - 1] for i in range(nx) for j in range(ny)], dtype=int),
                "left": np.array([[0, j, k] for j in range(ny) for k in range(nz)], dtype=int),
                "right": np.array([[nx - 1, j, k] for j in range(ny) for k in range(nz)], dtype=int),
                "front": np.array([[i, 0, k] for i in range(nx) for k in range(nz)], dtype=int),
                "back": np.array([[i, ny - 1, k] for i in range(nx) for k in range(nz)], dtype=int)}

    def create_grid_mask(self, solid_halo_voxels):
        return grid_mask(self.nx, self.ny, self.lattice, solid_halo_voxels, nz=self.nz)

    def _create_boundary_data(self):
        """``src/base.py:351-372`` followed by rule compilation."""
        self.BCs = []
        self.set_boundary_conditions()
        t0 = time.time()
        gm = self.create_grid_mask(solid_halo_voxels(self.BCs))
        for bc in self.BCs:
            assert bc.implementationStep in ['PostStreaming', 'PostCollision']
            bc.create_local_mask_and_normal_arrays(gm)
        self._compile_rules()
        print("Time to create the grid mask and boundary rules:", time.time() - t0)

    def _compile_rules(self):
        pass

    def distributed_array_init(self, shape, type, init_val=0, sharding=None):
        """``src/base.py:379-411``: a device field of ``shape`` filled with ``init_val``."""
        dt = torch_dtype(type)
        if len(shape) == 3:
            return Layout(shape[0], shape[1], dt).field(init_val, shape[2])
        if len(shape) == 4:
            return Layout(shape[0], shape[1], dt, nz=shape[2]).field(init_val, shape[3])
        x = init_val if isinstance(init_val, torch.Tensor) else torch.as_tensor(np.asarray(init_val))
        return torch.broadcast_to(x.to(device="cuda", dtype=dt), shape).clone()

    def initialize_macroscopic_fields(self):
        print("WARNING: Default initial conditions assumed: density = 1, velocity = 0")
        print("         To set explicit initial density and velocity, use self.initialize_macroscopic_fields.")
        return None, None

    def assign_fields_sharded(self):
        """``src/base.py:528-559``: default populations are the lattice weights."""
        rho0, u0 = self.initialize_macroscopic_fields()
        if rho0 is None or u0 is None:
            return self._layout.field(torch.as_tensor(self.w), self.q)
        return self.initialize_populations(rho0, u0)

    def initialize_populations(self, rho0, u0):
        return self.equilibrium(rho0, u0)

    def equilibrium(self, rho, u, cast_output=True):
        """``src/base.py:686-724`` (initialisation only; computed with device
        tensor algebra)."""
        L = self._layout
        rho = L.field(rho, 1)
        u = L.field(u, self.dim)
        c = torch.as_tensor(self.c, device=L.device, dtype=L.dtype)
        w = torch.as_tensor(self.w, device=L.device, dtype=L.dtype)
        cu = 3.0 * (u @ c)
        usqr = 1.5 * torch.sum(u * u, dim=-1, keepdim=True)
        return L.field(rho * w * (1.0 + cu * (1.0 + 0.5 * cu) - usqr), self.q)

    def set_boundary_conditions(self):
        pass

    def get_force(self):
        pass

    def output_data(self, **kwargs):
        pass

    def save_checkpoint(self, timestep, f):
        """The populations after ``timestep`` (the reference's orbax manager with
        ``max_to_keep=1``, ``src/base.py:82-87``: older checkpoints are removed)."""
        os.makedirs(self.checkpointDir, exist_ok=True)
        name = f"checkpoint_{timestep:08d}.pt"
        torch.save({"timestep": timestep, "f": f.detach().cpu()}, os.path.join(self.checkpointDir, name + ".tmp"))
        os.replace(os.path.join(self.checkpointDir, name + ".tmp"), os.path.join(self.checkpointDir, name))
        for old in os.listdir(self.checkpointDir):
            if old.startswith("checkpoint_") and old.endswith(".pt") and old != name:
                os.remove(os.path.join(self.checkpointDir, old))

    def load_latest_checkpoint(self):
        if not os.path.isdir(self.checkpointDir):
            return None
        names = sorted(n for n in os.listdir(self.checkpointDir) if n.startswith("checkpoint_") and n.endswith(".pt"))
        if not names:
            return None
        return torch.load(os.path.join(self.checkpointDir, names[-1]))
