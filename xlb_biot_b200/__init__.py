"""B200-native (sm_100a) lattice-Boltzmann Biot poroelasticity hot path.

Drop-in replacements for the solver modules of s-lunowa/xlb-biot:

=====================================  ==========================================
reference module                       this package
=====================================  ==========================================
``src.lattice``                        ``xlb_biot_b200.lattice``
``src.boundary_conditions``            ``xlb_biot_b200.boundary_conditions``
``src.base``                           ``xlb_biot_b200.base``
``src.elasticity``                     ``xlb_biot_b200.elasticity``
``src.darcy``                          ``xlb_biot_b200.darcy``
``src.poroelasticity``                 ``xlb_biot_b200.poroelasticity``
``src.models`` (D2Q9 BGK, KBC)         ``xlb_biot_b200.models``
``src.utils`` (Parameters, downsample) ``xlb_biot_b200.utils``
=====================================  ==========================================

``install_as_src()`` registers these modules under the reference's ``src.*``
names so unmodified scripts that do ``from src.elasticity import LBMElasticity``
run on the CUDA kernels.
"""
import importlib
import sys

__version__ = "1.0.0"

_MODULES = ("lattice", "boundary_conditions", "base", "elasticity", "darcy", "poroelasticity", "models",
            "utils")


def install_as_src():
    """Alias this package as the reference's ``src`` package."""
    pkg = sys.modules[__name__]
    sys.modules["src"] = pkg
    for m in _MODULES:
        sys.modules["src." + m] = importlib.import_module(__name__ + "." + m)
    return pkg
