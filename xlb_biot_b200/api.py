"""All public classes under the reference's names, in one namespace."""
from .lattice import Lattice, LatticeD2Q8, LatticeD2Q9, LatticeD3Q19, LatticeD3Q27  # noqa: F401
from .boundary_conditions import BoundaryCondition, BounceBackHalfway, BounceBack, EquilibriumBC  # noqa: F401
from .elasticity import (LBMElasticity, ElasticityBounceBackFullway, ElasticityBounceBack,  # noqa: F401
                         ElasticityAntiBounceBack)
from .darcy import (AdvectionDiffusionReactionBGK, ADR_AntiBounceBack, ADR_Neumann_BounceBack,  # noqa: F401
                    ADR_EquilibriumBC)
from .base import LBMBase  # noqa: F401
from .poroelasticity import LBMPoroelasticity, DivGradForce  # noqa: F401
from .utils import Parameters, downsample_field  # noqa: F401
from .models import BGKSim, KBCSim  # noqa: F401
