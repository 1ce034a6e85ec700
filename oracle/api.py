"""The oracle's classes under the reference's names (test infrastructure only)."""
from .lattice import Lattice, LatticeD2Q8, LatticeD2Q9, LatticeD3Q19, LatticeD3Q27, Policy  # noqa: F401
from .boundary_conditions import BoundaryCondition, BounceBackHalfway  # noqa: F401
from .elasticity import (LBMElasticity, ElasticityBounceBackFullway, ElasticityBounceBack,  # noqa: F401
                         ElasticityAntiBounceBack)
from .darcy import (AdvectionDiffusionReactionBGK, ADR_AntiBounceBack, ADR_Neumann_BounceBack,  # noqa: F401
                    ADR_EquilibriumBC)
from .poroelasticity import LBMPoroelasticity  # noqa: F401
from .models import BGKSim, KBCSim, BounceBack, EquilibriumBC  # noqa: F401
