"""``install_as_src()`` exposes every class the reference's example scripts
import from ``src.*`` (module aliasing only; no GPU needed)."""
import sys

import pytest

# (module, names) imported by the reference's examples: examples/elasticity/*.py,
# examples/darcy/*.py, examples/poroelasticity/*.py, examples/performance/MLUPS2d.py
EXAMPLE_IMPORTS = [
    ("src.lattice", ["LatticeD2Q8", "LatticeD2Q9"]),
    ("src.elasticity", ["LBMElasticity", "ElasticityBounceBackFullway", "ElasticityBounceBack",
                        "ElasticityAntiBounceBack"]),
    ("src.darcy", ["AdvectionDiffusionReactionBGK", "ADR_AntiBounceBack", "ADR_Neumann_BounceBack",
                   "ADR_EquilibriumBC"]),
    ("src.poroelasticity", ["LBMPoroelasticity"]),
    ("src.boundary_conditions", ["BoundaryCondition", "BounceBack", "BounceBackHalfway", "EquilibriumBC"]),
    ("src.models", ["BGKSim", "KBCSim"]),
    ("src.utils", ["Parameters", "downsample_field", "save_fields_vtk"]),
    ("src.base", ["LBMBase"]),
]


@pytest.fixture
def aliased():
    before = {k: v for k, v in sys.modules.items() if k == "src" or k.startswith("src.")}
    import xlb_biot_b200
    xlb_biot_b200.install_as_src()
    yield
    for k in [k for k in sys.modules if k == "src" or k.startswith("src.")]:
        del sys.modules[k]
    sys.modules.update(before)


@pytest.mark.parametrize("module,names", EXAMPLE_IMPORTS, ids=[m for m, _ in EXAMPLE_IMPORTS])
def test_example_imports_resolve(aliased, module, names):
    import importlib
    mod = importlib.import_module(module)
    assert mod.__name__.startswith("xlb_biot_b200.")
    missing = [n for n in names if not hasattr(mod, n)]
    assert not missing, missing
