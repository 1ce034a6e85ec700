"""Generate ``reference_fixtures.npz`` by running the reference's own solver
source (s-lunowa/xlb-biot ``src/*.py``, unmodified) on the golden cases.

JAX 0.5.3 is not installed (no network, here or on the GPU machines), so the
reference's modules are imported with the NumPy stand-in for the JAX API in
``jaxshim/`` first on ``sys.path`` (JAX's x64 mode, FP64 throughout).  The
stand-in replaces only the array library; every solver step, boundary
condition, multigrid recursion and coupling step that runs is the reference's
code.  Two hooks adapt the cases to it: inputs are converted to the stand-in's
array type (``golden_asarray``), and the per-cell relaxation case stores its
omega array on the solver directly (the reference's ``omega`` setter accepts
floats only, ``src/base.py:166-173``; its collision expressions broadcast an
array).

    python tests/golden/make_golden.py [--reference /path/to/xlb-biot] [--cases NAME ...]

``--cases`` regenerates only the named cases and keeps the others' arrays.
"""
import argparse
import json
import os
import sys
import time
from types import SimpleNamespace

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "reference_fixtures.npz")


def reference_namespace(root):
    sys.dont_write_bytecode = True           # the reference tree is read-only
    sys.path.insert(0, os.path.join(HERE, "jaxshim"))
    sys.path.insert(0, root)
    import jax
    jax.config.update("jax_enable_x64", True)
    import jax.numpy as jnp
    import src.boundary_conditions
    import src.darcy
    import src.elasticity
    import src.lattice
    import src.models
    import src.poroelasticity
    import src.utils
    ns = {}
    for mod in (src.lattice, src.boundary_conditions, src.elasticity, src.darcy, src.poroelasticity, src.utils,
                src.models):
        ns.update({k: getattr(mod, k) for k in dir(mod) if not k.startswith("_")})
    m = SimpleNamespace(**ns)
    m.golden_asarray = jnp.asarray
    m.golden_set_omega = lambda solver, om: setattr(solver, "_omega", om)
    return m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("XLB_BIOT_REFERENCE", "/root/reference"))
    ap.add_argument("--out", default=OUT)
    ap.add_argument("--cases", nargs="*", default=None)
    args = ap.parse_args()
    m = reference_namespace(args.reference)
    sys.path.insert(0, HERE)
    from cases import CASES
    import numpy as np
    arrays, manifest = {}, {}
    todo = CASES
    if args.cases:
        unknown = sorted(set(args.cases) - set(CASES))
        if unknown:
            raise SystemExit(f"unknown cases: {unknown}")
        with np.load(args.out) as old:
            for key in old.files:
                name = key.split("/")[0]
                if name in CASES and name not in args.cases:
                    arrays[key] = old[key]
                    manifest.setdefault(name, {})[key.split("/", 1)[1]] = list(old[key].shape)
        todo = {k: CASES[k] for k in args.cases}
    for name, case in todo.items():
        t0 = time.time()
        res = case(m)
        manifest[name] = {k: list(v.shape) for k, v in res.items()}
        for k, v in res.items():
            arrays[f"{name}/{k}"] = v
        print(f"{name}: {sorted(res)} ({time.time() - t0:.1f} s)", file=sys.stderr)
    np.savez_compressed(args.out, **arrays)
    with open(os.path.splitext(args.out)[0] + ".json", "w") as fh:
        json.dump({"generator": "tests/golden/make_golden.py", "source": "s-lunowa/xlb-biot src/*.py under the "
                   "NumPy stand-in for JAX (tests/golden/jaxshim), FP64", "cases": manifest}, fh, indent=1,
                  sort_keys=True)


if __name__ == "__main__":
    main()
