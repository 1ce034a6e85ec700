"""Host-side boundary preprocessing and rule compilation (CPU, no GPU).

The product's BC classes are preprocessed exactly as the solvers do and
compiled to per-cell rules; the rules, evaluated on random populations, must
equal the oracle's direct application of its own BC objects
(``apply_bc``, src/elasticity.py:1061-1091) in every boundary cell.
"""
import numpy as np
import pytest
import torch

import oracle.api as O
from oracle.boundary_conditions import apply_bc_list, create_grid_mask, solid_voxels
import xlb_biot_b200.lattice as GL
import xlb_biot_b200.boundary_conditions as GB
import xlb_biot_b200.elasticity as GE
import xlb_biot_b200.darcy as GD
from xlb_biot_b200.bc_compile import compile_rules, evaluate_rules
from problems import corner_fixed_classes


class _NS:
    pass


def _ns_product():
    m = _NS()
    for mod in (GE, GD, GB):
        for k in dir(mod):
            if not k.startswith("_"):
                setattr(m, k, getattr(mod, k))
    return m


G = _ns_product()


def _prep(bcs, nx, ny, lattice, mask_fn):
    gm = mask_fn(nx, ny, lattice, (solid_voxels if mask_fn is create_grid_mask else GB.solid_halo_voxels)(bcs))
    for bc in bcs:
        bc.create_local_mask_and_normal_arrays(gm)
    return bcs


def _scenarios():
    """(name, q, nx, ny, builder(m, lattice, gi, pp) -> list of BCs)."""
    def bbox(nx, ny):
        return {"bottom": np.array([[i, 0] for i in range(nx)]), "top": np.array([[i, ny - 1] for i in range(nx)]),
                "left": np.array([[0, i] for i in range(ny)]), "right": np.array([[nx - 1, i] for i in range(ny)])}

    def dirichlet_full(m, lat, gi, pp, nx, ny):
        b = bbox(nx, ny)
        rng = np.random.default_rng(0)
        return [m.ElasticityBounceBackFullway(tuple(b[s].T), gi, pp, 1e-3 * rng.standard_normal((len(b[s]), 2)))
                for s in ("left", "right", "bottom", "top")]

    def neumann(m, lat, gi, pp, nx, ny):
        b = bbox(nx, ny)
        rng = np.random.default_rng(1)
        return [m.ElasticityAntiBounceBack(tuple(b["left"].T), gi, pp, rng.standard_normal((ny - 2, 2))),
                m.ElasticityAntiBounceBack(tuple(b["right"].T), gi, pp, rng.standard_normal((ny - 2, 2))),
                m.ElasticityAntiBounceBack(tuple(b["bottom"].T), gi, pp, rng.standard_normal((nx - 2, 2))),
                m.ElasticityAntiBounceBack(tuple(b["top"].T), gi, pp, rng.standard_normal((nx - 2, 2)))]

    def halfway(m, lat, gi, pp, nx, ny):
        b = bbox(nx, ny)
        walls = np.concatenate((b["left"], b["right"], b["top"], b["bottom"]))
        return [m.ElasticityBounceBack(tuple(walls.T), gi, pp, np.array([0.3, -0.2]))]

    def terz_el(m, lat, gi, pp, nx, ny):
        b = bbox(nx, ny)
        _, _, AntiBB = corner_fixed_classes(m)
        T = np.stack((np.full((ny,), -1.0), np.zeros((ny,))), axis=-1)
        return [m.ElasticityBounceBackFullway(tuple(b["left"].T), gi, pp), AntiBB(tuple(b["right"].T), gi, pp, T)]

    def adr_anti(m, lat, gi, pp, nx, ny):
        b = bbox(nx, ny)
        walls = np.concatenate((b["left"], b["right"], b["top"], b["bottom"]))
        return [m.ADR_AntiBounceBack(tuple(walls.T), gi, pp, rho=0.7)]

    def adr_mixed(m, lat, gi, pp, nx, ny):
        b = bbox(nx, ny)
        BB, AntiBB, _ = corner_fixed_classes(m)
        return [BB(tuple(b["bottom"].T), gi, pp), AntiBB(tuple(b["top"].T), gi, pp),
                m.ADR_EquilibriumBC(tuple(b["left"].T), gi, pp, rho=0.25)]

    def cavity(m, lat, gi, pp, nx, ny):
        b = bbox(nx, ny)
        walls = np.concatenate((b["left"], b["right"], b["bottom"]))
        vel = np.zeros(b["top"].shape)
        vel[:, 0] = 0.1
        return [m.BounceBack(tuple(walls.T), gi, pp),
                m.EquilibriumBC(tuple(b["top"].T), gi, pp, np.ones((len(b["top"]), 1)), vel)]

    return [("dirichlet_fullway", 8, 10, 9, dirichlet_full), ("neumann_antibb", 8, 10, 9, neumann),
            ("halfway_bb", 8, 9, 8, halfway), ("terzaghi_elasticity", 8, 12, 4, terz_el),
            ("adr_anti_rho", 9, 10, 9, adr_anti), ("adr_mixed", 9, 11, 10, adr_mixed),
            ("lid_driven_cavity", 9, 10, 9, cavity)]


@pytest.mark.parametrize("name,q,nx,ny,builder", _scenarios(), ids=[s[0] for s in _scenarios()])
def test_compiled_rules_match_oracle(name, q, nx, ny, builder):
    olat = O.LatticeD2Q8("f64/f64") if q == 8 else O.LatticeD2Q9("f64/f64")
    glat = GL.LatticeD2Q8("f64/f64") if q == 8 else GL.LatticeD2Q9("f64/f64")
    opp = O.Policy("f64/f64")
    gpp = GB.PrecisionPolicy(np.float64, np.float64)
    obcs = _prep(builder(O, olat, {"nx": nx, "ny": ny, "nz": 0, "dim": 2, "lattice": olat}, opp, nx, ny),
                 nx, ny, olat, create_grid_mask)
    gbcs = _prep(builder(G, glat, {"nx": nx, "ny": ny, "nz": 0, "dim": 2, "lattice": glat}, gpp, nx, ny),
                 nx, ny, glat, GB.grid_mask)
    rng = np.random.default_rng(42)
    for step in ("PostCollision", "PostStreaming"):
        rules = compile_rules(gbcs, nx, ny, q, torch.float64, "cpu", step=step)
        fout = rng.standard_normal((nx, ny, q))
        fin = rng.standard_normal((nx, ny, q))
        ref = apply_bc_list(obcs, fout, fin, step)
        if rules.count == 0:
            assert np.array_equal(ref, fout)
            continue
        cx, cy = rules.cells[:, 0], rules.cells[:, 1]
        got = evaluate_rules(rules, fout[cx, cy], fin[cx, cy])
        np.testing.assert_allclose(got, ref[cx, cy], rtol=0, atol=1e-14)
        mask = np.ones((nx, ny), bool)
        mask[cx, cy] = False
        assert np.array_equal(ref[mask], fout[mask])


def test_rest_population_quirk_of_adr_antibb():
    """The reference's zero-padded ``imissing/iknown`` make ADR anti-bounce-back
    rewrite the D2Q9 rest population as ``-f*_0`` plus, with ``rho``, one
    ``2 w_0 rho`` per non-missing direction (scatter-add of duplicates)."""
    nx, ny = 8, 6
    glat = GL.LatticeD2Q9("f64/f64")
    gi = {"nx": nx, "ny": ny, "nz": 0, "dim": 2, "lattice": glat}
    left = np.array([[0, i] for i in range(ny)])
    bcs = _prep([GD.ADR_AntiBounceBack(tuple(left.T), gi, GB.PrecisionPolicy(np.float64, np.float64), rho=1.0)],
                nx, ny, glat, GB.grid_mask)
    rules = compile_rules(bcs, nx, ny, 9, torch.float64, "cpu", step="PostStreaming")
    r = list(map(tuple, rules.cells)).index((1, 2))    # a straight-wall cell
    assert rules.code_np[r, 0] == 9 + 0                  # -src[0]
    n_missing = int(bcs[0].imissingMask[list(map(tuple, np.array(bcs[0].indices).T)).index((1, 2))].sum())
    assert np.isclose(rules.cst_np[r, 0], (9 - n_missing) * 2 * 4.0 / 9.0)


def test_non_local_bc_is_rejected():
    class Shifty(GB.BoundaryCondition):
        def apply(self, fout, fin):
            return fout[(np.asarray(self.indices[0]) + 1) % 6, np.asarray(self.indices[1])]
    lat = GL.LatticeD2Q8("f64/f64")
    gi = {"nx": 6, "ny": 6, "nz": 0, "dim": 2, "lattice": lat}
    bc = Shifty((np.array([2, 3]), np.array([1, 1])), gi, GB.PrecisionPolicy(np.float64, np.float64))
    bc.create_local_mask_and_normal_arrays(GB.grid_mask(6, 6, lat, None))
    with pytest.raises(NotImplementedError):
        compile_rules([bc], 6, 6, 8, torch.float64, "cpu", step="PostStreaming")


@pytest.mark.parametrize("name,q,nx,ny,builder", _scenarios(), ids=[s[0] for s in _scenarios()])
def test_push_words_reproduce_stream_then_rules(name, q, nx, ny, builder):
    """The collide-and-push sweep's per-cell push words: pushing every
    post-collision population except the flagged directions, then letting each
    rule cell write the directions its post-streaming rules rebuild, writes every
    output exactly once and equals streaming followed by the rules."""
    glat = GL.LatticeD2Q8("f64/f64") if q == 8 else GL.LatticeD2Q9("f64/f64")
    gpp = GB.PrecisionPolicy(np.float64, np.float64)
    gbcs = _prep(builder(G, glat, {"nx": nx, "ny": ny, "nz": 0, "dim": 2, "lattice": glat}, gpp, nx, ny),
                 nx, ny, glat, GB.grid_mask)
    rules = compile_rules(gbcs, nx, ny, q, torch.float64, "cpu", step="PostStreaming")
    if rules.count == 0:
        return
    keep = 2 * q + 1
    if rules.push is None:       # a "current value" code transforms the streamed value: row-marching sweep
        assert np.any(rules.code_np == keep + 1) or np.any((rules.code_np == keep) & (rules.cst_np != 0))
        return
    c = np.asarray(glat.c, dtype=np.int64)
    rng = np.random.default_rng(5)
    post = rng.standard_normal((nx, ny, q))
    stream = np.stack([np.roll(post[..., i], (c[0, i], c[1, i]), axis=(0, 1)) for i in range(q)], -1)
    cx, cy = rules.cells[:, 0], rules.cells[:, 1]
    ref = stream.copy()
    ref[cx, cy] = evaluate_rules(rules, stream[cx, cy], post[cx, cy])
    words = rules.push.numpy().view(np.uint32).reshape(ny, nx).T
    out = np.zeros_like(post)
    count = np.zeros((nx, ny, q), dtype=np.int64)
    for x in range(nx):
        for y in range(ny):
            for i in range(q):
                if not (words[x, y] >> i) & 1:
                    z = ((x + c[0, i]) % nx, (y + c[1, i]) % ny)
                    out[z + (i,)] = post[x, y, i]
                    count[z + (i,)] += 1
    assert np.array_equal(((words >> 16) & 1).astype(bool)[cx, cy], np.ones(len(cx), bool))
    assert int(((words >> 16) & 1).sum()) == rules.count
    for r, (x, y) in enumerate(zip(cx, cy)):
        for d in range(q):
            code = int(rules.code_np[r, d])
            if code != keep:
                k = code if code < q else (code - q if code < 2 * q else 0)
                base = post[x, y, k] if code < q else (-post[x, y, k] if code < 2 * q else 0.0)
                out[x, y, d] = base + rules.cst_np[r, d]
                count[x, y, d] += 1
    assert np.all(count == 1)
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-14)
