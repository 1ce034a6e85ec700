"""The three-dimensional fluid sweep's host side on the CPU (no GPU).

``xlbb_fluid3_sweep`` collides every cell, applies the compiled PostCollision
rules, pushes each post-collision population to the cell it streams to unless
the cell's push word flags the direction, and lets every rule cell (flag bit
31) write the directions its PostStreaming rules rebuild.  Here that sweep is
emulated in NumPy from the product's compiled rules and push words of the
lid-driven cavity of ``examples/performance/MLUPS3d.py`` (D3Q19 and D3Q27) and
must equal the oracle's step (``src/base.py:809-846``: collision, PostCollision
BCs, streaming, PostStreaming BCs) to rounding, with every output written
exactly once.
"""
import numpy as np
import pytest
import torch

import oracle.api as O
import xlb_biot_b200.boundary_conditions as GB
import xlb_biot_b200.lattice as GL
from xlb_biot_b200.bc_compile import compile_rules, evaluate_rules
from xlb_biot_b200.workloads import lid_driven_cavity_3d


def _product_bcs(osim, lattice_name):
    """The product's BC objects on the oracle solver's boundary indices."""
    lat = getattr(GL, "Lattice" + lattice_name)("f64/f64")
    gi = {"nx": osim.nx, "ny": osim.ny, "nz": osim.nz, "dim": 3, "lattice": lat}
    pp = GB.PrecisionPolicy(np.float64, np.float64)
    bcs = []
    for bc in osim.BCs:
        idx = tuple(np.asarray(i) for i in bc.indices)
        if type(bc).__name__ == "BounceBack":
            bcs.append(GB.BounceBack(idx, gi, pp))
        else:                    # the lid: the equilibrium of rho = 1, u = (0.1, 0, 0)
            n = len(idx[0])
            u = np.zeros((n, 3))
            u[:, 0] = 0.1
            bcs.append(GB.EquilibriumBC(idx, gi, pp, np.ones((n, 1)), u))
    gm = GB.grid_mask(osim.nx, osim.ny, lat, GB.solid_halo_voxels(bcs), nz=osim.nz)
    for bc in bcs:
        bc.create_local_mask_and_normal_arrays(gm)
    return bcs, lat


def _bgk(f, c, w, omega):
    """The kernel's collision arithmetic (BGK, second-order equilibrium)."""
    rho = f.sum(-1, keepdims=True)
    u = (f @ c.T) / rho
    cu = 3.0 * (u @ c)
    usqr = 1.5 * (u * u).sum(-1, keepdims=True)
    feq = rho * w * (1.0 + cu * (1.0 + 0.5 * cu) - usqr)
    return f - omega * (f - feq)


@pytest.mark.parametrize("lattice_name", ["D3Q19", "D3Q27"])
def test_push_sweep_emulation_matches_oracle_step(lattice_name):
    nx, ny, nz = 6, 5, 7
    C, om = lid_driven_cavity_3d(O)
    olat = getattr(O, "Lattice" + lattice_name)("f64/f64")
    osim = C(lattice=olat, omega=om(nx), nx=nx, ny=ny, nz=nz, precision="f64/f64")
    q = olat.q
    rng = np.random.default_rng(11)
    f = osim.assign_fields_sharded() * (1.0 + 0.05 * rng.standard_normal((nx, ny, nz, q)))
    ref, _ = osim.step(f, 0)

    bcs, glat = _product_bcs(osim, lattice_name)
    pc = compile_rules(bcs, nx, ny, q, torch.float64, "cpu", step="PostCollision", nz=nz)
    ps = compile_rules(bcs, nx, ny, q, torch.float64, "cpu", step="PostStreaming", nz=nz)
    assert ps.push is not None and ps.count > 0
    c = np.asarray(glat.c, dtype=np.int64)
    w = np.asarray(glat.w, dtype=np.float64)

    post = _bgk(f, c.astype(np.float64), w, om(nx))
    if pc.count:
        x, y, z = pc.cells_nd.T
        post[x, y, z] = evaluate_rules(pc, post[x, y, z], f[x, y, z])
    # push words are indexed (y + ny z) nx + x
    words = ps.push.numpy().view(np.uint32).reshape(nz, ny, nx).transpose(2, 1, 0)
    out = np.zeros_like(post)
    count = np.zeros(post.shape, dtype=np.int64)
    X, Y, Z = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    for i in range(q):
        send = ((words >> i) & 1) == 0
        dst = ((X + c[0, i]) % nx, (Y + c[1, i]) % ny, (Z + c[2, i]) % nz)
        out[dst[0][send], dst[1][send], dst[2][send], i] = post[X[send], Y[send], Z[send], i]
        np.add.at(count, (dst[0][send], dst[1][send], dst[2][send], np.full(int(send.sum()), i)), 1)
    flag = ((words >> 31) & 1).astype(bool)
    x, y, z = ps.cells_nd.T
    assert flag[x, y, z].all() and int(flag.sum()) == ps.count
    keep = 2 * q + 1
    for r in range(ps.count):
        for d in range(q):
            code = int(ps.code_np[r, d])
            if code != keep:
                k = code if code < q else (code - q if code < 2 * q else 0)
                base = post[x[r], y[r], z[r], k] if code < q else (-post[x[r], y[r], z[r], k] if code < 2 * q
                                                                    else 0.0)
                out[x[r], y[r], z[r], d] = base + ps.cst_np[r, d]
                count[x[r], y[r], z[r], d] += 1
    assert np.array_equal(count, np.ones_like(count))
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-14)


def test_push_word_flag_bit_by_lattice():
    """The 2-D sweeps flag rule cells with bit 16 (q <= 16), the 3-D sweep with
    bit 31 (q = 19 and 27 use bits 0 .. 26 for directions)."""
    nx, ny, nz = 4, 4, 4
    C, om = lid_driven_cavity_3d(O)
    osim = C(lattice=O.LatticeD3Q27("f64/f64"), omega=om(nx), nx=nx, ny=ny, nz=nz, precision="f64/f64")
    bcs, _ = _product_bcs(osim, "D3Q27")
    ps = compile_rules(bcs, nx, ny, 27, torch.float64, "cpu", step="PostStreaming", nz=nz)
    words = ps.push.numpy().view(np.uint32)
    assert int(((words >> 31) & 1).sum()) == ps.count
    assert not np.any(words & np.uint32(((1 << 31) - 1) & ~((1 << 27) - 1)))
