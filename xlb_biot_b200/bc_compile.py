"""Compile an ordered list of boundary-condition objects into per-cell rules.

Every boundary condition of the Biot path is, cell by cell, an affine map of
the populations it reads (``fout`` = collision output or streamed values, and
``fin`` = the step input or post-collision values).  Applying a list of them in
order (``apply_bc``, ``src/elasticity.py:1061-1091``) is again affine per cell.
This module finds that map by probing the objects' own ``apply`` methods with
basis vectors once, then checks that every output direction is
``+-base + constant`` with ``base`` one of {same direction of fout, one
direction of fin, zero}.  The result is uploaded as a CSR-by-row rule table
(``XlbbRules`` in ``include/xlbb.h``) and applied inside the sweep kernels.

A random self-check at compile time compares the compiled rules with the
direct application of the BC list, so non-local or non-affine user BCs are
rejected instead of silently mis-compiled.
"""
import numpy as np
import torch

from . import _lib
from .boundary_conditions import apply_in_order


class CompiledRules:
    """Device-resident rule table of one grid and one phase."""

    def __init__(self, q, ny, cells, code, cst, dtype, device, nx=None, push=False, shape=None, cells_nd=None):
        """``cells``: (x, row) of every rule cell, row = y (2D) or y + ny * z
        (3D, ``shape`` = (nx, ny, nz)); ``cells_nd``: the same cells as (x, y[, z])."""
        self.q = q
        self.count = len(cells)
        self.nx = int(nx) if nx is not None else (int(cells[:, 0].max()) + 1 if len(cells) else 1)
        self.shape = tuple(shape) if shape is not None else (self.nx, ny)
        self.cells_nd = np.asarray(cells_nd) if cells_nd is not None else np.asarray(cells)
        order = np.lexsort((cells[:, 0], cells[:, 1])) if self.count else np.zeros(0, dtype=np.int64)
        cells = cells[order]
        self.cells = cells
        self.cells_nd = self.cells_nd[order] if self.count else self.cells_nd
        self.code_np = code[order]
        self.cst_np = cst[order]
        row_ptr = np.zeros(ny + 1, dtype=np.int32)
        if self.count:
            np.add.at(row_ptr, cells[:, 1] + 1, 1)
        row_ptr = np.cumsum(row_ptr).astype(np.int32)
        # one bit per cell and the index of the first rule of every 32-cell word:
        # the sweeps find a cell's rule as word_base + popcount(bits below it)
        self.words_per_row = (self.nx + 31) // 32
        if self.count:
            words = cells[:, 1] * self.words_per_row + cells[:, 0] // 32
            mask = np.zeros(ny * self.words_per_row, dtype=np.uint64)
            np.bitwise_or.at(mask, words, (np.uint64(1) << (cells[:, 0] % 32).astype(np.uint64)))
            first = np.full(ny * self.words_per_row, self.count, dtype=np.int64)
            np.minimum.at(first, words, np.arange(self.count))
            word_base = np.minimum.accumulate(first[::-1])[::-1].astype(np.int32)
            self.row_ptr = torch.as_tensor(row_ptr, device=device)
            self.cell_x = torch.as_tensor(cells[:, 0].astype(np.int32), device=device)
            self.code = torch.as_tensor(self.code_np.astype(np.uint8).reshape(-1), device=device)
            self.cst = torch.as_tensor(self.cst_np.reshape(-1), device=device).to(dtype)
            self.mask = torch.as_tensor(mask.astype(np.uint32).view(np.int32), device=device)
            self.word_base = torch.as_tensor(word_base, device=device)
        else:
            self.row_ptr = self.cell_x = self.code = self.cst = self.mask = self.word_base = None
        self.push = self._push_words(ny, device) if push and self.count else None

    def _push_words(self, ny, device):
        """Per-cell word of the collide-and-push sweep for post-streaming rules:
        bit d of cell x is set when x + c_d is a rule cell whose direction d is
        rebuilt from that cell's own values (source / zero codes), bit 16 on
        rule cells.  None when a "current value" code transforms the streamed
        value (negated, or with a constant): that sweep cannot apply it."""
        q, nx = self.q, self.nx
        keep, neg_keep = 2 * q + 1, 2 * q + 2
        code = self.code_np
        if np.any(code == neg_keep) or np.any((code == keep) & (self.cst_np != 0)):
            return None
        from .lattice import LatticeD2Q8, LatticeD2Q9, LatticeD3Q19, LatticeD3Q27
        lat = {8: LatticeD2Q8, 9: LatticeD2Q9, 19: LatticeD3Q19, 27: LatticeD3Q27}[q]
        c = np.asarray(lat("f64/f64").c, dtype=np.int64)
        shape = self.shape
        dim = len(shape)
        z = self.cells_nd.astype(np.int64)
        lin = np.ravel_multi_index(tuple(z[:, k] for k in range(dim)), shape, order="F")
        words = np.zeros(int(np.prod(shape)), dtype=np.uint32)
        # bit d: direction d of the cell is rebuilt at its destination; the flag
        # bit marks a rule cell (16 for the 2D lattices, 31 for the 3D ones)
        flag = np.uint32(1 << (16 if q <= 16 else 31))
        np.bitwise_or.at(words, lin, flag)
        for d in range(q):
            rebuilt = code[:, d] != keep
            src = tuple((z[rebuilt, k] - c[k, d]) % shape[k] for k in range(dim))
            np.bitwise_or.at(words, np.ravel_multi_index(src, shape, order="F"), np.uint32(1 << d))
        return torch.as_tensor(words.view(np.int32), device=device)

    def struct(self):
        if self.count == 0:
            return _lib.Rules(0, None, None, None, None, None, None, self.words_per_row, None)
        return _lib.Rules(self.count, self.row_ptr.data_ptr(), self.cell_x.data_ptr(), self.code.data_ptr(),
                          self.cst.data_ptr(), self.mask.data_ptr(), self.word_base.data_ptr(),
                          self.words_per_row, self.push.data_ptr() if self.push is not None else None)

    def restricted(self, nx, ny, dtype, device):
        """The same rules on a smaller grid: cells outside it are dropped (the
        reference's coarse-level gradient gathers clamp and scatters drop)."""
        keep = (self.cells[:, 0] < nx) & (self.cells[:, 1] < ny) if self.count else np.zeros(0, bool)
        return CompiledRules(self.q, ny, self.cells[keep], self.code_np[keep], self.cst_np[keep], dtype, device, nx,
                             push=self.push is not None)


def _run(bcs, fout, fin, step, names):
    return apply_in_order(bcs, fout, fin, implementation_step=step, names=names)


def compile_rules(bcs, nx, ny, q, dtype, device, step=None, names=None, check=True, nz=0):
    """Rules of ``bcs`` for one phase: ``step`` in {"PostCollision",
    "PostStreaming"} (apply_bc semantics) or ``names`` (the gradient's filter);
    ``nz > 0``: a three-dimensional grid (rows y + ny * z)."""
    shape = (nx, ny) if nz == 0 else (nx, ny, nz)
    dim = len(shape)
    rows = ny * (nz if nz else 1)
    if step is not None:
        active = [bc for bc in bcs if bc.implementationStep == step]
    else:
        active = [bc for bc in bcs if bc.name in names]
    cells = []
    for bc in active:
        idx = np.array(bc.indices, dtype=np.int64).reshape(dim, -1).T
        ok = np.logical_and.reduce([(idx[:, k] >= 0) & (idx[:, k] < shape[k]) for k in range(dim)])
        cells.append(idx[ok])
    if not cells or sum(len(c) for c in cells) == 0:
        return CompiledRules(q, rows, np.zeros((0, 2), np.int64), np.zeros((0, q), np.uint8), np.zeros((0, q)),
                             dtype, device, nx, shape=shape, cells_nd=np.zeros((0, dim), np.int64))
    cells = np.unique(np.vstack(cells), axis=0)
    at = tuple(cells[:, k] for k in range(dim))

    def probe(fout_vec, fin_vec):
        fout = np.zeros(shape + (q,))
        fin = np.zeros(shape + (q,))
        if fout_vec is not None:
            fout[at] = fout_vec
        if fin_vec is not None:
            fin[at] = fin_vec
        return _run(bcs, fout, fin, step, names)[at]

    c0 = probe(None, None)
    eye = np.eye(q)
    A = np.stack([probe(eye[k], None) - c0 for k in range(q)], axis=-1)   # (n, q_out, q_in)
    B = np.stack([probe(None, eye[k]) - c0 for k in range(q)], axis=-1)
    # (1 + c) - c is not exactly 1 in floating point: snap the probed
    # coefficients to integers (a genuine scaling survives and is rejected below)
    A = np.where(np.abs(A - np.round(A)) < 1e-9, np.round(A), A)
    B = np.where(np.abs(B - np.round(B)) < 1e-9, np.round(B), B)

    n = len(cells)
    code = np.empty((n, q), dtype=np.uint8)
    KEEP, NEG_KEEP, ZERO = 2 * q + 1, 2 * q + 2, 2 * q
    for d in range(q):
        a, b = A[:, d, :], B[:, d, :]
        a_other = a.copy()
        a_other[:, d] = 0
        nz_a = np.abs(a_other).sum(axis=1) > 0
        nb = (np.abs(b) > 0).sum(axis=1)
        ad = a[:, d]
        if np.any(nz_a):
            raise NotImplementedError("boundary rule mixes streamed directions; not representable")
        both = (ad != 0) & (nb > 0)
        if np.any(both) or np.any(nb > 1):
            raise NotImplementedError("boundary rule combines several sources; not representable")
        bk = np.argmax(np.abs(b), axis=1)
        bv = b[np.arange(n), bk]
        cd = np.full(n, ZERO, dtype=np.int64)
        cd[ad == 1] = KEEP
        cd[ad == -1] = NEG_KEEP
        cd[bv == 1] = bk[bv == 1]
        cd[bv == -1] = q + bk[bv == -1]
        bad = ((ad != 0) & (np.abs(ad) != 1)) | ((nb == 1) & (np.abs(bv) != 1))
        if np.any(bad):
            raise NotImplementedError("boundary rule scales a population; not representable")
        code[:, d] = cd
    # push words: post-streaming rules (collide-and-push sweep, transposed sweeps)
    # and the gradient's rules (its transposed stencil gathers the same way)
    cells2 = cells[:, :2].copy()
    if dim == 3:
        cells2[:, 1] = cells[:, 1] + ny * cells[:, 2]
    rules = CompiledRules(q, rows, cells2, code, c0, dtype, device, nx,
                          push=(step == "PostStreaming" or step is None), shape=shape, cells_nd=cells)
    if check:
        _self_check(bcs, shape, q, step, names, rules)
    return rules


def evaluate_rules(rules, cur, src):
    """Apply compiled rules to per-cell vectors (host; used by the compile-time
    self-check): ``cur``/``src`` are (n, q) arrays in ``rules.cells`` order."""
    q = rules.q
    code = rules.code_np.astype(np.int64)
    out = np.empty_like(cur)
    rows = np.arange(len(code))
    for d in range(q):
        cdv = code[:, d]
        k = np.where(cdv < q, cdv, np.where(cdv < 2 * q, cdv - q, 0))
        base = np.where(cdv < q, src[rows, k], np.where(cdv < 2 * q, -src[rows, k],
                        np.where(cdv == 2 * q, 0.0, np.where(cdv == 2 * q + 1, cur[:, d], -cur[:, d]))))
        out[:, d] = base + rules.cst_np[:, d]
    return out


def apply_rules_device(rules, fout, fin):
    """Apply compiled rules to device fields of shape (nx, ny, q) (``apply_bc``
    outside the fused sweep, e.g. to return post-collision populations)."""
    out = fout.clone()
    if rules.count == 0:
        return out
    q = rules.q
    at = tuple(torch.as_tensor(rules.cells_nd[:, k], device=fout.device) for k in range(rules.cells_nd.shape[1]))
    cur, src = fout[at], fin[at]
    code = rules.code.view(-1, q).long()
    k = torch.where(code < q, code, torch.where(code < 2 * q, code - q, torch.zeros_like(code)))
    s = torch.gather(src, 1, k)
    base = torch.where(code < q, s, torch.where(code < 2 * q, -s, torch.where(
        code == 2 * q, torch.zeros_like(s), torch.where(code == 2 * q + 1, cur, -cur))))
    out[at] = base + rules.cst.view(-1, q).to(fout.dtype)
    return out


def _self_check(bcs, shape, q, step, names, rules):
    if rules.count == 0:
        return
    rng = np.random.default_rng(1234)
    fout = rng.standard_normal(tuple(shape) + (q,))
    fin = rng.standard_normal(tuple(shape) + (q,))
    ref = _run(bcs, fout.copy(), fin, step, names)
    at = tuple(rules.cells_nd[:, k] for k in range(len(shape)))
    got = evaluate_rules(rules, fout[at], fin[at])
    scale = max(1.0, float(np.abs(ref[at]).max()))
    if not np.allclose(got, ref[at], rtol=0, atol=1e-12 * scale):
        raise NotImplementedError("boundary conditions are not cell-local affine maps; cannot compile them")
    mask = np.ones(tuple(shape), dtype=bool)
    mask[at] = False
    if not np.array_equal(ref[mask], fout[mask]):
        raise NotImplementedError("boundary conditions modify cells outside their index sets")
