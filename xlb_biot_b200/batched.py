"""Batched multigrid elasticity: many independent periodic instances.

The reference solves one elasticity problem per ``LBMElasticity`` object and
dispatches every sweep separately.  ``BatchedElasticity`` advances a whole
batch of periodic D2Q8 problems of different sizes and Lame parameters with
the reference's V-cycle (``src/elasticity.py:1221-1312``: damped smoothing,
residual, block-sum restriction, coarse solve from zero, injection), one
launch per sweep for all instances (``xlbb_batched_elast_sweep``: CTAs loop
over a work list of tiles) and the whole V-cycle captured once as a CUDA graph.
Per-instance FP64 residual norms (level-0 interior, as the reference's
``_mg_step`` returns) are reduced on the device; the host reads them once per
cycle to decide convergence.

Every instance may have its own number of levels (``levels="auto"`` halves each
grid down to a coarsest side of 3 to 5 cells, which keeps the V-cycle's
convergence factor independent of the grid size).  At a level that is the
coarsest one of some instances, those instances only smooth (the reference's
coarsest level: 2 * k_smooth damped sweeps), which the shared smoothing
launches already do; the residual, restriction and prolongation launches cover
the instances that go deeper.  With ``coarsest_precision="f64"`` each
instance's own coarsest level is FP64, so a level can hold an FP32 and an FP64
group, each with its own launches.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._common import require_finite
from .fields import pitch_for

_ALIGN = 64   # elements; keeps every instance's planes 256-byte aligned


def balanced_block_map(cells, per_block=1024):
    """Block map of ``xlbb_batched_prolong_add_map``: ceil(cells[k] / per_block)
    consecutive blocks for instance k, each the pair (k, first cell index).
    Returns (int32 array (nblocks, 2), int32 begin array (len(cells) + 1):
    instance k's blocks are begin[k] .. begin[k + 1])."""
    blocks, begin = [], [0]
    for k, n in enumerate(cells):
        blocks += [(k, e) for e in range(0, int(n), per_block)]
        begin.append(len(blocks))
    return np.asarray(blocks, dtype=np.int32).reshape(-1, 2), np.asarray(begin, dtype=np.int32)


def auto_levels(nx, ny, min_side=3):
    """Levels of the factor-2 hierarchy of an ``nx x ny`` grid whose coarsest
    side is the smallest one that is still >= ``min_side``."""
    levels = 1
    while nx % 2 == 0 and ny % 2 == 0 and min(nx, ny) // 2 >= min_side:
        nx, ny, levels = nx // 2, ny // 2, levels + 1
    return levels


class _Arena:
    """One buffer holding a field of ``c`` planes for the instances ``ids``
    (global instance numbers) of one level."""

    def __init__(self, ids, shapes, c, dtype, device):
        self.c = c
        self.pos = {g: k for k, g in enumerate(ids)}
        self.offsets, self.pitch, self.plane, self.shapes = [], [], [], []
        off = 0
        for g in ids:
            nx, ny = shapes[g]
            p = pitch_for(nx, dtype)
            pl = p * ny
            self.offsets.append(off)
            self.pitch.append(p)
            self.plane.append(pl)
            self.shapes.append((nx, ny))
            off += -(-c * pl // _ALIGN) * _ALIGN
        self.buf = torch.zeros(max(off, 1), dtype=dtype, device=device)

    def ptr(self, g):
        return self.buf.data_ptr() + self.offsets[self.pos[g]] * self.buf.element_size()

    def view(self, g):
        k = self.pos[g]
        nx, ny = self.shapes[k]
        return self.buf[self.offsets[k]:].as_strided((nx, ny, self.c), (1, self.pitch[k], self.plane[k]))


class _Launch:
    """Descriptor array + tile work list of one batched sweep launch; ``vec``:
    every instance qualifies for the four-column kernel."""

    def __init__(self, desc, tiles, ntiles, ctas, dcode, begin=None, vec=False):
        self.desc, self.tiles, self.ntiles, self.ctas, self.dcode, self.begin = desc, tiles, ntiles, ctas, dcode, begin
        self.vec = vec


class BatchedElasticity:
    """A batch of periodic elasticity problems solved by batched V-cycles.

    ``sizes``: list of (nx, ny); ``lams``, ``mus``: Lame parameters per
    instance; ``forces``: list of (nx, ny, 2) body forces (level 0 only, as in
    the reference).  ``levels``: one count for all instances, a list with one
    count per instance, or ``"auto"`` (``auto_levels`` of each size); every
    instance needs at least 2.  ``gamma``, ``k_smooth`` as the reference's
    ``MG_relaxation``, ``MG_n_smoothing`` (k_smooth even).
    ``coarsest_precision="f64"`` runs each instance's coarsest level in FP64;
    ``residual_precision="f64"`` computes the level-0 residual sweep of an FP32
    batch in FP64 arithmetic (FP32 storage).  ``vectorized``: FP32 launches
    whose instances all have widths divisible by 4 use the four-column kernel
    (``xlbb_batched_elast_sweep4``; same results).  ``persistent_tail``: from
    the top-most level where an instance's remaining levels fit in
    ``tail_smem`` bytes of shared memory, its V-cycle is finished by one
    launch for all instances (``xlbb_batched_tail``: a CTA per instance, the
    levels in shared memory; same results as the level-by-level launches).
    ``remove_mean``: ``solve`` ends with ``remove_mean_moment`` (the rigid
    displacement mode, zero in exact arithmetic, reset after FP32 drift)."""

    def __init__(self, sizes, lams, mus, forces, levels=5, gamma=0.75, k_smooth=2, precision="f32/f32",
                 coarsest_precision=None, residual_precision=None, strip_rows=16, ctas_per_sm=4, vectorized=True,
                 persistent_tail=True, tail_smem=100 * 1024, remove_mean=True):
        _lib.require_cuda()
        lib = _lib.lib()
        if k_smooth % 2:
            raise ValueError("the batched V-cycle keeps ping-pong parity: k_smooth must be even")
        self.n = len(sizes)
        sizes = [(int(nx), int(ny)) for nx, ny in sizes]
        if levels == "auto":
            lv = [auto_levels(nx, ny) for nx, ny in sizes]
        elif isinstance(levels, (list, tuple, np.ndarray)):
            lv = [int(v) for v in levels]
        else:
            lv = [int(levels)] * self.n
        if len(lv) != self.n or min(lv) < 2:
            raise ValueError("every instance needs at least 2 multigrid levels")
        for (nx, ny), L in zip(sizes, lv):
            den = 2 ** (L - 1)
            if nx % den or ny % den:
                raise ValueError("every size must be divisible by 2**(levels-1)")
        self.instance_levels = lv
        self.levels = max(lv)
        self.gamma, self.k_smooth = float(gamma), k_smooth
        self.lams, self.mus = [float(v) for v in lams], [float(v) for v in mus]
        dt = torch.float32 if precision == "f32/f32" else torch.float64
        coarse_dt = torch.float64 if coarsest_precision == "f64" else dt
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        self.ctas_per_sm = ctas_per_sm

        def dtype_of(g, l):
            return coarse_dt if l == lv[g] - 1 else dt

        # tail_start[g]: the first level of instance g handled by the persistent
        # tail (lv[g]: none); the level-by-level launches stop above it
        self.tail_start = list(lv)
        if persistent_tail:
            for g, (nx, ny) in enumerate(sizes):
                for l in range(1, lv[g]):
                    b = lib.xlbb_batched_tail_smem(_lib.dtype_code(dt), _lib.dtype_code(coarse_dt), nx >> l, ny >> l,
                                                   lv[g] - l)
                    if 0 < b <= tail_smem:
                        self.tail_start[g] = l
                        break
        self.batched_depth = max(self.tail_start)

        def act(g, l):
            return self.tail_start[g] > l

        # groups[l]: dtype -> instance ids at level l;  deeper[l]: ids that recurse below l
        self.groups, self.deeper, self.shapes = [], [], []
        for l in range(self.levels):
            shapes = {g: (sizes[g][0] >> l, sizes[g][1] >> l) for g in range(self.n) if lv[g] > l}
            self.shapes.append(shapes)
            grp = {}
            for g in sorted(shapes):
                grp.setdefault(dtype_of(g, l), []).append(g)
            self.groups.append(grp)
            self.deeper.append([g for g in sorted(shapes) if lv[g] > l + 1])
        self.X, self.Y, self.R = [], [], []
        for l in range(self.levels):
            self.X.append({d: _Arena(ids, self.shapes[l], 8, d, dev) for d, ids in self.groups[l].items()})
            self.Y.append({d: _Arena(ids, self.shapes[l], 8, d, dev) for d, ids in self.groups[l].items()})
            self.R.append({d: _Arena(ids, self.shapes[l], 8, d, dev) for d, ids in self.groups[l].items()}
                          if l > 0 else None)
        # residual buffers of the instances that recurse (always the bulk dtype)
        self.RES = [_Arena(self.deeper[l], self.shapes[l], 8, dt, dev) for l in range(self.levels - 1)]
        self.F = _Arena(list(range(self.n)), self.shapes[0], 2, dt, dev)
        for g, f in enumerate(forces):
            self.F.view(g).copy_(torch.as_tensor(np.asarray(f), device=dev))

        def launch(l, ids, d, src, dst, want_begin=False, code=None):
            recs = (_lib.BatchInstance * len(ids))()
            for k, g in enumerate(ids):
                nx, ny = self.shapes[l][g]
                resid = self.R[l][d].ptr(g) if l > 0 else None
                recs[k] = _lib.BatchInstance(src.ptr(g), dst.ptr(g), self.F.ptr(g) if l == 0 else None, resid,
                                             nx, ny, src.pitch[src.pos[g]], src.plane[src.pos[g]],
                                             self.lams[g], self.mus[g])
            code = _lib.dtype_code(d) if code is None else code
            desc = torch.empty(lib.xlbb_batch_desc_bytes(code) * len(ids), dtype=torch.uint8, device=dev)
            _lib.check(lib.xlbb_batch_upload(code, recs, len(ids), ctypes.c_void_p(desc.data_ptr()),
                                             _lib.stream_ptr()), "xlbb_batch_upload")
            tl, begin = [], [0]
            for k, g in enumerate(ids):
                nx, ny = self.shapes[l][g]
                rows = max(1, min(strip_rows, ny))
                nstrip = -(-ny // rows)
                for s in range(nstrip):
                    ys, ye = (s * ny) // nstrip, ((s + 1) * ny) // nstrip
                    for x0 in range(0, nx, 128):
                        tl.append((k, x0, ys, ye))
                begin.append(len(tl))
            tiles = torch.as_tensor(np.asarray(tl, dtype=np.int32).reshape(-1), device=dev)
            b = torch.as_tensor(np.asarray(begin, dtype=np.int32), device=dev) if want_begin else None
            # four-column kernel: FP32 (storage and arithmetic), widths (and so pitches and planes) multiples of 4
            vec = vectorized and code == _lib.XLBB_F32 and all(self.shapes[l][g][0] % 4 == 0 for g in ids)
            return _Launch(desc, tiles, len(tl), min(len(tl), ctas_per_sm * sms), code, b, vec)

        # smoothing launches (X->Y, Y->X) per level and dtype group; residual launch per level
        # (FP32 groups split into the instances the four-column kernel takes and the rest)
        self.smooth_xy, self.smooth_yx, self.res = [], [], []
        for l in range(self.levels):
            parts = []
            for d, ids in self.groups[l].items():
                ids = [g for g in ids if act(g, l)]
                if not ids:
                    continue
                if vectorized and d == torch.float32:
                    q4 = [g for g in ids if self.shapes[l][g][0] % 4 == 0]
                    parts += [(d, p) for p in (q4, [g for g in ids if g not in set(q4)]) if p]
                else:
                    parts.append((d, ids))
            self.smooth_xy.append([launch(l, ids, d, self.X[l][d], self.Y[l][d]) for d, ids in parts])
            self.smooth_yx.append([launch(l, ids, d, self.Y[l][d], self.X[l][d]) for d, ids in parts])
            if l < self.levels - 1:
                acc64 = l == 0 and residual_precision == "f64" and dt == torch.float32
                rids = [g for g in self.deeper[l] if act(g, l)]
                self.res.append(launch(l, rids, dt, self.X[l][dt], self.RES[l], want_begin=(l == 0),
                                       code=_lib.XLBB_F32_ACC64 if acc64 else None) if rids else None)
        if self.deeper[0] != list(range(self.n)):
            raise AssertionError("every instance recurses below level 0")
        # per-instance ranges of the level-0 residual sweep's partials (a partial per warp of each tile)
        self.tile_begin = self.res[0].begin * _lib.XLBB_BATCH_PARTS_PER_TILE
        self.tile_sumsq = torch.zeros(self.res[0].ntiles * _lib.XLBB_BATCH_PARTS_PER_TILE, dtype=torch.float64,
                                      device=dev)
        self.norm2 = torch.zeros(self.n, dtype=torch.float64, device=dev)
        # level-0 coarse correction: per instance [sum corr^2, sum f^2] (FP64)
        self.corr2 = torch.zeros((self.n, 2), dtype=torch.float64, device=dev)
        self._corr_parts = None       # sized below: 2 doubles per block of the level-0 prolongation maps

        def transfers(l, fine, coarse_arenas, d_coarse, src_is_res):
            ids = [g for g in self.deeper[l] if dtype_of(g, l + 1) == d_coarse and act(g, l)]
            if not ids:
                return None
            recs = (_lib.BatchTransfer * len(ids))()
            coarse = coarse_arenas[d_coarse]
            for k, g in enumerate(ids):
                nx, ny = self.shapes[l][g]
                recs[k] = _lib.BatchTransfer(fine.ptr(g), coarse.ptr(g), nx, ny, fine.pitch[fine.pos[g]],
                                             coarse.pitch[coarse.pos[g]], fine.plane[fine.pos[g]],
                                             coarse.plane[coarse.pos[g]])
            raw = bytes(recs)
            return (torch.as_tensor(np.frombuffer(raw, dtype=np.uint8).copy(), device=dev), len(ids),
                    _lib.dtype_code(dt), _lib.dtype_code(d_coarse), ids)

        def prolong_map(t, l):
            blocks, begin = balanced_block_map([self.shapes[l][g][0] * self.shapes[l][g][1] for g in t[4]])
            return (torch.as_tensor(blocks.reshape(-1), device=dev), len(blocks),
                    torch.as_tensor(begin, device=dev))

        self.t_restrict, self.t_prolong = [], []
        for l in range(self.levels - 1):
            dcs = sorted(set(dtype_of(g, l + 1) for g in self.deeper[l]), key=str)
            self.t_restrict.append([t for t in (transfers(l, self.RES[l], self.R[l + 1], d, True) for d in dcs) if t])
            self.t_prolong.append([t + prolong_map(t, l) for t in
                                   (transfers(l, self.X[l][dt], self.X[l + 1], d, False) for d in dcs) if t])
        # row r of corr2 belongs to instance _corr_ids[r] (transfer-list order)
        self._corr_ids = np.asarray([g for t in self.t_prolong[0] for g in t[4]])
        self._corr_parts = torch.zeros(2 * max(t[6] for t in self.t_prolong[0]), dtype=torch.float64, device=dev)
        # the persistent tail's records: top-level right-hand side and correction of every tail instance
        self.tail = None
        tail_ids = [g for g in range(self.n) if self.tail_start[g] < lv[g]]
        if tail_ids:
            recs = (_lib.BatchTail * len(tail_ids))()
            smem = 0
            for k, g in enumerate(tail_ids):
                t = self.tail_start[g]
                d = dtype_of(g, t)
                R, X = self.R[t][d], self.X[t][d]
                nx, ny = self.shapes[t][g]
                recs[k] = _lib.BatchTail(R.ptr(g), X.ptr(g), nx, ny, X.pitch[X.pos[g]], X.plane[X.pos[g]],
                                         lv[g] - t, self.lams[g], self.mus[g])
                if R.pitch[R.pos[g]] != X.pitch[X.pos[g]] or R.plane[R.pos[g]] != X.plane[X.pos[g]]:
                    raise AssertionError("tail right-hand side and correction differ in layout")
                smem = max(smem, lib.xlbb_batched_tail_smem(_lib.dtype_code(dt), _lib.dtype_code(coarse_dt),
                                                            nx, ny, lv[g] - t))
            buf = torch.as_tensor(np.frombuffer(bytes(recs), dtype=np.uint8).copy(), device=dev)
            self.tail = (buf, len(tail_ids), smem, _lib.dtype_code(dt), _lib.dtype_code(coarse_dt))
        # records of xlbb_batched_remove_mean_moment: every instance's level-0 populations
        self.remove_mean = bool(remove_mean)
        self._mean = []
        for d, ids in self.groups[0].items():
            arena = self.X[0][d]
            recs = (_lib.BatchTransfer * len(ids))()
            for k, g in enumerate(ids):
                nx, ny = self.shapes[0][g]
                recs[k] = _lib.BatchTransfer(arena.ptr(g), None, nx, ny, arena.pitch[arena.pos[g]], 0,
                                             arena.plane[arena.pos[g]], 0)
            blocks, begin = balanced_block_map([self.shapes[0][g][0] * self.shapes[0][g][1] for g in ids])
            self._mean.append((torch.as_tensor(np.frombuffer(bytes(recs), dtype=np.uint8).copy(), device=dev),
                               torch.as_tensor(blocks.reshape(-1), device=dev), len(blocks),
                               torch.as_tensor(begin, device=dev), len(ids),
                               torch.zeros(2 * len(blocks), dtype=torch.float64, device=dev),
                               torch.zeros(2 * len(ids), dtype=torch.float64, device=dev), _lib.dtype_code(d)))
        self.launches_per_cycle = 0
        self.graph = None

    def remove_mean_moment(self):
        """Sets the mean first moments of every instance's level-0 populations to
        zero (``xlbb_batched_remove_mean_moment``).  A periodic problem leaves
        the rigid displacement undetermined; the V-cycle from zero with a
        zero-mean force keeps it at zero in exact arithmetic, and this restores
        that invariant after FP32 rounding made it drift (a random walk that
        grows with the number of cycles).  ``solve`` calls it once at the end
        unless the batch was built with ``remove_mean=False``."""
        lib = _lib.lib()
        for rec, mp, nb, begin, ni, parts, sums, code in self._mean:
            _lib.check(lib.xlbb_batched_remove_mean_moment(
                code, ctypes.c_void_p(rec.data_ptr()), ctypes.c_void_p(mp.data_ptr()), nb,
                ctypes.c_void_p(parts.data_ptr()), ctypes.c_void_p(begin.data_ptr()), ni,
                ctypes.c_void_p(sums.data_ptr()), _lib.stream_ptr()), "xlbb_batched_remove_mean_moment")

    # ------------------------------------------------------------------ kernels
    def _sweep(self, l, ln, a, b, sumsq=False, zero_in=False):
        fn = "xlbb_batched_elast_sweep4" if ln.vec else "xlbb_batched_elast_sweep"
        _lib.check(getattr(_lib.lib(), fn)(
            ln.dcode, ctypes.c_void_p(ln.desc.data_ptr()), ctypes.c_void_p(ln.tiles.data_ptr()), ln.ntiles, ln.ctas,
            float(a), float(b), 1 if l == 0 else 0, 1 if l > 0 else 0, 0,
            ctypes.c_void_p(self.tile_sumsq.data_ptr()) if sumsq else None, 1 if zero_in else 0,
            _lib.stream_ptr()), fn)
        self.launches_per_cycle += 1

    def _smooth(self, l, from_zero=False):
        """k_smooth damped sweeps X->Y->X...; ``from_zero``: X holds zeros (a
        coarse level's correction starts from zero), so the first sweep takes
        its input as zero instead of reading a zero-filled X."""
        g = self.gamma
        for k in range(self.k_smooth):
            for ln in (self.smooth_xy[l] if k % 2 == 0 else self.smooth_yx[l]):
                self._sweep(l, ln, 1.0 - g, g, zero_in=from_zero and k == 0)

    def _tail(self):
        buf, count, smem, dcode, ccode = self.tail
        _lib.check(_lib.lib().xlbb_batched_tail(dcode, ccode, ctypes.c_void_p(buf.data_ptr()), count, smem,
                                                self.gamma, self.k_smooth, _lib.stream_ptr()), "xlbb_batched_tail")
        self.launches_per_cycle += 1

    def _level(self, l):
        """Level l of every instance still on the level-by-level launches; at
        the deepest such level the persistent tail runs the rest."""
        self._smooth(l, from_zero=l > 0)
        if l < self.levels - 1 and self.res[l] is not None:
            self._sweep(l, self.res[l], 1.0, -1.0, sumsq=(l == 0))
            if l == 0:
                _lib.check(_lib.lib().xlbb_segment_sum(
                    ctypes.c_void_p(self.tile_sumsq.data_ptr()), ctypes.c_void_p(self.tile_begin.data_ptr()),
                    self.n, ctypes.c_void_p(self.norm2.data_ptr()), _lib.stream_ptr()), "xlbb_segment_sum")
                self.launches_per_cycle += 1
            for buf, cnt, cf, cc, _ in self.t_restrict[l]:
                _lib.check(_lib.lib().xlbb_batched_restrict(cf, cc, ctypes.c_void_p(buf.data_ptr()), cnt,
                                                            _lib.stream_ptr()), "xlbb_batched_restrict")
                self.launches_per_cycle += 1
        if l + 1 < self.batched_depth:
            self._level(l + 1)          # its correction starts from zero (first sweep: zero input)
        elif self.tail is not None:
            self._tail()
        if l < self.levels - 1 and self.res[l] is not None:
            for k, (buf, cnt, cf, cc, _, bmap, nblocks, bbegin) in enumerate(self.t_prolong[l]):
                if l == 0:   # instances of transfer list k occupy rows offset.. of corr2
                    off = sum(t[1] for t in self.t_prolong[0][:k])
                    parts, norms = ctypes.c_void_p(self._corr_parts.data_ptr()), ctypes.c_void_p(
                        self.corr2.data_ptr() + 16 * off)
                    self.launches_per_cycle += 2
                else:
                    parts = norms = None
                    self.launches_per_cycle += 1
                _lib.check(_lib.lib().xlbb_batched_prolong_add_map(
                    cf, cc, ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(bmap.data_ptr()), nblocks, parts,
                    ctypes.c_void_p(bbegin.data_ptr()), cnt, norms, _lib.stream_ptr()), "xlbb_batched_prolong_add_map")
        self._smooth(l)

    def vcycle(self):
        """One V-cycle of every instance (graph replay after the first call).
        Leaves the level-0 residual norms^2 in ``norm2``."""
        if self.graph is None:
            x0 = self.X[0]
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self.launches_per_cycle = 0
                saved = {d: a.buf.clone() for d, a in x0.items()}
                self._level(0)            # warm-up outside the capture (module loading)
                for d, a in x0.items():
                    a.buf.copy_(saved[d])
            torch.cuda.current_stream().wait_stream(s)
            self.graph = torch.cuda.CUDAGraph()
            self.launches_per_cycle = 0
            with torch.cuda.graph(self.graph):
                self._level(0)
        self.graph.replay()

    def reset(self):
        for a in self.X[0].values():
            a.buf.zero_()

    def solve(self, tol=1e-5, max_cycles=100, criterion="residual", stall_cycles=3):
        """V-cycles from zero until every instance has converged.  Returns
        (cycles, per-instance measure).

        ``criterion="residual"``: the level-0 residual norm fell by ``tol``
        relative to the first cycle (the reference's measure).
        ``criterion="error"``: the estimated relative error of the populations,
        ``c * rho / (1 - rho)`` with ``c`` = ||coarse correction|| / ||f|| of the
        cycle and ``rho`` the observed contraction of ``c`` (capped at 0.95), is
        below ``tol``.  An instance whose ``c`` stops falling for
        ``stall_cycles`` cycles has reached the rounding floor of its precision
        and counts as converged (``self.stalled``).  ``self.converged_at`` holds
        each instance's cycle of convergence."""
        self.reset()
        self.converged_at = np.full(self.n, -1)
        self.stalled = np.zeros(self.n, dtype=bool)
        self.vcycle()
        cycles = 1
        if criterion == "residual":
            r0 = torch.sqrt(self.norm2).cpu().numpy()
            require_finite(r0, "level-0 residual norm of the first V-cycle", cycles)
            rel = np.ones(self.n)
            while cycles < max_cycles:
                self.vcycle()
                cycles += 1
                rel = torch.sqrt(self.norm2).cpu().numpy() / np.where(r0 > 0, r0, 1.0)
                require_finite(rel, "relative V-cycle residual", cycles)
                self.converged_at[(self.converged_at < 0) & (rel < tol)] = cycles
                if np.all(rel < tol):
                    break
            if self.remove_mean:
                self.remove_mean_moment()
            return cycles, rel
        if criterion != "error":
            raise ValueError("criterion must be 'residual' or 'error'")

        def corr():
            c = self.corr2.cpu().numpy()
            out = np.empty(self.n)
            out[self._corr_ids] = np.sqrt(c[:, 0] / np.where(c[:, 1] > 0, c[:, 1], 1.0))
            return out
        prev = corr()
        require_finite(prev, "relative coarse-grid correction", cycles)
        est = np.full(self.n, np.inf)
        flat = np.zeros(self.n, dtype=int)
        while cycles < max_cycles:
            self.vcycle()
            cycles += 1
            c = corr()
            require_finite(c, "relative coarse-grid correction", cycles)
            ratio = c / np.where(prev > 0, prev, 1.0)
            rho = np.minimum(ratio, 0.95)
            est = c * rho / (1.0 - rho)
            flat = np.where(ratio > 0.95, flat + 1, 0)
            newly = (self.converged_at < 0) & ((est < tol) | (flat >= stall_cycles))
            self.stalled |= newly & ~(est < tol)
            self.converged_at[newly] = cycles
            prev = c
            if np.all(self.converged_at >= 0):
                break
        if self.remove_mean:
            self.remove_mean_moment()
        return cycles, est

    def populations(self, i):
        """Level-0 populations of instance ``i`` (an (nx, ny, 8) view)."""
        (arena,) = self.X[0].values()
        return arena.view(i)

    def displacement(self, i):
        """Displacement of instance ``i``: the first two moments plus half the
        body force (``update_macroscopic``, ``src/elasticity.py:1002-1038``), FP64."""
        from .lattice import LatticeD2Q8
        c = torch.as_tensor(np.asarray(LatticeD2Q8("f64/f64").c, dtype=np.float64), device=self.device)
        f = self.populations(i).double()
        return torch.einsum("xyq,dq->xyd", f, c) + 0.5 * self.F.view(i).double()

    def lattice_updates_per_cycle(self):
        """Cell updates of one V-cycle summed over the batch (smoothing and
        residual sweeps; the reference's sweep count per level)."""
        total = 0
        for g in range(self.n):
            nx, ny = self.shapes[0][g]
            for l in range(self.instance_levels[g]):
                sweeps = 2 * self.k_smooth + (1 if l < self.instance_levels[g] - 1 else 0)
                total += sweeps * (nx >> l) * (ny >> l)
        return total
