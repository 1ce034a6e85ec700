"""Adjoint (reverse-mode) pieces of the Biot step: wrappers over the
hand-written transposed kernels of ``libxlbb.so``.

No counterpart in the reference, which has no gradients.  Every function takes
the adjoint of a forward call's output and returns (or accumulates) the
adjoints of its inputs; parameter gradients (per-cell lambda, mu of the
elasticity collision and omega of the Darcy BGK) accumulate in FP64 buffers.
The forward calls they transpose are the solvers' own: ``LBMElasticity._sweep``,
``AdvectionDiffusionReactionBGK._sweep`` / ``gradient`` / ``update_macroscopic``
and ``LBMElasticity.update_divergence`` / ``update_macroscopic``.
"""
import ctypes

import torch

from . import _lib


class ElastGrads:
    """Per-level FP64 accumulators of d/d lambda and d/d mu (one plane each,
    indexed like the level's fields)."""

    def __init__(self, el):
        self.lam = [f64_plane(el._L(l)) for l in range(el.levels)]
        self.mu = [f64_plane(el._L(l)) for l in range(el.levels)]

    def zero_(self):
        for t in self.lam + self.mu:
            t.zero_()


def f64_plane(L):
    """A zeroed FP64 (nx, ny, 1) plane with the element pitch of layout ``L``
    (the kernels index it with L's grid)."""
    buf = torch.zeros(L.plane, dtype=torch.float64, device=L.device)
    return buf.as_strided((L.nx, L.ny, 1), (1, L.pitch, L.plane))


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def elast_sweep_adjoint(el, level, lam_out, a=0.0, b=1.0, f_in=None, resid=None, fext=None, lam_resid=None,
                        want_force=False, grads=None):
    """Transpose of ``el._sweep(f_in, level, a, b, resid=resid, fext=fext)``.
    Returns (lam_f, lam_force or None); ``lam_resid`` (if given) accumulates
    -lam_g; ``grads`` (an ``ElastGrads``) accumulates d/d lambda, d/d mu of
    ``level``'s material (needs the forward inputs)."""
    L = el._L(level)
    lam_f = L.empty(8)
    lam_force = L.empty(2) if want_force else None
    if fext is not None and not L.conforms(fext, 2):
        fext = L.field(fext, 2)
    if getattr(el, "_acc64_all", False):
        raise NotImplementedError("the adjoint kernels compute in their storage type: use 'f32/f32' or 'f64/f64'")
    pc, ps = el._rules[level]
    force = el.force if level == 0 else None
    s = _lib.ElastSweepAdjoint(
        lam_out.data_ptr(), lam_f.data_ptr(), lam_resid.data_ptr() if lam_resid is not None else None,
        lam_force.data_ptr() if lam_force is not None else None,
        grads.lam[level].data_ptr() if grads is not None else None,
        grads.mu[level].data_ptr() if grads is not None else None,
        f_in.data_ptr() if f_in is not None else None, resid.data_ptr() if resid is not None else None,
        force.data_ptr() if force is not None else None, 1 if level == 0 else 0,
        fext.data_ptr() if fext is not None else None, float(a), float(b), pc.struct(), ps.struct())
    _lib.check(_lib.lib().xlbb_elast_sweep_adjoint(_lib.dtype_code(L.dtype), L.grid(), el._mats[level], s,
                                                   _lib.stream_ptr()), "xlbb_elast_sweep_adjoint")
    return lam_f, lam_force


def darcy_sweep_adjoint(da, lam_out, f_in=None, source=None, g_omega=None, want_source=False):
    """Transpose of ``da._sweep(f_in, source)`` (``source``: the external
    source).  Returns (lam_f, lam_source or None); ``g_omega`` accumulates."""
    L = da._layout
    lam_f = L.empty(9)
    lam_s = L.empty(1) if want_source else None
    s = _lib.DarcySweepAdjoint(
        lam_out.data_ptr(), lam_f.data_ptr(), lam_s.data_ptr() if lam_s is not None else None,
        g_omega.data_ptr() if g_omega is not None else None, f_in.data_ptr() if f_in is not None else None,
        float(da.omega), da.omega_field.data_ptr() if da.omega_field is not None else None,
        da.source.data_ptr() if da.source is not None else None,
        source.data_ptr() if source is not None else None, da._pc.struct(), da._ps.struct())
    _lib.check(_lib.lib().xlbb_darcy_sweep_adjoint(da._dcode, L.grid(), s, _lib.stream_ptr()),
               "xlbb_darcy_sweep_adjoint")
    return lam_f, lam_s


def gradient_adjoint(da, lam_grad, scale, lam_q, dtype=None):
    """lam_q += G^T lam_grad with G = ``da.gradient(., scale, dtype=dtype)`` on
    lam_grad's grid (any multigrid level)."""
    from .fields import Layout
    nx, ny = int(lam_grad.shape[0]), int(lam_grad.shape[1])
    dtype = da._dtype if dtype is None else dtype
    L = Layout(nx, ny, dtype)
    if not (L.conforms(lam_grad, 2) and L.conforms(lam_q, 1)):
        raise ValueError("gradient_adjoint: operands must be fields of the grid in the given precision")
    rules = da.gradient_rules(nx, ny, dtype)
    _lib.check(_lib.lib().xlbb_darcy_gradient_adjoint(_lib.dtype_code(dtype), L.grid(), lam_grad.data_ptr(),
                                                      float(scale), rules.struct(), lam_q.data_ptr(),
                                                      _lib.stream_ptr()), "xlbb_darcy_gradient_adjoint")
    return lam_q


def elast_moments_adjoint(el, level, lam_f, lam_eta=None, lam_div=None, f=None, grads=None):
    """lam_f += adjoint of eta's population part and of the divergence moment
    (``update_divergence``) on ``level``; ``grads`` accumulates the derivative
    of the divergence scale (needs the forward ``f``)."""
    L = el._L(level)
    use_g = grads is not None and lam_div is not None
    _lib.check(_lib.lib().xlbb_elast_moments_adjoint(
        _lib.dtype_code(L.dtype), L.grid(), el._mats[level], _p(f), _p(lam_eta), _p(lam_div),
        float(el._div_scale), lam_f.data_ptr(), grads.lam[level].data_ptr() if use_g else None,
        grads.mu[level].data_ptr() if use_g else None, _lib.stream_ptr()), "xlbb_elast_moments_adjoint")
    return lam_f


def darcy_moments_adjoint(da, lam_f, lam_rho=None, lam_grad=None, f=None, g_omega=None):
    """lam_f += adjoint of rho's population part and of grad = -3 omega sum c f;
    ``g_omega`` accumulates (needs the forward ``f``)."""
    L = da._layout
    _lib.check(_lib.lib().xlbb_darcy_moments_adjoint(
        da._dcode, L.grid(), _p(f), float(da.omega), _p(da.omega_field), _p(lam_rho), _p(lam_grad),
        lam_f.data_ptr(), g_omega.data_ptr() if g_omega is not None else None, _lib.stream_ptr()),
        "xlbb_darcy_moments_adjoint")
    return lam_f


def divgrad_adjoint(el, da, level, lam_ext, scale, lam_f, lam_fe=None, f=None, grads=None):
    """Transpose of the coupling force ext = fe + ``da.gradient(el.update_divergence(f,
    level), scale, dtype=level's)``: lam_f += div^T G^T lam_ext, lam_fe += lam_ext
    (if given); ``grads`` accumulates the divergence scale's derivative (needs f)."""
    L = el._L(level)
    rules = da.gradient_rules(L.nx, L.ny, L.dtype)
    _lib.check(_lib.lib().xlbb_divgrad_adjoint(
        _lib.dtype_code(L.dtype), L.grid(), el._mats[level], lam_ext.data_ptr(), float(scale), rules.struct(), _p(f),
        lam_f.data_ptr(), _p(lam_fe), grads.lam[level].data_ptr() if grads is not None else None,
        grads.mu[level].data_ptr() if grads is not None else None, _lib.stream_ptr()), "xlbb_divgrad_adjoint")
    return lam_f


def add_(dst, src):
    """dst += src for two fields of one layout (the library's axpby over the
    fields' planes, padding included)."""
    n = dst.shape[2] * dst.stride(2)
    if src.shape != dst.shape or src.stride() != dst.stride() or src.dtype != dst.dtype:
        raise ValueError("add_: fields of one layout expected")
    _lib.check(_lib.lib().xlbb_axpby(_lib.dtype_code(dst.dtype), n, 1.0, dst.data_ptr(), 1.0, src.data_ptr(),
                                     dst.data_ptr(), _lib.stream_ptr()), "xlbb_axpby")
    return dst
