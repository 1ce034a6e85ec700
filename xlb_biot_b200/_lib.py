"""ctypes binding of ``libxlbb.so`` (the C ABI declared in ``include/xlbb.h``).

There is no CPU fallback: if the library or a CUDA device is missing, every
solver call raises.  All calls are asynchronous on torch's current CUDA stream.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxlbb.so")

XLBB_F32, XLBB_F64, XLBB_F32_ACC64 = 0, 1, 2
XLBB_PROLONG_BLOCKS = 32
XLBB_BATCH_PARTS_PER_TILE = 32       # FP64 partials per tile of a batched sweep with sums
XLBB_OK, XLBB_EBADARG, XLBB_ELAUNCH, XLBB_ETIMEOUT, XLBB_ENONFINITE, XLBB_EUNSUPPORTED = 0, -1, -2, -3, -4, -5
ERRORS = {-1: "XLBB_EBADARG", -2: "XLBB_ELAUNCH", -3: "XLBB_ETIMEOUT", -4: "XLBB_ENONFINITE",
          -5: "XLBB_EUNSUPPORTED"}


class XlbbError(RuntimeError):
    """A negative status returned by the C ABI."""

    code = None


class NonFiniteError(XlbbError):
    """XLBB_ENONFINITE: a convergence norm became NaN or Inf (the iteration
    diverged, or a field or parameter holds non-finite values)."""

    code = XLBB_ENONFINITE


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("pitch", ctypes.c_int), ("plane", ctypes.c_longlong)]


class Grid3(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("pitch", ctypes.c_int),
                ("plane", ctypes.c_longlong)]


class Rules(ctypes.Structure):
    _fields_ = [("count", ctypes.c_int), ("row_ptr", ctypes.c_void_p), ("cell_x", ctypes.c_void_p),
                ("code", ctypes.c_void_p), ("cst", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("word_base", ctypes.c_void_p), ("words_per_row", ctypes.c_int), ("push", ctypes.c_void_p)]


class SweepConfig(ctypes.Structure):
    _fields_ = [("tx", ctypes.c_int), ("depth", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("min_rows", ctypes.c_int), ("pipeline", ctypes.c_int)]


class ElastMaterial(ctypes.Structure):
    _fields_ = [("lam", ctypes.c_double), ("mu", ctypes.c_double), ("lam_field", ctypes.c_void_p),
                ("mu_field", ctypes.c_void_p)]


class ElastSweep(ctypes.Structure):
    _fields_ = [("f_in", ctypes.c_void_p), ("f_out", ctypes.c_void_p), ("force", ctypes.c_void_p),
                ("use_force", ctypes.c_int), ("fext", ctypes.c_void_p), ("resid", ctypes.c_void_p),
                ("a", ctypes.c_double), ("b", ctypes.c_double), ("pc", Rules), ("ps", Rules),
                ("sumsq", ctypes.c_void_p), ("bx0", ctypes.c_int), ("bx1", ctypes.c_int),
                ("by0", ctypes.c_int), ("by1", ctypes.c_int), ("div_out", ctypes.c_void_p),
                ("sumsq_diff", ctypes.c_int)]


class DarcySweep(ctypes.Structure):
    _fields_ = [("f_in", ctypes.c_void_p), ("f_out", ctypes.c_void_p), ("omega", ctypes.c_double),
                ("omega_field", ctypes.c_void_p), ("source", ctypes.c_void_p), ("ext_source", ctypes.c_void_p),
                ("pc", Rules), ("ps", Rules), ("sumsq", ctypes.c_void_p), ("resid", ctypes.c_void_p)]


class BatchInstance(ctypes.Structure):
    _fields_ = [("f_in", ctypes.c_void_p), ("f_out", ctypes.c_void_p), ("force", ctypes.c_void_p),
                ("resid", ctypes.c_void_p), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("pitch", ctypes.c_int),
                ("plane", ctypes.c_longlong), ("lam", ctypes.c_double), ("mu", ctypes.c_double)]


class BatchTransfer(ctypes.Structure):
    _fields_ = [("fine", ctypes.c_void_p), ("coarse", ctypes.c_void_p), ("nx_f", ctypes.c_int),
                ("ny_f", ctypes.c_int), ("pitch_f", ctypes.c_int), ("pitch_c", ctypes.c_int),
                ("plane_f", ctypes.c_longlong), ("plane_c", ctypes.c_longlong)]


class ElastSweepAdjoint(ctypes.Structure):
    _fields_ = [("lam_out", ctypes.c_void_p), ("lam_f", ctypes.c_void_p), ("lam_resid", ctypes.c_void_p),
                ("lam_force", ctypes.c_void_p), ("g_lam", ctypes.c_void_p), ("g_mu", ctypes.c_void_p),
                ("f_in", ctypes.c_void_p), ("resid", ctypes.c_void_p), ("force", ctypes.c_void_p),
                ("use_force", ctypes.c_int), ("fext", ctypes.c_void_p), ("a", ctypes.c_double),
                ("b", ctypes.c_double), ("pc", Rules), ("ps", Rules)]


class BatchTail(ctypes.Structure):
    _fields_ = [("resid", ctypes.c_void_p), ("f_out", ctypes.c_void_p), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
                ("pitch", ctypes.c_int), ("plane", ctypes.c_longlong), ("levels", ctypes.c_int),
                ("lam", ctypes.c_double), ("mu", ctypes.c_double)]


class DarcySweepAdjoint(ctypes.Structure):
    _fields_ = [("lam_out", ctypes.c_void_p), ("lam_f", ctypes.c_void_p), ("lam_source", ctypes.c_void_p),
                ("g_omega", ctypes.c_void_p), ("f_in", ctypes.c_void_p), ("omega", ctypes.c_double),
                ("omega_field", ctypes.c_void_p), ("source", ctypes.c_void_p), ("ext_source", ctypes.c_void_p),
                ("pc", Rules), ("ps", Rules)]


P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double
PG = ctypes.POINTER(Grid)
SIGNATURES = {
    "xlbb_elast_sweep": (I, [I, PG, ctypes.POINTER(ElastMaterial), ctypes.POINTER(ElastSweep), P]),
    "xlbb_elast_sweep_pipeline": (I, [I, PG, ctypes.POINTER(ElastMaterial), ctypes.POINTER(ElastSweep)]),
    "xlbb_elast_sweep_ctas": (I, [I, PG]),
    "xlbb_elast_sweep_partials": (I, [I, PG, ctypes.POINTER(ElastMaterial), ctypes.POINTER(ElastSweep)]),
    "xlbb_darcy_sweep": (I, [I, PG, ctypes.POINTER(DarcySweep), P]),
    "xlbb_darcy_sweep_ctas": (I, [I, PG]),
    "xlbb_darcy_sweep_partials": (I, [I, PG, ctypes.POINTER(DarcySweep)]),
    "xlbb_darcy_sweep_pipeline": (I, [I, PG, ctypes.POINTER(DarcySweep)]),
    "xlbb_fluid_sweep": (I, [I, PG, ctypes.POINTER(DarcySweep), I, P]),
    "xlbb_fluid3_sweep": (I, [I, ctypes.POINTER(Grid3), ctypes.POINTER(DarcySweep), I, I, P]),
    "xlbb_darcy_sweep_residual_noalloc": (I, [I, PG, ctypes.POINTER(DarcySweep), P, P]),
    "xlbb_darcy_gradient": (I, [I, PG, P, D, ctypes.POINTER(Rules), P, P, P]),
    "xlbb_elast_divgrad": (I, [I, PG, ctypes.POINTER(ElastMaterial), D, P, D, ctypes.POINTER(Rules), P, P, P]),
    "xlbb_elast_sweep_divgrad": (I, [I, PG, ctypes.POINTER(ElastMaterial), ctypes.POINTER(ElastSweep), D, D,
                                     ctypes.POINTER(Rules), P]),
    "xlbb_elast_moments": (I, [I, PG, ctypes.POINTER(ElastMaterial), P, P, P, P, P, P, D, P]),
    "xlbb_elast_equilibrium": (I, [I, PG, ctypes.POINTER(ElastMaterial), P, P, P, P, P, P]),
    "xlbb_darcy_moments": (I, [I, PG, P, D, P, P, P, P, P, P]),
    "xlbb_restrict": (I, [I, I, PG, PG, I, I, I, I, I, P, P, P]),
    "xlbb_prolong_add": (I, [I, I, PG, PG, I, I, I, I, I, P, P, P]),
    "xlbb_reduce_sum": (I, [P, I, P, P]),
    "xlbb_batched_tail_smem": (I, [I, I, I, I, I]),
    "xlbb_batched_tail": (I, [I, I, P, I, I, D, I, P]),
    "xlbb_wait_selftest": (I, [ctypes.c_uint, P, P]),
    "xlbb_sumsq": (I, [I, PG, I, P, I, I, I, I, P, P]),
    "xlbb_sumsq_ctas": (I, [PG]),
    "xlbb_axpby": (I, [I, ctypes.c_longlong, D, P, D, P, P, P]),
    "xlbb_sweep_set_config": (I, [I, ctypes.POINTER(SweepConfig)]),
    "xlbb_sweep_get_config": (I, [I, ctypes.POINTER(SweepConfig)]),
    "xlbb_device_status": (I, [ctypes.POINTER(ctypes.c_int), I]),
    "xlbb_batch_desc_bytes": (I, [I]),
    "xlbb_batch_upload": (I, [I, ctypes.POINTER(BatchInstance), I, P, P]),
    "xlbb_batched_elast_sweep": (I, [I, P, P, I, I, D, D, I, I, I, P, I, P]),
    "xlbb_batched_elast_sweep4": (I, [I, P, P, I, I, D, D, I, I, I, P, I, P]),
    "xlbb_batched_restrict": (I, [I, I, P, I, P]),
    "xlbb_batched_prolong_add": (I, [I, I, P, I, P]),
    "xlbb_batched_prolong_add_norms": (I, [I, I, P, I, P, P, P]),
    "xlbb_batched_prolong_add_map": (I, [I, I, P, P, I, P, P, I, P, P]),
    "xlbb_segment_sum": (I, [P, P, I, P, P]),
    "xlbb_batched_remove_mean_moment": (I, [I, P, P, I, P, P, I, P, P]),
    "xlbb_elast_sweep_adjoint": (I, [I, PG, ctypes.POINTER(ElastMaterial), ctypes.POINTER(ElastSweepAdjoint), P]),
    "xlbb_darcy_sweep_adjoint": (I, [I, PG, ctypes.POINTER(DarcySweepAdjoint), P]),
    "xlbb_darcy_gradient_adjoint": (I, [I, PG, P, D, ctypes.POINTER(Rules), P, P]),
    "xlbb_elast_moments_adjoint": (I, [I, PG, ctypes.POINTER(ElastMaterial), P, P, P, D, P, P, P, P]),
    "xlbb_darcy_moments_adjoint": (I, [I, PG, P, D, P, P, P, P, P, P]),
    "xlbb_divgrad_adjoint": (I, [I, PG, ctypes.POINTER(ElastMaterial), P, D, ctypes.POINTER(Rules), P, P, P, P, P,
                                 P]),
    "xlbb_last_error": (ctypes.c_char_p, []),
    "xlbb_version": (I, []),
}

_lib = None


def lib():
    """Load ``libxlbb.so`` once.  Raises if it is missing (build it with
    ``python -m xlb_biot_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise XlbbError(f"CUDA library not built: {LIB_PATH} is missing "
                            "(run `python -m xlb_biot_b200.build`)")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def require_cuda():
    if not torch.cuda.is_available():
        raise XlbbError("xlb_biot_b200 needs a CUDA device: there is no CPU fallback")


def check(status, what):
    if status < 0:
        msg = lib().xlbb_last_error().decode()
        cls = NonFiniteError if status == XLBB_ENONFINITE else XlbbError
        err = cls(f"{what} failed with {ERRORS.get(status, status)}: {msg}")
        err.code = status
        raise err
    return status


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def dtype_code(dtype):
    if dtype == torch.float32:
        return XLBB_F32
    if dtype == torch.float64:
        return XLBB_F64
    raise XlbbError(f"unsupported dtype {dtype}")


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())
