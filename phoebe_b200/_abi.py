"""ctypes binding of libphx.so (the C ABI declared in include/phx_abi.h).

There is no fallback: if the library is missing or cannot be loaded, or no
sm_100 device is present, every call raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libphx.so")

PHX_OK = 0
PHX_ERR_ARG = 1
PHX_ERR_CUDA = 2
PHX_ERR_NOCONV = 3
PHX_ERR_STATE = 4
PHX_ERR_MESH = 5
PHX_ERR_NODEV = 6

PHX_SMEAR_GAUSSIAN = 0
PHX_SMEAR_ADAPTIVE = 1
PHX_PREC_FP64 = 0
PHX_PREC_SPLIT_BF16 = 1
PHX_PREC_SPLIT_TF32 = 2   # reserved, rejected
PHX_PREC_SPLIT_FP16 = 3

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p
_i = ctypes.c_int


class LwParams(ctypes.Structure):
    _fields_ = [("num_temperatures", ctypes.c_int), ("temperatures", _D),
                ("smearing", ctypes.c_int), ("sigma", ctypes.c_double),
                ("finalize", ctypes.c_int), ("q2_begin", ctypes.c_int), ("q2_end", ctypes.c_int),
                ("window_energy", _D), ("window_cut", _D),
                ("isotope_coupling", _D), ("boundary_length", ctypes.c_double)]


class LwStats(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_double), ("ms_vertex", ctypes.c_double),
                ("pairs", ctypes.c_longlong), ("kernel_launches", ctypes.c_int),
                ("pair_launches", ctypes.c_int), ("ms_pair", ctypes.c_double),
                ("plan_chunk", ctypes.c_int), ("plan_slots", ctypes.c_int), ("graph", ctypes.c_int),
                ("edge_events_peak", ctypes.c_longlong), ("edge_events_cap", ctypes.c_longlong),
                ("edge_overflow_chunks", ctypes.c_int), ("pairs_screened_out", ctypes.c_longlong),
                ("tile_rt", ctypes.c_int), ("tile_qp", ctypes.c_int)]


class ElParams(ctypes.Structure):
    _fields_ = [("num_temperatures", ctypes.c_int), ("temperatures", ctypes.POINTER(ctypes.c_double)),
                ("chemical_potential", ctypes.c_double), ("window", ctypes.c_double),
                ("smearing", ctypes.c_int), ("sigma", ctypes.c_double), ("norm", ctypes.c_double),
                ("num_k1", ctypes.c_int), ("k1_list", ctypes.POINTER(ctypes.c_int))]


# name -> argtypes (all return int unless listed in _RESTYPE)
SIGNATURES = {
    "phx_ctx_create": [_i, ctypes.POINTER(_VP)],
    "phx_ctx_destroy": [_VP],
    "phx_ctx_synchronize": [_VP],
    "phx_last_error": [_VP, ctypes.c_char_p, ctypes.c_size_t],
    "phx_version": [],
    "phx_ws_reorder": [_i, _D, _D, _I, _D, _I, _D, _D, _D],
    "phx_ph_h0_create": [_VP, _i, _D, _D, _D, _I, _D, ctypes.POINTER(_VP)],
    "phx_ph_h0_destroy": [_VP],
    "phx_ph_h0_num_bands": [_VP],
    "phx_ph_diag": [_VP, _i, _D, _i, _D, _D],
    "phx_ph_diag_velocities": [_VP, _i, _D, _D, _D, _D],
    "phx_bands_create_mesh": [_VP, _I, _i, ctypes.POINTER(_VP)],
    "phx_bands_create_from_host": [_VP, _I, _D, _i, _D, _D, _D, ctypes.POINTER(_VP)],
    "phx_bands_destroy": [_VP],
    "phx_bands_num_points": [_VP],
    "phx_bands_get": [_VP, _D, _D, _D],
    "phx_v3_create": [_VP, _i, _i, _i, _D, _D, _D, _D, _D, ctypes.POINTER(_VP)],
    "phx_v3_destroy": [_VP],
    "phx_v3_set_precision": [_VP, _i],
    "phx_v3_cache_d3": [_VP, _D],
    "phx_v3_couplings_sq": [_VP, _i, _D, _D, _I, _D, _i, _D, _I, _D, _I, _D, _D],
    "phx_v3_estimate_num_batches": [_VP, _i, _i, _I],
    "phx_ph_linewidths": [_VP, _VP, ctypes.POINTER(LwParams), _D, ctypes.POINTER(LwStats)],
    "phx_ph_linewidths_screened": [_VP, _VP, ctypes.POINTER(LwParams), _VP, ctypes.c_double, _D,
                                   ctypes.POINTER(LwStats)],
    "phx_ph_linewidths_d": [_VP, _VP, ctypes.POINTER(LwParams), _VP, ctypes.POINTER(LwStats)],
    "phx_ph_rta_kappa": [_VP, _i, _D, _D, ctypes.c_double, _D],
    "phx_ph_linewidths_static": [_VP, _VP, ctypes.POINTER(LwParams), _VP],
    "phx_ph_smatrix_create": [_VP, _VP, ctypes.POINTER(LwParams), ctypes.POINTER(_VP), ctypes.POINTER(LwStats)],
    "phx_smatrix_num_states": [_VP],
    "phx_smatrix_diagonal": [_VP, _D],
    "phx_smatrix_get_rows": [_VP, _i, _i, _D],
    "phx_smatrix_dot": [_VP, _i, _D, _i, _D],
    "phx_smatrix_dot_d": [_VP, _i, _VP, _i, _VP, ctypes.POINTER(ctypes.c_float)],
    "phx_smatrix_destroy": [_VP],
    "phx_smatrix_symmetrize": [_VP],
    "phx_smatrix_a2omega": [_VP],
    "phx_smatrix_diagonalize": [_VP, _i, _D, ctypes.POINTER(_i)],
    "phx_smatrix_relaxon_solve": [_VP, _i, _D, _D],
    "phx_ph_smatrix_dot": [_VP, _VP, ctypes.POINTER(LwParams), _i, _D, _D, ctypes.POINTER(LwStats)],
    "phx_ph_smatrix_dot_d": [_VP, _VP, ctypes.POINTER(LwParams), _i, _VP, _VP, ctypes.POINTER(LwStats)],
    "phx_el_h0_create": [_VP, _i, _i, _D, _D, _D, _D, ctypes.POINTER(_VP)],
    "phx_el_h0_destroy": [_VP],
    "phx_el_h0_num_bands": [_VP],
    "phx_el_diag": [_VP, _i, _D, _D, _D, _D],
    "phx_el_bands_create_mesh": [_VP, _I, _i, ctypes.POINTER(_VP)],
    "phx_elph_create": [_VP, _i, _i, _i, _i, _D, _D, _D, _D, ctypes.POINTER(ctypes.c_float),
                        ctypes.POINTER(_VP)],
    "phx_elph_destroy": [_VP],
    "phx_elph_cache_k1": [_VP, _D, _D, _i],
    "phx_elph_set_precision": [_VP, _i],
    "phx_elph_couplings_sq": [_VP, _i, _D, _D, _I, _i, _D, _D],
    "phx_el_linewidths": [_VP, _VP, _VP, ctypes.POINTER(ElParams), _D, ctypes.POINTER(LwStats)],
    "phx_mlp_create": [_VP, _i, _i, _i, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_VP)],
    "phx_mlp_destroy": [_VP],
    "phx_mlp_num_params": [_VP],
    "phx_mlp_get_params": [_VP, ctypes.POINTER(ctypes.c_float)],
    "phx_mlp_set_params": [_VP, ctypes.POINTER(ctypes.c_float)],
    "phx_mlp_infer": [_VP, _i, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "phx_mlp_grad": [_VP, _i, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                     ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "phx_mlp_train": [_VP, _i, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float), _i, _i,
                      ctypes.c_float, ctypes.c_ulonglong, ctypes.POINTER(ctypes.c_float)],
    "phx_diag_tc_gemm": [_VP, _i, _i, ctypes.POINTER(ctypes.c_float),
                         ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)],
    "phx_debug_set_split_edge_cap": [ctypes.c_uint],
}
_RESTYPE = {"phx_version": ctypes.c_char_p, "phx_mlp_num_params": ctypes.c_longlong}

_lib = None


class PhxError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("phx error %d: %s" % (status, msg))
        self.status = status


def load():
    """Load libphx.so; raises if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PhxError(PHX_ERR_NODEV, "libphx.so not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, ctypes.c_int)
        _lib = L
    return _lib


def last_error(ctx=None):
    buf = ctypes.create_string_buffer(1024)
    load().phx_last_error(ctx, buf, 1024)
    return buf.value.decode(errors="replace")


def check(status, ctx=None):
    if status != PHX_OK:
        raise PhxError(status, last_error(ctx))


def dptr(a):
    return a.ctypes.data_as(_D)


def iptr(a):
    return a.ctypes.data_as(_I)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def c128(a):
    """Complex array -> contiguous interleaved float64 view."""
    return np.ascontiguousarray(a, dtype=np.complex128).view(np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)
