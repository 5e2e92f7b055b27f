"""ctypes binding of libpipeflow_b200.so (the C ABI in include/pipeflow_b200.h).

The library is required: importing this module without the built library, or
calling into it without a CUDA device, raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpipeflow_b200.so"

PF_OK = 0
PF_ERR_ARG = -1
PF_ERR_CUDA = -2
PF_ERR_SINGULAR = -3
PF_ERR_NOMEM = -4
PF_ERR_STATE = -5
PF_ERR_CONVERGE = -6
PF_ERR_NODEVICE = -7
PF_ERR_CANCELLED = -8
PF_PREC_FP64 = 0
PF_PREC_MIXED = 1
PF_IO_TIME_FROM_FILE = 1
PF_UTIL_NONE = 0
PF_UTIL_CORIOLIS = 1
PF_UTIL_CARREAU_YASUDA = 2
PF_UTIL_LES = 3
UTIL_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_void_p)
KL = 4


class pf_config(C.Structure):
    _fields_ = [
        ("N", C.c_int), ("K", C.c_int), ("M", C.c_int), ("Mp", C.c_int),
        ("Re", C.c_double), ("alpha", C.c_double),
        ("dt", C.c_double), ("implicit", C.c_double), ("dterr", C.c_double),
        ("courant", C.c_double), ("maxdt", C.c_double),
        ("const_flux", C.c_int), ("mirrorsym", C.c_int), ("shiftrefl", C.c_int),
        ("shiftrott", C.c_int),
        ("r", C.POINTER(C.c_double)),
        ("precision", C.c_int),
    ]


class pf_tim_state(C.Structure):
    _fields_ = [
        ("t", C.c_double), ("dt", C.c_double), ("dterr", C.c_double),
        ("corr_dt", C.c_double), ("cfl_dt", C.c_double),
        ("it", C.c_int), ("step", C.c_int), ("cfl_dir", C.c_int),
        ("new_dt", C.c_int), ("pcn", C.c_int),
    ]


PF_LD_AUTO = 0
PF_LD_STREAMED = 1
PF_LD_REBUILT = 2
PF_LD_PAIRED = 3
PF_LD_WARPRING = 4


class pf_tuning(C.Structure):
    _fields_ = [("ld_solver", C.c_int), ("nl_mc", C.c_int), ("nl_zc", C.c_int), ("nl_fused", C.c_int)]


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
D = C.c_double
DP = C.POINTER(C.c_double)
I = C.c_int
IP = C.POINTER(C.c_int)

# name -> argtypes (all return int unless listed in _RESTYPES)
_SIGS = {
    "pf_last_error": [],
    "pf_version": [IP, IP],
    "pf_ctx_create": [C.POINTER(pf_config), I, PP],
    "pf_ctx_destroy": [P],
    "pf_ctx_reconfigure": [P, C.POINTER(pf_config)],
    "pf_ctx_set_stream": [P, P],
    "pf_ctx_set_tuning": [P, C.POINTER(pf_tuning)],
    "pf_ctx_get_tuning": [P, C.POINTER(pf_tuning)],
    "pf_nl_passes": [P, C.POINTER(C.c_int)],
    "pf_ctx_sync": [P],
    "pf_ctx_dims": [P, IP, IP, IP, IP],
    "pf_ctx_device_bytes": [P, C.POINTER(C.c_ulonglong)],
    "pf_mes_get": [P, DP, DP, DP, DP, DP, DP],
    "pf_mes_compute": [I, DP, DP, DP, DP, DP, DP, DP],
    "pf_coll_create": [P, PP],
    "pf_coll_destroy": [P],
    "pf_coll_upload": [P, DP, DP],
    "pf_coll_download": [P, DP, DP],
    "pf_phys_create": [P, PP],
    "pf_phys_destroy": [P],
    "pf_phys_upload": [P, DP],
    "pf_phys_download": [P, DP],
    "pf_var_coll_init": [P],
    "pf_var_coll_copy": [P, P],
    "pf_var_coll_add": [P, P],
    "pf_var_coll_sub": [P, P],
    "pf_var_coll_dmult": [D, P],
    "pf_var_coll_neg": [P, P],
    "pf_var_coll_meshmult": [I, P, P],
    "pf_var_coll_curl": [P, P, P, P, P, P],
    "pf_var_coll_grad": [P, P, P, P],
    "pf_var_coll_div": [P, P, P, P],
    "pf_var_coll_shift": [D, D, P, P],
    "pf_var_imposesym": [I, P, P, P],
    "pf_var_coll_norm": [P, DP, DP, DP],
    "pf_tra_coll2phys": [P, P],
    "pf_tra_phys2coll": [P, P],
    "pf_tra_coll2phys_noalloc": [I, I, I, P, P, P, P],
    "pf_tim_get": [P, C.POINTER(pf_tim_state)],
    "pf_tim_set": [P, C.POINTER(pf_tim_state)],
    "pf_tim_mesh_init": [P, I, D, D, PP],
    "pf_mesh_destroy": [P],
    "pf_mesh_download": [P, DP],
    "pf_tim_lumesh_init": [P, I, I, D, D, PP],
    "pf_lumesh_destroy": [P],
    "pf_lumesh_download": [P, DP, IP],
    "pf_tim_lumesh_invert": [I, P, P],
    "pf_tim_meshmult": [I, P, P, P, P],
    "pf_tim_zerobc": [P],
    "pf_tim_nlincorr": [P, P],
    "pf_tim_measurecorr": [P, P, P],
    "pf_tim_check_cgce": [P],
    "pf_tim_new_tstep": [P],
    "pf_vel_coll": [P, I, PP],
    "pf_vel_phys": [P, I, PP],
    "pf_vel_set_state": [P, DP, DP, DP, DP, DP, DP],
    "pf_vel_get_state": [P, DP, DP, DP, DP, DP, DP],
    "pf_vel_get_state_async": [P, DP, DP, DP, DP, DP, DP],
    "pf_vel_get_scalars": [P, DP, DP],
    "pf_vel_imposesym": [P],
    "pf_vel_matrices": [P],
    "pf_vel_transform": [P],
    "pf_vel_nonlinear": [P],
    "pf_vel_transform_nonlinear": [P],
    "pf_vel_predictor": [P],
    "pf_vel_corrector": [P],
    "pf_vel_maxtstep": [P],
    "pf_vel_influence_download": [P, DP, DP],
    "pf_timestep": [P, IP],
    "pf_steporbit": [P, I],
    "pf_util_set": [P, I, DP, I],
    "pf_util_set_callback": [P, P, P],
    "pf_util": [P, I],
    "pf_util_nu_stats": [P, DP, DP, DP],
    "pf_io_save_state": [P, C.c_char_p],
    "pf_io_load_state": [P, C.c_char_p, I, IP],
    "pf_state_write": [C.c_char_p, I, I, I, I, DP, DP, DP, DP, DP, DP, DP, DP],
    "pf_state_read": [C.c_char_p, I, I, I, I, DP, DP, DP, DP, DP, DP, DP, DP, IP],
    "pf_orbit_set_scales": [P, DP, D],
    "pf_orbit_vec_len": [P, C.POINTER(C.c_longlong)],
    "pf_orbit_rtz2vec": [P, P],
    "pf_orbit_vec2rtz": [P, P],
    "pf_orbit_dotprod": [P, I, P, P, DP],
    "pf_orbit_shiftdir": [P, I, P, P],
    "pf_orbit_step": [P, I, P, P],
    "pf_diag_energy": [P, DP],
    "pf_diag_friction": [P, DP, DP, DP],
    "pf_batch_create": [I, C.POINTER(pf_config), I, PP],
    "pf_batch_destroy": [P],
    "pf_batch_pipe": [P, I, PP],
    "pf_batch_matrices": [P],
    "pf_batch_step": [P, I, I, C.POINTER(C.c_longlong)],
    "pf_batch_sync": [P],
    "pf_batch_stream": [P, PP],
    "pf_batch_io_bytes": [P, C.POINTER(C.c_ulonglong)],
    "pf_batch_put_states": [P, I, P],
    "pf_batch_step_io": [P, I, I, I, C.POINTER(C.c_longlong)],
    "pf_batch_get_states": [P, I, P],
    "pf_batch_io_wait": [P, I],
    "pf_batch_io_sync": [P],
    "pf_batch_prof_enable": [P, I],
    "pf_batch_prof_read": [P, I, DP, C.POINTER(C.c_ulonglong)],
    "pf_batch_prof_read_staged": [P, I, DP, C.POINTER(C.c_ulonglong)],
    "pf_batch_launches": [P, C.POINTER(C.c_ulonglong)],
    "pf_batch_size": [P, C.POINTER(I)],
    "pf_batch_attach": [P, P],
    "pf_batch_detach": [P, P],
    "pf_batch_set_graphs": [P, I],
    "pf_serve_create": [I, C.c_ulonglong, I, I, PP],
    "pf_serve_destroy": [P],
    "pf_serve_submit": [P, C.POINTER(pf_config), I, DP, DP, DP, DP, DP, DP, C.POINTER(C.c_longlong)],
    "pf_serve_step": [P, C.POINTER(I), C.POINTER(I)],
    "pf_serve_finished": [P, C.POINTER(C.c_longlong), I, C.POINTER(I)],
    "pf_serve_result": [P, C.c_longlong, DP, DP, DP, DP, DP, DP],
    "pf_serve_cancel": [P, C.c_longlong],
    "pf_serve_stats": [P, C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(C.c_ulonglong),
                       C.POINTER(C.c_longlong)],
    "pf_serve_batch": [P, PP],
    "pf_batch_staged": [P, C.POINTER(I)],
    "pf_batch_set_worklist": [P, I],
    "pf_batch_get_worklist": [P, C.POINTER(I)],
    "pf_ctx_launches": [P, C.POINTER(C.c_ulonglong)],
    "pf_prof_enable": [P, I],
    "pf_prof_read": [P, I, DP, C.POINTER(C.c_ulonglong)],
}
_RESTYPES = {"pf_last_error": C.c_char_p}

_lib = None


def load() -> C.CDLL:
    """Load the library once and attach prototypes; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with "
            "`python softx-d-17-00015_b200/build.py` (no CPU fallback exists)")
    lib = C.CDLL(str(LIB_PATH))
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, C.c_int)
    _lib = lib
    return lib


def declared_symbols():
    return list(_SIGS)
