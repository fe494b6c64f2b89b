"""ctypes binding of the C ABI in include/kratos_b200.h (libkrb200.so)."""
import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
# KRATOS_B200_VARIANT=nofma selects the parity build (no fused multiply-add,
# the reference's own CPU arithmetic), used by tests only
_VARIANT = os.environ.get("KRATOS_B200_VARIANT", "")
LIB_PATH = os.path.join(_PKG, "libkrb200%s.so" % ("_" + _VARIANT if _VARIANT else ""))

KR_ABI_VERSION = 7
KR_FLAG_HALO_ALL, KR_FLAG_BOXES, KR_FLAG_UNFUSED = 2, 4, 8
BC_KINDS = {"per": 0, "out": 1, "ref": 2, "fre": 3, "fixd": 4}
KR_RIEMANN_DEFAULT, KR_RIEMANN_HLLE, KR_RIEMANN_LEARNED = 0, 1, 2
KR_INTEGRATOR_RK2, KR_INTEGRATOR_VL2 = 0, 1


class kr_cfg(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_int),
        ("mhd", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("riemann", ctypes.c_int),
        ("nb", ctypes.c_int * 3),
        ("n", ctypes.c_int * 3),
        ("x_min", ctypes.c_double * 3),
        ("x_max", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("rho_floor", ctypes.c_double),
        ("tmp_floor", ctypes.c_double),
        ("dt_init", ctypes.c_double),
        ("dt_expand", ctypes.c_double),
        ("device", ctypes.c_int),
        ("bc", ctypes.c_int * 6),
        ("w_fix", ctypes.c_double * 5),
        ("b_fix", ctypes.c_double * 3),
        ("flags", ctypes.c_int),
        ("n_ranks", ctypes.c_int),
        ("rank", ctypes.c_int),
        ("sel_period", ctypes.c_int),
        ("integrator", ctypes.c_int),
        ("reserved", ctypes.c_int * 2),
    ]


class kr_region(ctypes.Structure):
    _fields_ = [
        ("level", ctypes.c_int),
        ("x_min", ctypes.c_double * 3),
        ("x_max", ctypes.c_double * 3),
    ]


# name -> (restype, argtypes); every symbol include/kratos_b200.h declares
_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
SIGNATURES = {
    "kr_cfg_default": (None, [ctypes.POINTER(kr_cfg)]),
    "kr_ctx_create": (_vp, [ctypes.POINTER(kr_cfg)]),
    "kr_ctx_destroy": (None, [_vp]),
    "kr_ctx_create_refined": (_vp, [ctypes.POINTER(kr_cfg), ctypes.c_int, ctypes.POINTER(kr_region)]),
    "kr_block_info": (ctypes.c_int, [_vp, _vp, _vp]),
    "kr_last_error": (ctypes.c_char_p, [_vp]),
    "kr_set_stream": (ctypes.c_int, [_vp, _vp]),
    "kr_init_problem": (ctypes.c_int, [_vp, ctypes.c_char_p, ctypes.c_uint64]),
    "kr_box_params": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_int, ctypes.c_double, _dp]),
    "kr_init_boxes": (ctypes.c_int, [_vp, ctypes.c_uint64, _vp]),
    "kr_box_times": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "kr_set_state": (ctypes.c_int, [_vp, _vp, _vp]),
    "kr_get_state": (ctypes.c_int, [_vp, _vp, _vp]),
    "kr_step": (ctypes.c_int, [_vp, ctypes.c_int]),
    "kr_get_time": (ctypes.c_int, [_vp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_longlong)]),
    "kr_set_time": (ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    "kr_status": (ctypes.c_int, [_vp]),
    "kr_launches_per_step": (ctypes.c_int, [_vp]),
    "kr_profile_step": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    "kr_c2p_dt_noalloc": (ctypes.c_int, [ctypes.POINTER(kr_cfg), _vp, _vp, _vp, _vp, _vp]),
    "kr_set_selector": (ctypes.c_int, [_vp, _vp, ctypes.c_float]),
    "kr_selector_stats": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong),
                                         ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]),
    "kr_selector_collect": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_uint, ctypes.c_uint64,
                                           ctypes.c_longlong, _vp, ctypes.POINTER(ctypes.c_longlong)]),
    "kr_mlp_param_count": (ctypes.c_int, []),
    "kr_mlp_init": (None, [_vp, ctypes.c_uint64]),
    "kr_mlp_grad": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _vp, ctypes.c_float, _vp,
                                   ctypes.POINTER(ctypes.c_double), ctypes.c_int]),
    "kr_mlp_train": (ctypes.c_int, [_vp, _vp, ctypes.c_longlong, _vp, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_float, ctypes.POINTER(ctypes.c_double),
                                    ctypes.c_int]),
    "kr_mlp_infer": (ctypes.c_int, [_vp, ctypes.c_longlong, _vp, _vp, ctypes.c_int]),
    "kr_learn_last_error": (ctypes.c_char_p, []),
    "kr_diagnostics": (ctypes.c_int, [_vp, _dp, _dp]),
    "kr_shard_owner": (ctypes.c_int, [ctypes.POINTER(kr_cfg), _vp]),
    "kr_halo_counts": (ctypes.c_int, [ctypes.POINTER(kr_cfg), _vp, _vp]),
    "kr_shard_blocks": (ctypes.c_int, [_vp, _vp]),
    "kr_comm_unique_id": (ctypes.c_int, [_vp]),
    "kr_comm_init": (ctypes.c_int, [_vp, _vp]),
    "kr_group_step": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    "kr_batch_create": (_vp, [_vp, ctypes.c_int]),
    "kr_batch_destroy": (None, [_vp]),
    "kr_batch_last_error": (ctypes.c_char_p, [_vp]),
    "kr_batch_step": (ctypes.c_int, [_vp, ctypes.c_int]),
    "kr_batch_launches_per_step": (ctypes.c_int, [_vp]),
    "kr_batch_get_grid": (ctypes.c_int, [_vp, _vp]),
    "kr_batch_set_grid": (ctypes.c_int, [_vp, _vp]),
    "kr_batch_autotune": (ctypes.c_int, [_vp, ctypes.c_char_p, _vp]),
    "kr_batch_profile_step": (ctypes.c_int, [_vp, ctypes.c_int, _vp]),
}

_lib = None


class EngineMissing(RuntimeError):
    pass


def lib():
    """Load libkrb200.so.  There is no fallback: without the compiled engine
    every entry point raises."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineMissing("%s is missing; build it with `python -m kratos_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib
