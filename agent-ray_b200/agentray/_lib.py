"""Loader for libagentray.so (the C ABI in include/agentray.h).

The library is built in-tree (agent-ray_b200/libagentray.so).  There is no
fallback: if it is missing or fails to load, every entry point raises.
"""
import ctypes as C
import os

from . import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libagentray.so")

# Every symbol include/agentray.h declares, with its ctypes signature.
SIGNATURES = {
    "ar_last_error": (C.c_char_p, []),
    "ar_abi_version": (C.c_int, []),
    "ar_context_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "ar_context_destroy": (C.c_int, [C.c_void_p]),
    "ar_context_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "ar_context_synchronize": (C.c_int, [C.c_void_p]),
    "ar_scene_create": (C.c_int, [C.c_void_p, C.POINTER(A.SceneDesc), C.POINTER(C.c_void_p)]),
    "ar_scene_destroy": (C.c_int, [C.c_void_p]),
    "ar_scene_build_accel": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(A.AccelOpts)]),
    "ar_context_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(A.Tuning)]),
    "ar_film_to_rgb8": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.c_float,
                                  C.c_float, C.c_void_p, C.c_uint32]),
    "ar_film_save_exr": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32,
                                   C.c_char_p]),
    "ar_context_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(A.Tuning)]),
    "ar_autotune": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(A.CameraDesc), C.POINTER(A.TuneOpts),
                              C.POINTER(A.TuneResult)]),
    "ar_scene_get_stats": (C.c_int, [C.c_void_p, C.POINTER(A.SceneStats)]),
    "ar_trace_closest": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(A.RayBatch), C.c_void_p, C.c_void_p,
                                   C.c_uint32]),
    "ar_trace_any": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(A.RayBatch), C.c_void_p, C.c_uint32]),
    "ar_render_samples": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(A.CameraDesc), C.POINTER(A.IntegratorCfg),
                                    C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32]),
    "ar_render": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(A.CameraDesc), C.POINTER(A.IntegratorCfg),
                            C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32]),
    "ar_poisson_reconstruct": (C.c_int, [C.c_void_p, C.POINTER(A.IntegratorCfg), C.c_uint32, C.c_uint32,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                         C.POINTER(C.c_double)]),
    "ar_poisson_sor_static": (C.c_int, [C.POINTER(A.IntegratorCfg), C.c_uint32, C.c_uint32, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "ar_server_create": (C.c_int, [C.c_void_p, C.POINTER(A.ServerOpts), C.POINTER(C.c_void_p)]),
    "ar_server_destroy": (C.c_int, [C.c_void_p]),
    "ar_job_submit": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(A.CameraDesc), C.POINTER(A.IntegratorCfg),
                                C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32, C.POINTER(C.c_uint64)]),
    "ar_job_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(A.JobInfo)]),
    "ar_job_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.c_double, C.POINTER(A.JobInfo)]),
    "ar_job_cancel": (C.c_int, [C.c_void_p, C.c_uint64]),
    "ar_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(A.ServerStats)]),
    "ar_server_now_ms": (C.c_double, [C.c_void_p]),
    "ar_server_debug_dump": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint32]),
    "ar_get_render_stats": (C.c_int, [C.c_void_p, C.POINTER(A.RenderStats)]),
    "ar_profile_enable": (C.c_int, [C.c_void_p, C.c_int]),
    "ar_profile_reset": (C.c_int, [C.c_void_p]),
    "ar_profile_read": (C.c_int, [C.c_void_p, C.c_char_p, C.c_uint32, C.POINTER(C.c_double),
                                  C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
}

_lib = None


class AgentRayError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"agentray error {code}: {msg}")
        self.code = code


def lib():
    """Loads libagentray.so once; raises if it is absent (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C agent-ray_b200`")
        lb = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lb, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lb
    return _lib


def check(status):
    if status != A.AR_OK:
        msg = lib().ar_last_error()
        raise AgentRayError(status, msg.decode() if msg else "")
    return status
