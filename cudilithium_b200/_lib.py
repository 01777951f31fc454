"""ctypes binding of the in-tree CUDA library (C ABI of ``include/cudilithium.h``).

There is no fallback: if ``libcudilithium_b200.so`` is missing or fails to load, importing this
module raises, so nothing can silently run on the CPU.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_int, c_int32, c_size_t, c_uint8, c_uint16, c_uint32, c_void_p
from pathlib import Path

# CUDIL_LIB selects another build of the library (for example the bounds-checked
# libcudilithium_b200_bc.so); default: the in-tree libcudilithium_b200.so
LIB_PATH = (Path(os.environ["CUDIL_LIB"]) if os.environ.get("CUDIL_LIB")
            else Path(__file__).resolve().parent / "libcudilithium_b200.so")

CUDIL_OK = 0
CUDIL_ERR_INVALID = -1
CUDIL_ERR_CUDA = -2
CUDIL_ERR_TIMEOUT = -3
CUDIL_ERR_BUDGET = -4

_ERRORS = {
    CUDIL_ERR_INVALID: "invalid argument",
    CUDIL_ERR_CUDA: "CUDA error",
    CUDIL_ERR_TIMEOUT: "device wait timed out",
    CUDIL_ERR_BUDGET: "device-memory budget exceeded",
}


class CudilError(RuntimeError):
    def __init__(self, code: int, what: str):
        super().__init__(f"{what}: {_ERRORS.get(code, 'error')} ({code})")
        self.code = code


class cudil_params(ctypes.Structure):
    _fields_ = [(n, c_int) for n in (
        "mode", "k", "l", "eta", "tau", "beta", "gamma1", "gamma2", "omega",
        "pk_bytes", "sk_bytes", "sig_bytes", "polyz_packed", "polyw1_packed", "polyeta_packed")]


class cudil_sign_lut_element(ctypes.Structure):
    _fields_ = [("done_flag", c_int32), ("nonce", c_uint16)]


class cudil_copy_lut_element(ctypes.Structure):
    _fields_ = [("exec_idx", c_size_t), ("sign_idx", c_size_t)]


class cudil_task_lut(ctypes.Structure):
    _fields_ = [
        ("sign_lut", POINTER(cudil_sign_lut_element)),
        ("sign_lut_len", c_size_t),
        ("h_exec_lut", c_void_p),
        ("h_done_lut", c_void_p),
        ("h_copy_lut", c_void_p),
        ("d_exec_lut", c_void_p),
        ("d_done_lut", c_void_p),
        ("d_copy_lut", c_void_p),
    ]


class cudil_serve_config(ctypes.Structure):
    _fields_ = [("device_budget_bytes", c_size_t), ("path", c_int32), ("slots_per_lane", c_int32),
                ("max_batch", c_int32), ("engine_threads", c_int32), ("engine_spec_slots", c_int32),
                ("plain_exec_threshold", c_int32), ("max_mlen", c_uint32), ("lane_slots_by_load", c_uint32)]


class cudil_serve_stats(ctypes.Structure):
    _fields_ = [("wall_s", ctypes.c_double), ("batches", c_size_t), ("slots", c_size_t),
                ("device_bytes", c_size_t), ("host_stage_s", ctypes.c_double), ("device_wait_s", ctypes.c_double),
                ("host_post_s", ctypes.c_double)]


# Every symbol the public header declares, with its ctypes signature.
SIGNATURES = {
    "cudil_version": (c_char_p, []),
    "cudil_last_error": (c_char_p, []),
    "cudil_get_params": (c_int, [c_int, POINTER(cudil_params)]),
    "cudil_keypair_row_bytes": (c_size_t, [c_int]),
    "cudil_sign_row_bytes": (c_size_t, [c_int, c_size_t]),
    "cudil_sign_temp_row_bytes": (c_size_t, [c_int]),
    "cudil_verify_row_bytes": (c_size_t, [c_int, c_size_t]),
    "cudil_keypair": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p, c_size_t]),
    "cudil_keypair_from_seed": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p]),
    "cudil_keypair_dev": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p, c_size_t]),
    "cudil_sign": (c_int, [c_int, c_void_p, c_size_t, POINTER(c_size_t), c_void_p, c_size_t, c_size_t, c_void_p,
                           c_void_p, c_size_t, c_void_p, c_size_t, POINTER(cudil_task_lut), c_size_t, c_size_t,
                           c_void_p]),
    "cudil_sign_randomized": (c_int, [c_int, c_void_p, c_size_t, POINTER(c_size_t), c_void_p, c_size_t, c_size_t,
                                      c_void_p, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p, c_size_t,
                                      POINTER(cudil_task_lut), c_size_t, c_size_t, c_void_p]),
    "cudil_sign_dev_randomized": (c_int, [c_int, c_void_p, c_size_t, c_void_p, c_size_t, c_size_t, c_void_p, c_void_p,
                                          c_size_t, c_void_p, c_size_t, c_void_p, c_size_t, POINTER(cudil_task_lut),
                                          c_size_t, c_size_t, c_void_p]),
    "cudil_sign_dev": (c_int, [c_int, c_void_p, c_size_t, c_void_p, c_size_t, c_size_t, c_void_p, c_void_p, c_size_t,
                               c_void_p, c_size_t, POINTER(cudil_task_lut), c_size_t, c_size_t, c_void_p]),
    "cudil_verify": (c_int, [c_int, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p, c_size_t, c_size_t, c_void_p,
                             c_void_p, c_size_t, c_size_t, c_void_p]),
    "cudil_verify_dev": (c_int, [c_int, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p, c_size_t, c_size_t,
                                 c_void_p, c_void_p, c_size_t, c_size_t, c_void_p]),
    "cudil_crypto_sign": (c_int, [c_int, c_void_p, c_size_t, POINTER(c_size_t), c_void_p, c_size_t, c_size_t, c_void_p,
                                  c_void_p, c_size_t, c_void_p, c_size_t, POINTER(cudil_task_lut), c_size_t, c_size_t,
                                  c_void_p]),
    "cudil_crypto_sign_open": (c_int, [c_int, c_void_p, c_size_t, POINTER(c_size_t), c_void_p, c_void_p, c_size_t,
                                       c_size_t, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p]),
    "cudil_sig_check": (c_int, [c_int, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p]),
    "cudil_sk_check": (c_int, [c_int, c_void_p, c_void_p, c_size_t, c_void_p]),
    "cudil_ntt_mul": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "cudil_sign_dev_varlen": (c_int, [c_int, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p, c_size_t, c_void_p,
                                      c_void_p, c_size_t, c_void_p, c_size_t, POINTER(cudil_task_lut), c_size_t,
                                      c_size_t, c_void_p]),
    "cudil_verify_dev_varlen": (c_int, [c_int, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p, c_size_t, c_void_p,
                                        c_size_t, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p]),
    "cudil_verify_noalloc_max_batch": (c_size_t, [c_int, c_size_t]),
    "cudil_verify_noalloc": (c_int, [c_int, c_void_p, c_void_p, c_size_t, c_size_t, c_void_p, c_size_t, c_size_t,
                                     c_void_p, c_size_t, c_void_p]),
    "cudil_engine_create": (c_int, [POINTER(c_void_p), c_int, c_size_t, c_size_t, c_int, c_size_t]),
    "cudil_engine_destroy": (c_int, [c_void_p]),
    "cudil_engine_device_bytes": (c_size_t, [c_void_p]),
    "cudil_engine_set_secret_keys": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p]),
    "cudil_engine_update_secret_keys": (c_int, [c_void_p, c_void_p, c_size_t, c_size_t, c_void_p]),
    "cudil_engine_attach_keys": (c_int, [c_void_p, c_void_p]),
    "cudil_engine_set_public_keys": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p]),
    "cudil_engine_sign": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_size_t,
                                  c_void_p]),
    "cudil_engine_sign_randomized": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p,
                                             c_void_p, c_size_t, c_void_p]),
    "cudil_engine_verify": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p,
                                    c_size_t, c_void_p]),
    "cudil_engine_last_status": (c_int, [c_void_p, POINTER(ctypes.c_ulonglong), POINTER(c_uint32)]),
    "cudil_engine_last_work": (c_int, [c_void_p, POINTER(ctypes.c_ulonglong), POINTER(ctypes.c_ulonglong)]),
    "cudil_engine_last_phases": (c_int, [c_void_p, POINTER(ctypes.c_ulonglong), POINTER(c_uint32)]),
    "cudil_engine_set_spec_slots": (c_int, [c_void_p, c_uint32]),
    "cudil_engine_set_sign_kernel": (c_int, [c_void_p, c_int]),
    "cudil_engine_set_limits": (c_int, [c_void_p, c_uint32, c_uint32, c_uint32]),
    "cudil_engine_sign_seeded": (c_int, [c_void_p, c_void_p, c_void_p, c_size_t, c_void_p, c_void_p, c_void_p,
                                         c_void_p, ctypes.c_ulonglong, c_size_t, c_void_p]),
    "cudil_derive_rhoprime": (c_int, [c_void_p, c_size_t, c_void_p, ctypes.c_ulonglong, c_size_t, c_void_p]),
    "cudil_bounds_check_status": (c_int, [POINTER(c_uint32), c_int]),
    "cudil_engine_last_nonces": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p]),
    "cudil_engine_set_large_batch": (c_int, [c_void_p, c_size_t, c_int, c_uint32]),
    "cudil_engine_last_jobs": (c_int, [c_void_p, POINTER(ctypes.c_ulonglong)]),
    "cudil_engine_info": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "cudil_serve_trace": (c_int, [POINTER(cudil_serve_config), POINTER(c_void_p), POINTER(c_void_p),
                                  POINTER(c_size_t), c_void_p, c_size_t, c_void_p, c_void_p, c_void_p, c_size_t,
                                  c_void_p, POINTER(cudil_serve_stats)]),
    "cudil_alu_peak": (c_int, [c_void_p, c_int, c_int, c_void_p, POINTER(ctypes.c_double)]),
    "cudil_launch_count": (ctypes.c_ulonglong, []),
    "cudil_kernel_timing": (None, [c_int]),
    "cudil_kernel_count": (c_int, []),
    "cudil_kernel_name": (c_char_p, [c_int]),
    "cudil_kernel_stats": (c_int, [c_int, POINTER(ctypes.c_double), POINTER(ctypes.c_ulonglong)]),
    "cudil_kernel_stats_reset": (None, []),
}


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python cudilithium_b200/build.py` "
            "(the CUDA path has no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(code: int, what: str) -> None:
    if code != CUDIL_OK:
        if code == CUDIL_ERR_CUDA:
            what = f"{what} [{lib.cudil_last_error().decode()}]"
        raise CudilError(code, what)


def kernel_stats() -> dict:
    """{kernel name: (total device ms, launches)} accumulated while cudil_kernel_timing(1) was on."""
    out = {}
    for i in range(lib.cudil_kernel_count()):
        ms, n = ctypes.c_double(0), ctypes.c_ulonglong(0)
        lib.cudil_kernel_stats(i, ctypes.byref(ms), ctypes.byref(n))
        if n.value:
            out[lib.cudil_kernel_name(i).decode()] = (ms.value, n.value)
    return out


def params(mode: int) -> cudil_params:
    p = cudil_params()
    check(lib.cudil_get_params(mode, ctypes.byref(p)), f"cudil_get_params({mode})")
    return p
