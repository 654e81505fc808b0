"""Loads libghive_b200.so and declares the C-ABI prototypes.

The product path has no fallback: if the CUDA library is missing this module
raises, it never substitutes a CPU implementation.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libghive_b200.so")

_lib = None

P, I32, I64 = C.c_void_p, C.c_int32, C.c_int64

_PROTOS = {
    "ghb_abi_version": (I32, []),
    "ghb_ctx_create": (I32, [I32, I64, C.POINTER(C.c_void_p)]),
    "ghb_ctx_destroy": (I32, [P]),
    "ghb_last_error": (C.c_char_p, [P]),
    "ghb_sync": (I32, [P, P]),
    "ghb_kernel_launches": (I64, [P]),
    "ghb_ctx_set_spin_limit": (I32, [P, I32]),
    "ghb_ctx_set_log": (I32, [P, C.c_char_p, I32, C.c_double]),
    "ghb_filter": (I32, [P, P, P, I32, P, I32, P, I64, P, P]),
    "ghb_filter_groupby": (I32, [P, P, P, I32, P, I32, P, I32, P, I64, P, P, P]),
    "ghb_join_build": (I32, [P, P, P, I32, P, C.POINTER(C.c_void_p), P]),
    "ghb_join_table_free": (I32, [P, P]),
    "ghb_join_table_info": (I32, [P, P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]),
    "ghb_join_probe": (I32, [P, P, P, I32, P, P, I32, P, P, P, I64, P, P]),
    "ghb_sort": (I32, [P, P, P, P, I32, P, I32, P, P, P, P, P]),
    "ghb_filter_groupby_noalloc": (I32, [P, P, I32, P, I32, P, I32, P, I64, P, P, P]),
    "ghb_batch_groupby_create": (I32, [P, P, I32, I32, P, I32, P, I32, P, P, P,
                                       C.POINTER(C.c_void_p)]),
    "ghb_batch_launch": (I32, [P, P]),
    "ghb_jit_groupby_source": (I32, [P, P, I32, P, I32, P, I32, I32, C.c_char_p, I64]),
    "ghb_jit_compile_source": (I32, [C.c_char_p, C.POINTER(I64), C.c_char_p, I64]),
    "ghb_server_create": (I32, [I32, P, C.POINTER(C.c_void_p)]),
    "ghb_server_add_join_table": (I32, [P, P, P, I32, C.c_float, C.POINTER(I32)]),
    "ghb_server_submit": (I32, [P, P, C.POINTER(C.c_uint64)]),
    "ghb_server_wait": (I32, [P, C.c_uint64, P]),
    "ghb_server_release": (I32, [P, C.c_uint64]),
    "ghb_server_stats": (I32, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(I64)]),
    "ghb_server_last_error": (C.c_char_p, [P]),
    "ghb_server_destroy": (I32, [P]),
    "ghb_batch_describe": (I32, [P, C.c_char_p, I64]),
    "ghb_batch_destroy": (I32, [P]),
    "ghb_filter_host": (I32, [P, P, P, I32, P, I32, P, I64, C.POINTER(I64)]),
    "ghb_filter_groupby_host": (I32, [P, P, P, I32, P, I32, P, I32, P, I64, C.POINTER(I64), P]),
    "ghb_hash_join_host": (I32, [P, P, P, I32, P, I32, P, P, I32, P, P, P, I64,
                                 C.POINTER(I64), P]),
    "ghb_sort_host": (I32, [P, P, P, P, I32, P, I32, P, P, P, P]),
    "ghb_gtables_table": (I32, [P, I32, P, I32, C.POINTER(I32), C.POINTER(I64)]),
    "ghb_run_plan": (I32, [P, P, I32, P, I32, P]),
    "ghb_plan_result_free": (I32, [P]),
}


class GhbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%s)" % (msg, abi.STATUS_NAMES.get(code, code)))
        self.code = code


def lib():
    """The loaded library; raises ImportError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libghive_b200.so is not built (run `python -m ghive_b200.build`); "
                              "there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(L, name)
            fn.restype, fn.argtypes = res, args
        _lib = L
    return _lib


def declared_symbols():
    """Names of the functions include/ghive_b200.h declares."""
    import re
    hdr = os.path.join(os.path.dirname(HERE), "include", "ghive_b200.h")
    with open(hdr) as f:
        txt = f.read()
    return sorted(set(re.findall(r"^\s*(?:int32_t|int64_t|const char\*)\s+(ghb_\w+)\s*\(", txt, re.M)))
