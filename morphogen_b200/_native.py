"""ctypes binding of libmorphogen_gpu.so (the C ABI in include/morphogen_gpu.h).

The shared library is the product: every scan runs in its sm_100a kernels.
There is no fallback.  If the library is missing, importing this module's
loader raises, and calls fail with the library's own error codes.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path
from typing import Sequence

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libmorphogen_gpu.so"

MG_OK = 0
MG_EINVAL = 1
MG_EKEY = 2
MG_ERANGE = 3
MG_ENOMEM = 4
MG_ECUDA = 5
MG_ETIMEDOUT = 6
MG_ENODEV = 7
MG_EBUSY = 8
MAX_DOMAIN_BITS = 32
MAX_ROW_BYTES = 4096

# Every symbol include/morphogen_gpu.h declares.
EXPORTED = (
    "mg_context_create", "mg_context_destroy", "mg_last_error", "mg_device_info",
    "mg_table_create", "mg_table_create_range", "mg_table_first_row", "mg_table_destroy", "mg_table_write_rows", "mg_table_read_rows",
    "mg_table_fill_splitmix", "mg_table_xor_rows", "mg_table_rows", "mg_table_row_bytes",
    "mg_table_device_ptr", "mg_table_delta_reserve", "mg_table_delta_push", "mg_table_delta_count",
    "mg_table_delta_clear", "mg_table_delta_merge", "mg_table_epoch", "mg_key_size", "mg_key_check", "mg_keygen", "mg_scan",
    "mg_batch_create", "mg_batch_destroy", "mg_batch_set_keys", "mg_batch_set_shape", "mg_batch_set_kernel",
    "mg_batch_autotune",
    "mg_batch_launch", "mg_batch_launch_graph", "mg_batch_read", "mg_batch_sync",
    "mg_batch_shares_device", "mg_batch_plan", "mg_batch_last_kernel_ns", "mg_batch_last_scan_ns",
    "mg_eval_points", "mg_prg_peak", "mg_scan_noalloc",
    "mg_server_create", "mg_server_destroy", "mg_server_submit", "mg_server_wait", "mg_server_pause",
    "mg_server_resume", "mg_server_get_stats", "mg_server_reset_stats",
)


class MgError(RuntimeError):
    """A failing library call: `.code` is the MG_E* status."""

    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code
        self.message = message


class DriverError(MgError):
    """CUDA/device failure (the reference's cudarc DriverError)."""


class GpuDpfError(MgError):
    """Key or index error (the reference's GpuDpfError, dpf.rs:9-15)."""


class Timeout(MgError):
    pass


class Timing(C.Structure):
    _fields_ = [("h2d_ns", C.c_uint64), ("kernel_ns", C.c_uint64), ("d2h_ns", C.c_uint64),
                ("total_ns", C.c_uint64)]


class PlanInfo(C.Structure):
    _fields_ = [("subtree_bits", C.c_uint32), ("keys_per_cta", C.c_uint32), ("grid", C.c_uint32),
                ("items", C.c_uint32), ("segments", C.c_uint32), ("smem_bytes", C.c_uint32),
                ("kernel", C.c_uint32), ("frontier_nodes", C.c_uint32), ("kernels", C.c_uint32)]


KERNEL_AUTO, KERNEL_CTA, KERNEL_WARP = 0, 1, 2


class ServerConfig(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("max_keys_per_pass", C.c_uint32), ("memory_reserve", C.c_uint64)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("failed", C.c_uint64), ("passes", C.c_uint64),
                ("keys_completed", C.c_uint64), ("pending", C.c_uint32), ("in_flight", C.c_uint32),
                ("wall_s", C.c_double), ("p50_ms", C.c_double), ("p95_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("max_ms", C.c_double)]


_lib = None
_lock = threading.Lock()


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m morphogen_b200.build` "
                "(the sm_100a library is required; there is no CPU fallback)")
        L = C.CDLL(str(LIB_PATH))
        vp, u8p, u64p = C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.c_uint64)
        sz = C.c_size_t
        sig = {
            "mg_context_create": ([C.c_int, C.POINTER(vp)], C.c_int),
            "mg_context_destroy": ([vp], C.c_int),
            "mg_last_error": ([], C.c_char_p),
            "mg_device_info": ([vp, C.POINTER(C.c_int), u64p, u64p], C.c_int),
            "mg_table_create": ([vp, C.c_uint64, C.c_uint32, C.POINTER(vp)], C.c_int),
            "mg_table_create_range": ([vp, C.c_uint64, C.c_uint64, C.c_uint32, C.POINTER(vp)], C.c_int),
            "mg_table_first_row": ([vp], C.c_uint64),
            "mg_table_destroy": ([vp], C.c_int),
            "mg_table_write_rows": ([vp, C.c_uint64, vp, C.c_uint64], C.c_int),
            "mg_table_read_rows": ([vp, C.c_uint64, vp, C.c_uint64], C.c_int),
            "mg_table_fill_splitmix": ([vp, C.c_uint64], C.c_int),
            "mg_table_xor_rows": ([vp, u64p, vp, C.c_uint64], C.c_int),
            "mg_table_rows": ([vp], C.c_uint64),
            "mg_table_row_bytes": ([vp], C.c_uint32),
            "mg_table_device_ptr": ([vp], vp),
            "mg_table_delta_reserve": ([vp, C.c_uint32], C.c_int),
            "mg_table_delta_push": ([vp, u64p, vp, C.c_uint32], C.c_int),
            "mg_table_delta_count": ([vp], C.c_uint32),
            "mg_table_delta_clear": ([vp], C.c_int),
            "mg_table_delta_merge": ([vp], C.c_int),
            "mg_table_epoch": ([vp], C.c_uint64),
            "mg_key_size": ([C.c_uint32], sz),
            "mg_key_check": ([u8p, sz, C.POINTER(C.c_uint32), u8p], C.c_int),
            "mg_keygen": ([C.c_uint32, C.c_uint64, u8p, u8p, u8p, u8p], C.c_int),
            "mg_scan": ([vp, C.POINTER(vp), C.POINTER(u8p), C.POINTER(sz), C.c_uint32, u8p,
                         C.c_uint32, C.POINTER(Timing)], C.c_int),
            "mg_batch_create": ([vp, C.POINTER(vp)], C.c_int),
            "mg_batch_destroy": ([vp], C.c_int),
            "mg_batch_set_keys": ([vp, C.POINTER(vp), C.POINTER(u8p), C.POINTER(sz), C.c_uint32], C.c_int),
            "mg_batch_set_shape": ([vp, C.c_uint32, C.c_uint32], C.c_int),
            "mg_batch_set_kernel": ([vp, C.c_int], C.c_int),
            "mg_batch_autotune": ([vp, C.c_uint32, C.POINTER(PlanInfo), C.POINTER(C.c_double)], C.c_int),
            "mg_batch_launch": ([vp, vp], C.c_int),
            "mg_batch_launch_graph": ([vp, vp], C.c_int),
            "mg_batch_read": ([vp, u8p, vp], C.c_int),
            "mg_batch_sync": ([vp, C.c_uint32], C.c_int),
            "mg_batch_shares_device": ([vp, C.POINTER(vp), C.POINTER(sz)], C.c_int),
            "mg_batch_plan": ([vp, C.POINTER(PlanInfo)], C.c_int),
            "mg_batch_last_kernel_ns": ([vp, u64p], C.c_int),
            "mg_batch_last_scan_ns": ([vp, u64p], C.c_int),
            "mg_prg_peak": ([vp, C.c_uint32, C.POINTER(C.c_double)], C.c_int),
            "mg_eval_points": ([vp, u8p, sz, u64p, C.c_uint64, u8p], C.c_int),
            "mg_server_create": ([vp, C.POINTER(ServerConfig), C.POINTER(vp)], C.c_int),
            "mg_server_destroy": ([vp], C.c_int),
            "mg_server_submit": ([vp, C.POINTER(vp), C.POINTER(u8p), C.POINTER(sz), C.c_uint32, u64p], C.c_int),
            "mg_server_wait": ([vp, C.c_uint64, u8p, C.c_uint32, C.POINTER(C.c_double)], C.c_int),
            "mg_server_pause": ([vp, C.c_uint32], C.c_int),
            "mg_server_resume": ([vp], C.c_int),
            "mg_server_get_stats": ([vp, C.POINTER(ServerStats)], C.c_int),
            "mg_server_reset_stats": ([vp], C.c_int),
            "mg_scan_noalloc": ([C.c_int, vp, C.c_uint64, C.c_uint32, C.POINTER(u8p), C.POINTER(sz),
                                 C.c_uint32, vp, vp], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
        return _lib


def last_error() -> str:
    msg = lib().mg_last_error()
    return msg.decode() if msg else ""


def check(rc: int) -> None:
    if rc == MG_OK:
        return
    msg = last_error()
    if rc in (MG_EKEY, MG_ERANGE):
        raise GpuDpfError(rc, msg)
    if rc == MG_ETIMEDOUT:
        raise Timeout(rc, msg)
    if rc in (MG_ECUDA, MG_ENODEV, MG_ENOMEM):
        raise DriverError(rc, msg)
    raise MgError(rc, msg)


def u8ptr(buf) -> C.POINTER(C.c_uint8):
    """Pointer to the bytes of a bytes/bytearray/numpy buffer (caller keeps it alive)."""
    if isinstance(buf, bytes):
        return C.cast(C.c_char_p(buf), C.POINTER(C.c_uint8))
    import numpy as np
    arr = buf if isinstance(buf, np.ndarray) else np.frombuffer(buf, np.uint8)
    return arr.ctypes.data_as(C.POINTER(C.c_uint8))


class KeyArray:
    """C arrays of key pointers and lengths for one call (keeps the bytes alive)."""

    def __init__(self, keys: Sequence[bytes]):
        self.keys = [k if type(k) is bytes else bytes(k) for k in keys]
        n = len(self.keys)
        # A char* array holds references to the bytes objects; the C side
        # sees the same pointers as const uint8_t* const*.
        self._arr = (C.c_char_p * n)(*self.keys)
        self.ptrs = C.cast(self._arr, C.POINTER(C.POINTER(C.c_uint8)))
        self.lens = (C.c_size_t * n)(*[len(k) for k in self.keys])
        self.n = n
