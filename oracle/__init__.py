"""CPU oracle for the per-server ChaCha8-DPF PIR answer path.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU baseline / reference arm import this package, and only as the checker or
the timed CPU restatement of the reference.  The product
(morphogen_b200, libmorphogen_gpu.so) never imports, loads or calls it.

The C code in mg_oracle.c restates the reference's CPU algorithm
(crates/morphogen-gpu-dpf/src/{chacha_prg,dpf,kernel}.rs and
crates/morphogen-server/src/scan.rs:434-485), function by function with
file:line citations.  How it is pinned: tests/test_oracle.py (ChaCha20 against
OpenSSL through the `cryptography` package, the reference's own DPF property
tests) and the GPU test that compares page-mode shares with the reference's own
CUDA kernels built into oracle/_ref.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libmg_oracle.so"
MAX_LEVELS = 64


class _Key(C.Structure):
    _fields_ = [
        ("root_seed", C.c_uint32 * 4),
        ("root_t", C.c_uint8),
        ("party", C.c_uint8),
        ("domain_bits", C.c_uint32),
        ("cw_seed", (C.c_uint32 * 4) * MAX_LEVELS),
        ("cw_tl", C.c_uint8 * MAX_LEVELS),
        ("cw_tr", C.c_uint8 * MAX_LEVELS),
        ("final_cw", C.c_uint32 * 4),
    ]


def build() -> Path:
    """Compile the oracle with the committed Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        u8p = C.POINTER(C.c_uint8)
        u32p = C.POINTER(C.c_uint32)
        u64p = C.POINTER(C.c_uint64)
        kp = C.POINTER(_Key)
        L.mgo_chacha_block.argtypes = [u32p, C.c_uint32, u32p, C.c_int, u32p]
        L.mgo_prg_expand.argtypes = [u32p, u32p, u32p, u8p, u8p]
        L.mgo_key_from_bytes.argtypes = [u8p, C.c_size_t, kp]
        L.mgo_key_to_bytes.argtypes = [kp, u8p]
        L.mgo_key_to_bytes.restype = C.c_size_t
        L.mgo_eval.argtypes = [kp, C.c_uint64, u32p]
        L.mgo_eval_subtree.argtypes = [kp, C.c_uint64, C.c_uint64, u32p]
        L.mgo_keygen.argtypes = [C.c_uint32, C.c_uint64, u32p, u32p, kp, kp]
        L.mgo_scan_fused.argtypes = [kp, C.c_int, u8p, C.c_uint64, C.c_uint32, C.c_uint64, u8p, C.c_int]
        L.mgo_scan_fused_avx512.argtypes = [kp, C.c_int, u8p, C.c_uint64, C.c_uint32, C.c_uint64, u8p, C.c_int]
        L.mgo_avx512_available.argtypes = []
        L.mgo_scan_pointwise.argtypes = [kp, u8p, C.c_uint64, C.c_uint32, u8p]
        L.mgo_delta_apply.argtypes = [kp, C.c_int, u64p, u8p, C.c_uint64, C.c_uint32, u8p]
        L.mgo_fill_splitmix.argtypes = [u8p, C.c_uint64, C.c_uint64, C.c_uint64]
        L.mgo_splitmix_word.argtypes = [C.c_uint64, C.c_uint64]
        L.mgo_splitmix_word.restype = C.c_uint64
        L.mgo_fill_lcg.argtypes = [u8p, C.c_uint64, C.c_uint64]
        L.mgo_fill_test_rows.argtypes = [u8p, C.c_uint64, C.c_uint32]
        _lib = L
    return _lib


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(C.POINTER(C.c_uint32))


def _u8(a):
    a = np.ascontiguousarray(a, dtype=np.uint8)
    return a, a.ctypes.data_as(C.POINTER(C.c_uint8))


def chacha_block(key8, counter: int, nonce3, double_rounds: int = 4) -> np.ndarray:
    k, kp = _u32(key8)
    n, np_ = _u32(nonce3)
    out = np.zeros(16, np.uint32)
    lib().mgo_chacha_block(kp, counter, np_, double_rounds, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out


def prg_expand(seed4):
    s, sp = _u32(seed4)
    L = np.zeros(4, np.uint32)
    R = np.zeros(4, np.uint32)
    lt, rt = C.c_uint8(), C.c_uint8()
    lib().mgo_prg_expand(sp, L.ctypes.data_as(C.POINTER(C.c_uint32)),
                         R.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(lt), C.byref(rt))
    return L, R, lt.value, rt.value


def parse_key(key: bytes) -> _Key:
    k = _Key()
    b, bp = _u8(np.frombuffer(bytes(key), np.uint8))
    rc = lib().mgo_key_from_bytes(bp, len(key), C.byref(k))
    if rc != 0:
        raise ValueError(f"oracle: malformed key ({rc})")
    return k


def key_to_bytes(k: _Key) -> bytes:
    buf = np.zeros(19 + 18 * MAX_LEVELS + 16, np.uint8)
    n = lib().mgo_key_to_bytes(C.byref(k), buf.ctypes.data_as(C.POINTER(C.c_uint8)))
    return buf[:n].tobytes()


def keygen(domain_bits: int, target: int, seed0, seed1) -> tuple[bytes, bytes]:
    """generate_chacha_dpf_keys with the two 128-bit root seeds given as 4 u32 words."""
    s0, p0 = _u32(seed0)
    s1, p1 = _u32(seed1)
    k0, k1 = _Key(), _Key()
    rc = lib().mgo_keygen(domain_bits, target, p0, p1, C.byref(k0), C.byref(k1))
    if rc != 0:
        raise ValueError(f"oracle: keygen rejected ({rc})")
    return key_to_bytes(k0), key_to_bytes(k1)


def eval_point(key: bytes, index: int) -> bytes:
    k = parse_key(key)
    out = np.zeros(4, np.uint32)
    lib().mgo_eval(C.byref(k), index, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    return out.tobytes()


def eval_subtree(key: bytes, start: int, n: int) -> np.ndarray:
    k = parse_key(key)
    out = np.zeros(n * 4, np.uint32)
    rc = lib().mgo_eval_subtree(C.byref(k), start, n, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    if rc != 0:
        raise ValueError("oracle: bad subtree")
    return out.view(np.uint8).reshape(n, 16)


def _keys_array(keys):
    arr = (_Key * len(keys))()
    for i, kb in enumerate(keys):
        arr[i] = parse_key(kb)
    return arr


def avx512_available() -> bool:
    return bool(lib().mgo_avx512_available())


def scan_fused(keys, rows: np.ndarray, row_bytes: int, row_base: int = 0, nthreads: int = 0,
               avx512: bool = False) -> list[bytes]:
    """eval_fused_3dpf_cpu generalised: one share of row_bytes per key.
    avx512: the AND/XOR loop in 512-bit registers, eight rows per step (the
    shape of the reference server's AVX-512 scan); same result."""
    rows = np.ascontiguousarray(rows, dtype=np.uint8).reshape(-1)
    nrows = rows.size // row_bytes
    karr = _keys_array(keys)
    out = np.zeros(len(keys) * row_bytes, np.uint8)
    fn = lib().mgo_scan_fused_avx512 if avx512 else lib().mgo_scan_fused
    rc = fn(karr, len(keys), rows.ctypes.data_as(C.POINTER(C.c_uint8)), nrows,
            row_bytes, row_base, out.ctypes.data_as(C.POINTER(C.c_uint8)), nthreads)
    if rc == -2:
        raise RuntimeError("oracle: this CPU has no AVX-512F")
    if rc != 0:
        raise ValueError("oracle: scan precondition failed (more rows than domain size?)")
    return [out[i * row_bytes:(i + 1) * row_bytes].tobytes() for i in range(len(keys))]


def scan_pointwise(key: bytes, rows: np.ndarray, row_bytes: int) -> bytes:
    rows = np.ascontiguousarray(rows, dtype=np.uint8).reshape(-1)
    k = parse_key(key)
    out = np.zeros(row_bytes, np.uint8)
    lib().mgo_scan_pointwise(C.byref(k), rows.ctypes.data_as(C.POINTER(C.c_uint8)), rows.size // row_bytes,
                             row_bytes, out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out.tobytes()


def delta_apply(keys, row_idx, diffs: np.ndarray, row_bytes: int) -> list[bytes]:
    idx = np.ascontiguousarray(row_idx, dtype=np.uint64)
    diffs = np.ascontiguousarray(diffs, dtype=np.uint8).reshape(-1)
    karr = _keys_array(keys)
    out = np.zeros(len(keys) * row_bytes, np.uint8)
    lib().mgo_delta_apply(karr, len(keys), idx.ctypes.data_as(C.POINTER(C.c_uint64)),
                          diffs.ctypes.data_as(C.POINTER(C.c_uint8)), idx.size, row_bytes,
                          out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return [out[i * row_bytes:(i + 1) * row_bytes].tobytes() for i in range(len(keys))]


def fill_splitmix(byte_offset: int, nbytes: int, seed: int) -> np.ndarray:
    buf = np.zeros(nbytes, np.uint8)
    lib().mgo_fill_splitmix(buf.ctypes.data_as(C.POINTER(C.c_uint8)), byte_offset, nbytes, seed)
    return buf


def splitmix_word(seed: int, index: int) -> int:
    return int(lib().mgo_splitmix_word(seed, index))


def fill_lcg(nbytes: int, seed: int) -> np.ndarray:
    buf = np.zeros(nbytes, np.uint8)
    lib().mgo_fill_lcg(buf.ctypes.data_as(C.POINTER(C.c_uint8)), nbytes, seed)
    return buf


def fill_test_rows(nrows: int, row_bytes: int) -> np.ndarray:
    buf = np.zeros(nrows * row_bytes, np.uint8)
    lib().mgo_fill_test_rows(buf.ctypes.data_as(C.POINTER(C.c_uint8)), nrows, row_bytes)
    return buf


# ---- the reference's own CUDA kernels (built by oracle/ref_build.py) -------

REF_LIB_PATH = HERE / "_ref" / "libmg_refkernels.so"
REF_MAX_DOMAIN_BITS = 25
REF_PAGE_BYTES = 4096
_ref = None


def ref_available() -> bool:
    return REF_LIB_PATH.exists()


def ref_lib():
    global _ref
    if _ref is None:
        L = C.CDLL(str(REF_LIB_PATH))
        L.ref_key_pod.argtypes = [C.POINTER(C.c_uint8), C.c_size_t, C.POINTER(C.c_uint8)]
        L.ref_scan.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.POINTER(C.c_uint8),
                               C.POINTER(C.c_uint8), C.c_int, C.POINTER(C.c_float)]
        _ref = L
    return _ref


def ref_scan(kind: int, keys, db_dev_ptr: int, num_pages: int, reps: int = 1):
    """Run the reference kernel over num_pages 4096-byte pages at db_dev_ptr.
    kind 0: baseline fused_batch_pir_kernel_1 (3 keys); kind 1: optimized
    kernel with batch = len(keys) / 3 in {1, 2, 4}.  Returns (shares, best ms)."""
    L = ref_lib()
    nk = len(keys)
    if nk % 3:
        raise ValueError("the reference kernels take 3 keys per query")
    pods = np.zeros(nk * 488, np.uint8)
    for i, k in enumerate(keys):
        kb = np.frombuffer(bytes(k), np.uint8)
        if kb[18] > REF_MAX_DOMAIN_BITS:
            raise ValueError("the reference kernel evaluates at most 25 levels")
        rc = L.ref_key_pod(kb.ctypes.data_as(C.POINTER(C.c_uint8)), kb.size,
                           pods[i * 488:].ctypes.data_as(C.POINTER(C.c_uint8)))
        if rc:
            raise ValueError("malformed key")
    out = np.zeros(nk * REF_PAGE_BYTES, np.uint8)
    ms = C.c_float()
    rc = L.ref_scan(kind, nk // 3, C.c_void_p(db_dev_ptr), num_pages, pods.ctypes.data_as(C.POINTER(C.c_uint8)),
                    out.ctypes.data_as(C.POINTER(C.c_uint8)), reps, C.byref(ms))
    if rc:
        raise RuntimeError(f"reference kernel launch failed (cudaError {rc})")
    return [out[i * REF_PAGE_BYTES:(i + 1) * REF_PAGE_BYTES].tobytes() for i in range(nk)], ms.value
