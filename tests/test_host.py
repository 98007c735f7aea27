"""Host logic that runs without a GPU: the C-ABI library loads and exports
every symbol include/*.h declares, key generation / parsing match the oracle
byte for byte, and the reference's host policy helpers behave as its own
tests require (crates/morphogen-gpu-dpf/src/kernel.rs:1405-1441)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, oracle_keypair, seeded_roots

from morphogen_b200 import _native as N
from morphogen_b200 import gpu_dpf as G


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(mg_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(N.EXPORTED)


def test_library_is_sm100a_build():
    # The library embeds only sm_100a code: cuobjdump is not used; the build
    # recipe is checked instead.
    from morphogen_b200 import build
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)
    assert N.LIB_PATH.exists()


@pytest.mark.parametrize("d,target", [(1, 0), (1, 1), (8, 42), (20, 12345), (25, (1 << 25) - 1),
                                      (31, 1 << 30), (32, (1 << 32) - 1)])
def test_keygen_matches_oracle(oracle_mod, d, target):
    s0, s1 = seeded_roots(d, target & 0xFFFF)
    r0, r1 = s0.tobytes(), s1.tobytes()
    n = G.key_size(d)
    b0 = (C.c_uint8 * n)()
    b1 = (C.c_uint8 * n)()
    N.check(N.lib().mg_keygen(d, target, N.u8ptr(r0), N.u8ptr(r1), b0, b1))
    o0, o1 = oracle_mod.keygen(d, target, s0, s1)
    assert bytes(b0) == o0 and bytes(b1) == o1


def test_generate_keys_seeded_and_unseeded(oracle_mod):
    p = G.ChaChaParams(12)
    rng = np.random.default_rng(0)
    k0, k1 = G.generate_chacha_dpf_keys(p, 1000, rng)
    assert not k0.is_party1() and k1.is_party1() and k0.domain_bits == 12
    for i in (999, 1000, 1001):
        x = bytes(a ^ b for a, b in zip(oracle_mod.eval_point(k0.to_bytes(), i),
                                        oracle_mod.eval_point(k1.to_bytes(), i)))
        assert x == (b"\xff" * 16 if i == 1000 else bytes(16))
    u0, _ = G.generate_chacha_dpf_keys(p, 1000)
    assert u0.to_bytes() != k0.to_bytes()
    with pytest.raises(G.GpuDpfError):
        G.generate_chacha_dpf_keys(p, 4096)


def test_params_bounds():
    assert G.ChaChaParams(10).max_pages() == 1024
    for bad in (0, 33):
        with pytest.raises(G.GpuDpfError):
            G.ChaChaParams(bad)


def test_key_parsing_and_errors(oracle_mod):
    k0, _ = oracle_keypair(oracle_mod, 10, 42)
    key = G.ChaChaKey.from_bytes(k0)
    assert key.to_bytes() == k0 and key.domain_bits == 10 and key.party == 0
    assert len(key.correction_words) == 10 and key.final_cw == k0[-16:]
    with pytest.raises(G.GpuDpfError) as e:
        G.ChaChaKey(k0[:20])
    assert e.value.code == N.MG_EKEY and "too short" in e.value.message
    with pytest.raises(G.GpuDpfError) as e:
        G.ChaChaKey(k0 + b"\0")
    assert e.value.code == N.MG_EKEY and "length" in e.value.message
    # 40 levels: a well-formed reference key, beyond the device path's 32.
    big = bytearray(19 + 18 * 40 + 16)
    big[18] = 40
    with pytest.raises(G.GpuDpfError) as e:
        G.ChaChaKey(bytes(big))
    assert e.value.code == N.MG_ERANGE


def test_tiled_launch_batch_sizes_respect_requested_tile_limit():
    assert G.plan_tiled_launch_batch_sizes(17, 4) == [4, 4, 4, 4, 1]
    assert G.plan_tiled_launch_batch_sizes(6, 3) == [2, 2, 2]


def test_tiled_launch_batch_sizes_default_to_supported_minimum_when_zero():
    assert G.plan_tiled_launch_batch_sizes(5, 0) == [1, 1, 1, 1, 1]


def test_workspace_pool_size_defaults_and_clamps():
    assert G.parse_workspace_pool_size(None) == G.DEFAULT_WORKSPACE_POOL_SIZE
    assert G.parse_workspace_pool_size("0") == G.DEFAULT_WORKSPACE_POOL_SIZE
    assert G.parse_workspace_pool_size("999") == G.MAX_WORKSPACE_POOL_SIZE
    assert G.parse_workspace_pool_size("bad") == G.DEFAULT_WORKSPACE_POOL_SIZE
    assert G.parse_workspace_pool_size("6") == 6


def test_workspace_pool_slot_wraps_with_modulo():
    assert [G.select_workspace_pool_slot(t, 4) for t in (0, 1, 3, 4, 9)] == [0, 1, 3, 0, 1]


def test_context_create_reports_missing_device_cleanly():
    h = C.c_void_p()
    rc = N.lib().mg_context_create(0, C.byref(h))
    if rc == N.MG_OK:  # a GPU is visible: nothing to check here
        N.lib().mg_context_destroy(h)
        return
    assert rc == N.MG_ENODEV and N.last_error()


def test_null_arguments_are_rejected():
    lib = N.lib()
    assert lib.mg_context_create(0, None) == N.MG_EINVAL
    assert lib.mg_scan(None, None, None, None, 0, None, 0, None) == N.MG_EINVAL
    assert lib.mg_key_check(None, 0, None, None) == N.MG_EINVAL
    assert lib.mg_key_size(31) == 19 + 18 * 31 + 16
