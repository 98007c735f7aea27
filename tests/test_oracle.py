"""The CPU oracle, pinned: ChaCha core vs OpenSSL ChaCha20 fixtures, and the
reference's own DPF / fused-scan property tests restated
(crates/morphogen-gpu-dpf/src/dpf.rs:434-609, chacha_prg.rs:186-262,
kernel.rs:1385-1561)."""
import json
from pathlib import Path

import numpy as np
import pytest

from conftest import oracle_keypair, seeded_roots, xor_bytes

GOLDEN = Path(__file__).with_name("golden")
ONES = b"\xff" * 16
ZERO = bytes(16)


def test_chacha20_matches_openssl_fixtures(oracle_mod):
    cases = json.loads((GOLDEN / "chacha20_openssl.json").read_text())["cases"]
    assert len(cases) >= 20
    for c in cases:
        key = np.frombuffer(bytes.fromhex(c["key"]), np.uint32)
        nonce = np.frombuffer(bytes.fromhex(c["nonce"]), np.uint32)
        got = oracle_mod.chacha_block(key, c["counter"], nonce, double_rounds=10).tobytes()
        assert got.hex() == c["block"]


def test_prg_expand_is_chacha8_of_doubled_seed(oracle_mod):
    # chacha_prg.rs:153-178: key = seed||seed, nonce 0, counters 0/1.
    seed = np.array([0x12345678, 0x9ABCDEF0, 0xFEDCBA98, 0x76543210], np.uint32)
    L, R, lt, rt = oracle_mod.prg_expand(seed)
    key = np.concatenate([seed, seed])
    b0 = oracle_mod.chacha_block(key, 0, np.zeros(3, np.uint32), 4)
    b1 = oracle_mod.chacha_block(key, 1, np.zeros(3, np.uint32), 4)
    assert (L == b0[:4]).all() and (R == b0[4:8]).all()
    assert lt == (b1[0] & 1) and rt == (b1[1] & 1)
    # prg_deterministic / children differ / control bits binary (chacha_prg.rs:210-251)
    L2, R2, lt2, rt2 = oracle_mod.prg_expand(seed)
    assert (L == L2).all() and (R == R2).all() and (lt, rt) == (lt2, rt2)
    assert not (L == R).all()
    zL, zR, _, _ = oracle_mod.prg_expand(np.zeros(4, np.uint32))
    assert zL.any() and zR.any()  # chacha8_known_vector (chacha_prg.rs:254-262)


@pytest.mark.parametrize("d,target,points", [
    (8, 42, range(256)),                              # dpf_correctness_8bit
    (10, 500, [0, 1, 100, 500, 1000, 1023]),          # dpf_correctness_10bit
    (16, 32000, [0, 1, 32000, 65534, 65535]),         # dpf_correctness_16bit
])
def test_dpf_correctness(oracle_mod, d, target, points):
    k0, k1 = oracle_keypair(oracle_mod, d, target, seed=d)
    for i in points:
        x = xor_bytes(oracle_mod.eval_point(k0, i), oracle_mod.eval_point(k1, i))
        assert x == (ONES if i == target else ZERO), i


@pytest.mark.parametrize("bits", [4, 8, 12, 16])
def test_dpf_boundary_cases(oracle_mod, bits):
    mx = 1 << bits
    for j, target in enumerate([0, mx // 2, mx - 1]):
        k0, k1 = oracle_keypair(oracle_mod, bits, target, seed=bits, i=j)
        assert xor_bytes(oracle_mod.eval_point(k0, target), oracle_mod.eval_point(k1, target)) == ONES
        other = (target + 1) % mx
        assert xor_bytes(oracle_mod.eval_point(k0, other), oracle_mod.eval_point(k1, other)) == ZERO


def test_keygen_party_bits_and_rejections(oracle_mod):
    k0, k1 = oracle_keypair(oracle_mod, 8, 42)
    assert (k0[17], k1[17]) == (0, 1) and (k0[18], k1[18]) == (8, 8)
    assert len(k0) == 19 + 18 * 8 + 16
    s0, s1 = seeded_roots(0, 0)
    for d, t in [(8, 300), (0, 0), (33, 0)]:  # key_generation_rejects_out_of_range, params bounds
        with pytest.raises(ValueError):
            oracle_mod.keygen(d, t, s0, s1)


def test_full_eval_matches_point_eval(oracle_mod):
    k0, _ = oracle_keypair(oracle_mod, 8, 100)
    full = oracle_mod.eval_subtree(k0, 0, 256)
    for i in range(256):
        assert full[i].tobytes() == oracle_mod.eval_point(k0, i)


def test_subtree_matches_point_eval_deep(oracle_mod):
    k0, _ = oracle_keypair(oracle_mod, 31, 123456789, seed=5)
    start = 3 * 2048 + (1 << 30)
    sub = oracle_mod.eval_subtree(k0, start, 2048)
    for i in [0, 1, 777, 2046, 2047]:
        assert sub[i].tobytes() == oracle_mod.eval_point(k0, start + i)


def test_serialization_roundtrip(oracle_mod):
    k0, k1 = oracle_keypair(oracle_mod, 10, 42)
    for k in (k0, k1):
        assert oracle_mod.key_to_bytes(oracle_mod.parse_key(k)) == k
    with pytest.raises(ValueError):
        oracle_mod.parse_key(k0[:-1])
    with pytest.raises(ValueError):
        oracle_mod.parse_key(k0[:20])


def _pages(oracle_mod, n, row_bytes=4096):
    return oracle_mod.fill_test_rows(n, row_bytes).reshape(n, row_bytes)


def test_single_dpf_recovers_target_page(oracle_mod):
    pages = _pages(oracle_mod, 256)
    k0, k1 = oracle_keypair(oracle_mod, 8, 42)
    r = xor_bytes(oracle_mod.scan_pointwise(k0, pages, 4096), oracle_mod.scan_pointwise(k1, pages, 4096))
    assert r == pages[42].tobytes()


@pytest.mark.parametrize("d,npages,targets", [
    (8, 256, [10, 100, 200]),      # fused_3dpf_recovers_all_targets
    (10, 500, [5, 150, 300]),      # fused_handles_non_power_of_two_pages
    (12, 4096, [2048, 100, 3000]),  # tile_processing_correctness
])
def test_fused_recovers_targets(oracle_mod, d, npages, targets):
    pages = _pages(oracle_mod, npages)
    pairs = [oracle_keypair(oracle_mod, d, t, seed=d, i=j) for j, t in enumerate(targets)]
    a = oracle_mod.scan_fused([p[0] for p in pairs], pages, 4096)
    b = oracle_mod.scan_fused([p[1] for p in pairs], pages, 4096)
    for j, t in enumerate(targets):
        assert xor_bytes(a[j], b[j]) == pages[t].tobytes()
    # fused == pointwise, key by key
    for j in range(3):
        assert a[j] == oracle_mod.scan_pointwise(pairs[j][0], pages, 4096)


def test_fused_rejects_more_rows_than_domain(oracle_mod):
    k0, _ = oracle_keypair(oracle_mod, 4, 3)
    with pytest.raises(ValueError):
        oracle_mod.scan_fused([k0], _pages(oracle_mod, 17, 32), 32)


@pytest.mark.parametrize("row_bytes", [16, 32, 48, 64, 256])
def test_row_mode_recovers_target_row(oracle_mod, row_bytes):
    n = 3000
    rows = oracle_mod.fill_splitmix(0, n * row_bytes, 7).reshape(n, row_bytes)
    k0, k1 = oracle_keypair(oracle_mod, 12, 2999, seed=row_bytes)
    a = oracle_mod.scan_fused([k0], rows, row_bytes)[0]
    b = oracle_mod.scan_fused([k1], rows, row_bytes)[0]
    assert xor_bytes(a, b) == rows[2999].tobytes()


def test_row_base_window_equals_slice_of_full_scan(oracle_mod):
    # The CPU baseline times an aligned window of a larger domain; the window
    # scan must equal the same rows' contribution to a full scan.
    row_bytes, n, base = 32, 8192, 16384
    rows = oracle_mod.fill_splitmix(base * row_bytes, n * row_bytes, 3).reshape(n, row_bytes)
    k0, _ = oracle_keypair(oracle_mod, 20, 77, seed=9)
    win = oracle_mod.scan_fused([k0], rows, row_bytes, row_base=base)[0]
    masks = oracle_mod.eval_subtree(k0, base, n)
    acc = np.zeros(row_bytes, np.uint8)
    for i in range(n):
        acc ^= rows[i] & np.tile(masks[i], row_bytes // 16)
    assert win == acc.tobytes()


def test_delta_is_linear(oracle_mod):
    # Scanning (table XOR delta) == scanning table, XOR the delta scan (scan.rs:434-485).
    row_bytes, n = 32, 1024
    rows = oracle_mod.fill_splitmix(0, n * row_bytes, 11).reshape(n, row_bytes).copy()
    idx = np.array([5, 77, 1023, 77], np.uint64)
    diffs = oracle_mod.fill_splitmix(0, idx.size * row_bytes, 12).reshape(-1, row_bytes)
    keys = [oracle_keypair(oracle_mod, 10, t, seed=4, i=t)[0] for t in (5, 77, 500)]
    base = oracle_mod.scan_fused(keys, rows, row_bytes)
    delta = oracle_mod.delta_apply(keys, idx, diffs, row_bytes)
    patched = rows.copy()
    for i, r in enumerate(idx):
        patched[r] ^= diffs[i]
    after = oracle_mod.scan_fused(keys, patched, row_bytes)
    for j in range(3):
        assert xor_bytes(base[j], delta[j]) == after[j]


def test_generators(oracle_mod):
    # SplitMix64 stream: any byte range regenerates identically.
    full = oracle_mod.fill_splitmix(0, 4096, 42)
    part = oracle_mod.fill_splitmix(1000, 333, 42)
    assert (full[1000:1333] == part).all()
    w = oracle_mod.splitmix_word(42, 3)
    assert full[24:32].tobytes() == int(w).to_bytes(8, "little")
    # LCG fill (chunked_matrix.rs:83-93)
    state, ref = 7, []
    for _ in range(64):
        state = (state * 6364136223846793005 + 1) % (1 << 64)
        ref.append(state >> 56)
    assert oracle_mod.fill_lcg(64, 7).tolist() == ref
    # make_test_pages pattern (kernel.rs:1390-1403)
    p = oracle_mod.fill_test_rows(300, 64).reshape(300, 64)
    assert p[299, 0] == 299 & 0xFF and p[299, 1] == 1 and p[299, 5] == (299 + 5) & 0xFF


def test_nonbinary_t_bytes_follow_reference_semantics(oracle_mod):
    # from_bytes accepts any t byte (dpf.rs:277-316); a node corrects itself
    # only when t == 1 (dpf.rs:122).  A t_cw byte of 3 makes the child's t
    # differ from 1 even when its low bit is set.
    k0, _ = oracle_keypair(oracle_mod, 6, 9)
    b = bytearray(k0)
    b[16] = 1  # root_t
    for lvl in range(6):
        b[19 + 18 * lvl + 16] = 3
        b[19 + 18 * lvl + 17] = 2
    k = bytes(b)
    full = oracle_mod.eval_subtree(k, 0, 64)
    for i in range(64):
        assert full[i].tobytes() == oracle_mod.eval_point(k, i)


def test_oracle_matches_reference_kernel_fixtures(oracle_mod):
    """Shares recorded from the reference's own CUDA kernel
    (cuda/fused_kernel.cu, fused_batch_pir_kernel_1, built for sm_100a and run
    on a B200 by tests/golden/make_ref_fixtures.py) for make_test_pages pages
    (kernel.rs:1390-1403): the oracle reproduces every one."""
    import hashlib
    data = json.loads((GOLDEN / "ref_kernel_pages.json").read_text())
    assert len(data["cases"]) >= 4
    for case in data["cases"]:
        pages = oracle_mod.fill_test_rows(case["pages"], 4096)
        keys = [bytes.fromhex(k) for k in case["keys"]]
        got = oracle_mod.scan_fused(keys, pages, 4096)
        for j, share in enumerate(got):
            assert hashlib.sha256(share).hexdigest() == case["sha256"][j]
            assert share[:64].hex() == case["head"][j] and share[-64:].hex() == case["tail"][j]
            if "shares" in case:
                assert share.hex() == case["shares"][j]


@pytest.mark.parametrize("row_bytes,nrows", [(16, 4099), (32, 5001), (64, 3000), (256, 1027), (48, 700), (4096, 40)])
def test_avx512_scan_variant_equals_scalar(oracle_mod, row_bytes, nrows):
    # The CPU baseline's AVX-512-shaped AND/XOR loop gives the scalar path's shares.
    if not oracle_mod.avx512_available():
        pytest.skip("no AVX-512F on this CPU")
    from conftest import oracle_keypair
    d = max(13, (nrows - 1).bit_length())
    rows = oracle_mod.fill_splitmix(0, nrows * row_bytes, 900 + row_bytes)
    keys = [oracle_keypair(oracle_mod, d, (97 * j) % nrows, seed=901, i=j)[0] for j in range(3)]
    want = oracle_mod.scan_fused(keys, rows, row_bytes)
    assert oracle_mod.scan_fused(keys, rows, row_bytes, avx512=True) == want
    # a window that starts mid-tile
    assert (oracle_mod.scan_fused(keys, rows[row_bytes * 37:], row_bytes, row_base=37, avx512=True)
            == oracle_mod.scan_fused(keys, rows[row_bytes * 37:], row_bytes, row_base=37))
