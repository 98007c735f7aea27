"""Generate tests/golden/chacha20_openssl.json: ChaCha20 keystream blocks from
OpenSSL (through the `cryptography` package), used to pin the oracle's ChaCha
core.  The reference ships no ChaCha known-answer vectors
(crates/morphogen-gpu-dpf/src/chacha_prg.rs:254-262 only checks "not zero"),
so the pin is an independent ChaCha20 implementation: the oracle's block
function run with 10 double rounds must reproduce these bytes, and the
reference's ChaCha8 is the same function with 4 double rounds.

Run: python tests/golden/make_golden.py
"""
import json
import random
from pathlib import Path

from cryptography.hazmat.primitives.ciphers import Cipher, algorithms


def block(key: bytes, counter: int, nonce: bytes) -> bytes:
    enc = Cipher(algorithms.ChaCha20(key, counter.to_bytes(4, "little") + nonce), mode=None).encryptor()
    return enc.update(bytes(64))


def main():
    rng = random.Random(8439)
    cases = [
        # RFC 8439 section 2.3.2 inputs.
        (bytes(range(32)), 1, bytes.fromhex("000000090000004a00000000")),
        # The PRG's shape: key = seed || seed, nonce 0, counters 0 and 1.
        (bytes(16) * 2, 0, bytes(12)),
        (bytes(16) * 2, 1, bytes(12)),
    ]
    for _ in range(13):
        seed = rng.randbytes(16)
        cases.append((seed + seed, rng.choice([0, 1]), bytes(12)))
    for _ in range(8):
        cases.append((rng.randbytes(32), rng.randrange(1 << 32), rng.randbytes(12)))
    out = [{"key": k.hex(), "counter": c, "nonce": n.hex(), "block": block(k, c, n).hex()}
           for k, c, n in cases]
    path = Path(__file__).with_name("chacha20_openssl.json")
    path.write_text(json.dumps({"source": "OpenSSL ChaCha20 via cryptography", "cases": out}, indent=1) + "\n")
    print(path, len(out))


if __name__ == "__main__":
    main()
