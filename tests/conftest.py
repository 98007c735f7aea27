import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def scanner():
    from morphogen_b200.gpu_dpf import GpuScanner
    s = GpuScanner(0)
    yield s
    s.close()


def seeded_roots(seed: int, i: int):
    """Two 128-bit root seeds (4 u32 words each) for key pair i of a seeded run."""
    rng = np.random.default_rng([seed, i])
    return rng.integers(0, 2**32, 4, dtype=np.uint32), rng.integers(0, 2**32, 4, dtype=np.uint32)


def oracle_keypair(oracle, d: int, target: int, seed: int = 0, i: int = 0):
    s0, s1 = seeded_roots(seed, i)
    return oracle.keygen(d, target, s0, s1)


def xor_bytes(a: bytes, b: bytes) -> bytes:
    return (np.frombuffer(a, np.uint8) ^ np.frombuffer(b, np.uint8)).tobytes()
