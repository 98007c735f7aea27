"""morphogen_b200 -- B200-native (sm_100a) per-server PIR answer path.

A drop-in for the reference's morphogen-gpu-dpf scan path: ChaCha8 GGM DPF
keys (unchanged wire format) are expanded over the whole row domain on the
GPU, every HBM-resident row is AND-masked with its 16-byte DPF output and
XOR-accumulated into the server's response share.  The compute lives in
libmorphogen_gpu.so (C ABI: include/morphogen_gpu.h); this package is the
host-side mirror of the reference's Rust interface.
"""
from .gpu_dpf import (  # noqa: F401
    ChaChaKey,
    ChaChaParams,
    CorrectionWord,
    DriverError,
    GpuDpfError,
    GpuPageMatrix,
    GpuScanner,
    KernelTiming,
    PirResult,
    Workspace,
    generate_chacha_dpf_keys,
    plan_tiled_launch_batch_sizes,
)

__all__ = [
    "ChaChaKey", "ChaChaParams", "CorrectionWord", "DriverError", "GpuDpfError", "GpuPageMatrix",
    "GpuScanner", "KernelTiming", "PirResult", "Workspace", "generate_chacha_dpf_keys",
    "plan_tiled_launch_batch_sizes",
]
