"""Build oracle/_ref/libmg_refkernels.so: the reference's own CUDA kernels
(crates/morphogen-gpu-dpf/cuda/fused_kernel.cu and fused_kernel_optimized.cu,
compiled unmodified from the reference tree for sm_100a) linked with the
launch harness oracle/ref_harness.cu.  Test infrastructure only: it is the
checker for page-mode parity and the timed reference GPU kernel, never part
of the product.  The reference sources are read where they lie; nothing is
copied into this repository.  Without the reference tree (the GPU box) the
prebuilt library is used as is.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
# The reference checkout (read-only); MORPHOGEN_REFERENCE_DIR overrides the
# location this recipe was written against.
REF_ROOT = Path(os.environ.get("MORPHOGEN_REFERENCE_DIR", "/root/reference"))
REF_CUDA = REF_ROOT / "crates" / "morphogen-gpu-dpf" / "cuda"
OUT = HERE / "_ref" / "libmg_refkernels.so"
SOURCES = [HERE / "ref_harness.cu", REF_CUDA / "fused_kernel.cu", REF_CUDA / "fused_kernel_optimized.cu"]


def build_if_present(force: bool = False) -> Path | None:
    if not REF_CUDA.exists():
        return OUT if OUT.exists() else None
    if OUT.exists() and not force and all(OUT.stat().st_mtime >= s.stat().st_mtime for s in SOURCES):
        return OUT
    OUT.parent.mkdir(parents=True, exist_ok=True)
    nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
    # -O3 as the reference's build.rs (build.rs:18-26), SASS for sm_100a.
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
           "-shared", "-cudart", "static", "-o", str(OUT), *map(str, SOURCES)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("building the reference kernels failed")
    return OUT


if __name__ == "__main__":
    print(build_if_present(force="--force" in sys.argv))
