"""Builds libor_ecycle.so in-tree for sm_100a (nvcc cross-compiles without a GPU).

    python -m openradioss_b200.build [--verbose]
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = [os.path.join(HERE, "csrc", "ecycle.cu"), os.path.join(HERE, "csrc", "ecycle_noalloc.cu")]
DEPS = SRC + [os.path.join(HERE, "csrc", "ecycle_kernels.cuh"), os.path.join(HERE, "csrc", "persistent_kernel.cuh"),
              os.path.join(HERE, "csrc", "shell_adjoint.cuh"), os.path.join(HERE, "csrc", "adjoint_kernels.cuh"),
              os.path.join(HERE, "..", "include", "or_ecycle.h")]
OUT = os.path.join(HERE, "libor_ecycle.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
         # single precision only (the split form's FP32 kernels): fast sqrt/div/exp/log,
         # FP32 denormals flushed; FP64 arithmetic is unaffected
         "--use_fast_math"]


# Parity variant: the same sources with floating-point contraction off (no FMA, in
# FP64 and FP32 alike) and IEEE division and square root, the arithmetic of the
# oracle (built with -ffp-contract=off).  Used only by the test that separates the
# effect of FMA contraction from that of the assembly order.
OUT_NOFMA = os.path.join(HERE, "libor_ecycle_nofma.so")
FLAGS_NOFMA = [f for f in FLAGS if f != "--use_fast_math"] + ["-fmad=false"]


def needs_build(out=OUT):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(f) > t for f in DEPS)


def build(verbose=False, force=False, variant=None):
    """Builds libor_ecycle.so (variant None) or the parity variant ("nofma")."""
    out, flags = (OUT_NOFMA, FLAGS_NOFMA) if variant == "nofma" else (OUT, FLAGS)
    if not force and not needs_build(out):
        return out
    cmd = [NVCC, *flags, *(["-Xptxas", "-v"] if verbose else []), "-o", out, *SRC]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose:
        sys.stderr.write(r.stdout + r.stderr)
    return out


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True,
                variant="nofma" if "--nofma" in sys.argv else None))
