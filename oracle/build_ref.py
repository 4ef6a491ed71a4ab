"""Build oracle/_ref/libgscp_ref.so: the reference's own Gaussian rasteriser
(gscp/csrc/gscp_rasterizer/{forward,backward,rasterizer_impl}.cu, compiled
from the sources where they lie in the reference tree (``PTYCHO_REFERENCE``,
default /root/reference), with the reference's
nvcc flags -O3 --use_fast_math, gscp/csrc/setup.py:25-27) plus the C entry
points of oracle/gscp_ref_shim.cu.  TEST ONLY: the parity tests load it as a
checker.  Skipped (returns None) when the reference tree or nvcc is absent,
e.g. on a machine that only received the built library.

    python oracle/build_ref.py
"""
from __future__ import annotations

import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("PTYCHO_REFERENCE", "/root/reference")
REF = os.path.join(REF_ROOT, "gscp", "csrc", "gscp_rasterizer")
OUT = os.path.join(HERE, "_ref", "libgscp_ref.so")
SOURCES = ["forward.cu", "backward.cu", "rasterizer_impl.cu"]


def build(force: bool = False):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.isdir(REF) or not os.path.exists(nvcc):
        return None
    srcs = [os.path.join(REF, s) for s in SOURCES] + [os.path.join(HERE, "gscp_ref_shim.cu")]
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(s) for s in srcs):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--use_fast_math", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-I" + REF, *srcs, "-o", OUT, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building the reference rasteriser failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(force=True))
