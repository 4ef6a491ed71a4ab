"""Build libptycho_b200.so in-tree for sm_100a (B200).

    python conventional-ptychography-reconstruction_b200/csrc/build.py [-v] [--force]

Every ``*.cu`` file in this folder is compiled by ``nvcc`` with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into an object file
under ``_build/`` and linked into ``../libptycho_b200.so``.  Objects are rebuilt
when their source or any header in this folder (or ``include/``) is newer.
``fastabi.c`` (a CPython fast-call binding of the per-step entry points) is
compiled by the host C compiler into ``../_fastabi<EXT_SUFFIX>``.
No GPU is needed: nvcc cross-compiles.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
OUT = os.path.join(PKG, "libptycho_b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include"), "-I" + HERE]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def _deps_mtime() -> float:
    hdrs = glob.glob(os.path.join(HERE, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    return max([os.path.getmtime(h) for h in hdrs] + [0.0])


def _compile(src: str, verbose: bool, force: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps_mtime())):
        return obj
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build_fastabi(force: bool = False) -> str:
    """The CPython binding module (host C code, no CUDA)."""
    src = os.path.join(HERE, "fastabi.c")
    out = os.path.join(PKG, "_fastabi" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cc = os.environ.get("CC") or shutil.which("gcc") or "cc"
    cmd = [cc, "-O2", "-shared", "-fPIC", "-I" + sysconfig.get_paths()["include"], src, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building {src} failed:\n{r.stdout}\n{r.stderr}")
    return out


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(HERE, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs) or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, force), srcs))
    if (force or not os.path.exists(OUT)
            or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs)):
        cmd = [nvcc(), *ARCH, "-shared", "-o", OUT, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_fastabi(force)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register usage")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))
