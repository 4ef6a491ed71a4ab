"""Build libptycho_b200.so in-tree for sm_100a (B200).

    python conventional-ptychography-reconstruction_b200/csrc/build.py [-v] [--force]

Every ``*.cu`` file in this folder is compiled by ``nvcc`` with
``-gencode arch=compute_100a,code=sm_100a -lineinfo -O3`` into an object file
under ``_build/`` and linked into ``../libptycho_b200.so``.  Objects are rebuilt
when their source or any header in this folder (or ``include/``) is newer.
``fastabi.c`` (a CPython fast-call binding of the per-step entry points) is
compiled by the host C compiler into ``../_fastabi<EXT_SUFFIX>``, and
``torch_ext.cpp`` (the fused loss's autograd node, host C++ against libtorch)
by the host C++ compiler into ``../_torchext<EXT_SUFFIX>``.
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


def build_torchext(force: bool = False) -> str:
    """The torch autograd node of the fused loss (host C++ against libtorch,
    no CUDA code: it calls libptycho_b200.so through bound addresses)."""
    import torch

    src = os.path.join(HERE, "torch_ext.cpp")
    out = os.path.join(PKG, "_torchext" + sysconfig.get_config_var("EXT_SUFFIX"))
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    cuda_home = os.environ.get("CUDA_HOME") or "/usr/local/cuda"
    incs = [os.path.join(os.path.dirname(torch.__file__), "include"),
            os.path.join(os.path.dirname(torch.__file__), "include", "torch", "csrc", "api", "include"),
            os.path.join(cuda_home, "include"), sysconfig.get_paths()["include"]]
    libdir = os.path.join(os.path.dirname(torch.__file__), "lib")
    abi = int(bool(torch._C._GLIBCXX_USE_CXX11_ABI))
    # the system g++ (libtorch's own compiler family): a toolchain whose link
    # path holds only a static libstdc++ would put a second copy of the C++
    # runtime (locale, iostream state) into the module, next to the process's
    # shared one -- formatting an error message then crashes.  PTYCHO_CXX
    # overrides; the result is checked below either way.
    cxx = os.environ.get("PTYCHO_CXX") or shutil.which("g++", path="/usr/bin:/bin") or shutil.which("g++") or "c++"
    cmd = [cxx, "-O2", "-std=c++17", "-shared", "-fPIC", "-w", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
           "-DTORCH_EXTENSION_NAME=_torchext", "-DTORCH_API_INCLUDE_EXTENSION_H",
           *["-I" + i for i in incs], src, "-o", out, "-L" + libdir, "-Wl,-rpath," + libdir,
           "-lc10", "-lc10_cuda", "-ltorch", "-ltorch_cpu", "-ltorch_cuda", "-ltorch_python"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building {src} failed:\n{r.stdout}\n{r.stderr}")
    own = runtime_copies(out)
    if own:
        os.remove(out)
        raise RuntimeError(f"{cxx} linked C++ runtime code into {out} ({own[0]} ...); "
                           "set PTYCHO_CXX to a g++ that links libstdc++ as a shared library")
    return out


def runtime_copies(so: str) -> list:
    """Text symbols of the C++ runtime (std::basic_ostream, std::locale, codecvt ...)
    that `so` defines itself instead of taking from the shared libstdc++."""
    nm = shutil.which("nm")
    if nm is None:
        return []
    r = subprocess.run([nm, "-C", "--defined-only", so], capture_output=True, text=True)
    bad = ("std::basic_ostream", "std::ostream::", "std::locale::", "std::__codecvt", "std::codecvt",
           "std::ios_base::")
    return [ln.split(" ", 2)[-1] for ln in r.stdout.splitlines()
            if " T " in ln and any(b in ln for b in bad)]


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
    build_torchext(force)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-v", "--verbose", action="store_true", help="print ptxas register usage")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))
