"""Build libdeltamic_b200.so in-tree with nvcc for sm_100a.

    python -m deltamic_b200.build          # or __graft_entry__.build()

The library is a plain C-ABI shared object (no torch headers): every ``.cu`` file
under ``csrc/`` is compiled with ``-gencode arch=compute_100a,code=sm_100a`` and
linked with the static CUDA runtime into ``deltamic_b200/lib/``.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIBNAME = "libdeltamic_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
              "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found (set $NVCC)")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h"))
                  + glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h")))


def lib_path() -> str:
    return os.path.join(LIBDIR, LIBNAME)


def up_to_date() -> bool:
    out = lib_path()
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(p) <= t for p in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every csrc/*.cu into one shared library; returns its path."""
    if not force and up_to_date():
        return lib_path()
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(LIBDIR, "_obj")
    os.makedirs(objdir, exist_ok=True)
    cmds, objs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmds.append([nvcc(), *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj])
        objs.append(obj)
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd))
    # one nvcc per source file, several at once
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=not verbose), cmds)):
            if r.returncode != 0:
                if r.stderr:
                    sys.stderr.write(r.stderr.decode(errors="replace"))
                raise subprocess.CalledProcessError(r.returncode, r.args)
    tmp = lib_path() + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib_path())
    return lib_path()


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
