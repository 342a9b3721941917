"""Build libcoffee_b200.so in-tree with nvcc for sm_100a.

    python -m coffee_b200.build [--verbose-ptxas]

The library is compiled for B200 only (-gencode arch=compute_100a,code=sm_100a)
and placed next to this file, where coffee_b200._lib loads it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libcoffee_b200.so")

SOURCES = ["coffee_abi.cu", "coffee_params.cpp", "axisym.cu", "gr.cu", "yee.cu",
           "coffee_noalloc.cu", "surrogate.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newest_input() -> float:
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    paths += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(p) for p in paths if os.path.isfile(p))


def build(force: bool = False, ptxas_verbose: bool = False, log=None, defines=(),
          out: str | None = None) -> str:
    """Compile the library; `defines` (e.g. ["COFFEE_F32_STY=4"]) override
    tile-shape macros, `out` writes the library elsewhere than LIB.  Each
    source is compiled to an object by its own nvcc process, in parallel,
    and the objects are linked into the shared library."""
    target = out or LIB
    if not force and not defines and os.path.exists(target) and \
            os.path.getmtime(target) >= _newest_input():
        return target
    nvcc = nvcc_path()
    objdir = target + ".objs"
    os.makedirs(objdir, exist_ok=True)
    common = [nvcc, "-O3", "-std=c++17", *ARCH, "-lineinfo",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
              "-I", INCLUDE, "-I", CSRC, "-DCOFFEE_BUILDING_LIBRARY"] + [f"-D{d}" for d in defines]
    if ptxas_verbose:
        common += ["-Xptxas", "-v"]
    objs = [os.path.join(objdir, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    procs = [subprocess.Popen(common + ["-c", os.path.join(CSRC, s), "-o", o],
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
             for s, o in zip(SOURCES, objs)]
    failed, texts = [], []
    for s, p in zip(SOURCES, procs):
        text = p.communicate()[0]
        texts.append(text)
        if p.returncode != 0:
            failed.append(f"{s}: nvcc exited {p.returncode}\n{text[-6000:]}")
    if log is not None:
        log.write("".join(texts))
    if failed:
        raise RuntimeError("\n".join(failed))
    cmd = [nvcc, *ARCH, "--shared", "-o", target + ".tmp"] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{(r.stdout + r.stderr)[-6000:]}")
    os.replace(target + ".tmp", target)
    return target


if __name__ == "__main__":
    verbose = "--verbose-ptxas" in sys.argv
    build(force=True, ptxas_verbose=verbose, log=sys.stdout if verbose else None)
    print(LIB)
