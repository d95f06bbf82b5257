"""Build recipe for libsod2d_b200.so (sm_100a) — compiled in-tree with nvcc.

    python -m sod2d_refmap_b200.build         # or sod2d_refmap_b200.build.build()
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsod2d_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(HERE, "..", "include", "sod2d_b200.h")]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, extra: list | None = None) -> str:
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(CSRC, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
               "-rdc=false", "-c", src, "-o", obj] + (extra or [])
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True), src))
        objs.append(obj)
    failed = False
    for p, src in procs:
        out, _ = p.communicate()
        if out.strip():
            sys.stderr.write(out)
        if p.returncode != 0:
            failed = True
            sys.stderr.write(f"nvcc failed on {src}\n")
    if failed:
        raise RuntimeError("libsod2d_b200 build failed")
    cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    _check_resolved(LIB)
    return LIB


def _check_resolved(lib: str) -> None:
    """A shared library links with undefined symbols and fails only when loaded; refuse a build
    that leaves one of the library's own (namespace sod) functions undefined, e.g. a declaration
    in one source file that no longer matches its definition in another."""
    try:
        out = subprocess.run(["nm", "-C", "-u", lib], capture_output=True, text=True, check=True).stdout
    except (OSError, subprocess.CalledProcessError):
        return  # no nm on this machine: nothing to check with
    missing = [ln.strip() for ln in out.splitlines() if "sod::" in ln]
    if missing:
        os.remove(lib)
        raise RuntimeError("libsod2d_b200 has undefined internal symbols:\n  " + "\n  ".join(missing))


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
