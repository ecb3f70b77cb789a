"""Builds the sm_100a shared library ``liar_b200/libliar_gpu.so`` from ``liar_b200/csrc``.

The library is a plain C-ABI shared object (include/liar_gpu.h): nvcc compiles the CUDA
kernels for sm_100a only and the host C++ (tree builder, entry points) with the same
invocation. The CUDA runtime is linked statically, so the library needs nothing from the
Python environment. Run ``python -m liar_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
LIB = HERE / "libliar_gpu.so"
STAMP = HERE / ".libliar_gpu.stamp"
# the benchmark's L2 bandwidth probe, a separate library outside the C ABI
PROBE_SRC = HERE / "probe" / "l2_read.cu"
PROBE_LIB = HERE / "libliar_probe.so"

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off",
    "-Xptxas", "-O3",
    "--expt-relaxed-constexpr",
    "-ftz=false", "-prec-div=true", "-prec-sqrt=true", "-fmad=true",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def sources() -> list[Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _digest() -> str:
    h = hashlib.sha256()
    for p in sorted(list(CSRC.glob("*")) + list(INCLUDE.glob("*.h"))):
        if p.is_file():
            h.update(p.name.encode())
            h.update(p.read_bytes())
    h.update(" ".join(NVCC_FLAGS).encode())
    return h.hexdigest()


def build_probe(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the L2 bandwidth probe library unless it is newer than its source."""
    if not force and PROBE_LIB.exists() and PROBE_LIB.stat().st_mtime >= PROBE_SRC.stat().st_mtime:
        return PROBE_LIB
    tmp = PROBE_LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), *NVCC_FLAGS, "-shared", str(PROBE_SRC), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, PROBE_LIB)
    return PROBE_LIB


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compiles the library unless it is up to date; returns its path."""
    build_probe(force=force, verbose=verbose)
    digest = _digest()
    if not force and LIB.exists() and STAMP.exists() and STAMP.read_text().strip() == digest and not extra_flags:
        return LIB
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.name + ".o")
        cmd = [_nvcc(), *NVCC_FLAGS, *(extra_flags or []), "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stdout.write(out.decode(errors="replace"))
        if p.returncode:
            failed.append(src.name)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(tmp), *map(str, objs), "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    STAMP.write_text(digest)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
