"""Builds the CPU oracle ``oracle/liboracle.so`` (test infrastructure only).

The oracle restates the reference's hot-path arithmetic in plain C++ (see the header of each
``oracle/*.cpp``). It is compiled with ``-ffp-contract=off`` and without ``-ffast-math`` so
that every single-precision product and sum is rounded exactly as written, which is what
makes the GPU's explicitly rounded triangle test bit-comparable to it.

The reference itself cannot be built in this container: its geometry core (QBVH, triangle
test, kd-tree) lives in the Lass library pinned as lass/1.11.0-250+g078d9309
(conanfile.py:39), which is neither vendored nor installed, so there is no ``oracle/_ref``.
"""
from __future__ import annotations

import hashlib
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
STAMP = HERE / ".liboracle.stamp"
FLAGS = ["-O3", "-std=c++17", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread"]


def sources() -> list[Path]:
    return sorted(HERE.glob("*.cpp"))


def _digest() -> str:
    h = hashlib.sha256()
    # the sources, and the C ABI header whose struct layouts they check
    for p in sources() + sorted(HERE.glob("*.h")) + sorted((HERE.parent / "include").glob("*.h")):
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(" ".join(FLAGS).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> Path:
    digest = _digest()
    if not force and LIB.exists() and STAMP.exists() and STAMP.read_text().strip() == digest:
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = ["g++", *FLAGS, *map(str, sources()), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    STAMP.write_text(digest)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
