"""Builds libostc_b200.so in-tree with nvcc for sm_100a (no JIT cache, no pip install)."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = ["csrc/host.cpp", "csrc/chem.cpp", "csrc/ostc_air.cu", "csrc/ostc_noalloc.cu"]
OUT = PKG / "libostc_b200.so"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    headers = sorted((PKG / "csrc").glob("*.h")) + sorted((PKG / "csrc").glob("*.cuh"))
    deps = [PKG / s for s in SOURCES] + headers + [ROOT / "include" / "ostc.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return OUT
    cmd = [nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-I", str(ROOT / "include"), "-shared",
           *[str(PKG / s) for s in SOURCES], "-o", str(OUT)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc build of libostc_b200.so failed")
    if verbose:
        sys.stdout.write(r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
