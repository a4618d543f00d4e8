"""Builds libostc_b200.so in-tree with nvcc for sm_100a (no JIT cache, no pip install)."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
SOURCES = ["csrc/host.cpp", "csrc/chem.cpp", "csrc/ostc_b200.cu", "csrc/ostc_noalloc.cu"]
OUT = PKG / "libostc_b200.so"
OUT_CHECKED = PKG / "libostc_b200_checked.so"  # -DOSTC_BOUNDS_CHECK: index-checked accessors


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build(out: Path = OUT) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    headers = sorted((PKG / "csrc").glob("*.h")) + sorted((PKG / "csrc").glob("*.cuh"))
    deps = [PKG / s for s in SOURCES] + headers + [ROOT / "include" / "ostc.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> Path:
    out = OUT_CHECKED if checked else OUT
    if not force and not needs_build(out):
        return out
    cmd = [nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-I", str(ROOT / "include"), "-shared",
           *(["-DOSTC_BOUNDS_CHECK"] if checked else []), *[str(PKG / s) for s in SOURCES], "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc build of {out.name} failed")
    if verbose:
        sys.stdout.write(r.stdout + r.stderr)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
