"""Build the unichem shared library in-tree for sm_100a.

    python -m unicorn_b200.build [--verbose]

Regenerates the mechanism tables and the species-update program from
``unicorn_b200/mech/sandiego52.json`` when they are older than it, then
compiles ``unicorn_b200/csrc/unichem.cu`` with nvcc into
``unicorn_b200/libunichem.so``.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libunichem.so"
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(p).exists():
        raise RuntimeError("nvcc not found: the unichem CUDA library cannot be built")
    return p


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted((CSRC / "generated").glob("*")) + \
        [ROOT / "include" / "unichem.h"]


def regenerate():
    from unicorn_b200.mech import codegen
    gen = [CSRC / "generated" / "mech_tables.h", CSRC / "generated" / "update_program.cuh",
           CSRC / "generated" / "update_program_tr.cuh"]
    src = [codegen.MECH, Path(codegen.__file__)]
    if any(not g.exists() for g in gen) or max(s.stat().st_mtime for s in src) > min(g.stat().st_mtime for g in gen):
        codegen.main()


def build(verbose: bool = False, force: bool = False) -> Path:
    regenerate()
    newest = max(s.stat().st_mtime for s in sources())
    if LIB.exists() and LIB.stat().st_mtime >= newest and not force:
        return LIB
    cmd = [nvcc(), *NVCC_FLAGS, "-I", str(ROOT / "include"), "-o", str(LIB), str(CSRC / "unichem.cu")]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed to build libunichem.so")
    if verbose:
        sys.stderr.write(res.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))
