"""Build recipe for libarcb200.so (the C-ABI library of the B200 PIC hot path).

Compiles the CUDA sources under arcwarden_b200/csrc for sm_100a only and links
cuFFT. The library is built in-tree (arcwarden_b200/libarcb200.so) so it travels
with the source tree; nothing is installed into site-packages.

    python -m arcwarden_b200.build            # build if stale
    python -m arcwarden_b200.build --force    # rebuild
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libarcb200.so"
SOURCES = ["aw_abi.cu", "aw_particles.cu", "aw_deposit.cu", "aw_spectral.cu", "aw_noalloc.cu", "aw_resort.cu", "aw_adjoint.cu", "aw_adjoint_darwin.cu", "aw_ensemble.cu", "aw_checkpoint.cu"]
HEADERS = ["aw_device.cuh", "aw_internal.h"]

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    deps = [CSRC / s for s in SOURCES] + [CSRC / h for h in HEADERS] + [ROOT / "include" / "arcb200.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    procs = []
    for s in SOURCES:
        o = objdir / (Path(s).stem + ".o")
        objs.append(o)
        cmd = [NVCC, *ARCH, *FLAGS, "-I", str(ROOT / "include"), "-c", str(CSRC / s), "-o", str(o)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = []
    for s, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode != 0:
            sys.stdout.write(out)
        if p.returncode != 0:
            failed.append(s)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(tmp),
           "-lcufft", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv or "--verbose" in sys.argv)
    print(LIB)
