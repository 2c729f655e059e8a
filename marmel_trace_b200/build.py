"""Build libmtgpu.so (the sm_100a renderer core) in-tree with nvcc.

Usage: python -m marmel_trace_b200.build [--force]

Every translation unit is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a). The FP64 kernel unit is compiled
with --fmad=false so double arithmetic rounds exactly as the reference's C
build does; the FP32 units keep FMA contraction. The build is skipped when
the recorded digest of every source and header is unchanged.
"""
from __future__ import annotations

import concurrent.futures
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libmtgpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-I", str(INCLUDE), "-I", str(CSRC)]

# (source, extra flags)
UNITS = [
    ("mt_api.cu", []),
    ("mt_kernels_f32.cu", []),
    ("mt_kernels_f64.cu", ["--fmad=false"]),
    ("mt_wavefront.cu", []),
    ("mt_wavefront_f64.cu", ["--fmad=false"]),
    ("mt_noalloc.cu", []),
    ("mt_batch.cu", []),
    ("mt_adjoint.cu", []),
    ("mt_adjoint_f64.cu", ["--fmad=false"]),
    ("mt_bvh.cpp", []),
    ("mt_bvh_gpu.cu", ["--fmad=false"]),
    ("mt_probe.cu", []),
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libmtgpu.so")


def _digest() -> str:
    h = hashlib.sha256()
    files = sorted(CSRC.glob("*")) + sorted(INCLUDE.glob("*.h")) + [Path(__file__)]
    for f in files:
        if f.is_file():
            h.update(f.name.encode())
            h.update(f.read_bytes())
    return h.hexdigest()


def _compile(nvcc: str, src: str, extra: list[str]) -> Path:
    obj = BUILD / (src + ".o")
    cmd = [nvcc, *ARCH, *COMMON, *extra, "-c", str(CSRC / src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, verbose: bool = True) -> Path:
    """Compile and link libmtgpu.so; returns its path."""
    stamp = BUILD / "digest.txt"
    digest = _digest()
    if not force and LIB.exists() and stamp.exists() and stamp.read_text().strip() == digest:
        return LIB
    nvcc = _nvcc()
    BUILD.mkdir(parents=True, exist_ok=True)
    if verbose:
        print(f"[mtgpu] compiling {len(UNITS)} units for sm_100a ...", file=sys.stderr)
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(lambda u: _compile(nvcc, u[0], u[1]), UNITS))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    stamp.write_text(digest)
    if verbose:
        print(f"[mtgpu] built {LIB}", file=sys.stderr)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
