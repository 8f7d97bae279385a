"""Build the in-tree shared libraries of gpu_compressstore2_b200 with nvcc for sm_100a.

libcompressstore.so  : the product (C ABI of include/compressstore.h)
libcs_cubflagged.so  : CUB DeviceSelect::Flagged comparator used by the bench and tests

Usage: python -m gpu_compressstore2_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-Xptxas",
    "-v" if os.environ.get("CS_PTXAS_VERBOSE") else "-O3",
]

LIBS = {
    "libcompressstore.so": ["cs_api.cu", "cs_kernels.cu", "cs_compact.cu", "cs_tuning.cu", "cs_plan.cu",
                            "cs_batch.cu", "cs_server.cu", "cs_host.cu", "cs_noalloc.cu", "cs_pattern.cu",
                            "cs_predicate.cu"],
    "libcs_cubflagged.so": ["cs_cub_flagged.cu"],
}


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _deps(srcs: list[str]) -> list[Path]:
    deps = [CSRC / s for s in srcs]
    return deps + _headers()


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _compile(src: str, obj: Path, verbose: bool) -> None:
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-I", str(INCLUDE), "-I", str(CSRC), "-c", str(CSRC / src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_lib(name: str, force: bool = False, verbose: bool = False) -> Path:
    """Compile the stale objects of one library in parallel, then link it."""
    srcs = LIBS[name]
    out = PKG / name
    if not force and not _stale(out, _deps(srcs)):
        return out
    build_dir = PKG / "_build"
    build_dir.mkdir(exist_ok=True)
    headers = _headers()
    objs, todo = [], []
    for s in srcs:
        obj = build_dir / (Path(s).stem + ".o")
        objs.append(str(obj))
        if force or _stale(obj, [CSRC / s, *headers]):
            todo.append((s, obj))
    workers = max(1, min(len(todo), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        for f in [ex.submit(_compile, s, obj, verbose) for s, obj in todo]:
            f.result()
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-cudart", "static", *objs, "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, out)
    return out


def build_all(force: bool = False, verbose: bool = False) -> list[Path]:
    return [build_lib(name, force=force, verbose=verbose) for name in LIBS]


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv, verbose=True):
        print("built", p)
