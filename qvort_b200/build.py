"""Build libqvort_b200.so (the C-ABI library of include/qv.h) in-tree for sm_100a.

Every CUDA source under qvort_b200/csrc is compiled by nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared
library next to this file, so the built artefact travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "libqvort_b200.so"
BUILD = HERE / "_build"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr",
    "-I", str(HERE.parent / "include"),
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


# Per-file extra flags.  The per-point kernels (ghosts, LIA finite differences,
# Adams-Bashforth, energy) follow the reference's FP64 operation order with one
# rounding per operation, so FMA contraction is switched off there.
FILE_FLAGS = {"qv_points.cu": ["--fmad=false"], "qv_line.cu": ["--fmad=false"]}


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


RUNNER_SRC = HERE / "host" / "qvort_run.cpp"
RUNNER = HERE / "qvort_run"


def build_runner() -> Path:
    """The C++ driver executable, linked against the library (rpath = its folder)."""
    if RUNNER.exists() and RUNNER.stat().st_mtime >= max(RUNNER_SRC.stat().st_mtime,
                                                        OUT.stat().st_mtime):
        return RUNNER
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-I", str(HERE.parent / "include"), str(RUNNER_SRC),
           "-L", str(HERE), "-lqvort_b200", "-Wl,-rpath,$ORIGIN", "-o", str(RUNNER)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"qvort_run build failed:\n{r.stdout}\n{r.stderr}")
    return RUNNER


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name.replace(".", "_") + ".o")
    deps = [src] + sorted(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "qv.h"]
    if obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return obj
    cmd = [_nvcc(), *NVCC_FLAGS, *FILE_FLAGS.get(src.name, []), "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    stamp = BUILD / "flags.txt"
    flags = repr((NVCC_FLAGS, FILE_FLAGS))
    if not stamp.exists() or stamp.read_text() != flags:
        force = True
    if force:
        for o in BUILD.glob("*.o"):
            o.unlink()
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not OUT.exists() or OUT.stat().st_mtime < newest:
        tmp = OUT.with_suffix(".so.tmp")
        cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
               "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, OUT)
    stamp.write_text(flags)
    build_runner()
    return OUT


if __name__ == "__main__":
    p = build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(p)
