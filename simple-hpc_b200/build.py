"""Build the B200 solver library (libsgpu.so) and the `simple` driver in place.

nvcc compiles every CUDA source for sm_100a only. The FP64 path is bit-identical to the reference's
serial code, so those sources are compiled with --fmad=false (the reference's own CUDA build uses
the same flag, CMakeLists.txt:83-84) and host code with -ffp-contract=off. Object files go to
_obj/ next to this file; the library and the driver binary are written beside it, so they travel
with the repository snapshot to the GPU machine.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OBJ = HERE / "_obj"
LIB = HERE / "libsgpu.so"
EXE = HERE / "simple"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = "-fPIC,-ffp-contract=off,-O2,-Wall"
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", HOST_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}"]
# Sources whose arithmetic must match the reference bit for bit: no fused multiply-add contraction.
EXACT = ["--fmad=false"]
# Sources that compute in reduced precision (FP32 / BF16) where contraction is allowed.
FAST: list[str] = []

SOURCES = {
    "params.cpp": EXACT,
    "solver.cu": EXACT,
    "phases.cu": EXACT,
    "reduce.cu": EXACT,
    "mg.cu": EXACT,
    "cg.cu": EXACT,
    "fused.cu": EXACT,
    "mg_fast.cu": EXACT,
    "mixed.cu": EXACT,
    "io.cpp": EXACT,
    "noalloc.cu": EXACT,
    "cnn.cu": FAST,
    "conv_tc.cu": FAST,
    "mg32.cu": FAST,
    "mg_fast32.cu": FAST,
    "mixed32.cu": FAST,
}
DRIVER = ["driver.cpp"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def git_hash() -> str:
    try:
        r = subprocess.run(["git", "-C", str(HERE), "rev-parse", "--short", "HEAD"],
                           capture_output=True, text=True, timeout=10)
        return r.stdout.strip() or "unknown"
    except (OSError, subprocess.SubprocessError):
        return "unknown"


def _compile(src: Path, flags: list[str], verbose: bool) -> Path:
    obj = OBJ / (src.name + ".o")
    deps = [src] + sorted(CSRC.glob("*.hpp")) + sorted(CSRC.glob("*.cuh")) + [INCLUDE / "sgpu.h"]
    # sources that #include another .cu (the FP32 units) depend on it too
    deps += [CSRC / m for m in re.findall(r'#include "([\w.]+\.cu)"', src.read_text())]
    if obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps if d.exists()):
        return obj
    lang = ["-x", "cu"] if src.suffix == ".cu" else ["-x", "c++"]
    cmd = [nvcc(), *ARCH, *COMMON, *flags, *lang, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, file=sys.stderr)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    srcs = [(CSRC / name, flags) for name, flags in SOURCES.items() if (CSRC / name).exists()]
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda a: _compile(a[0], a[1], verbose), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *map(str, objs), "-o", str(LIB),
               "-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    drv = [CSRC / d for d in DRIVER if (CSRC / d).exists()]
    if drv:
        dflags = EXACT + [f'-DSIMPLE_GIT_HASH="{git_hash()}"', '-DSIMPLE_COMPILER="nvcc 12.9 (sm_100a)"']
        dobjs = [_compile(d, dflags, verbose) for d in drv]
        if not EXE.exists() or EXE.stat().st_mtime < max(o.stat().st_mtime for o in dobjs + [LIB]):
            cmd = [nvcc(), *ARCH, *map(str, dobjs), "-o", str(EXE), f"-L{HERE}", "-lsgpu",
                   "-Xlinker", "-rpath,$ORIGIN"]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"driver link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
