"""Build the CUDA library (libcubature_b200.so) in-tree for sm_100a.

Compiles old-gpuintegration_b200/csrc/capi.cu and one instantiation unit per
dimension (capi_dim.cu with -DCUB_DIM=N) in parallel with nvcc, then links a
shared library next to the Python package.  Objects are rebuilt only when a
source or header is newer.

    python old-gpuintegration_b200/build.py [--jobs J] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OBJ = PKG / "_build"
LIB = PKG / "cubature" / "libcubature_b200.so"
DIMS = range(2, 9)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
    "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}",
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps() -> list[Path]:
    return sorted(list(INCLUDE.rglob("*.h")) + list(INCLUDE.rglob("*.hpp")) +
                  list(INCLUDE.rglob("*.cuh")) + list(CSRC.glob("*.h")))


def _stale(obj: Path, src: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def units() -> list[tuple[Path, Path, list[str]]]:
    out = [(CSRC / "capi.cu", OBJ / "capi.o", []),
           (CSRC / "noalloc.cu", OBJ / "noalloc.o", []),
           (CSRC / "peak.cu", OBJ / "peak.o", []),
           (CSRC / "capi_tables.cu", OBJ / "capi_tables.o", []),
           (CSRC / "graph.cu", OBJ / "graph.o", []),
           (CSRC / "mlp.cu", OBJ / "mlp.o", [])]
    for n in DIMS:
        out.append((CSRC / "capi_dim.cu", OBJ / f"capi_dim{n}.o", [f"-DCUB_DIM={n}"]))
    return out


# Example programs of the C++ front end (include/cubature/gpucuhre.cuh),
# built as executables next to their sources; one dimension each.
EXAMPLES = [(PKG / "examples" / "ref_api_example.cu", PKG / "examples" / "ref_api_example",
             ["-DCUB_FRONT_MIN_DIM=3", "-DCUB_FRONT_MAX_DIM=3"])]


def build(jobs: int | None = None, verbose: bool = False, extra: list[str] | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    deps = _deps()
    cc = nvcc()
    todo = [(s, o, d) for s, o, d in units() if _stale(o, s, deps)]

    def compile_one(item):
        src, obj, defs = item
        cmd = [cc, *NVCC_FLAGS, *(extra or []), *defs, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {obj.name}:\n{r.stderr[-4000:]}")
        return obj

    def link_example(item):
        src, exe, defs = item
        cmd = [cc, *NVCC_FLAGS, *(extra or []), *defs, str(src), "-o", str(exe), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {exe.name}:\n{r.stderr[-4000:]}")
        return exe

    examples = [e for e in EXAMPLES if _stale(e[1], e[0], deps)]
    if todo or examples:
        jobs = jobs or max(1, min(len(todo) + len(examples), os.cpu_count() or 1))
        with ThreadPoolExecutor(jobs) as ex:
            futs = [ex.submit(compile_one, t) for t in todo]
            futs += [ex.submit(link_example, e) for e in examples]
            for f in futs:
                f.result()
    objs = [o for _, o, _ in units()]
    if todo or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        LIB.parent.mkdir(exist_ok=True)
        cmd = [cc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    print(build(args.jobs, args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
