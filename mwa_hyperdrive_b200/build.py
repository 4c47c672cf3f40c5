"""Build libhdc.so (all CUDA sources under csrc/) for sm_100a with nvcc.

The library is built in-tree (mwa_hyperdrive_b200/libhdc.so) so that it
travels with the source tree; it is not installed anywhere else.
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libhdc.so"
OBJ = PKG / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-Wall", "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (Path(c).exists() or c == "nvcc"):
            return c
    return "nvcc"


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "hdc.h"]
    return any(d.stat().st_mtime > obj.stat().st_mtime for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> Path:
    OBJ.mkdir(exist_ok=True)
    srcs = sources()
    objs = [OBJ / (s.stem + ".o") for s in srcs]

    def compile_one(pair):
        src, obj = pair
        if not force and not _stale(obj, src):
            return None
        cmd = [nvcc(), *ARCH, *NVCC_FLAGS, *extra_flags, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        return (src.name, r.stderr)

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, zip(srcs, objs)))
    if verbose:
        for res in results:
            if res and res[1].strip():
                print(f"--- {res[0]}\n{res[1]}", file=sys.stderr)
    relink = force or not OUT.exists() or any(o.stat().st_mtime > OUT.stat().st_mtime for o in objs)
    if relink:
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(OUT)
