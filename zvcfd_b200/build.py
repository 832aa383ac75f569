"""Build ``libzvfv_b200.so`` in-tree with nvcc for sm_100a (B200).

``python -m zvcfd_b200.build`` (or :func:`build`) regenerates the element-table header,
compiles every ``csrc/*.cu`` to an object in ``csrc/_build/`` (in parallel, only when a
source or header is newer than its object) and links the shared library next to this
file, where :mod:`zvcfd_b200._lib` loads it.
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = CSRC / "_build"
LIB = HERE / "libzvfv_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-extended-lambda", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-O3"]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    p = Path(cuda) / "bin" / "nvcc"
    return str(p) if p.exists() else "nvcc"


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def build(verbose: bool = False, force: bool = False, jobs: int | None = None) -> Path:
    from zvcfd_b200.topology import write_header

    write_header()
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    nvcc = _nvcc()
    todo = []
    objs = []
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src, headers):
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        cmd = [nvcc, *ARCH, *FLAGS, "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stderr}")
        return src.name

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            for name in ex.map(compile_one, todo):
                if verbose:
                    print("compiled", name, flush=True)
    if force or todo or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime
                                                   for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
        if verbose:
            print("linked", LIB, flush=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
