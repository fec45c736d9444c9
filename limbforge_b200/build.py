"""Builds limbforge_b200/liblimbforge_b200.so in place: every CUDA/C++ source under csrc/
compiled for sm_100a (nvcc -gencode arch=compute_100a,code=sm_100a), translation units in
parallel, objects cached under limbforge_b200/_build (rebuilt when a source or any header is
newer than the object)."""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblimbforge_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -compress-mode=size: the fatbinaries of the 31 widths' kernels shrink about 8x against the default mode, which keeps
# the library small enough to ship in-tree.
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp", "-compress-mode=size",
         f"-I{os.path.join(ROOT, 'include')}", f"-I{CSRC}", "--expt-relaxed-constexpr"]


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(src: str, obj: str, newest_header: float) -> bool:
    """An object is stale when it, or the dependency list nvcc wrote beside it, is missing, or
    when the source or any header it included is newer."""
    dep = obj + ".d"
    if not os.path.exists(obj) or not os.path.exists(dep):
        return True
    t = os.path.getmtime(obj)
    text = open(dep).read().replace("\\\n", " ")
    files = text.split(":", 1)[1].split() if ":" in text else []
    for f in [src] + files:
        if not os.path.exists(f) or os.path.getmtime(f) > t:
            return True
    return False


def _compile(src: str, obj: str, verbose: bool) -> str:
    cmd = [NVCC, *ARCH, *FLAGS, "-MD", "-MF", obj + ".d", "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stderr[-6000:]}")
    return r.stderr


def build(jobs: int | None = None, verbose: bool = False, force: bool = False) -> str:
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    newest = max((os.path.getmtime(h) for h in _headers()), default=0.0)
    # without the object directory (a copy of the tree that carries only the built library), a library newer
    # than every source and header is current; with it, every object is checked against its dependencies
    if not force and not os.path.isdir(OBJ) and os.path.exists(LIB) and \
            os.path.getmtime(LIB) >= max([newest] + [os.path.getmtime(x) for x in sources]):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    objs, todo = [], []
    for s in sources:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(s, o, newest):
            todo.append((s, o))
    if todo:
        # the widest element-wise groups dominate; start them first
        todo.sort(key=lambda so: -os.path.getsize(so[0]) - (10**6 if "_ew_" in so[0] else 0))
        with cf.ThreadPoolExecutor(max_workers=jobs or max(2, os.cpu_count() or 2)) as ex:
            futs = {ex.submit(_compile, s, o, verbose): s for s, o in todo}
            for f in cf.as_completed(futs):
                log = f.result()
                if verbose and log:
                    sys.stderr.write(log)
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fopenmp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))
