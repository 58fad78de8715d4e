"""Build libgbs_b200.so in-tree: every CUDA source compiled for sm_100a with nvcc.

    python -m gbskernels_b200.build            (or gbskernels_b200.build.build())

Translation units compile in parallel; objects go to gbskernels_b200/_build/ and
the shared library to gbskernels_b200/libgbs_b200.so.  A unit is rebuilt only when
it or a header is newer than its object.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libgbs_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: every fused multiply-add is an explicit fma() in the source, so the
# rounding of a value does not depend on the kernel it is inlined into.
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
           "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (CUDA toolkit required to build libgbs_b200.so)")


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, src: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    nvcc = _nvcc()
    BUILD.mkdir(exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h"))
    srcs = _sources()
    objs = [BUILD / (s.stem + ".o") for s in srcs]

    def compile_one(pair):
        src, obj = pair
        if not _stale(obj, src, headers):
            return None
        cmd = [nvcc, *ARCH, *NVFLAGS, "-I", str(CSRC), "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stderr[-4000:]}")
        return (src.name, r.stderr)

    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 4))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        for res in ex.map(compile_one, zip(srcs, objs)):
            if res and verbose:
                print(f"[build] {res[0]}", res[1][-2000:], file=sys.stderr)
    build_host_helper()
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    return LIB


def build_host_helper() -> Path | None:
    """The CPython helper of the binding (_hostptr.c: matrix addresses of a batch in
    one C loop), compiled with the host C compiler.  Optional: without it the
    binding walks the batch in Python."""
    import sysconfig
    src = HERE / "_hostptr.c"
    out = HERE / ("_hostptr" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))
    inc = sysconfig.get_paths().get("include")
    cc = shutil.which("gcc") or shutil.which("cc")
    if not cc or not inc or not (Path(inc) / "Python.h").exists():
        return None
    if out.exists() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    r = subprocess.run([cc, "-O2", "-shared", "-fPIC", "-I", inc, str(src), "-o", str(out)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"building {src.name} failed:\n{r.stderr[-4000:]}")
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
