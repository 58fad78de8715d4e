"""The hafnian workspace layout holds every access of the binary64 power loop.

On the 8-tile path the power loop stores and reads whole live column tiles (the
columns s .. 4 ntn - 1 hold zeros) and d is zero-padded to whole tiles, so the
loop stays inside the warp's shared workspace only if the strides and regions of
`haf_layout` are large enough for every subset size of a launch.  The layout
functions are __host__ __device__; tests/layout_host.cu compiles them for the host
and checks every (launch maximum, subset size) pair up to the cap, plain and
certified.  Needs nvcc (present wherever the library is built) but no GPU."""

from __future__ import annotations

import ctypes
import shutil
import subprocess
from pathlib import Path

import pytest

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def layoutlib():
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else None)
    if nvcc is None:
        pytest.skip("nvcc not available")
    out = HERE / "_build" / "liblayouthost.so"
    out.parent.mkdir(exist_ok=True)
    src = HERE / "layout_host.cu"
    csrc = HERE.parent / "gbskernels_b200" / "csrc"
    deps = [src, *csrc.glob("*.cuh")]
    if not out.exists() or out.stat().st_mtime < max(p.stat().st_mtime for p in deps):
        cmd = [nvcc, "-x", "cu", "-O1", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
               "-gencode", "arch=compute_100a,code=sm_100a", "-I", str(csrc), str(src), "-o", str(out)]
        subprocess.run(cmd, check=True, capture_output=True)
    lib = ctypes.CDLL(str(out))
    lib.t_haf_layout_check.argtypes = [ctypes.c_char_p, ctypes.c_int]
    lib.t_haf_layout_check.restype = ctypes.c_int
    return lib


def test_layout_holds_every_live_tile_access(layoutlib):
    msg = ctypes.create_string_buffer(256)
    bad = layoutlib.t_haf_layout_check(msg, 256)
    assert bad == 0, msg.value.decode()
