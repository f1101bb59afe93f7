"""Build recipe of libash3d_b200.so (sm_100a only).

    nvcc -gencode arch=compute_100a,code=sm_100a -O3 --fmad=false -lineinfo \
         -Xcompiler -fPIC -shared csrc/*.cu -o libash3d_b200.so

--fmad=false keeps every product and sum separately rounded, as the
reference's CPU arithmetic is; divisions stay IEEE (the default -prec-div).
"""
from __future__ import annotations

import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
SRCS = ["a3g_api.cu", "k_advect.cu", "k_diffuse.cu", "k_reduce.cu", "a3g_noalloc.cu"]
OUT = HERE / "libash3d_b200.so"
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-std=c++17",
              "-lineinfo", "-Xcompiler", "-fPIC", "-shared"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [HERE / "csrc" / s for s in SRCS] + [HERE / "csrc" / "a3g_internal.cuh",
                                               HERE / "csrc" / "exact_div.cuh",
                                               HERE.parent / "include" / "ash3d_b200.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    if not force and not needs_build():
        return OUT
    cmd = [nvcc(), *NVCC_FLAGS, "-o", str(OUT), *[str(HERE / "csrc" / s) for s in SRCS]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
