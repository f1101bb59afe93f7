"""Build recipe of libash3d_b200.so (sm_100a only).

    nvcc -gencode arch=compute_100a,code=sm_100a -O3 --fmad=false -lineinfo \
         -Xcompiler -fPIC -c csrc/<each>.cu -o _build/<each>.o     (in parallel)
    nvcc -gencode arch=compute_100a,code=sm_100a -shared _build/*.o -o libash3d_b200.so

--fmad=false keeps every product and sum separately rounded, as the
reference's CPU arithmetic is; divisions stay IEEE (the default -prec-div).
"""
from __future__ import annotations

import concurrent.futures
import pathlib
import shutil
import subprocess
import sys

HERE = pathlib.Path(__file__).resolve().parent
SRCS = ["k_advect_x.cu", "k_advect_y.cu", "k_advect_z.cu", "k_advect.cu", "k_diffuse.cu", "k_reduce.cu",
        "a3g_api.cu", "a3g_inverse.cu", "a3g_noalloc.cu"]
OUT = HERE / "libash3d_b200.so"
OBJ_DIR = HERE / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [*ARCH, "-O3", "--fmad=false", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return p


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = [HERE / "csrc" / s for s in SRCS] + [HERE / "csrc" / "a3g_internal.cuh", HERE / "csrc" / "k_advect.cuh",
                                               HERE / "csrc" / "exact_div.cuh", HERE / "csrc" / "tma.cuh",
                                               HERE.parent / "include" / "ash3d_b200.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    if not force and not needs_build():
        return OUT
    OBJ_DIR.mkdir(exist_ok=True)
    objs = [OBJ_DIR / (pathlib.Path(s).stem + ".o") for s in SRCS]
    cmds = [[nvcc(), *NVCC_FLAGS, "-c", str(HERE / "csrc" / s), "-o", str(o)] for s, o in zip(SRCS, objs)]
    if verbose:
        for c in cmds:
            print(" ".join(c), file=sys.stderr)
    with concurrent.futures.ThreadPoolExecutor(len(cmds)) as ex:
        for f in [ex.submit(subprocess.check_call, c) for c in cmds]:
            f.result()
    link = [nvcc(), *ARCH, "-shared", "-o", str(OUT), *[str(o) for o in objs]]
    if verbose:
        print(" ".join(link), file=sys.stderr)
    subprocess.check_call(link)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
