"""Build libfqxv_rans_gpu.so for sm_100a with nvcc, in-tree.

    python -m fqxv_b200.build            # build if sources changed
    python -m fqxv_b200.build --force    # rebuild
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libfqxv_rans_gpu.so")
SOURCES = ["rans_encode.cu", "rans_decode.cu", "rans_capi.cu", "rans_noalloc.cu", "rans_server.cu",
           "rans_x.cu", "rans_tuning.cu", "frame_kernels.cu", "frame_capi.cu", "tok_capi.cu", "streams_capi.cu",
           "perm_capi.cu"]
HEADERS = ["rans_internal.cuh", "rans_common.cuh", "rans_ctx.cuh", "frame_internal.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _inputs() -> list[str]:
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    inc = os.path.join(ROOT, "include")
    files += [os.path.join(inc, f) for f in sorted(os.listdir(inc)) if f.endswith(".h")]
    files.append(os.path.abspath(__file__))
    return files


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
                    "-I", os.path.join(ROOT, "include")]
    if verbose:
        flags += ["-Xptxas", "-v"]
    for src in SOURCES:
        obj = os.path.join(OUT_DIR, src.replace(".cu", ".o"))
        cmd = [nvcc(), "-c", os.path.join(CSRC, src), "-o", obj] + flags
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, r.stdout, r.stderr))
        if verbose:
            sys.stderr.write(r.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
