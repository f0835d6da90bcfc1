"""Builds libms_gpu.so (all CUDA sources, sm_100a) in-tree with nvcc."""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libms_gpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
         "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(HERE, "..", "include", "ms_gpu.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(src), _headers_mtime()):
        return obj
    cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stderr}")
    if verbose or "spill" in r.stderr.lower() and "0 bytes spill" not in r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = _sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB, *objs]
        subprocess.run(cmd, check=True)
    _build_examples()
    return LIB


def _build_examples() -> None:
    """The C++ drop-in examples, linked against libms_gpu.so."""
    ex = os.path.join(HERE, "examples")
    out = os.path.join(ex, "bin")
    os.makedirs(out, exist_ok=True)
    for src in sorted(f for f in os.listdir(ex) if f.endswith(".cpp")):
        binp = os.path.join(out, src[:-4])
        srcp = os.path.join(ex, src)
        hdr = os.path.join(HERE, "include", "morphstore_b200", "morphstore.h")
        if os.path.exists(binp) and os.path.getmtime(binp) > max(os.path.getmtime(srcp), os.path.getmtime(hdr),
                                                                   os.path.getmtime(LIB)):
            continue
        cmd = ["g++", "-std=c++14", "-O2", "-Wall", "-I", os.path.join(HERE, "..", "include"),
               "-I", os.path.join(HERE, "include"), srcp, "-o", binp, "-L", HERE, "-lms_gpu",
               "-Wl,-rpath,$ORIGIN/../.."]
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
