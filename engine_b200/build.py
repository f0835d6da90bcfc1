"""Builds libms_gpu.so (all CUDA sources, sm_100a) in-tree with nvcc."""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
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


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(path: str, seen=None) -> set:
    """The file and every local header it includes, transitively."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for inc in _INCLUDE.findall(f.read()):
            _deps(os.path.join(os.path.dirname(path), inc), seen)
    return seen


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) > max(os.path.getmtime(d) for d in _deps(src)):
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
    _build_reference_sources()
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


# The reference's own example query and operator known-answer tests, compiled
# against the reference's headers with the processing style changed to
# gpu_b200 and ve_gpu_b200.h put in front (-include).  The only edit to each
# source is the style token: `using ve = scalar<v64<uint64_t> >;` in the
# example, every `scalar<v64<uint64_t>>` in the tests.  The edited text is
# piped to g++ and never written out; only the binaries are kept (bin/ref_*).
# Built where the reference tree is present (MS_REFERENCE_DIR); the binaries
# travel with the library.
REFERENCE_SOURCES = [
    ("select_sum_query", "src/examples/select_sum_query.cpp", "using ve = scalar<v64<uint64_t> >;",
     "using ve = gpu_b200<v512<uint64_t> >;"),
] + [(f"kat_{n}", f"test/core/operators/{n}.cpp", "scalar<v64<uint64_t>>", "gpu_b200<v512<uint64_t>>")
     for n in ("select_test", "project_test", "agg_sum_whole_column_test", "agg_sum_group_based_test",
               "group_unary_test", "group_binary_test", "intersect_test")]


def _build_reference_sources() -> None:
    ref = os.environ.get("MS_REFERENCE_DIR")
    if not ref or not os.path.isdir(os.path.join(ref, "include", "core")):
        return
    root = os.path.dirname(HERE)
    gen = os.path.join(root, "oracle", "_ref", "gen")
    if not os.path.exists(os.path.join(gen, "core", "morphing", "vbp_routines.h")):
        subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle"), f"MS_REFERENCE_DIR={ref}",
                        os.path.join(gen, "core", "morphing", "vbp_routines.h")], check=True)
    out = os.path.join(HERE, "examples", "bin")
    os.makedirs(out, exist_ok=True)
    hdr = os.path.join(HERE, "include", "morphstore_b200", "ve_gpu_b200.h")
    flags = ["-std=c++14", "-O2", "-DMSV_NO_SELFMANAGED_MEMORY", "-DMSV_NO_LOG", "-DMSV_MEMORY_MANAGER_ALIGNMENT_BYTE=64",
             "-Wno-ignored-attributes", "-I", gen, "-I", os.path.join(ref, "include"),
             "-I", os.path.join(root, "include"), "-I", os.path.join(HERE, "include")]

    def one(item):
        name, rel, old, new = item
        src = os.path.join(ref, rel)
        binp = os.path.join(out, "ref_" + name)
        deps = [src, hdr, LIB, os.path.join(root, "include", "ms_gpu.h")]
        if os.path.exists(binp) and os.path.getmtime(binp) > max(os.path.getmtime(d) for d in deps):
            return
        text = open(src).read()
        if text.count(old) < 1 or (name == "select_sum_query" and text.count(old) != 1):
            raise RuntimeError(f"{rel}: processing-style token not found as expected")
        cmd = ["g++", *flags, "-I", os.path.dirname(src), "-include", hdr, "-x", "c++", "-", "-o", binp,
               "-L", HERE, "-lms_gpu", "-Wl,-rpath,$ORIGIN/../.."]
        r = subprocess.run(cmd, input=text.replace(old, new), capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"g++ failed for {rel}:\n{r.stderr[-4000:]}")

    with cf.ThreadPoolExecutor(max_workers=8) as ex:
        list(ex.map(one, REFERENCE_SOURCES))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
