"""The reference's own code on the GPU through the gpu_b200 processing style
(engine_b200/include/morphstore_b200/ve_gpu_b200.h).

* The reference's operator known-answer tests (test/core/operators/*_test.cpp)
  and its example query (src/examples/select_sum_query.cpp), compiled from the
  reference's sources with only the processing-style token changed
  (engine_b200/build.py REFERENCE_SOURCES), run on the GPU and must pass /
  print the right sum.  The example draws its data from a clock-seeded
  generator, so it runs with MSV_GPU_B200_DUMP_DIR set: the binding writes
  every operator's input and output columns, and the expected positions,
  values and sum are recomputed from the dumped inputs by the oracle.
* oracle/ref_style_diff runs the reference's operator templates with the
  reference's AVX-512 style and with gpu_b200 on the same columns and
  compares every output.

The binaries are built where the reference tree is present and travel with
the library; without them these tests skip.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "engine_b200", "examples", "bin")
KATS = ["select_test", "project_test", "agg_sum_whole_column_test", "agg_sum_group_based_test", "group_unary_test",
        "group_binary_test", "intersect_test"]


def _bin(name):
    p = os.path.join(BIN, "ref_" + name)
    if not os.path.exists(p):
        pytest.skip("reference-source binaries are built only where the reference tree is present")
    return p


@pytest.mark.parametrize("name", KATS)
def test_reference_known_answer_test_on_gpu_style(ms, name):
    r = subprocess.run([_bin("kat_" + name)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert "* Overall: ok" in r.stdout, r.stdout[-3000:]


def _read_col(path):
    with open(path, "rb") as f:
        count, used = np.frombuffer(f.read(16), dtype=np.uint64)
        data = np.frombuffer(f.read(int(used)), dtype=np.uint8)
    return int(count), data


def test_reference_example_query_on_gpu_style(ms, orc, tmp_path):
    env = dict(os.environ, MSV_GPU_B200_DUMP_DIR=str(tmp_path))
    r = subprocess.run([_bin("select_sum_query")], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    m = re.search(r"^\s*0\s+\.*(\d+)\s*$", r.stdout, re.M)
    assert m, r.stdout
    printed = int(m.group(1))
    trace = [ln.split() for ln in open(tmp_path / "trace.txt").read().splitlines()]
    files = {(t[1], t[2]): tmp_path / t[8] for t in trace}
    assert [t[1] for t in trace] == ["select", "select", "project", "project", "project", "agg_sum", "agg_sum"]
    n, x8 = _read_col(files[("select", "in")])
    x = x8.view(np.uint64)
    _, y8 = _read_col(files[("project", "data")])
    y = y8.view(np.uint64)
    assert n == 100_000_000 and len(y) == n
    # SELECT SUM(baseCol2) WHERE baseCol1 = 150
    want_pos = orc.select(O.CMP_EQ, 150, x)
    want_vals = y[want_pos.astype(np.int64)]
    want_sum = int(want_vals.sum(dtype=np.uint64))
    k, p8 = _read_col(files[("select", "out")])
    assert np.array_equal(p8.view(np.uint64)[:k], want_pos)
    k, v8 = _read_col(files[("project", "out")])
    assert np.array_equal(v8.view(np.uint64)[:k], want_vals)
    _, s8 = _read_col(files[("agg_sum", "out")])
    assert int(s8.view(np.uint64)[0]) == want_sum == printed


def test_reference_operators_cpu_style_vs_gpu_style(ms):
    path = os.path.join(ROOT, "oracle", "_ref", "ref_style_diff")
    if not os.path.exists(path):
        pytest.skip("built only where the reference tree is present")
    if not O.host_has_avx512():
        pytest.skip("the reference's AVX-512 style needs an AVX-512 host")
    r = subprocess.run([path], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, "\n".join(ln for ln in r.stdout.splitlines() if ln.startswith("FAIL"))[-4000:] + \
        r.stderr[-2000:]
    assert re.search(r"^0 of (\d+) cases differ$", r.stdout, re.M), r.stdout[-2000:]
