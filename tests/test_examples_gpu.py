"""The C++ drop-in examples (engine_b200/examples), built against the
drop-in header and libms_gpu.so, run on the GPU and check themselves."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "engine_b200", "examples", "bin")


@pytest.mark.parametrize("prog,args", [("select_sum_query", ["2000003"]), ("kat_test", []),
                                       ("star_and_batch", ["1000003"])])
def test_example_runs(ms, prog, args):
    path = os.path.join(BIN, prog)
    if not os.path.exists(path):
        pytest.fail(f"{prog} was not built (python engine_b200/build.py)")
    r = subprocess.run([path, *args], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, MSV_GPU_ARENA_BYTES=str(4 << 30)))
    assert r.returncode == 0, r.stdout + r.stderr
