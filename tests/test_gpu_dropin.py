"""The drop-in claim with a real C++ caller: the reference's own benchmark
of its C-ABI (layer/bvh_bench.cu:1-97: terrain BLAS builds of 20K-1.6M
triangles, cudaBVH_tracePrimary at 512^2..2048^2, cudaBVH_traceToRGBA at
1080p) compiled unchanged against include/cuda_bvh_backend.h and linked to
libcudabvh_b200.so (oracle/_ref/bvh_bench_b200, made by `make -C oracle
ref`), run on the GPU: it must finish cleanly and report rays per second
for every row."""
import re
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

BENCH = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "bvh_bench_b200"


def test_reference_bvh_bench_runs_on_the_library(cuda):
    if not BENCH.exists():
        pytest.fail(f"{BENCH} not built (make -C oracle ref, where the reference sources are mounted)")
    r = subprocess.run([str(BENCH)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    rows = re.findall(r"║\s*(\d+)x\s*(\d+)\s*║\s*(\d+)K\s*║\s*(\d+)x\s*(\d+)\s*║\s*([\d.]+)\s*║", r.stdout)
    assert len(rows) == 18, r.stdout
    assert all(float(mrs) > 0 for *_, mrs in rows), rows
    assert "Build failed" not in r.stdout
    m = re.search(r"1920x1080 @ (\d+)K tris: ([\d.]+) ms/frame", r.stdout)
    assert m and float(m.group(2)) > 0, r.stdout
