"""The C-ABI library: loads, exports every declared symbol, and the
host-only entry points behave like the reference (no GPU needed)."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O
from rtb200 import lib

GOLD = Path(__file__).resolve().parent / "golden"


def test_library_loads_and_exports_every_declared_symbol():
    L = lib.load()
    declared = lib.declared_symbols()
    assert "cudaBVH_build" in declared and "cudaBVH_traceClosest" in declared
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing


def test_reference_header_symbols_all_present():
    # the 21 entry points of the reference's layer/cuda_bvh_backend.h:21-141
    ref = ["cudaBVH_build", "cudaBVH_destroy", "cudaBVH_tracePrimary", "cudaBVH_traceDiffuse",
           "cudaBVH_traceToRGBA", "cudaBVH_traceToGPUPtr", "cudaBVH_traceToGPUAsync", "cudaBVH_traceToHostPtr",
           "cudaBVH_importBufferFd", "cudaBVH_getBounds", "cudaBVH_getNumTris", "cudaBVH_getNumBVH4Nodes",
           "cudaBVH_getNumCWBVHNodes", "cudaBVH_getNodeData", "cudaBVH_getTriData", "cudaBVH_getStacklessBVH2",
           "cudaBVH_getPackedTris", "cudaBVH_resetDevice", "cudaBVH_buildFromAABBs", "cudaBVH_buildTLASFast",
           "cudaBVH_readGPUMemoryFd"]
    assert len(set(ref)) == 21
    L = lib.load()
    assert all(hasattr(L, s) for s in ref)


def test_null_and_empty_inputs_fail_cleanly():
    L = lib.load()
    assert L.cudaBVH_build(None, 0) is None
    assert "empty" in lib.last_error()
    assert L.cudaBVH_buildFromAABBs(None, 5) is None
    L.cudaBVH_destroy(None)  # no-op
    assert L.cudaBVH_getNumTris(None) == 0
    assert L.cudaBVH_getNumCWBVHNodes(None) == 0
    assert L.cudaBVH_getNodeData(None) is None
    p = C.POINTER(C.c_uint32)()
    assert L.cudaBVH_getStacklessBVH2(None, C.byref(p)) == 0 and not p
    assert L.cudaBVH_traceClosest(None, None, 1, None, None) == -1
    assert L.cudaBVH_traceAnyHost(None, None, 1, None) == -1
    assert L.cudaBVH_tracePrimary(None, 16, 0.0, 0.0, 0.0, None) == 0.0
    pn = C.POINTER(C.c_uint32)()
    assert L.cudaBVH_buildTLASFast(None, 3, C.byref(pn), None) == 0
    assert L.cudaTLAS_build(None, 0, None, 0) is None
    assert L.cudaTLAS_setTransforms(None, None, 0) == -1
    assert "one instance record per TLAS instance" in lib.last_error()


@pytest.mark.parametrize("path", sorted(GOLD.glob("ref_tlasfast_*.npz")), ids=lambda p: p.stem)
def test_tlas_fast_matches_reference_except_skips(path):
    """Host-only entry point: node bytes equal the reference's in every word
    but the skip pointer, which equals the repaired export."""
    g = np.load(path)
    nodes, ordered = lib.tlas_fast(g["aabbs"])
    assert np.array_equal(ordered, g["ordered"])
    ref = g["nodes"].reshape(-1, 8)
    mine = nodes.reshape(-1, 8)
    assert np.array_equal(mine[:, :7], ref[:, :7])
    assert np.array_equal(nodes, O.fix_skips(g["nodes"]))


REF_OUT = Path(__file__).resolve().parents[1] / "oracle" / "_ref"


def _nm(path, *flags):
    import subprocess
    r = subprocess.run(["nm", "-D", *flags, str(path)], capture_output=True, text=True, check=True)
    return {ln.split()[-1].split("@")[0] for ln in r.stdout.splitlines() if ln.strip()}


def test_reference_caller_and_shim_link_against_the_library():
    """The reference's own C-ABI caller (layer/bvh_bench.cu, compiled unchanged
    against include/cuda_bvh_backend.h) and its OptiX shim (linked as
    OptiX_Shim/build_shim.sh:18-21 does, with this library in place of
    cuda_bvh_backend.o) resolve every backend symbol they import from
    libcudabvh_b200.so.  Built by `make -C oracle ref` from the reference
    sources; the GPU run of the caller is tests/test_gpu_dropin.py."""
    import subprocess
    bench, shim = REF_OUT / "bvh_bench_b200", REF_OUT / "libnvoptix_shim_b200.so"
    if not bench.exists() or not shim.exists():
        pytest.skip("oracle/_ref caller and shim are built only where the reference sources are mounted")
    exported = _nm(lib.LIB_PATH, "--defined-only")
    wanted = {s for s in _nm(bench, "--undefined-only") if s.startswith("cudaBVH_")}
    assert {"cudaBVH_build", "cudaBVH_tracePrimary", "cudaBVH_traceToRGBA", "cudaBVH_destroy"} <= wanted
    assert wanted <= exported, wanted - exported
    for f in (bench, shim):
        ldd = subprocess.run(["ldd", str(f)], capture_output=True, text=True, check=True).stdout
        line = next(ln for ln in ldd.splitlines() if "libcudabvh_b200.so" in ln)
        assert "not found" not in line and Path(line.split("=>")[1].split("(")[0].strip()).resolve() == \
            lib.LIB_PATH.resolve()
    assert "optixQueryFunctionTable" in _nm(shim, "--defined-only")
