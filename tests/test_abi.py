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
