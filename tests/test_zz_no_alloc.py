"""The allocation-free entry point matches the allocating one.

cc_transport_photons_device_noalloc serves callers that cannot let the
library allocate device memory (an application that owns every device
allocation, or a pipeline that forbids cudaMalloc/cudaFree while it runs).
Its scratch is a static device array shared by all calls, so this test
calls it twice in a row and compares both results with
cc_transport_photons_device on the same photons and seed; the second call
runs on a stream of the caller's, and the device's free memory must not
change across it.  It lives in its own file, collected last, and runs
alone in a fresh process too.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GEOMS = [
    {"name": "room", "shape": "box", "material": "air", "center": [0, 0, 0], "size_cm": [120, 100, 90]},
    {"name": "slab", "shape": "box", "material": "water", "center": [0, 0, 0], "size_cm": [30, 30, 20]},
    {"name": "ball", "shape": "sphere", "material": "bone", "center": [5, -3, 2], "radius_cm": 6},
    {"name": "rod", "shape": "cylinder", "material": "lead", "axis": "x", "center": [0, 8, -4],
     "radius_cm": 1.5, "height_cm": 25},
]


def _photons(torch, n):
    d = torch.tensor([1.0, 0.05, 0.02], dtype=torch.float64)
    d = d / d.norm()
    pos = torch.tensor([-55.0, 1.0, 2.0], dtype=torch.float64).repeat(n, 1).cuda().contiguous()
    dirv = d.repeat(n, 1).cuda().contiguous()
    en = torch.full((n,), 80.0, dtype=torch.float64, device="cuda")
    return pos, dirv, en


def _outputs(torch, n):
    return (torch.zeros(n, dtype=torch.int32, device="cuda"), torch.zeros(n, dtype=torch.uint8, device="cuda"),
            torch.zeros(n, dtype=torch.uint8, device="cuda"))


def test_noalloc_matches_allocating_entry_point():
    torch = pytest.importorskip("torch")
    from chatcarlo_b200 import _native as N
    from chatcarlo_b200.geometry import Geometry
    from chatcarlo_b200.transport import default_engine

    eng = default_engine()
    geom = Geometry(GEOMS)
    ts, th = eng.tables(geom.materials(), need_muen=False)
    sh = eng.scene(geom, ts)
    lib = eng.lib
    n, seed = 300_000, 1234
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    try:
        ref_pos, ref_dir, ref_en = _photons(torch, n)
        ref_nsc, ref_abs, ref_esc = _outputs(torch, n)
        ref_edep = np.zeros(len(ts.names))
        ref_nfl = C.c_int64()
        N.check(lib.cc_transport_photons_device(eng.ctx, sh, th, None, n, ptr(ref_pos), ptr(ref_dir), ptr(ref_en),
                                                seed, 0, 1, ptr(ref_nsc), ptr(ref_abs), ptr(ref_esc),
                                                N.dptr(ref_edep), C.byref(ref_nfl)))
        torch.cuda.synchronize()
        for call in range(2):
            pos, dirv, en = _photons(torch, n)
            nsc, absd, esc = _outputs(torch, n)
            edep = np.zeros(len(ts.names))
            nfl = C.c_int64()
            # call 0 on the legacy default stream, call 1 on a stream of the
            # caller's; the second call allocates nothing on the device
            stream = torch.cuda.Stream() if call == 1 else None
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            N.check(lib.cc_transport_photons_device_noalloc(
                sh, th, n, ptr(pos), ptr(dirv), ptr(en), seed, 0, 1, ptr(nsc), ptr(absd), ptr(esc),
                N.dptr(edep), C.byref(nfl), C.c_void_p(stream.cuda_stream) if stream is not None else None))
            torch.cuda.synchronize()
            if call == 1:
                assert torch.cuda.mem_get_info()[0] == free_before
            # same kernel code and the same per-history Philox streams: identical photons
            assert torch.equal(pos, ref_pos), call
            assert torch.equal(dirv, ref_dir), call
            assert torch.equal(en, ref_en), call
            assert torch.equal(nsc, ref_nsc), call
            assert torch.equal(absd, ref_abs), call
            assert torch.equal(esc, ref_esc), call
            assert nfl.value == ref_nfl.value, call
            # deposited energy: FP64 sums in a different atomic order
            np.testing.assert_allclose(edep, ref_edep, rtol=1e-9, atol=0.0, err_msg=str(call))
            assert edep.sum() > 0
    finally:
        lib.cc_scene_destroy(sh)
