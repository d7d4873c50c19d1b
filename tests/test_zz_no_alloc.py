"""u1_measure_noalloc: the measurement for callers that cannot allocate.

Some callers cannot call cudaMalloc, for example code confined to memory its
host framework hands out, or loops that cannot accept a cudaMalloc that may
synchronise the device.  u1_measure_noalloc runs the same fused plaquette +
Polyakov kernel as u1_measure_async with its scratch in a fixed device array
inside the library (lattices up to V/2 = 1,048,576 sites).  Here it is called
through the C ABI, twice in a row per lattice, and checked

* bit for bit against u1_measure_async (same kernel, grid and block order,
  so any stale partial sum or wrong block count in the shared array shows);
  the largest lattice runs first, so a smaller one that read leftovers of it
  would differ;
* against the FP64 oracle's plaquettes and Polyakov loop of the same
  configuration, within the measurement tolerance of the other GPU tests;
* for allocating nothing: the library's count of device blocks and the
  device's free memory are unchanged across a call made after the first
  (the first call on a device may load the kernel's module).

The file is collected last, so a stop-at-first-failure run has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

from latticeu1_b200 import _lib
from latticeu1_b200._lib import lib, u1_geom

TOL = 2e-6  # the measurement tolerance used by the other GPU tests
LIMIT = 1 << 20  # V/2 sites the fixed array serves


def _geom(dims, N, beta=1.0, aniso=1.0):
    return u1_geom(dims=dims, N=(C.c_int * 4)(*(list(N) + [0] * (4 - len(N)))), beta=beta, aniso=aniso)


@pytest.mark.parametrize("N", [(32, 32, 32, 66), (48, 48, 48, 48)])
def test_noalloc_rejects_lattice_above_limit_before_device_work(N):
    """V/2 above the fixed array's capacity is refused by the host-side check,
    which runs before any CUDA call (the pointers are never touched)."""
    g = _geom(4, N)
    dummy = C.c_void_p(256)
    rc = lib.u1_measure_noalloc(dummy, C.byref(g), dummy, None)
    assert rc == _lib.U1_ERR_INVALID
    assert "too large" in _lib.last_error()


# largest first: 32^3 x 64 is exactly at the limit (V/2 = 1,048,576)
CASES = [(4, (32, 32, 32, 64), 1.0, 1.0), (4, (16, 16, 16, 16), 1.0, 1.0), (3, (12, 8, 0, 10), 2.0, 1.3)]


@pytest.mark.gpu
def test_noalloc_matches_measure_on_two_calls():
    import torch

    from latticeu1_b200 import Context, Lattice, Rng
    from oracle.oracle import Oracle

    ctx = Context(0)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    want = torch.zeros(6, dtype=torch.float64, device="cuda")
    for case, (dims, N, beta, aniso) in enumerate(CASES):
        lat = Lattice(ctx, dims, N, beta, aniso)
        assert case > 0 or lat.Vh == LIMIT
        rng = Rng(ctx, 100 + case)
        lat.hot_start(rng)
        lat.update(rng, 1, 4)
        lat.measure_async(want.data_ptr())  # the existing entry point (library-owned scratch)
        torch.cuda.synchronize()
        w = want.cpu().numpy()
        g = _geom(dims, N, beta, aniso)
        for call in range(2):
            out.fill_(np.nan)
            torch.cuda.synchronize()
            blocks, free = _lib.device_allocations(), torch.cuda.mem_get_info()[0]
            rc = lib.u1_measure_noalloc(C.c_void_p(lat.links_ptr()), C.byref(g), C.c_void_p(out.data_ptr()), None)
            assert rc == 0, _lib.last_error()
            torch.cuda.synchronize()
            if call == 1:
                assert _lib.device_allocations() == blocks
                assert torch.cuda.mem_get_info()[0] == free
            got = out.cpu().numpy()
            assert np.array_equal(got, w), (case, call, got, w)
        th = lat.export_angles()
        o = Oracle(dims, N, beta, aniso)
        ss, st = o.plaquette(th)
        pl = o.polyakov(th)
        if dims > 2:
            assert abs(complex(got[0], got[1]) - ss) < TOL, (case, got, ss)
        assert abs(complex(got[2], got[3]) - st) < TOL, (case, got, st)
        assert abs(complex(got[4], got[5]) - pl) < TOL, (case, got, pl)
        lat.close()
        rng.close()
