"""Failure detection without a GPU fault.

* Allocation failures are injected on the host through the library's device
  allocator hook (u1_set_device_allocator): a fake allocator refuses the k-th
  request, for every k a lattice / rng / batch workload makes.  Each refused
  call returns U1_ERR_NOMEM, the object it worked on stays usable (the same
  call succeeds when repeated), and once every object is destroyed the
  library holds no device memory (no leak).  The GPU part runs in a child
  process, so that no other test's objects hold memory from the allocator.
* The persistent sweep's bounded neighbour wait is made to run out with a
  tile that never publishes its phases and a short poll limit: the kernel
  returns, the next synchronous call reports U1_ERR_CUDA, and the same
  lattice then runs a correct sweep (bit-identical to the phase kernels).
"""
import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_allocator_hook_host_logic():
    """No device needed: both functions or neither, and the hook can be
    installed and removed while the library holds no device memory."""
    from latticeu1_b200 import _lib
    alloc = _lib.DEV_ALLOC_FN(lambda user, n, out: 1)
    free = _lib.DEV_FREE_FN(lambda user, p: None)
    assert _lib.device_allocations() == 0
    assert _lib.lib.u1_set_device_allocator(alloc, _lib.NO_FREE, None) == _lib.U1_ERR_INVALID
    assert _lib.lib.u1_set_device_allocator(_lib.NO_ALLOC, free, None) == _lib.U1_ERR_INVALID
    assert _lib.lib.u1_set_device_allocator(alloc, free, None) == _lib.U1_OK
    assert _lib.lib.u1_set_device_allocator(_lib.NO_ALLOC, _lib.NO_FREE, None) == _lib.U1_OK


def _child_injection() -> None:
    """Run the workload once per injection point k = 1, 2, ... until a run
    makes fewer than k requests; print a summary line."""
    os.environ["U1_TUNE"] = "0"
    import torch

    from latticeu1_b200 import Batch, Context, Lattice, Rng, U1Error, _lib
    torch.cuda.init()
    live = {}
    st = {"n": 0, "fail": 0, "injected": 0}

    def alloc(user, nbytes, out):
        st["n"] += 1
        if st["n"] == st["fail"]:
            st["injected"] += 1
            return 1
        p = torch.cuda.caching_allocator_alloc(max(int(nbytes), 1), device=0)
        live[p] = nbytes
        out[0] = p
        return 0

    def release(user, p):
        live.pop(p)
        torch.cuda.caching_allocator_delete(p)

    a_fn, r_fn = _lib.DEV_ALLOC_FN(alloc), _lib.DEV_FREE_FN(release)
    _lib.check(_lib.lib.u1_set_device_allocator(a_fn, r_fn, None), "u1_set_device_allocator")
    ctx = Context(0)
    geoms = [(4, (8, 8, 8, 8), 1.0), (4, (6, 6, 6, 8), 1.1)]
    k, refused = 0, []
    while True:
        k += 1
        st.update(n=0, fail=k, injected=0)
        o = {}
        steps = [
            ("lattice", lambda: o.__setitem__("lat", Lattice(ctx, 4, (8, 8, 8, 8), 1.0))),
            ("rng", lambda: o.__setitem__("rng", Rng(ctx, 5))),
            ("hot_start", lambda: o["lat"].hot_start(o["rng"])),
            ("update", lambda: o["lat"].update(o["rng"], 1, 4)),
            ("measure", lambda: o["lat"].measure()),
            ("export", lambda: o["lat"].export_angles()),
            ("poly_corr", lambda: o["lat"].poly_corr(True)),
            ("multilevel", lambda: o["lat"].multilevel(o["rng"], 1, 1, 2, 1, 1, 1)),
            ("batch", lambda: o.__setitem__("batch", Batch(ctx, geoms, seed=3))),
            ("batch_sweep", lambda: (o["batch"].hot_start(), o["batch"].update(1, 4, measure=True),
                                     o["batch"].measure())),
        ]
        for name, fn in steps:
            before = st["injected"]
            try:
                fn()
            except U1Error as e:
                assert st["injected"] == before + 1, f"k={k} {name}: failure without injection: {e}"
                assert e.code == _lib.U1_ERR_NOMEM, f"k={k} {name}: status {e.code}, not U1_ERR_NOMEM: {e}"
                refused.append(name)
                fn()  # the object is still usable: the same call now succeeds
            else:
                assert st["injected"] == before, f"k={k} {name}: an injected failure was not reported"
        m = o["lat"].measure()
        assert 0.0 < m["plaq_ss"].real < 2.0
        for name in ("batch", "lat", "rng"):
            o.pop(name).close()
        torch.cuda.synchronize()
        assert _lib.device_allocations() == 0 and not live, (k, _lib.device_allocations(), len(live))
        if st["n"] < k:  # this run had no k-th request: every injection point is covered
            break
    _lib.check(_lib.lib.u1_set_device_allocator(_lib.NO_ALLOC, _lib.NO_FREE, None), "u1_set_device_allocator")
    print(f"INJECTION_OK points={k - 1} refused={sorted(set(refused))}")


@pytest.mark.gpu
def test_injected_allocation_failures_no_leak():
    env = {**os.environ, "PYTHONPATH": str(ROOT)}
    r = subprocess.run([sys.executable, str(Path(__file__).resolve()), "inject"], cwd=str(ROOT), env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0 and "INJECTION_OK" in r.stdout, (r.stdout[-3000:], r.stderr[-3000:])
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("INJECTION_OK")][0]
    points = int(line.split()[1].split("=")[1])
    assert points >= 10, line
    for step in ("lattice", "rng", "measure", "multilevel", "batch"):
        assert step in line, line


@pytest.mark.gpu
def test_wave_wait_runs_out_and_lattice_recovers(ctx):
    from latticeu1_b200 import Lattice, Rng, U1Error
    dims, N, beta = 4, (16, 16, 8, 8), 1.0
    lat = Lattice(ctx, dims, N, beta)
    try:
        lat.set_variant(4)
    except U1Error:
        pytest.skip("persistent sweep not usable on this device")
    with pytest.raises(U1Error):
        lat.set_wave_wait(0, N[2] * N[3])  # tiles are the (x2, x3) planes
    rng = Rng(ctx, 12)
    lat.hot_start(rng)
    th0 = lat.export_angles()
    lat.set_wave_wait(4096, 5)
    lat.update(rng, 1, 4)  # asynchronous: returns before the waits run out
    with pytest.raises(U1Error) as e:
        lat.synchronize()
    assert e.value.code == -2 and "ran out" in str(e.value)
    lat.synchronize()  # the condition was cleared by the report
    # the same lattice, default waits: a correct sweep again
    lat.set_wave_wait(0, -1)
    lat.import_angles(th0)
    ra, rb = Rng(ctx, 40), Rng(ctx, 40)
    lat.update(ra, 1, 4)
    ref = Lattice(ctx, dims, N, beta)
    ref.set_variant(1)
    ref.import_angles(th0)
    ref.update(rb, 1, 4)
    assert np.array_equal(lat.export_angles(), ref.export_angles())


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "inject":
    sys.path.insert(0, str(ROOT))
    _child_injection()
