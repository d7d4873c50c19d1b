"""The checked build (libu1b200_check.so, -DU1_BOUNDS_CHECK) and the static
phase-dependency check.

* static (CPU): for every phase (parity p, direction mu) of the checkerboard
  update, the staple of a link (x, mu) with x of parity p reads no link
  (mu, p, y) with y != x, so the links one phase writes are never read by
  another update of the same phase.  The neighbour indices come from the
  FP64 oracle's restatement of the reference's EO indexing
  (include/index.h:114-153, pinned to the reference's own tables by
  test_oracle_pin) and the staple's six links per plaquette pair
  (include/staple.h:79-102).  Every extent the library accepts (even, >= 2)
  passes; an odd extent, which u1_geom_validate refuses, is shown to break
  the decomposition.
* checked build (GPU, child process with U1_CHECKED=1): every update
  variant, the batched kernels (two lanes of chain groups), the measuring
  phases, windowed Metropolis,
  multilevel sub-updates and full-size four-site phases (32^4 in one wave,
  40^4 in several) run with bounds, alignment and race checks on
  every link access; no violation and no race may occur, the phase count
  must match the phases launched, and the links and measurements must be
  bit-identical to the normal build's.  The checker itself is exercised by
  u1_check_selftest (two refused accesses, two races, planted in its marks
  and never dereferenced).
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# (dims, N as the ABI takes it: Nx, Ny, Nz, Nt; beta, aniso)
GEOMS = [
    (4, (8, 8, 8, 8), 1.0, 1.0),
    (4, (16, 6, 4, 4), 1.05, 1.5),
    (4, (6, 4, 4, 8), 1.1, 1.0),
    (4, (4, 2, 2, 6), 0.9, 2.0),   # extents 2: x + e and x - e are the same site
    (3, (8, 6, 0, 10), 1.2, 0.8),
    (2, (16, 0, 0, 12), 2.0, 1.0),
]
BATCH = [(4, (8, 8, 8, 8), 1.0, 1.0), (4, (16, 4, 4, 4), 1.1, 1.0), (4, (6, 4, 4, 8), 0.9, 1.2),
         (4, (4, 2, 2, 6), 1.0, 2.0)] + [(4, (16, 16, 16, 16), 0.95, 1.0)] * 3  # 2 MiB groups: 4 groups, 2 lanes
SWEEPS = ((1, 4), (2, 0), (0, 3))


# ----------------------------------------------------------------- static check
def _grid(dims: int, N) -> list[int]:
    """The reference's Grid[] mapping (src/parameters.cu:150-161)."""
    Nx, Ny, Nz, Nt = N
    return {2: [Nx, Nt], 3: [Nx, Ny, Nt], 4: [Nx, Ny, Nz, Nt]}[dims]


def phase_conflicts_eo(o) -> tuple[int, int]:
    """Over all phases (p, mu): reads, by the staple of link (x, mu) with x of
    parity p, of a link (mu, p, y), y != x (a link the same phase writes),
    and the number of reads checked.  Links are the oracle's EO link indices
    eo + parity V/2 + dir V (reference include/index.h:114-153); the six
    links per plaquette pair are those of include/staple.h:79-102:
    U_nu(x+mu), U_mu(x+nu), U_nu(x) and U_nu(x+mu-nu), U_mu(x-nu), U_nu(x-nu)."""
    V, Vh, d = o.V, o.Vh, o.dims
    bad = checked = 0
    for p in (0, 1):
        for mu in range(d):
            lo, hi = mu * V + p * Vh, mu * V + (p + 1) * Vh  # the links this phase writes
            for i in range(Vh):
                own = mu * V + p * Vh + i
                for nu in range(d):
                    if nu == mu:
                        continue
                    xm = o.index_eo_neg(i, p, mu, 1)
                    xn = o.index_eo_neg(i, p, nu, 1)
                    xd = o.index_eo_neg(i, p, nu, -1)
                    xmd = o.index_eo_neg(i, p, mu, 1, nu, -1)
                    reads = (nu * V + xm, mu * V + xn, nu * V + p * Vh + i, nu * V + xmd, mu * V + xd, nu * V + xd)
                    for link in reads:
                        checked += 1
                        if lo <= link < hi and link != own:
                            bad += 1
    return bad, checked


def phase_conflicts(grid: list[int]) -> int:
    """The same count on site coordinates (any extents, odd ones included:
    the oracle's indexing refuses those), parity (sum x) & 1."""
    d = len(grid)

    def shift(y, k, s):
        y = list(y)
        y[k] = (y[k] + s) % grid[k]
        return tuple(y)

    sites = list(np.ndindex(*grid))
    bad = 0
    for p in (0, 1):
        own = [x for x in sites if sum(x) % 2 == p]
        for mu in range(d):
            written = {(mu, x) for x in own}
            for x in own:
                xm = shift(x, mu, 1)
                for nu in range(d):
                    if nu == mu:
                        continue
                    for link in ((nu, xm), (mu, shift(x, nu, 1)), (nu, x), (nu, shift(xm, nu, -1)),
                                 (mu, shift(x, nu, -1)), (nu, shift(x, nu, -1))):
                        if link in written and link != (mu, x):
                            bad += 1
    return bad


@pytest.mark.parametrize("geom", GEOMS, ids=lambda g: f"{g[0]}d-{'x'.join(map(str, g[1]))}")
def test_static_phase_dependencies(geom):
    from oracle.oracle import Oracle
    dims, N = geom[:2]
    o = Oracle(dims, N, 1.0)
    bad, checked = phase_conflicts_eo(o)
    assert checked == 2 * dims * o.Vh * (dims - 1) * 6
    assert bad == 0
    assert phase_conflicts(_grid(dims, N)) == 0


def test_static_check_finds_odd_extent():
    """A planted defect: with an odd extent a site and its neighbour across
    the boundary share a parity, so a phase reads links it writes (the
    reason u1_geom_validate requires even extents)."""
    from latticeu1_b200 import _lib
    g = _lib.u1_geom(4, (_lib.C.c_int * 4)(4, 4, 4, 5), 1.0, 1.0)
    assert _lib.lib.u1_geom_validate(_lib.C.byref(g), None) == _lib.U1_ERR_INVALID
    assert phase_conflicts([4, 4, 4, 5]) > 0
    assert phase_conflicts([4, 4, 4, 4]) == 0


def test_checked_library_exports():
    """The checked library is built and exports every symbol of the header."""
    import re
    lib_path = ROOT / "latticeu1_b200" / "lib" / "libu1b200_check.so"
    assert lib_path.exists(), "build it with python latticeu1_b200/build.py --checked"
    import ctypes
    lib = ctypes.CDLL(str(lib_path))
    names = re.findall(r"\b(u1_\w+)\s*\(", (ROOT / "include" / "u1_b200.h").read_text())
    missing = [n for n in set(names) if not hasattr(lib, n)]
    assert not missing, missing


# --------------------------------------------------------------- checked build
def run_workload(out: Path) -> dict:
    """The workload both builds run; returns the expected phase counts per
    section and saves the links and measurements to `out`."""
    import torch

    from latticeu1_b200 import Batch, Context, Lattice, Rng, U1Error, _lib
    ctx = Context(0)
    res: dict[str, np.ndarray] = {}
    phases = {"lattice": 0}
    meas = torch.zeros(8, dtype=torch.float64, device="cuda")
    for gi, (dims, N, beta, aniso) in enumerate(GEOMS):
        pair_ok = (N[0] // 2) % 2 == 0
        quad_ok = (N[0] // 2) % 4 == 0
        for v in (3,) + ((1, 2) if pair_ok else ()) + ((5,) if quad_ok else ()) + (4,):
            lat = Lattice(ctx, dims, N, beta, aniso)
            try:
                lat.set_variant(v)
            except U1Error:
                lat.close()
                continue
            rng = Rng(ctx, 77 + gi)
            lat.hot_start(rng)
            for m, o in SWEEPS:
                lat.update(rng, m, o)
                phases["lattice"] += 0 if v == 4 else 2 * dims * (m + o)
            lat.update_measure(rng, 1, 4, meas.data_ptr())
            phases["lattice"] += 0 if v == 4 else 2 * dims * 5
            torch.cuda.synchronize()
            res[f"meas_{gi}_{v}"] = meas.cpu().numpy().copy()
            for met, p, mu in ((True, 1, dims - 1), (False, 0, 0)):
                lat.update_phase(rng, met, p, mu)
                phases["lattice"] += 1
            res[f"links_{gi}_{v}"] = lat.export_angles()
            lat.close()
            rng.close()
    # full-size four-site phases: 32^4 (one wave, SM-local block order) and
    # 40^4 (several waves, launch order)
    for L in (32, 40):
        lat = Lattice(ctx, 4, (L,) * 4, 1.0)
        lat.set_variant(5)
        lat.set_block(128)
        rng = Rng(ctx, 11)
        lat.hot_start(rng)
        lat.update_measure(rng, 1, 4, meas.data_ptr())
        phases["lattice"] += 2 * 4 * 5
        torch.cuda.synchronize()
        res[f"meas_{L}"] = meas.cpu().numpy().copy()
        res[f"links_{L}"] = lat.export_angles()
        lat.close()
        rng.close()
    report = {"lattice": None}
    if _lib.CHECKED:
        report["lattice"] = _lib.check_report(ctx.handle, reset=True)
    # windowed multi-hit Metropolis
    lat = Lattice(ctx, 4, (8, 8, 8, 8), 1.0)
    lat.set_variant(5)
    lat.set_metropolis(0.6, 3)
    rng = Rng(ctx, 5)
    lat.hot_start(rng)
    lat.update(rng, 2, 1)
    phases["window"] = 2 * 4 * 3
    res["links_window"] = lat.export_angles()
    lat.close()
    rng.close()
    if _lib.CHECKED:
        report["window"] = _lib.check_report(ctx.handle, reset=True)
    # multilevel sub-updates (frozen time slices)
    lat = Lattice(ctx, 4, (4, 4, 4, 8), 0.95)
    rng = Rng(ctx, 9)
    lat.hot_start(rng)
    res["multilevel"] = lat.multilevel(rng, 2, 2, 2, 2, 1, 2)
    res["links_multilevel"] = lat.export_angles()
    lat.close()
    rng.close()
    if _lib.CHECKED:
        report["multilevel"] = _lib.check_report(ctx.handle, reset=True)
    # batched chains (four-, two- and one-site groups)
    b = Batch(ctx, BATCH, seed=21)
    b.configure(2)
    assert b.groups >= 3 and b.lanes == 2
    b.hot_start()
    b.update(1, 4, measure=True)
    b.update(0, 2)
    res["batch_meas"] = b.measure_raw()
    links = b.export_all()  # queued on the batch's stream
    torch.cuda.synchronize()
    res["batch_links"] = links.cpu().numpy()
    phases["batch"] = sum(2 * 4 * (m + o) for m, o in ((1, 4), (0, 2))) * b.groups
    b.close()
    if _lib.CHECKED:
        report["batch"] = _lib.check_report(ctx.handle, reset=True)
        report["selftest"] = _lib.check_selftest(ctx.handle)
    np.savez(out / ("checked.npz" if _lib.CHECKED else "normal.npz"), **res)
    return {"phases": phases, "report": report}


@pytest.mark.gpu
def test_checked_build_clean_and_bit_identical(tmp_path):
    normal = run_workload(tmp_path)
    env = {**os.environ, "PYTHONPATH": str(ROOT), "U1_CHECKED": "1"}
    r = subprocess.run([sys.executable, str(Path(__file__).resolve()), "run", str(tmp_path)], cwd=str(ROOT),
                       env=env, capture_output=True, text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-3000:])
    checked = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    rep = checked["report"]
    st = rep["selftest"]
    assert st["bad"] == 2 and st["races"] == 2 and st["marked"] == 4 and st["phases"] == 1, st
    assert st["first_bad_half"] == 16 and st["first_bad_idx"] in (14, 1) and st["first_bad_kind"] == 0, st
    assert st["first_race_link"] in (3, 5), st
    for section in ("lattice", "window", "multilevel", "batch"):
        s = rep[section]
        assert s["bad"] == 0, (section, s)
        assert s["races"] == 0, (section, s)
        assert s["marked"] > 0, (section, s)
        if section in checked["phases"]:
            assert s["phases"] == checked["phases"][section], (section, s, checked["phases"])
        else:
            assert s["phases"] > 0, (section, s)
    assert checked["phases"] == normal["phases"]
    a = np.load(tmp_path / "normal.npz")
    b = np.load(tmp_path / "checked.npz")
    assert sorted(a.files) == sorted(b.files)
    for k in a.files:
        assert np.array_equal(a[k], b[k], equal_nan=True), k  # 2D: no spatial plaquettes, SS is NaN as in the reference


if __name__ == "__main__" and len(sys.argv) > 2 and sys.argv[1] == "run":
    print(json.dumps(run_workload(Path(sys.argv[2]))))
