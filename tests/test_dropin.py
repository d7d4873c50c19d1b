"""Drop-in checks of the C++ API shim (latticeu1_b200/shim): code written
against the reference's driver surface (namespace U1, reference u1.cpp)
compiles and links against libu1shim.so + libu1b200.so unchanged.

* tests/dropin/driver.cpp (this repository's own driver using that API)
  compiles on the CPU; on the GPU its results equal the Python host layer's
  bit for bit (same kernels behind both);
* the reference's unmodified u1.cpp, compiled in place by `make -C oracle
  dropin REF=<reference source tree>` into oracle/_ref/u1_dropin, runs its full hard-coded workload
  (24^3 x 12, 1000 sweeps, Poly2, Poly2 multihit, MultiLevel) on the GPU and
  writes the reference's output files.
"""
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
SHIM_INC = ROOT / "latticeu1_b200" / "shim" / "include"
LIBDIR = ROOT / "latticeu1_b200" / "lib"
DRIVER = ROOT / "tests" / "dropin" / "driver.cpp"
REF_DROPIN = ROOT / "oracle" / "_ref" / "u1_dropin"


def _compile_driver(out: Path) -> Path:
    exe = out / "driver"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + str(SHIM_INC), str(DRIVER), "-L" + str(LIBDIR), "-lu1shim",
                    "-lu1b200", "-Wl,-rpath," + str(LIBDIR), "-o", str(exe)], check=True)
    return exe


def test_driver_compiles_against_shim(tmp_path):
    assert (LIBDIR / "libu1shim.so").exists(), "run latticeu1_b200/build.py"
    exe = _compile_driver(tmp_path)
    assert exe.exists()


def test_shim_headers_cover_reference_driver_includes():
    """Every project header the reference driver includes has a shim header."""
    names = ["timer.h", "alloc.h", "complex.h", "parameters.h", "random.h", "update.h", "plaquette.h",
             "polyakov.h", "multilevel.h", "array.h", "actime.h"]
    for n in names:
        assert (SHIM_INC / n).exists(), n


def _parse(stdout: str):
    out = {}
    for line in stdout.splitlines():
        parts = line.split()
        if parts and parts[0] in ("SWEEP", "POLY2MH", "MULTILEVEL"):
            key = parts[0] if parts[0] != "SWEEP" else f"SWEEP{parts[1]}"
            vals = parts[2:] if parts[0] == "SWEEP" else parts[1:]
            out[key] = np.array([float(v) for v in vals])
    return out


@pytest.mark.gpu
def test_driver_matches_python_host_layer(tmp_path):
    from latticeu1_b200 import Context, Lattice, Rng
    exe = _compile_driver(tmp_path)
    res = subprocess.run([str(exe), "4321"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr + res.stdout
    got = _parse(res.stdout)
    ctx = Context(0)
    lat = Lattice(ctx, 4, (8, 6, 6, 8), 1.0)
    rng = Rng(ctx, 4321)
    lat.hot_start(rng)
    for it in range(1, 4):
        lat.update(rng, 1, 4)
        m = lat.measure()
        want = np.array([m["plaq_ss"].real, m["plaq_ss"].imag, m["plaq_st"].real, m["plaq_st"].imag,
                         m["poly"].real, m["poly"].imag])
        np.testing.assert_array_equal(got[f"SWEEP{it}"], want)
    c = lat.poly_corr(True)
    np.testing.assert_array_equal(got["POLY2MH"], np.stack([c.real, c.imag], -1).reshape(-1))
    ml = lat.multilevel(rng, 2, 1, 3, 1, 1, 2)
    np.testing.assert_array_equal(got["MULTILEVEL"], np.stack([ml.real, ml.imag], -1).reshape(-1))
    assert (tmp_path / "Pot_mhit_8_6_6_8_beta_1_xi_1_mtr_1_ovr_4_iter_3.dat").exists()
    assert (tmp_path / "Pot_mlevel_8_6_6_8_beta_1_xi_1_mtr_1_ovr_4_iter_3_2_1_3_1_1_2.dat").exists()


@pytest.mark.gpu
@pytest.mark.skipif(not REF_DROPIN.exists(), reason="oracle/_ref/u1_dropin not built (reference sources absent)")
def test_reference_driver_runs_unmodified(tmp_path):
    res = subprocess.run([str(REF_DROPIN)], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:] + res.stdout[-2000:]
    name = "24_24_24_12_beta_1_xi_1_mtr_1_ovr_3"
    plaq = np.loadtxt(tmp_path / f"plaq_{name}.dat")
    assert plaq.shape == (11, 5)  # iter, SS re, SS im, ST re, ST im at iter 0, 100, ..., 1000
    assert np.allclose(plaq[0, 1:], 0.0)  # cold start: 1 - e^{i0} = 0
    # beta = 1.0 (cold start): ordered side of the transition, 1-<cos P> well below the hot value 1
    assert 0.1 < plaq[-1, 1] < 0.6 and 0.1 < plaq[-1, 3] < 0.6
    for pref in ("Pot_", "Pot_mhit_"):
        c = np.loadtxt(tmp_path / f"{pref}{name}_iter_1000.dat")
        assert c.shape == (12, 3) and np.all(np.isfinite(c))
    ml = np.loadtxt(tmp_path / f"Pot_mlevel_{name}_iter_1000_10_1_20_1_2_5.dat")
    assert ml.shape == (12, 3) and np.all(np.isfinite(ml))
    assert re.search(r"Time: [0-9.eE+-]+ s", res.stdout)


@pytest.mark.gpu
def test_timing_driver_reference_vs_dropin(tmp_path):
    """tests/dropin/timing_driver.cpp (the reference driver's workload through
    its namespace U1 API) built against the reference's own objects and
    against the drop-in shim: both run, agree on the physics scale, and the
    drop-in is faster.  Writes the timings to $U1_REF_TIMING_OUT when set."""
    import json
    import os
    import subprocess
    ref_exe = ROOT / "oracle" / "_ref" / "timing_reference"
    our_exe = ROOT / "oracle" / "_ref" / "timing_dropin"
    if not (ref_exe.exists() and our_exe.exists()):
        pytest.skip("timing drivers not built (make -C oracle timing REF=<reference source tree>)")
    out = {}
    for name, exe in (("reference", ref_exe), ("dropin", our_exe)):
        r = subprocess.run([str(exe)], cwd=tmp_path, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        lines = {ln.split()[0]: ln.split()[1:] for ln in r.stdout.splitlines() if ln.strip()}
        out[name] = {"time_s": float(lines["TIME"][0]), "plaq_ss": float(lines["SWEEP"][1]),
                     "plaq_st": float(lines["SWEEP"][2])}
    # independent chains at the same beta: equilibrium plaquettes agree to a few 1e-3
    assert abs(out["reference"]["plaq_ss"] - out["dropin"]["plaq_ss"]) < 0.01
    assert out["dropin"]["time_s"] < out["reference"]["time_s"]
    path = os.environ.get("U1_REF_TIMING_OUT")
    if path:
        d = {}
        if os.path.exists(path):
            with open(path) as f:
                d = json.load(f)
        d["driver_24x24x24x12_1000_sweeps"] = out
        with open(path, "w") as f:
            json.dump(d, f, indent=1)
