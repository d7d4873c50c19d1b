"""Run the REFERENCE's own CUDA build (oracle/_ref/libu1ref.so, GPU side of
oracle/ref/ref_harness.cu) in a child process.  TEST INFRASTRUCTURE ONLY:
used by tests/test_ref_cuda.py to compare the sm_100a kernels with the
reference's kernels on the same B200 and to time the reference build.

The reference keeps process-global state (PARAMS, __constant__ memory, its
tune cache) and exits on CUDA errors, so every task runs in a fresh child:

    python -m oracle.ref_gpu <task> <in.npz> <out.npz>

tasks: measure | or_pass | poly2 | multilevel | multilevel_timing | timing | chain |
       convert | plaq_fields
"""
from __future__ import annotations

import ctypes as C
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent


def run(task: str, inputs: dict, timeout: float = 600.0) -> dict:
    with tempfile.TemporaryDirectory() as d:
        fin, fout = Path(d) / "in.npz", Path(d) / "out.npz"
        np.savez(fin, **inputs)
        res = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", task, str(fin), str(fout)], cwd=d,
                             env={**__import__("os").environ, "PYTHONPATH": str(ROOT)}, capture_output=True,
                             text=True, timeout=timeout)
        if res.returncode != 0:
            raise RuntimeError(f"reference task {task} failed: {res.stderr[-3000:]}\n{res.stdout[-3000:]}")
        out = np.load(fout)
        return {k: out[k] for k in out.files}


def _child(task: str, fin: str, fout: str) -> None:
    from oracle.oracle import Ref
    d = np.load(fin)
    dims = int(d["dims"])
    N = [int(v) for v in d["N"]]
    beta, aniso = float(d["beta"]), float(d["aniso"])
    lib = Ref.lib()
    _dp = C.POINTER(C.c_double)
    lib.ref_gpu_start(0)
    lib.ref_gpu_setup(dims, N[0], N[1], N[2], N[3], beta, aniso, int(d.get("metrop", 1)), int(d.get("ovrn", 4)))
    out = {}
    lat = np.ascontiguousarray(d["lat"], dtype=np.float64) if "lat" in d.files else None
    R = (N[0]) // 2
    if task == "measure":
        m = np.zeros(6)
        lib.ref_gpu_measure(lat.ctypes.data_as(_dp), m.ctypes.data_as(_dp))
        out["m"] = m
    elif task == "or_pass":
        o = np.zeros_like(lat)
        lib.ref_gpu_update(lat.ctypes.data_as(_dp), o.ctypes.data_as(_dp), 0, int(d["passes"]), 0, 1, 1234)
        out["lat"] = o
    elif task == "poly2":
        for mh in (0, 1):
            c = np.zeros(2 * R)
            lib.ref_gpu_poly2(lat.ctypes.data_as(_dp), mh, c.ctypes.data_as(_dp))
            out[f"c{mh}"] = c
    elif task == "multilevel":
        c = np.zeros(2 * R)
        a = [int(v) for v in d["args"]]  # n4, k4, n2, k2, metrop, ovrn
        lib.ref_gpu_multilevel(lat.ctypes.data_as(_dp), *a, 1234, c.ctypes.data_as(_dp))
        out["c"] = c
    elif task == "multilevel_timing":
        import time
        c = np.zeros(2 * R)
        a = [int(v) for v in d["args"]]  # n4, k4, n2, k2, metrop, ovrn
        # first call: the reference tunes its kernels on first use
        lib.ref_gpu_multilevel(lat.ctypes.data_as(_dp), 1, a[1], 2, a[3], a[4], a[5], 1234, c.ctypes.data_as(_dp))
        t0 = time.perf_counter()
        lib.ref_gpu_multilevel(lat.ctypes.data_as(_dp), *a, 1234, c.ctypes.data_as(_dp))
        out["s"] = np.array([time.perf_counter() - t0])
        out["c"] = c
    elif task == "chain":
        n = int(d["sweeps"])
        o = np.zeros(6 * n)
        lib.ref_gpu_chain(lat.ctypes.data_as(_dp), int(d["metrop"]), int(d["ovrn"]), n, int(d.get("seed", 1234)),
                          o.ctypes.data_as(_dp))
        out["obs"] = o.reshape(n, 6)
    elif task == "convert":
        # only EO -> NO: the reference's NO -> EO kernel writes past the end of
        # its output (src/convertOrder.cu:49-58), so it is never run
        if int(d["eo_to_no"]) != 1:
            raise SystemExit("convert: only eo_to_no = 1 (the reference's NO -> EO direction writes out of bounds)")
        o = np.zeros_like(lat)
        lib.ref_gpu_convert(lat.ctypes.data_as(_dp), int(d["eo_to_no"]), o.ctypes.data_as(_dp))
        out["lat"] = o
    elif task == "plaq_fields":
        st = int(d["spacetime"])
        V = int(np.prod([n for n in N if n > 0]))
        size = V if st else V // N[3]
        f = np.zeros(12 * size)
        m = np.zeros(12)
        lib.ref_gpu_plaq_fields(lat.ctypes.data_as(_dp), st, f.ctypes.data_as(_dp), m.ctypes.data_as(_dp))
        out["field"] = (f[0::2] + 1j * f[1::2]).reshape(6, size)
        out["means"] = m[0::2] + 1j * m[1::2]
    elif task == "timing":
        warm, n = int(d["warmup"]), int(d["sweeps"])
        ms = lib.ref_gpu_update(lat.ctypes.data_as(_dp), None, int(d["metrop"]), int(d["ovrn"]), warm, n, 1234)
        out["ms"] = np.array([ms])
    else:
        raise SystemExit(f"unknown task {task}")
    np.savez(fout, **out)


if __name__ == "__main__":
    _child(sys.argv[1], sys.argv[2], sys.argv[3])
