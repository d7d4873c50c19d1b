"""The reference's OWN CUDA build (compiled in place into oracle/_ref) run on
the same B200 as the sm_100a kernels: results on identical configurations,
and throughput of its UpdateLattice on the 32^4 workload.

Deterministic comparisons (no RNG involved): the fused measurement, one
overrelaxation pass, Poly2 (plain and multihit), MultiLevel with no
updates (metrop = ovrn = 0), which pins the multilevel tensor contraction
to the reference implementation itself, and the format kernels
(LatticeConvert, src/convertOrder.cu:32-63,135-145; PlaquetteFields,
src/plaquette_comps.cu:34-107,216-227).
"""
import json
import os
import time

import numpy as np
import pytest

from oracle.oracle import Oracle, Ref, wrap_diff

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not Ref.available(), reason="oracle/_ref not built (reference sources absent)")]


def _inputs(dims, N, beta, aniso, lat, **kw):
    return dict(dims=dims, N=np.array(list(N) + [0] * (4 - len(N))), beta=beta, aniso=aniso, lat=lat, **kw)


@pytest.fixture(scope="module")
def ref_gpu():
    from oracle import ref_gpu
    return ref_gpu


@pytest.mark.parametrize("dims,N,beta,aniso", [(4, (8, 6, 6, 8), 1.0, 1.0), (4, (6, 6, 6, 8), 0.9, 2.0),
                                                (3, (8, 8, 0, 6), 2.0, 1.0)])
def test_measure_or_poly2_vs_reference_cuda(ctx, ref_gpu, dims, N, beta, aniso):
    from latticeu1_b200 import Lattice, Rng
    lat = Lattice(ctx, dims, N, beta, aniso)
    o = Oracle(dims, N, beta, aniso)
    th = np.random.default_rng(dims).uniform(0, 2 * np.pi, lat.nlinks) * 0.5
    lat.import_angles(th)
    th = lat.export_angles()  # exactly the configuration the GPU holds
    r = ref_gpu.run("measure", _inputs(dims, N, beta, aniso, th))["m"]
    m = lat.measure()
    got = np.array([m["plaq_ss"].real, m["plaq_ss"].imag, m["plaq_st"].real, m["plaq_st"].imag, m["poly"].real,
                    m["poly"].imag])
    if dims == 2:
        got, r = got[2:], r[2:]
    np.testing.assert_allclose(got, r, rtol=0, atol=2e-6)
    ref_or = ref_gpu.run("or_pass", _inputs(dims, N, beta, aniso, th, passes=1))["lat"]
    lat.update(Rng(ctx, 1), 0, 1)
    diff = wrap_diff(lat.export_angles(), ref_or)
    # whole pass: same bound as the golden pass (ill-conditioned links with
    # tiny |S| spread their FP32 error to links updated later in the pass)
    assert np.median(diff) < 1e-6 and np.mean(diff < 1e-5) > 0.95 and diff.max() < 5e-3, (diff.max(),
                                                                                           np.mean(diff < 1e-5))
    lat.import_angles(th)
    c = ref_gpu.run("poly2", _inputs(dims, N, beta, aniso, th))
    for mh in (0, 1):
        want = c[f"c{mh}"][0::2] + 1j * c[f"c{mh}"][1::2]
        got = lat.poly_corr(bool(mh))
        np.testing.assert_allclose(got, want, rtol=0, atol=3e-5 * np.abs(want).max())


@pytest.mark.parametrize("dims,N", [(4, (8, 6, 4, 10)), (3, (6, 8, 0, 4)), (2, (10, 0, 0, 6))])
def test_convert_order_vs_reference_cuda(ctx, ref_gpu, dims, N):
    """u1_convert_order EO -> NO against the reference's LatticeConvert(lat,
    true), bit for bit (a permutation of FP64 angles); NO -> EO is its exact
    inverse.  The reference's NO -> EO direction is not run: it writes
    out[id + parity V/2 + dir V] with the natural-order index id < V
    (src/convertOrder.cu:49-58), a wrong permutation that runs past the end of
    the output array by up to V/2 elements."""
    import torch
    from latticeu1_b200.lattice import convert_order
    n = int(np.prod([v for v in N if v > 0])) * dims
    th = np.random.default_rng(11 + dims).uniform(0, 2 * np.pi, n)
    want_no = ref_gpu.run("convert", _inputs(dims, N, 1.0, 1.0, th, eo_to_no=1))["lat"]
    t = torch.tensor(th, dtype=torch.float64, device="cuda")
    got_no = convert_order(t, dims, N, eo_to_no=True)
    assert np.array_equal(got_no.cpu().numpy(), want_no)
    back = convert_order(torch.tensor(want_no, dtype=torch.float64, device="cuda"), dims, N, eo_to_no=False)
    assert torch.equal(back, t)


@pytest.mark.parametrize("spacetime", [True, False])
def test_plaquette_fields_vs_reference_cuda(ctx, ref_gpu, spacetime):
    """u1_plaquette_fields against the reference's PlaquetteFields
    (evenoddOrder = true: the lattice in the EO layout, fields in natural
    site order), per site and time-averaged per spatial site: every
    component within 1e-6 (FP32 links against FP64 angles) and the six
    component means within 1e-6."""
    from latticeu1_b200 import Lattice, Rng
    N = (8, 6, 4, 10)
    lat = Lattice(ctx, 4, N, 1.0)
    rng = Rng(ctx, 6)
    lat.hot_start(rng)
    lat.update(rng, 1, 3)
    th = lat.export_angles()
    r = ref_gpu.run("plaq_fields", _inputs(4, N, 1.0, 1.0, th, spacetime=int(spacetime)))
    f, m = lat.plaquette_fields(spacetime=spacetime)
    f = f.cpu().numpy()
    assert f.shape == r["field"].shape
    assert np.abs(f - r["field"]).max() < 1e-6
    assert np.abs(m - r["means"]).max() < 1e-6


def _jackknife_mean(x, nbins=25):
    """Mean and jackknife error over nbins consecutive bins (binning absorbs
    the autocorrelation when a bin is much longer than tau_int)."""
    x = np.asarray(x, dtype=np.float64)
    b = x[: len(x) // nbins * nbins].reshape(nbins, -1).mean(axis=1)
    loo = (b.sum() - b) / (nbins - 1)
    return b.mean(), np.sqrt((nbins - 1) / nbins * np.sum((loo - loo.mean()) ** 2))


@pytest.mark.parametrize("dims,N,beta,aniso,start", [(4, (8, 8, 8, 8), 0.9, 1.0, "hot"),
                                                      (4, (8, 8, 8, 8), 1.1, 1.0, "cold"),
                                                      (4, (6, 6, 6, 12), 2.0, 2.0, "cold"),
                                                      (2, (16, 0, 0, 16), 4.0, 1.0, "hot")])
def test_long_run_statistics_vs_reference_cuda_and_oracle(ctx, ref_gpu, dims, N, beta, aniso, start):
    """Long runs (2500 sweeps of 1 Metropolis + 4 OR from the same start
    configuration, the first 250 dropped): <Re P_SS>, <Re P_ST> and <|L|>
    of our chain agree with the reference's own CUDA build (its MRG32k3a
    stream) and with the FP64 oracle's chain (Philox) within 4.5 combined
    jackknife errors.  In the Coulomb phase the chains start cold: from a
    hot start a small lattice can stay for thousands of sweeps in a
    metastable state with a trapped defect (each chain in a different one),
    which shifts the spatial and temporal plaquettes apart."""
    import torch
    from latticeu1_b200 import Lattice, Rng
    nsw, therm = 2500, 250
    lat = Lattice(ctx, dims, N, beta, aniso)
    rng = Rng(ctx, 77)
    if start == "hot":
        lat.hot_start(rng)
    else:
        lat.cold_start()
    th0 = lat.export_angles()
    out = torch.zeros((nsw, 6), dtype=torch.float64, device="cuda")
    for s in range(nsw):
        lat.update_measure(rng, 1, 4, out[s].data_ptr())
    ours = out.cpu().numpy()[therm:]
    ref = ref_gpu.run("chain", _inputs(dims, N, beta, aniso, th0, metrop=1, ovrn=4, sweeps=nsw))["obs"][therm:]
    o = Oracle(dims, N, beta, aniso)
    th = th0.copy()
    orc, pass_ = [], 10 ** 6
    for s in range(nsw):
        pass_ = o.update_philox(th, 4242, pass_, 1, 4)
        if s >= therm:
            ss, st = o.plaquette(th)
            lp = o.polyakov(th)
            orc.append((ss.real, ss.imag, st.real, st.imag, lp.real, lp.imag))
    orc = np.asarray(orc)
    cols = ([0] if dims > 2 else []) + [2]
    for name, series in [(f"Re P[{c}]", lambda a, c=c: a[:, c]) for c in cols] + \
                        [("|L|", lambda a: np.hypot(a[:, 4], a[:, 5]))]:
        mo, eo = _jackknife_mean(series(ours))
        for other, arr in (("reference CUDA", ref), ("FP64 oracle", orc)):
            mr, er = _jackknife_mean(series(arr))
            assert abs(mo - mr) < 4.5 * np.hypot(eo, er) + 1e-6, (name, other, mo, eo, mr, er)


def test_multilevel_vs_reference_cuda(ctx, ref_gpu):
    from latticeu1_b200 import Lattice, Rng
    dims, N, beta = 4, (6, 4, 4, 8), 1.1
    lat = Lattice(ctx, dims, N, beta)
    th = np.random.default_rng(3).uniform(0, 2 * np.pi, lat.nlinks) * 0.4
    lat.import_angles(th)
    th = lat.export_angles()
    args = np.array([2, 1, 3, 1, 0, 0])
    c = ref_gpu.run("multilevel", _inputs(dims, N, beta, 1.0, th, args=args))["c"]
    want = c[0::2] + 1j * c[1::2]
    got = lat.multilevel(Rng(ctx, 1), *[int(a) for a in args])
    np.testing.assert_allclose(got, want, rtol=1e-4, atol=1e-6 * np.abs(want).max())


def test_multilevel_statistics_vs_reference_cuda(ctx, ref_gpu):
    """MultiLevel with updates (n4 = 4, k4 = 1, n2 = 10, k2 = 1, 1 Metropolis
    + 2 OR per sub-update) on 10 configurations of one thermalised chain
    (8^3 x 8, beta = 1.1), once by this library and once by the reference's
    own CUDA MultiLevel from the same configuration: the mean C(r) over the
    configurations agree within 4 combined errors (spread over the
    configurations), r = 1..3, and both agree with the single-level multihit
    estimator (Poly2) of the same configurations within its larger error."""
    from latticeu1_b200 import Lattice, Rng
    dims, N, beta = 4, (8, 8, 8, 8), 1.1
    args = [4, 1, 10, 1, 1, 2]
    lat = Lattice(ctx, dims, N, beta)
    rng = Rng(ctx, 21)
    lat.cold_start()
    for _ in range(300):
        lat.update(rng, 1, 4)
    ours, ref, single = [], [], []
    for k in range(10):
        for _ in range(20):
            lat.update(rng, 1, 4)
        th = lat.export_angles()
        ours.append(lat.multilevel(Rng(ctx, 500 + k), *args)[:3].real)
        c = ref_gpu.run("multilevel", _inputs(dims, N, beta, 1.0, th, args=np.array(args)))["c"]
        ref.append(c[0:6:2])
        single.append(lat.poly_corr(True)[:3].real)
    ours, ref, single = np.asarray(ours), np.asarray(ref), np.asarray(single)
    n = len(ours)
    mo, eo = ours.mean(0), ours.std(0, ddof=1) / np.sqrt(n)
    mr, er = ref.mean(0), ref.std(0, ddof=1) / np.sqrt(n)
    ms, es = single.mean(0), single.std(0, ddof=1) / np.sqrt(n)
    assert np.all(mo > 0) and np.all(np.diff(mo) < 0), mo
    assert np.all(np.abs(mo - mr) < 4 * np.hypot(eo, er)), (mo, eo, mr, er)
    assert np.all(np.abs(mo - ms) < 4 * np.hypot(eo, es)), (mo, eo, ms, es)


def test_throughput_vs_reference_cuda(ctx, ref_gpu):
    """UpdateLattice(1 Metropolis + 4 OR) at 32^4 on the same B200: the
    reference's CUDA build (FP64, after its own autotuning in the warm-up)
    against the sm_100a path through the Python host layer."""
    import torch

    from latticeu1_b200 import Lattice, Rng
    L = 32
    sweeps = 20
    lat = Lattice(ctx, 4, (L, L, L, L), 1.0)
    rng = Rng(ctx, 7)
    lat.hot_start(rng)
    th = lat.export_angles()
    r = ref_gpu.run("timing", _inputs(4, (L, L, L, L), 1.0, 1.0, th, warmup=3, sweeps=sweeps, metrop=1, ovrn=4))
    ref_ms = float(r["ms"][0]) / sweeps
    for _ in range(3):
        lat.update(rng, 1, 4)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s = torch.cuda.Stream()
    lat.set_stream(s.cuda_stream)
    with torch.cuda.stream(s):
        lat.update(rng, 1, 4)
        e0.record(s)
        for _ in range(sweeps):
            lat.update(rng, 1, 4)
        e1.record(s)
        s.synchronize()
    ours_ms = e0.elapsed_time(e1) / sweeps
    lu = L ** 4 * 4 * 5
    result = {"workload": "32^4 beta=1 UpdateLattice(1 Metropolis + 4 OR)", "reference_cuda_ms_per_sweep": ref_ms,
              "reference_cuda_link_updates_per_s": lu / (ref_ms * 1e-3), "ours_ms_per_sweep": ours_ms,
              "ours_link_updates_per_s": lu / (ours_ms * 1e-3), "speedup": ref_ms / ours_ms}
    print(json.dumps(result))
    out = os.environ.get("U1_REF_TIMING_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(result, f, indent=1)
    assert ours_ms < ref_ms, result


def test_multilevel_throughput_vs_reference_cuda(ctx, ref_gpu):
    """MultiLevel at 24^3 x 32, beta = 0.95 (n4 = 1, k4 = 1, n2 = 20, k2 = 1,
    1 Metropolis + 4 OR per sub-update): the reference's CUDA build (after a
    first call that tunes its kernels) against u1_multilevel, wall clock of
    one call each on the same B200 and configuration."""
    import torch

    from latticeu1_b200 import Lattice, Rng
    N = (24, 24, 24, 32)
    lat = Lattice(ctx, 4, N, 0.95)
    rng = Rng(ctx, 5)
    lat.hot_start(rng)
    for _ in range(20):
        lat.update(rng, 1, 4)
    th = lat.export_angles()
    args = np.array([1, 1, 20, 1, 1, 4])
    r = ref_gpu.run("multilevel_timing", _inputs(4, N, 0.95, 1.0, th, args=args))
    ref_s = float(r["s"][0])
    lat.multilevel(rng, 1, 1, 2, 1, 1, 4)  # warm-up (graph capture, allocations)
    torch.cuda.synchronize()
    # best of three calls: run after the other tests of this file, a single
    # timed call once took 0.11 s against 0.008 s when the test runs alone
    times = []
    for _ in range(3):
        t0 = time.perf_counter()
        lat.multilevel(rng, *[int(a) for a in args])
        times.append(time.perf_counter() - t0)
    ours_s = min(times)
    assert ours_s < ref_s, times
    result = {"workload": "24^3x32 beta=0.95 MultiLevel(n4=1,k4=1,n2=20,k2=1,metrop=1,ovrn=4)",
              "reference_cuda_s": ref_s, "ours_s": ours_s, "speedup": ref_s / ours_s}
    print(json.dumps(result))
    out = os.environ.get("U1_REF_TIMING_OUT")
    if out:
        d = {}
        if os.path.exists(out):
            with open(out) as f:
                d = json.load(f)
        d["multilevel"] = result
        with open(out, "w") as f:
            json.dump(d, f, indent=1)
