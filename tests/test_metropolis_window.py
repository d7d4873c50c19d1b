"""Windowed multi-hit Metropolis (u1_lattice_set_metropolis): hit h proposes
theta' = theta + delta (2u - 1) (theta' = 2 pi u for delta = 0) with the
staple held fixed.  The reference has one whole-circle proposal per link and
pass (src/update.cu:181-182); that stays the default and the parity runs use
it, while this mode is checked separately against the FP64 oracle:

  * CPU: the oracle's windowed chains reproduce the exact 2D plaquette, and
    delta = 0 with one hit is the reference proposal bit for bit;
  * GPU: every Metropolis phase against the oracle drawing the same Philox
    numbers (links within 1e-6 rad, accept flips only at the FP32 decision
    margin), all kernel variants and graphs bit-identical, and the 8^4
    beta = 1 cold-start chain (delta = pi/2, 1 hit + 4 OR, 1000 sweeps)
    against the oracle's chain within statistical errors.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from tests.test_gpu_core import check_phase, exact_2d_plaquette

HALF_PI = np.pi / 2


def _binned(x, nbins):
    x = np.asarray(x)[: len(x) // nbins * nbins].reshape(nbins, -1).mean(axis=1)
    return x.mean(), x.std(ddof=1) / np.sqrt(nbins)


def test_oracle_delta0_single_hit_is_reference_proposal():
    o = Oracle(4, (6, 4, 4, 8), 1.1)
    lat = o.hot_start(3)
    a, b = lat.copy(), lat.copy()
    o.metropolis_philox(a, 3, 1)
    o.metropolis_hits(b, 3, 1, 0.0, 1)
    np.testing.assert_array_equal(a, b)
    c = lat.copy()
    o.metropolis_hits(c, 3, 1, 0.0, 2)  # a second hit draws new numbers
    assert not np.array_equal(a, c)


@pytest.mark.parametrize("L,beta,delta,nhits", [(16, 2.0, HALF_PI, 1), (16, 2.0, 1.0, 3), (16, 4.0, np.pi / 4, 2)])
def test_oracle_window_chain_exact_2d(L, beta, delta, nhits):
    """Pure windowed Metropolis (no OR) samples the Wilson action: the 2D
    plaquette equals the exact finite-volume Bessel result."""
    o = Oracle(2, (L, 0, 0, L), beta)
    lat = o.hot_start(7)
    vals = []
    for s in range(3000):
        o.metropolis_hits(lat, 7, s + 1, delta, nhits)
        if s >= 300:
            vals.append(1.0 - o.plaquette(lat)[1].real)
    m, e = _binned(vals, 27)
    ex = exact_2d_plaquette(beta, L * L)
    assert abs(m - ex) < 4 * e + 2e-5, (m, e, ex)


# ------------------------------------------------------------------ GPU
@pytest.mark.gpu
@pytest.mark.parametrize("dims,N,beta,aniso,delta,nhits", [
    (4, (8, 8, 8, 8), 1.0, 1.0, HALF_PI, 1),
    (4, (4, 6, 6, 8), 1.1, 2.0, HALF_PI, 3),
    (4, (6, 6, 4, 8), 1.0, 1.0, 1.0, 2),      # N0/2 odd: one-site kernel
    (3, (8, 6, 0, 8), 2.0, 1.5, np.pi / 4, 2),
    (2, (16, 0, 0, 16), 4.0, 1.0, HALF_PI, 1),
    (2, (14, 0, 0, 10), 3.0, 1.0, 0.0, 3),    # whole-circle multi-hit
])
def test_window_phases_vs_oracle(ctx, dims, N, beta, aniso, delta, nhits):
    """Every Metropolis phase of 3 sweeps (and the OR phases between them),
    each from the GPU's own configuration, against the FP64 oracle drawing
    the same Philox numbers for every hit."""
    from latticeu1_b200 import Lattice, Rng
    lat, o = Lattice(ctx, dims, N, beta, aniso), Oracle(dims, N, beta, aniso)
    lat.set_metropolis(delta, nhits)
    assert lat.metropolis == (pytest.approx(delta), nhits)
    rng = Rng(ctx, 4242)
    lat.hot_start(rng)
    for _ in range(20):
        lat.update(rng, 1, 2)
    flips = 0
    for _ in range(3):
        seed, p0 = rng.state
        for p in (0, 1):
            for mu in range(dims):
                flips += check_phase(lat, o, rng, True, p, mu, seed=seed, pass_=p0, delta=delta, nhits=nhits)[0]
        rng.set_state(seed, p0 + 1)
        for p in (0, 1):
            for mu in range(dims):
                check_phase(lat, o, rng, False, p, mu)
    assert flips <= 2 * nhits, flips


@pytest.mark.gpu
def test_window_variants_graphs_and_fused_measurement_bit_identical(ctx):
    """Windowed sweeps: kernel variants, graph vs direct launches and the
    measured sweep (last pass Metropolis, so it runs the windowed measuring
    kernels) give bit-identical links."""
    import torch
    from latticeu1_b200 import Lattice, Rng
    geom = (4, (8, 8, 8, 8), 1.0)
    ref = None
    for variant, graphs in [(1, True), (2, True), (3, True), (5, True), (1, False)]:
        lat = Lattice(ctx, *geom)
        lat.set_variant(variant)
        lat.set_graphs(graphs)
        lat.set_metropolis(HALF_PI, 2)
        rng = Rng(ctx, 99)
        lat.hot_start(rng)
        for _ in range(3):
            lat.update(rng, 2, 1)
        lat.update(rng, 1, 0)
        got = lat.export_angles()
        if ref is None:
            ref = got
        np.testing.assert_array_equal(got, ref)
    a, b = Lattice(ctx, *geom), Lattice(ctx, *geom)
    for x in (a, b):
        x.set_metropolis(1.0, 3)
    ra, rb = Rng(ctx, 5), Rng(ctx, 5)
    a.hot_start(ra)
    b.hot_start(rb)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    for metrop, ovrn in [(1, 0), (2, 0), (1, 2)]:
        a.update_measure(ra, metrop, ovrn, out.data_ptr())
        b.update(rb, metrop, ovrn)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(a.export_angles(), b.export_angles())
        want, got = b.measure(), out.cpu().numpy()
        assert abs(complex(got[0], got[1]) - want["plaq_ss"]) < 2e-6
        assert abs(complex(got[2], got[3]) - want["plaq_st"]) < 2e-6
        assert abs(complex(got[4], got[5]) - want["poly"]) < 2e-6
    # the whole-circle single hit is the default path: same links as never setting it
    c, d = Lattice(ctx, *geom), Lattice(ctx, *geom)
    c.set_metropolis(0.0, 1)
    rc, rd = Rng(ctx, 6), Rng(ctx, 6)
    c.hot_start(rc)
    d.hot_start(rd)
    c.update(rc, 1, 1)
    d.update(rd, 1, 1)
    np.testing.assert_array_equal(c.export_angles(), d.export_angles())


@pytest.mark.gpu
def test_window_argument_errors(ctx):
    from latticeu1_b200 import Lattice, U1Error
    lat = Lattice(ctx, 4, (4, 4, 4, 4), 1.0)
    for delta, nhits in [(-0.1, 1), (3.2, 1), (float("nan"), 1), (1.0, 0), (1.0, 128)]:
        with pytest.raises(U1Error):
            lat.set_metropolis(delta, nhits)
    assert lat.metropolis == (0.0, 1)


@pytest.mark.gpu
def test_cold_start_8x4_window_chain_vs_oracle(ctx):
    """8^4, beta = 1.0, cold start, per sweep 1 Metropolis (delta = pi/2,
    1 hit) + 4 OR, plaquettes and Polyakov loop measured every sweep, 1000
    sweeps: the GPU chain and the FP64 oracle chain (same Philox seed; they
    decorrelate within a few sweeps) agree within statistical errors."""
    import torch
    from latticeu1_b200 import Lattice, Rng
    N, beta, seed, nsw, therm = (8, 8, 8, 8), 1.0, 1234, 1000, 200
    lat = Lattice(ctx, 4, N, beta)
    lat.set_metropolis(HALF_PI, 1)
    rng = Rng(ctx, seed)
    lat.cold_start()
    out = torch.zeros((nsw, 6), dtype=torch.float64, device="cuda")
    for s in range(nsw):
        lat.update_measure(rng, 1, 4, out[s].data_ptr())
    g = out.cpu().numpy()[therm:]
    o = Oracle(4, N, beta)
    th = np.zeros(o.nlinks)
    ref = []
    pass_ = 0
    for s in range(nsw):
        pass_ = o.update_philox(th, seed, pass_, 1, 4, delta=HALF_PI, nhits=1)
        if s >= therm:
            ss, st = o.plaquette(th)
            ref.append((1.0 - ss.real, 1.0 - st.real, abs(o.polyakov(th))))
    ref = np.asarray(ref)
    for k, col in enumerate((0, 2)):  # 1 - Re P = <cos theta_P>
        mg, eg = _binned(1.0 - g[:, col], 20)
        mo, eo = _binned(ref[:, k], 20)
        assert abs(mg - mo) < 4 * np.hypot(eg, eo) + 1e-5, (k, mg, eg, mo, eo)
    lg, elg = _binned(np.hypot(g[:, 4], g[:, 5]), 10)
    lo, elo = _binned(ref[:, 2], 10)
    assert abs(lg - lo) < 5 * np.hypot(elg, elo) + 1e-3, (lg, elg, lo, elo)
