"""GPU parity of the sm_100a kernels (through the C ABI) against the FP64
oracle, the golden fixtures made by the reference, and exact 2D results.

Tolerances (FP32 links vs FP64 oracle):
  * link angles after 1-5 passes: <= 1e-5 rad, wrap-aware;
  * plaquette / Polyakov means:   <= 2e-6 absolute;
  * Philox uniforms and the hot-start counters: bit-exact.
"""
import numpy as np
import pytest

from latticeu1_b200 import Lattice, Rng, U1Error
from oracle.oracle import Oracle, wrap_diff
from tests.conftest import GOLDEN_NAMES, load_golden

pytestmark = pytest.mark.gpu

ANGLE_TOL = 1e-5


def _pair(ctx, dims, N, beta, aniso=1.0):
    return Lattice(ctx, dims, N, beta, aniso), Oracle(dims, N, beta, aniso)


def _from_golden(ctx, d):
    N = [int(v) for v in d["N"]]
    return _pair(ctx, int(d["dims"]), N, float(d["beta"]), float(d["aniso"]))


def test_import_export_roundtrip(ctx):
    lat, o = _pair(ctx, 4, (6, 4, 8, 4), 1.0)
    th = np.random.default_rng(0).uniform(0, 2 * np.pi, lat.nlinks)
    lat.import_angles(th)
    back = lat.export_angles()
    assert wrap_diff(back, th).max() < 2e-7
    assert back.min() >= 0.0 and back.max() < 2 * np.pi + 1e-12


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_overrelax_golden(ctx, name):
    """One overrelaxation pass vs the reference's own CPU result."""
    d = load_golden(name)
    lat, _ = _from_golden(ctx, d)
    lat.import_angles(d["lat0"])
    rng = Rng(ctx, 1)
    lat.update(rng, 0, 1)
    assert wrap_diff(lat.export_angles(), d["after_or"]).max() < ANGLE_TOL


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_metropolis_shared_stream_golden(ctx, name):
    """One Metropolis pass fed the reference's recorded (theta', b) stream."""
    d = load_golden(name)
    lat, _ = _from_golden(ctx, d)
    lat.import_angles(d["lat0"])
    rng = Rng(ctx, 1)
    rng.set_replay(d["pairs"])
    lat.update(rng, 1, 0)
    diff = wrap_diff(lat.export_angles(), d["after_met"])
    assert diff.max() < ANGLE_TOL, f"{(diff > ANGLE_TOL).sum()} links differ (accept flips)"


@pytest.mark.parametrize("dims,N,beta,aniso", [(4, (8, 8, 8, 8), 1.0, 1.0), (4, (4, 6, 6, 8), 1.1, 2.0),
                                                (3, (8, 6, 0, 8), 2.0, 1.5), (2, (16, 0, 0, 16), 4.0, 1.0)])
@pytest.mark.parametrize("sweeps", [1, 3, 5])
def test_sweeps_shared_stream_vs_oracle(ctx, dims, N, beta, aniso, sweeps):
    """1-5 sweeps of 1 Metropolis + 4 OR with a shared stream reproduce the
    FP64 oracle link by link within 1e-5 rad."""
    lat, o = _pair(ctx, dims, N, beta, aniso)
    rs = np.random.default_rng(sweeps)
    th = rs.uniform(0, 2 * np.pi, lat.nlinks)
    pairs = np.stack([rs.uniform(0, 2 * np.pi, (sweeps, lat.nlinks)), rs.uniform(0, 1, (sweeps, lat.nlinks))], -1)
    lat.import_angles(th)
    rng = Rng(ctx, 1)
    rng.set_replay(pairs)
    ref = th.copy()
    for s in range(sweeps):
        lat.update(rng, 1, 4)
        o.metropolis_pairs(ref, pairs[s].reshape(-1))
        for _ in range(4):
            o.overrelax(ref)
    diff = wrap_diff(lat.export_angles(), ref)
    assert np.quantile(diff, 0.999) < ANGLE_TOL and diff.max() < 1e-3, (diff.max(), (diff > ANGLE_TOL).sum())


def test_philox_uniforms_bit_exact(ctx):
    lat, o = _pair(ctx, 4, (4, 6, 8, 4), 1.0)
    rng = Rng(ctx, 0x1234_5678_9ABC)
    for pass_, p, mu in [(0, 0, 0), (7, 1, 3), (2 ** 33 + 5, 0, 2)]:
        gpu = rng.debug_uniforms(lat, pass_, p, mu)
        cpu = o.philox_uniforms(0x1234_5678_9ABC, pass_, p, mu)
        np.testing.assert_array_equal(gpu, cpu)


def test_hot_start_counters(ctx):
    lat, o = _pair(ctx, 4, (4, 6, 8, 4), 1.0)
    rng = Rng(ctx, 77)
    lat.hot_start(rng)
    assert rng.state == (77, 1)
    want = o.hot_start(77, pass_=0)
    assert wrap_diff(lat.export_angles(), want).max() < 2e-6


@pytest.mark.parametrize("dims,N,beta", [(4, (8, 8, 8, 8), 1.0), (4, (6, 4, 4, 12), 0.9), (3, (8, 6, 0, 8), 2.0)])
def test_philox_chain_vs_oracle(ctx, dims, N, beta):
    """Production (Philox) Metropolis + OR: GPU and oracle draw the same numbers."""
    lat, o = _pair(ctx, dims, N, beta)
    rng = Rng(ctx, 2024)
    lat.hot_start(rng)
    ref = o.hot_start(2024, 0)
    p = 1
    for _ in range(3):
        lat.update(rng, 1, 4)
        p = o.update_philox(ref, 2024, p, 1, 4)
    assert rng.state[1] == p
    diff = wrap_diff(lat.export_angles(), ref)
    assert np.quantile(diff, 0.999) < ANGLE_TOL, diff.max()


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_measure_golden(ctx, name):
    d = load_golden(name)
    lat, o = _from_golden(ctx, d)
    lat.import_angles(d["lat0"])
    m = lat.measure()
    ss, st = o.plaquette(d["lat0"])
    if int(d["dims"]) == 2:
        assert np.isnan(m["plaq_ss"].real)
    else:
        assert abs(m["plaq_ss"] - ss) < 2e-6
    assert abs(m["plaq_st"] - st) < 2e-6
    assert abs(m["poly"] - d["poly"][0]) < 2e-6
    assert lat.plaquette()[1] == m["plaq_st"] and lat.polyakov() == m["poly"]


def test_measure_deterministic_and_large(ctx):
    lat, o = _pair(ctx, 4, (16, 16, 16, 16), 1.0)
    th = np.random.default_rng(3).uniform(0, 2 * np.pi, lat.nlinks)
    lat.import_angles(th)
    a, b = lat.measure(), lat.measure()
    assert a == b
    ss, st = o.plaquette(th)
    assert abs(a["plaq_ss"] - ss) < 2e-6 and abs(a["plaq_st"] - st) < 2e-6
    assert abs(a["poly"] - o.polyakov(th)) < 2e-6


@pytest.mark.parametrize("multihit", [False, True])
@pytest.mark.parametrize("dims,N,beta,aniso", [(4, (8, 6, 6, 8), 1.0, 1.0), (4, (6, 6, 6, 4), 0.8, 2.0),
                                                (3, (8, 6, 0, 6), 2.0, 1.0), (2, (12, 0, 0, 8), 3.0, 1.0)])
def test_poly_corr_vs_oracle(ctx, dims, N, beta, aniso, multihit):
    lat, o = _pair(ctx, dims, N, beta, aniso)
    th = np.random.default_rng(9).uniform(0, 2 * np.pi, lat.nlinks) * 0.3  # smoother field: larger P
    lat.import_angles(th)
    got = lat.poly_corr(multihit)
    want = o.poly_corr(th, multihit)
    scale = np.abs(want).max()
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-5 * scale + 1e-300)


def test_multilevel_vs_oracle_or_only(ctx):
    """metrop = 0 makes the multilevel estimator deterministic: compare with FP64."""
    lat, o = _pair(ctx, 4, (4, 4, 4, 8), 1.2)
    th = np.random.default_rng(4).uniform(0, 2 * np.pi, lat.nlinks) * 0.4
    lat.import_angles(th)
    rng = Rng(ctx, 5)
    got = lat.multilevel(rng, 2, 1, 3, 1, 0, 2)
    want, _ = o.multilevel(th, 5, 0, 2, 1, 3, 1, 0, 2)
    np.testing.assert_allclose(got, want, rtol=2e-4, atol=1e-12 * np.abs(want).max())
    # the caller's lattice is untouched
    assert wrap_diff(lat.export_angles(), th).max() < 2e-7


def test_multilevel_vs_oracle_with_metropolis(ctx):
    lat, o = _pair(ctx, 4, (4, 4, 4, 8), 1.0)
    th = np.random.default_rng(6).uniform(0, 2 * np.pi, lat.nlinks)
    lat.import_angles(th)
    rng = Rng(ctx, 8)
    got = lat.multilevel(rng, 2, 1, 2, 1, 1, 2)
    want, pass_end = o.multilevel(th, 8, 0, 2, 1, 2, 1, 1, 2)
    assert rng.state[1] == pass_end
    np.testing.assert_allclose(got, want, rtol=2e-3, atol=1e-10 * np.abs(want).max())


def exact_2d_plaquette(beta, V):
    from scipy import special
    n = np.arange(-30, 31)
    In = special.iv(n, beta)
    num = np.sum(In ** (V - 1) * 0.5 * (special.iv(n - 1, beta) + special.iv(n + 1, beta)))
    return float(num / np.sum(In ** V))


@pytest.mark.parametrize("L,beta", [(16, 2.0), (32, 4.0), (32, 6.0)])
def test_2d_exact_plaquette(ctx, L, beta):
    lat = Lattice(ctx, 2, (L, 0, 0, L), beta)
    rng = Rng(ctx, 31 + L)
    lat.hot_start(rng)
    vals = []
    for s in range(3000):
        lat.update(rng, 1, 2)
        if s >= 500:
            vals.append(1.0 - lat.plaquette()[1].real)
    x = np.asarray(vals).reshape(25, -1).mean(axis=1)
    m, e = x.mean(), x.std(ddof=1) / 5.0
    ex = exact_2d_plaquette(beta, L * L)
    assert abs(m - ex) < 4 * e + 2e-5, (m, e, ex)


def test_errors_are_status_codes(ctx):
    with pytest.raises(U1Error) as ei:
        Lattice(ctx, 4, (8, 7, 8, 8), 1.0)
    assert ei.value.code == -1
    lat = Lattice(ctx, 4, (4, 4, 4, 6), 1.0)
    with pytest.raises(U1Error) as ei:
        lat.multilevel(Rng(ctx, 1), 1, 1, 1, 1, 1, 1)
    assert "multiple of 4" in str(ei.value)
    rng = Rng(ctx, 1)
    rng.set_replay(np.zeros((1, lat.nlinks, 2)))
    lat.update(rng, 1, 0)
    with pytest.raises(U1Error) as ei:
        lat.update(rng, 1, 0)
    assert ei.value.code == -5
