"""Pin the FP64 oracle (oracle/u1_oracle.cpp) before trusting it.

1. Golden fixtures produced by the reference's own code (tests/golden/).
2. The reference's own CPU functions run live (oracle/_ref, when built).
3. Known answers: Philox4x32-10 test vectors published with Random123
   (Salmon et al., SC'11), Bessel ratios from scipy, the exact 2D plaquette.
"""
import numpy as np
import pytest
from scipy import special

from oracle.oracle import Oracle, Ref
from tests.conftest import GOLDEN_NAMES, load_golden


def _oracle_for(d):
    return Oracle(int(d["dims"]), [int(v) for v in d["N"]], float(d["beta"]), float(d["aniso"]))


def test_philox_known_answers():
    # Random123 kat_vectors, philox4x32_10
    assert Oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert Oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert Oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_golden_indexing_bit_exact(name):
    d = load_golden(name)
    o = _oracle_for(d)
    dims = o.dims
    for p in (0, 1):
        for i in range(o.Vh):
            assert o.index_eo(i, p) == list(d["coords"][p, i])
            for mu in range(dims):
                assert o.index_eo_neg(i, p, mu, -1) == d["nbr"][p, i, mu, 0]
                assert o.index_eo_neg(i, p, mu, 1) == d["nbr"][p, i, mu, 1]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_golden_staple_and_updates(name):
    d = load_golden(name)
    o = _oracle_for(d)
    lat0 = d["lat0"].copy()
    st = np.array([[[o.staple(lat0, i, p, mu) for i in range(o.Vh)] for mu in range(o.dims)] for p in (0, 1)])
    np.testing.assert_array_equal(st, d["staple"])
    l = lat0.copy()
    o.overrelax(l)
    np.testing.assert_array_equal(l, d["after_or"])
    l = lat0.copy()
    o.metropolis_pairs(l, d["pairs"].reshape(-1))
    np.testing.assert_array_equal(l, d["after_met"])


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_golden_measurements(name):
    d = load_golden(name)
    o = _oracle_for(d)
    lat0 = d["lat0"]
    ss, st = o.plaquette(lat0)
    dims = o.dims
    nss = (dims - 1) * (dims - 2) // 2
    nst = dims - 1
    # the reference CPU plaquette returns <cos P>, <sin P> over all plaquettes
    ss_re = 0.0 if nss == 0 else ss.real
    ss_im = 0.0 if nss == 0 else ss.imag
    mean_cos = 1.0 - (nss * ss_re + nst * st.real) / (nss + nst)
    mean_sin = -(nss * ss_im + nst * st.imag) / (nss + nst)
    assert abs(mean_cos - d["plaq_cos_sin"][0]) < 1e-13
    assert abs(mean_sin - d["plaq_cos_sin"][1]) < 1e-13
    if nss == 0:
        assert np.isnan(ss.real)  # reference normalises SS by 1/(V*0)
    assert abs(o.polyakov(lat0) - d["poly"][0]) < 1e-13
    if "multihit" in d:
        mh = np.array([[o.multihit(lat0, i, p) for i in range(o.Vh)] for p in (0, 1)])
        np.testing.assert_allclose(mh, d["multihit"], rtol=1e-12, atol=1e-15)


@pytest.mark.skipif(not Ref.available(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("dims,N,beta,aniso", [(4, (4, 4, 6, 8), 0.9, 1.3), (3, (4, 6, 0, 4), 1.7, 1.0),
                                                (2, (6, 0, 0, 10), 3.0, 1.0)])
def test_live_reference_cpu(dims, N, beta, aniso):
    """Oracle vs the reference's own FP64 CPU functions over several sweeps."""
    o, r = Oracle(dims, N, beta, aniso), Ref(dims, N, beta, aniso)
    rng = np.random.default_rng(5)
    lat_o = rng.uniform(0, 2 * np.pi, o.nlinks)
    lat_r = lat_o.copy()
    pairs = r.record_pairs(99, 3)
    r.seed_cpu(1, 99)
    for s in range(3):
        o.metropolis_pairs(lat_o, pairs[s].reshape(-1))
        r.metropolis(lat_r)
        for _ in range(2):
            o.overrelax(lat_o)
            r.overrelax(lat_r)
    np.testing.assert_array_equal(lat_o, lat_r)
    assert abs(o.polyakov(lat_o) - r.polyakov(lat_r)) < 1e-13
    for p in (0, 1):
        for i in range(0, o.Vh, 7):
            if dims == 4:
                assert abs(o.multihit(lat_o, i, p) - r.multihit(lat_r, i, p)) < 1e-14


@pytest.mark.parametrize("d", [1, 2, 3, 5, 6, 7, 12, 16, 24, 31, 48, 100, 1000, 65535, 123457, 2 ** 20 + 1])
def test_fast_division_used_by_kernels(d):
    rs = np.random.default_rng(d)
    ns = np.concatenate([np.arange(0, 5000), rs.integers(0, 2 ** 31, 5000), [2 ** 31 - 1, 2 ** 31 - 2]])
    for n in ns:
        assert Oracle.fastdiv(int(n), d) == int(n) // d


@pytest.mark.parametrize("x", [1e-4, 0.3, 1.0, 2.5, 6.0, 12.0, 24.0])
def test_bessel_ratio(x):
    assert abs(Oracle.bessel_ratio(x) - special.iv(1, x) / special.iv(0, x)) < 1e-13


def exact_2d_plaquette(beta: float, V: int) -> float:
    """<cos theta_P> on a periodic 2D lattice of V plaquettes:
    sum_n I_n^{V-1} (I_{n-1}+I_{n+1})/2 / sum_n I_n^V (all at beta), with every
    I_n divided by I_0 so the powers stay finite."""
    n = np.arange(-40, 41)
    r = special.ive(n, beta) / special.ive(0, beta)
    rm = special.ive(n - 1, beta) / special.ive(0, beta)
    rp = special.ive(n + 1, beta) / special.ive(0, beta)
    return float(np.sum(r ** (V - 1) * 0.5 * (rm + rp)) / np.sum(r ** V))


def test_exact_2d_plaquette_large_volume_limit():
    for beta in (2.0, 4.0, 6.0):
        assert abs(exact_2d_plaquette(beta, 1024) - special.iv(1, beta) / special.iv(0, beta)) < 1e-10


def binned_mean_err(x, nbins=20):
    x = np.asarray(x)
    b = x[: len(x) // nbins * nbins].reshape(nbins, -1).mean(axis=1)
    return b.mean(), b.std(ddof=1) / np.sqrt(nbins)


def test_oracle_2d_exact_plaquette():
    """Oracle Philox chain on 2D 16x16 at beta=2 reproduces the exact plaquette."""
    beta = 2.0
    o = Oracle(2, (16, 0, 0, 16), beta)
    lat = o.hot_start(seed=3)
    p = 1
    vals = []
    for sweep in range(1500):
        p = o.update_philox(lat, 3, p, 1, 2)
        if sweep >= 200:
            _, st = o.plaquette(lat)
            vals.append(1.0 - st.real)
    m, e = binned_mean_err(vals)
    exact = exact_2d_plaquette(beta, 256)
    assert abs(m - exact) < 4 * e + 1e-4, (m, e, exact)
