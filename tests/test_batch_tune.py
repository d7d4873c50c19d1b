"""Update-kernel variants, the autotuner and batched chains (GPU).

* every update variant (two sites per thread with and without the register
  cap, one site per thread) gives bit-identical links;
* tuning restores the lattice and the rng pass counter, and caches its pick
  in $U1_RESOURCE_PATH/u1b200_tunecache.tsv;
* chain c of a batch is bit-identical to a single lattice driven by an rng
  with the same seed and chain number first_chain + c, and its measurement
  agrees with the FP64 oracle to 2e-6.
"""
import numpy as np
import pytest

from latticeu1_b200 import Batch, Lattice, Rng, U1Error
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

# (dims, N, beta, aniso); Nx = 6 gives Nx/2 odd (two-site kernels invalid)
VARIANT_GEOMS = [
    (4, (8, 8, 8, 8), 1.0, 1.0),
    (4, (16, 6, 4, 4), 1.05, 1.5),  # N0/2 = 8: quads inside and at the ends of a row
    (4, (12, 8, 4, 6), 0.9, 1.3),
    (4, (6, 4, 4, 8), 1.1, 1.0),
    (3, (8, 8, 0, 12), 1.2, 0.8),
    (2, (16, 0, 0, 8), 2.0, 1.0),
]


def _run(ctx, geom, variant, seed=77, chain=0, sweeps=((1, 4), (2, 0), (0, 3))):
    dims, N, beta, aniso = geom
    lat = Lattice(ctx, dims, N, beta, aniso)
    lat.set_variant(variant)
    rng = Rng(ctx, seed)
    rng.set_chain(chain)
    lat.hot_start(rng)
    for m, o in sweeps:
        lat.update(rng, m, o)
    return lat, rng


@pytest.mark.parametrize("geom", VARIANT_GEOMS, ids=lambda g: f"{g[0]}d-{'x'.join(map(str, g[1]))}")
def test_variants_bit_identical(ctx, geom):
    pair_ok = (geom[1][0] // 2) % 2 == 0
    quad_ok = (geom[1][0] // 2) % 4 == 0
    results = {}
    for v in (1, 2, 3, 5):
        if (not pair_ok and v in (1, 2)) or (not quad_ok and v == 5):
            with pytest.raises(U1Error):
                Lattice(ctx, *geom[:2], geom[2], geom[3]).set_variant(v)
            continue
        lat, _ = _run(ctx, geom, v)
        results[v] = lat.export_angles()
    base = results[3]
    for v, th in results.items():
        assert np.array_equal(th, base), f"variant {v} differs from the one-site kernel"


@pytest.mark.parametrize("geom", VARIANT_GEOMS[:3], ids=lambda g: f"{g[0]}d-{'x'.join(map(str, g[1]))}")
def test_block_sizes_bit_identical(ctx, geom):
    """Every threads-per-block setting of the phase kernels gives the same
    links (the kernels index sites from blockDim; ragged last blocks)."""
    pair_ok = (geom[1][0] // 2) % 2 == 0
    quad_ok = (geom[1][0] // 2) % 4 == 0
    base = _run(ctx, geom, 3)[0].export_angles()
    for v in ((1, 2, 3) if pair_ok else (3,)) + ((5,) if quad_ok else ()):
        for t in (32, 64, 96, 128, 224):
            dims, N, beta, aniso = geom
            lat = Lattice(ctx, dims, N, beta, aniso)
            lat.set_variant(v)
            lat.set_block(t)
            assert lat.block == t
            rng = Rng(ctx, 77)
            lat.hot_start(rng)
            for m, o in ((1, 4), (2, 0), (0, 3)):
                lat.update(rng, m, o)
            assert np.array_equal(lat.export_angles(), base), (v, t)
    for bad in (0, 16, 48, 288, 512):
        with pytest.raises(U1Error):
            Lattice(ctx, *geom[:2], geom[2], geom[3]).set_block(bad)


def test_graphs_and_variants_agree(ctx):
    geom = (4, (8, 8, 8, 8), 1.0, 1.0)
    a, _ = _run(ctx, geom, 1)
    dims, N, beta, aniso = geom
    b = Lattice(ctx, dims, N, beta, aniso)
    b.set_graphs(False)
    b.set_variant(3)
    rng = Rng(ctx, 77)
    b.hot_start(rng)
    for m, o in ((1, 4), (2, 0), (0, 3)):
        b.update(rng, m, o)
    assert np.array_equal(a.export_angles(), b.export_angles())


def test_tune_restores_state_and_caches(ctx, tmp_path, monkeypatch):
    monkeypatch.setenv("U1_RESOURCE_PATH", str(tmp_path))
    lat = Lattice(ctx, 4, (8, 8, 8, 12), 1.0)
    rng = Rng(ctx, 5)
    lat.hot_start(rng)
    lat.set_variant(3)
    lat.update(rng, 1, 2)
    th0 = lat.export_angles()
    st0 = rng.state
    best = lat.tune(rng)
    assert best in (1, 2, 3, 5)
    assert lat.variant == best and lat.block in (64, 96, 128, 192, 256)
    assert np.array_equal(lat.export_angles(), th0)
    assert rng.state == st0
    cache = tmp_path / "u1b200_tunecache.tsv"
    assert cache.exists()
    lines = [ln.split("\t") for ln in cache.read_text().splitlines()]
    assert any(ln[0].endswith("|update|4|8x8x8x12") and int(ln[1]) == best and int(ln[3]) == lat.block
               for ln in lines)
    # the tuned lattice continues the same chain as an untuned one
    ref = Lattice(ctx, 4, (8, 8, 8, 12), 1.0)
    ref.set_variant(3)
    rng2 = Rng(ctx, 5)
    ref.hot_start(rng2)
    ref.update(rng2, 1, 2)
    lat.update(rng, 1, 4)
    ref.update(rng2, 1, 4)
    assert np.array_equal(lat.export_angles(), ref.export_angles())


def test_auto_variant_tunes_on_first_update(ctx, monkeypatch, tmp_path):
    monkeypatch.setenv("U1_RESOURCE_PATH", str(tmp_path))
    monkeypatch.delenv("U1_TUNE", raising=False)
    lat = Lattice(ctx, 4, (8, 8, 8, 8), 1.0)
    assert lat.variant == 0
    rng = Rng(ctx, 9)
    lat.hot_start(rng)
    lat.update(rng, 1, 1)
    assert lat.variant in (1, 2, 3, 5)
    ref, _ = _run(ctx, (4, (8, 8, 8, 8), 1.0, 1.0), 3, seed=9, sweeps=((1, 1),))
    assert np.array_equal(lat.export_angles(), ref.export_angles())


BATCH_SETS = {
    "4d-groups": [(4, (24, 24, 24, 24), 0.9 + 0.05 * k) for k in range(8)],  # 85 MB: three groups, two lanes
    "4d-mixed": [(4, (8, 8, 8, 8), 1.0), (4, (12, 8, 4, 8), 0.85, 1.2), (4, (8, 4, 4, 16), 1.15)],
    "4d-odd-row": [(4, (6, 6, 4, 4), 1.0), (4, (8, 8, 8, 8), 0.9)],
    "3d": [(3, (8, 8, 0, 8), 1.2), (3, (16, 12, 0, 8), 1.6, 0.9)],
    "2d": [(2, (16, 0, 0, 16), 2.0), (2, (8, 0, 0, 32), 3.0)],
}


@pytest.mark.parametrize("name", list(BATCH_SETS))
def test_batch_matches_single_lattices(ctx, name):
    geoms = BATCH_SETS[name]
    seed, first = 2024, 17
    b = Batch(ctx, geoms, seed=seed, first_chain=first)
    if name == "4d-groups":
        assert b.groups == 3 and b.lanes == 2
    b.hot_start()
    plan = ((1, 4, False), (2, 0, False), (1, 2, True))
    for m, o, meas in plan:
        b.update(m, o, measure=meas)
    fused = b.results_raw()
    now = b.measure_raw()
    assert np.array_equal(fused, now, equal_nan=True)  # 2D: no SS plaquettes (NaN)
    assert b.pass_count() == 1 + 1 + 2 + 1
    for c, g in enumerate(geoms):
        dims, N, beta = g[0], g[1], g[2]
        aniso = g[3] if len(g) > 3 else 1.0
        lat = Lattice(ctx, dims, N, beta, aniso)
        rng = Rng(ctx, seed)
        rng.set_chain(first + c)
        lat.hot_start(rng)
        for m, o, _ in plan:
            lat.update(rng, m, o)
        th = b.export_angles(c)
        assert np.array_equal(th, lat.export_angles()), f"chain {c} differs from its single lattice"
        single = lat.measure()
        row = now[c]
        if dims > 2:
            assert row[0] == single["plaq_ss"].real and row[1] == single["plaq_ss"].imag
        assert row[2] == single["plaq_st"].real and row[3] == single["plaq_st"].imag
        assert row[4] == single["poly"].real and row[5] == single["poly"].imag
        o = Oracle(dims, N, beta, aniso)
        ss, st = o.plaquette(th)
        poly = o.polyakov(th)
        if dims > 2:
            assert abs(row[0] - ss.real) < 2e-6 and abs(row[1] - ss.imag) < 2e-6
        assert abs(row[2] - st.real) < 2e-6 and abs(row[3] - st.imag) < 2e-6
        assert abs(row[4] - poly.real) < 2e-6 and abs(row[5] - poly.imag) < 2e-6


def test_batch_import_export_and_errors(ctx):
    geoms = [(4, (8, 8, 8, 8), 1.0), (4, (8, 8, 8, 4), 1.0)]
    b = Batch(ctx, geoms, seed=3)
    th = np.random.default_rng(1).uniform(0, 2 * np.pi, b.nlinks(1))
    b.import_angles(1, th)
    back = b.export_angles(1)
    d = np.abs(np.angle(np.exp(1j * (back - th))))
    assert d.max() < 2e-7
    assert np.all(b.export_angles(0) == 0.0)  # cold
    with pytest.raises(U1Error):
        Batch(ctx, [(4, (8, 8, 8, 8), 1.0), (3, (8, 8, 0, 8), 1.0)])
    with pytest.raises(U1Error):
        Batch(ctx, [(4, (8, 8, 8, 8), 1.0)] * 2, first_chain=65535)
    with pytest.raises(U1Error):
        Batch(ctx, [(4, (7, 8, 8, 8), 1.0)])
    with pytest.raises(ValueError):
        b.import_angles(0, th[:10])


# geometries where the persistent sweep (variant 4) fits: N0/2 * N1 / 2 threads in [64, 256]
WAVE_GEOMS = [(4, (16, 16, 8, 8), 1.0, 1.0), (4, (32, 16, 6, 4), 0.9, 1.4), (4, (32, 32, 32, 32), 1.0, 1.0)]


@pytest.mark.parametrize("geom", WAVE_GEOMS, ids=lambda g: "x".join(map(str, g[1])))
def test_wave_sweep_bit_identical(ctx, geom):
    """The persistent sweep gives the phase kernels' links bit for bit, for
    mixed, Metropolis-only and overrelaxation-only sweeps."""
    dims, N, beta, aniso = geom
    sweeps = ((1, 4), (2, 0), (0, 3), (1, 1))
    ref, rr = _run(ctx, geom, 1, seed=31, sweeps=sweeps)
    lat = Lattice(ctx, dims, N, beta, aniso)
    try:
        lat.set_variant(4)
    except U1Error:
        pytest.skip("persistent sweep not usable on this device")
    rng = Rng(ctx, 31)
    lat.hot_start(rng)
    for m, o in sweeps:
        lat.update(rng, m, o)
    assert np.array_equal(lat.export_angles(), ref.export_angles())
    assert rng.state == rr.state


@pytest.mark.parametrize("geom", WAVE_GEOMS[:2], ids=lambda g: "x".join(map(str, g[1])))
def test_wave_measured_sweep(ctx, geom):
    import torch
    dims, N, beta, aniso = geom
    a = Lattice(ctx, dims, N, beta, aniso)
    b = Lattice(ctx, dims, N, beta, aniso)
    try:
        a.set_variant(4)
    except U1Error:
        pytest.skip("persistent sweep not usable on this device")
    b.set_variant(1)
    ra, rb = Rng(ctx, 8), Rng(ctx, 8)
    a.hot_start(ra)
    b.hot_start(rb)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    for m, o in ((1, 4), (2, 0)):
        a.update_measure(ra, m, o, out.data_ptr())
        b.update(rb, m, o)
        torch.cuda.synchronize()
        assert np.array_equal(a.export_angles(), b.export_angles())
        want = b.measure()
        got = out.cpu().numpy()
        assert abs(complex(got[0], got[1]) - want["plaq_ss"]) < 2e-6
        assert abs(complex(got[2], got[3]) - want["plaq_st"]) < 2e-6
        assert abs(complex(got[4], got[5]) - want["poly"]) < 2e-6


# a batch whose groups differ: 16^4 chains (2 MiB each, four sites per
# thread allowed), 12^3 x 8 chains (N0/2 = 6: two sites per thread at most),
# 6^4 chains (N0/2 odd: one site per thread only); 9.4 MiB of links
TUNE_SET = ([(4, (16, 16, 16, 16), 0.9 + 0.02 * k) for k in range(4)] + [(4, (12, 12, 12, 8), 1.0, 1.3)] * 3 +
            [(4, (6, 6, 6, 6), 1.1)] * 3)


def _batch_run(ctx, layout=None, tune=False, lanes=None):
    b = Batch(ctx, TUNE_SET, seed=77, first_chain=3)
    if lanes is not None:
        b.set_lanes(lanes)
    if layout is not None:
        b.configure(*layout)
    if tune:
        b.tune()
    b.hot_start()
    for m, o, meas in ((1, 4, True), (2, 1, False), (1, 4, True)):
        b.update(m, o, measure=meas)
    return b, np.concatenate([b.export_angles(c) for c in range(b.n)]), b.results_raw()


def test_batch_layouts_bit_identical(ctx):
    """Every chain-group size, per-group kernel / block size and lane count
    gives the same links and measurements bit for bit; choices a group's
    chains do not allow fall back to the default."""
    base, th0, m0 = _batch_run(ctx)
    assert [g[2] for g in base.layout()] == [3]  # one group holding 6^4 chains: one site per thread
    layouts = [(4, ()),  # 4 MiB groups, default kernels
               # 1 MiB: each 16^4 chain alone, two 12^3x8 chains, then 12^3x8 + 3 x 6^4
               (1, ((5, 64), (5, 96), (1, 256), (3, 96), (1, 192), (3, 64))),
               # 2 MiB: the last group mixes 12^3x8 and 6^4 chains, which refuse (5, 128)
               (2, ((5, 128), (1, 64), (3, 256), (5, 64), (5, 128))),
               (64, ((3, 128),))]
    for layout, lanes in [(lay, ln) for lay in layouts for ln in (1, 2)]:
        b, th, m = _batch_run(ctx, layout, lanes=lanes)
        assert b.lanes == lanes
        lay = b.layout()
        if layout[0] == 1:
            assert [(g[2], g[3]) for g in lay] == list(layout[1])
        if layout[0] == 2:
            assert lay[-1][2:] == (3, 256)
        assert lay[0][0] == 0 and lay[-1][1] == b.n
        for c0, c1, v, t in lay:  # only choices the chains allow
            assert v in (1, 3, 5) and 32 <= t <= (128 if v == 5 else 256)
            for c in range(c0, c1):
                h = TUNE_SET[c][1][0] // 2
                assert (v != 5 or h % 4 == 0) and (v != 1 or h % 2 == 0)
        assert np.array_equal(th, th0), (layout, lanes)
        assert np.array_equal(m, m0, equal_nan=True), (layout, lanes)
        assert b.pass_count() == base.pass_count(), (layout, lanes)
    for bad in (0, 3):
        with pytest.raises(U1Error):
            base.set_lanes(bad)


def test_batch_tune_and_cache(ctx, monkeypatch, tmp_path):
    """u1_batch_tune picks a group size, a lane count and a per-group kernel /
    block size, keeps the Markov chains bit for bit, and caches the result in
    $U1_RESOURCE_PATH; a second batch of the same extents applies it."""
    monkeypatch.setenv("U1_RESOURCE_PATH", str(tmp_path))
    _, th0, m0 = _batch_run(ctx)
    b, th, m = _batch_run(ctx, tune=True)
    assert np.array_equal(th, th0) and np.array_equal(m, m0, equal_nan=True)
    lay = b.layout()
    f = tmp_path / "u1b200_batch_tunecache.tsv"
    assert f.exists()
    rows = [r.split("\t") for r in f.read_text().splitlines() if r and not r.startswith("#")]
    assert len(rows) == 1 and int(rows[0][1]) in (32, 48, 64, 80, 96)
    assert rows[0][2] == ",".join(f"{v}:{t}" for _, _, v, t in lay)
    assert int(rows[0][4]) == b.lanes in (1, 2)
    b2 = Batch(ctx, TUNE_SET, seed=5)
    b2.set_lanes(3 - b.lanes)
    assert b2.tune() == int(rows[0][1])
    assert b2.layout() == lay and b2.lanes == b.lanes
    assert len([r for r in f.read_text().splitlines() if r]) == 1  # applied from the cache, not re-tuned


def test_quad_multi_wave_bit_identical(ctx):
    """A four-site phase larger than one wave (40^4: 2500 blocks of 128
    threads, launch order) gives the two-site kernel's links bit for bit.
    The measured sweep's sums are
    bit-identical between block sizes of the four-site kernel; against the
    two-site kernel they agree to rounding (its per-thread partial sums hold
    two sites instead of four)."""
    import torch
    N = (40, 40, 40, 40)
    res = []
    for variant, block in ((5, 128), (5, 64), (1, 256)):
        lat = Lattice(ctx, 4, N, 1.0)
        lat.set_variant(variant)
        lat.set_block(block)
        rng = Rng(ctx, 404)
        lat.hot_start(rng)
        lat.update(rng, 1, 4)
        out = torch.zeros(6, dtype=torch.float64, device="cuda")
        lat.update_measure(rng, 2, 1, out.data_ptr())
        torch.cuda.synchronize()
        res.append((lat.export_angles(), out.cpu().numpy(), rng.state))
        lat.close()
    for th, m, st in res[1:]:
        assert np.array_equal(th, res[0][0])
        assert st == res[0][2]
    assert np.array_equal(res[1][1], res[0][1])
    assert np.abs(res[2][1] - res[0][1]).max() < 1e-9
