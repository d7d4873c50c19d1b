"""GPU checks of the formats around the update path.

* EO <-> natural order conversion: an exact permutation, equal to a numpy
  restatement of the reference's kernel_convert_EO_NO;
* per-site plaquette fields: within 1e-6 of an FP64 numpy restatement of
  kernel_plaquette_comps (both orders: per site and time averages), and their
  means equal the field means;
* checkpoints: an exact checkpoint resumes the chain bit for bit; the angle
  section matches export_angles and reads with numpy; numpy-written
  checkpoints load; geometry mismatches are rejected.
"""
import numpy as np
import pytest
import torch

from latticeu1_b200 import Lattice, Rng, U1Error
from latticeu1_b200.checkpoint import grid_of, read_checkpoint, write_checkpoint
from latticeu1_b200.lattice import convert_order
from tests.torch_ref import link_index

pytestmark = pytest.mark.gpu

COMPS = [(0, 3), (1, 3), (2, 3), (1, 2), (2, 0), (0, 1)]


def _coords(grid):
    axes = [np.arange(n) for n in grid]
    # natural order: x0 fastest
    X = np.stack(np.meshgrid(*axes, indexing="ij"), 0)
    return X.transpose(0, 4, 3, 2, 1).reshape(4, -1)


def _eo_to_no(th, dims, grid):
    V = int(np.prod(grid))
    X = _coords(grid)
    out = np.empty_like(th)
    for mu in range(dims):
        out[mu * V:(mu + 1) * V] = th[link_index(grid, X, mu)]
    return out


@pytest.mark.parametrize("dims,N", [(4, (8, 6, 4, 10)), (3, (6, 8, 0, 4)), (2, (10, 0, 0, 6))])
def test_convert_order(ctx, dims, N):
    grid = grid_of(dims, N)
    n = int(np.prod(grid)) * dims
    th = np.random.default_rng(2).uniform(0, 2 * np.pi, n)
    t = torch.tensor(th, dtype=torch.float64, device="cuda")
    no = convert_order(t, dims, N, eo_to_no=True)
    assert np.array_equal(no.cpu().numpy(), _eo_to_no(th, dims, grid))
    back = convert_order(no, dims, N, eo_to_no=False)
    assert torch.equal(back, t)


def _plaq_field_ref(th, grid):
    X = _coords(grid)
    out = []
    e = np.eye(4, dtype=np.int64)
    for mu, nu in COMPS:
        tp = (th[link_index(grid, X, mu)] + th[link_index(grid, X + e[mu][:, None], nu)]
              - th[link_index(grid, X + e[nu][:, None], mu)] - th[link_index(grid, X, nu)])
        out.append(1.0 - np.exp(1j * tp))
    return np.stack(out, 0)


def test_plaquette_fields(ctx):
    N = (8, 6, 4, 6)
    lat = Lattice(ctx, 4, N, 1.0)
    rng = Rng(ctx, 4)
    lat.hot_start(rng)
    lat.update(rng, 1, 2)
    th = lat.export_angles()
    grid = grid_of(4, N)
    ref = _plaq_field_ref(th, grid)
    f, m = lat.plaquette_fields(spacetime=True)
    f = f.cpu().numpy()
    assert np.abs(f - ref).max() < 1e-6
    assert np.abs(m - f.mean(axis=1)).max() < 1e-12
    fs, ms = lat.plaquette_fields(spacetime=False)
    Vs = grid[0] * grid[1] * grid[2]
    ref_s = ref.reshape(6, grid[3], Vs).mean(axis=1)
    assert np.abs(fs.cpu().numpy() - ref_s).max() < 1e-6
    assert np.abs(ms - m).max() < 1e-6
    # the class means of the fields are the plaquette measurement (SS from (1,2),(2,0),(0,1) with
    # (2,0) the conjugate orientation of (0,2))
    meas = lat.measure()
    st = m[0:3].mean()
    ss = (m[3] + np.conj(m[4]) + m[5]) / 3
    assert abs(st - meas["plaq_st"]) < 2e-6 and abs(ss - meas["plaq_ss"]) < 2e-6


def test_plaquette_fields_4d_only(ctx):
    lat = Lattice(ctx, 3, (4, 4, 0, 4), 1.0)
    with pytest.raises(U1Error):
        lat.plaquette_fields()


def test_checkpoint_exact_resume(ctx, tmp_path):
    N = (8, 8, 8, 8)
    a = Lattice(ctx, 4, N, 1.1, 1.3)
    ra = Rng(ctx, 99)
    ra.set_chain(5)
    a.hot_start(ra)
    a.update(ra, 1, 4)
    p = tmp_path / "run.u1ck"
    a.save(p, ra, exact=True)
    a.update(ra, 1, 4)
    a.update(ra, 2, 1)
    b = Lattice(ctx, 4, N, 0.5)  # coupling comes from the file
    rb = Rng(ctx, 1)
    b.load(p, rb)
    assert rb.state == (99, 1 + 1) and b.beta == 1.1 and b.aniso == 1.3
    b.update(rb, 1, 4)
    b.update(rb, 2, 1)
    assert np.array_equal(a.export_angles(), b.export_angles())
    d = read_checkpoint(p)
    assert d["chain"] == 5 and d["flags"] == 1 and d["links"].shape == (a.nlinks, 2)


def test_checkpoint_angles_and_numpy_interop(ctx, tmp_path):
    N = (6, 4, 4, 8)
    a = Lattice(ctx, 4, N, 1.0)
    r = Rng(ctx, 3)
    a.hot_start(r)
    p = tmp_path / "ang.u1ck"
    a.save(p, r, exact=False)
    d = read_checkpoint(p)
    assert np.array_equal(d["angles"], a.export_angles()) and d["flags"] == 0
    b = Lattice(ctx, 4, N, 1.0)
    b.load(p)
    assert np.abs(np.angle(np.exp(1j * (b.export_angles() - d["angles"])))).max() < 2e-7
    th = np.random.default_rng(5).uniform(0, 2 * np.pi, a.nlinks)
    q = tmp_path / "np.u1ck"
    write_checkpoint(q, th, 4, grid_of(4, N), 1.0, seed=8, pass_=3)
    b.load(q, r)
    assert r.state == (8, 3)
    assert np.abs(np.angle(np.exp(1j * (b.export_angles() - th)))).max() < 2e-7
    c = Lattice(ctx, 4, (6, 4, 4, 4), 1.0)
    with pytest.raises(U1Error):
        c.load(q)
