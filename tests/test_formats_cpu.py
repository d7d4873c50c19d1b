"""Checkpoint files without a GPU: the numpy writer/reader and the library's
header parser (u1_checkpoint_info, host only) agree; corruption is caught."""
import numpy as np
import pytest

from latticeu1_b200 import U1Error
from latticeu1_b200.checkpoint import grid_of, read_checkpoint, write_checkpoint
from latticeu1_b200.lattice import checkpoint_info


@pytest.mark.parametrize("dims,N", [(4, (4, 6, 8, 4)), (3, (6, 4, 0, 8)), (2, (8, 0, 0, 6))])
def test_numpy_writer_reader_and_library_info(tmp_path, dims, N):
    grid = grid_of(dims, N)
    n = int(np.prod(grid)) * dims
    th = np.random.default_rng(0).uniform(0, 2 * np.pi, n)
    p = tmp_path / "c.u1ck"
    write_checkpoint(p, th, dims, grid, 1.25, 1.5, seed=77, pass_=12, chain=3)
    d = read_checkpoint(p)
    assert np.array_equal(d["angles"], th)
    assert d["grid"] == grid and d["dims"] == dims and d["seed"] == 77 and d["pass"] == 12 and d["chain"] == 3
    info = checkpoint_info(p)
    assert info["dims"] == dims and info["beta"] == 1.25 and info["aniso"] == 1.5
    assert info["seed"] == 77 and info["pass"] == 12 and info["chain"] == 3 and info["flags"] == 0
    expect = list(N) + [0] * (4 - len(N))
    assert list(info["N"]) == expect


def test_corruption_detected(tmp_path):
    grid = (4, 4, 4, 4)
    th = np.random.default_rng(1).uniform(0, 2 * np.pi, 256 * 4)
    p = tmp_path / "c.u1ck"
    write_checkpoint(p, th, 4, grid, 1.0)
    raw = bytearray(p.read_bytes())
    raw[200] ^= 0xFF
    p.write_bytes(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        read_checkpoint(p)
    bad = tmp_path / "bad.u1ck"
    bad.write_bytes(b"NOTACKPT" + bytes(200))
    with pytest.raises(U1Error):
        checkpoint_info(bad)
    with pytest.raises(ValueError):
        read_checkpoint(bad)
