"""Version-1 configuration checkpoints, readable and writable without a GPU.

The library writes them with u1_checkpoint_save (Lattice.save) and reads them
with u1_checkpoint_load (Lattice.load); this module parses and writes the
same files with numpy, e.g. to bring configurations in or out of other tools.

Layout (little endian): a 128-byte header
    magic "U1B200CK", u32 version = 1, u32 header bytes = 128, i32 dims,
    i32 Grid[4], u32 0, f64 beta, f64 aniso, u64 seed, u64 pass, u32 chain,
    u32 flags (bit 0: exact float2 links follow), u64 nlinks,
    u32 crc32(angles), u32 crc32(links), 32 zero bytes
then nlinks f64 angles in [0, 2 pi) in the reference's even/odd layout
theta[eo + parity V/2 + mu V] (include/index.h:114-153), then, with flag
bit 0, nlinks float2 (cos, sin) links in the same order.  The CRC is the
IEEE CRC-32 (zlib.crc32).  Grid uses the reference's direction mapping
(2D: (Nx, Nt, 1, 1); 3D: (Nx, Ny, Nt, 1); src/parameters.cu:146-208).
"""
from __future__ import annotations

import struct
import zlib
from pathlib import Path

import numpy as np

MAGIC = b"U1B200CK"
_HDR = struct.Struct("<8sIIi4iIddQQIIQII32x")
assert _HDR.size == 128


def grid_of(dims: int, N) -> tuple[int, int, int, int]:
    """Reference Grid from the ABI's (Nx, Ny, Nz, Nt)."""
    N = list(N) + [0] * (4 - len(N))
    if dims == 2:
        return (N[0], N[3], 1, 1)
    if dims == 3:
        return (N[0], N[1], N[3], 1)
    return (N[0], N[1], N[2], N[3])


def read_checkpoint(path) -> dict:
    data = Path(path).read_bytes()
    if len(data) < 128:
        raise ValueError("checkpoint: file shorter than its header")
    (magic, version, hbytes, dims, g0, g1, g2, g3, _res, beta, aniso, seed, pass_, chain, flags, nlinks,
     crc_a, crc_l) = _HDR.unpack_from(data, 0)
    if magic != MAGIC or version != 1 or hbytes != 128:
        raise ValueError("checkpoint: not a version-1 checkpoint")
    na = 8 * nlinks
    nl = 8 * nlinks if flags & 1 else 0
    if len(data) < 128 + na + nl:
        raise ValueError("checkpoint: truncated file")
    ang_b = data[128:128 + na]
    if zlib.crc32(ang_b) != crc_a:
        raise ValueError("checkpoint: angle checksum mismatch")
    out = {"dims": dims, "grid": (g0, g1, g2, g3), "beta": beta, "aniso": aniso, "seed": seed, "pass": pass_,
           "chain": chain, "flags": flags, "angles": np.frombuffer(ang_b, dtype="<f8").copy()}
    if flags & 1:
        lb = data[128 + na:128 + na + nl]
        if zlib.crc32(lb) != crc_l:
            raise ValueError("checkpoint: link checksum mismatch")
        out["links"] = np.frombuffer(lb, dtype="<f4").reshape(-1, 2).copy()
    return out


def write_checkpoint(path, angles, dims: int, grid, beta: float, aniso: float = 1.0, seed: int = 0,
                     pass_: int = 0, chain: int = 0) -> None:
    """Angles only (no exact links): loading rebuilds the links from them."""
    ang = np.ascontiguousarray(np.mod(np.asarray(angles, dtype=np.float64), 2 * np.pi), dtype="<f8")
    V = int(np.prod(grid))
    if ang.size != V * dims:
        raise ValueError(f"expected {V * dims} angles, got {ang.size}")
    ab = ang.tobytes()
    hdr = _HDR.pack(MAGIC, 1, 128, dims, *[int(x) for x in grid], 0, float(beta), float(aniso), int(seed),
                    int(pass_), int(chain), 0, ang.size, zlib.crc32(ab), 0)
    tmp = Path(str(path) + ".tmp")
    tmp.write_bytes(hdr + ab)
    tmp.replace(path)
