"""Generate the golden fixtures in tests/golden/ from the REFERENCE's own code.

Run where the reference sources exist and oracle/_ref/libu1ref.so is built
(`make -C oracle ref REF=<reference source tree>`):
    python tests/golden/make_golden.py

For each geometry the fixture holds a seeded random lattice and what the
reference's own FP64 CPU functions (reference src/update.cu:51-98,
src/plaquette.cu:32-57, src/polyakov.cu:33-49, include/staple.h:79-102,
include/lattice_functions.h:92-105, include/index.h:114-153) return on it:
the EO index table, staples, one overrelaxation pass, one Metropolis pass
with the recorded (new theta, b) stream, plaquette, Polyakov loop and the
multihit means.  The fixtures pin the oracle (tests/test_oracle_pin.py) and
the GPU kernels where the reference is not available.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Ref  # noqa: E402

GEOMS = {
    "g4d": dict(dims=4, N=(4, 6, 8, 4), beta=1.3, aniso=1.7, seed=11),
    "g4d_iso": dict(dims=4, N=(6, 4, 4, 8), beta=1.0, aniso=1.0, seed=12),
    "g3d": dict(dims=3, N=(6, 4, 0, 8), beta=2.1, aniso=0.8, seed=13),
    "g2d": dict(dims=2, N=(8, 0, 0, 6), beta=4.0, aniso=1.0, seed=14),
}


def make(name: str, dims: int, N, beta: float, aniso: float, seed: int) -> dict:
    ref = Ref(dims, N, beta, aniso)
    rng = np.random.default_rng(seed)
    lat0 = rng.uniform(0.0, 2.0 * np.pi, ref.nlinks)
    out = {"dims": dims, "N": np.array(list(N) + [0] * (4 - len(N))), "beta": beta, "aniso": aniso, "lat0": lat0}
    # EO index table and +-1 neighbours
    coords = np.array([[ref.index_eo(i, p) for i in range(ref.Vh)] for p in (0, 1)], dtype=np.int32)
    nbr = np.zeros((2, ref.Vh, dims, 2), dtype=np.int32)
    for p in (0, 1):
        for i in range(ref.Vh):
            for mu in range(dims):
                nbr[p, i, mu, 0] = ref.index_eo_neg(i, p, mu, -1)
                nbr[p, i, mu, 1] = ref.index_eo_neg(i, p, mu, 1)
    out["coords"], out["nbr"] = coords, nbr
    st = np.zeros((2, dims, ref.Vh), dtype=np.complex128)
    for p in (0, 1):
        for mu in range(dims):
            for i in range(ref.Vh):
                st[p, mu, i] = ref.staple(lat0, i, p, mu)
    out["staple"] = st
    l = lat0.copy()
    ref.overrelax(l)
    out["after_or"] = l
    pairs = ref.record_pairs(seed, 1)
    ref.seed_cpu(1, seed)
    l = lat0.copy()
    ref.metropolis(l)
    out["pairs"], out["after_met"] = pairs, l
    c, s = ref.plaquette(lat0)
    out["plaq_cos_sin"] = np.array([c, s])
    out["poly"] = np.array([ref.polyakov(lat0)])
    if dims == 4:
        mh = np.zeros((2, ref.Vh), dtype=np.complex128)
        for p in (0, 1):
            for i in range(ref.Vh):
                mh[p, i] = ref.multihit(lat0, i, p)
        out["multihit"] = mh
    return out


def main() -> None:
    here = Path(__file__).resolve().parent
    for name, kw in GEOMS.items():
        data = make(name, **kw)
        np.savez_compressed(here / f"{name}.npz", **data)
        print("wrote", here / f"{name}.npz")


if __name__ == "__main__":
    main()
