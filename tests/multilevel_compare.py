"""Multilevel against single-level Polyakov correlators at equal wall time
(test infrastructure; the 24^3 x 32, beta = 0.95 configuration).

Both estimators measure C(r) = <P(x) P*(x + r e_i)>, r = 1..12, on one B200:

* multilevel: u1_multilevel(n4 = 100, k4 = 1, n2 = 200, k2 = 1, 1 Metropolis +
  4 OR per sub-update) with analytic multihit temporal links (reference
  MultiLevel, src/multilevel.cu:639-732), once per configuration of a chain
  (`--gap` sweeps apart); errors: jackknife over the configurations;
* single-level: u1_poly_corr(multihit = 1) (reference Poly2(lat, true),
  src/polyakov.cu:618-654) after every sweep of the same chain, run for the
  wall time the multilevel estimates took; errors: binned jackknife (20 bins).

    python -m tests.multilevel_compare --configs 12 --out RESULT.json

prints a markdown table with the error of each estimator per r and their
ratio (single-level error / multilevel error at equal wall time).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def jackknife_bins(x: np.ndarray, nbins: int) -> tuple[np.ndarray, np.ndarray]:
    """Mean and jackknife error per column over nbins consecutive bins."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x) // nbins * nbins
    b = x[:n].reshape(nbins, -1, *x.shape[1:]).mean(axis=1)
    loo = (b.sum(axis=0) - b) / (nbins - 1)
    return x[:n].mean(axis=0), np.sqrt((nbins - 1) / nbins * ((loo - loo.mean(axis=0)) ** 2).sum(axis=0))


def run(configs: int, gap: int, therm: int, n4: int, n2: int, seed: int = 2024) -> dict:
    import torch

    from latticeu1_b200 import Context, Lattice, Rng
    ctx = Context(0)
    N, beta = (24, 24, 24, 32), 0.95
    lat = Lattice(ctx, 4, N, beta)
    rng = Rng(ctx, seed)
    lat.hot_start(rng)
    for _ in range(therm):
        lat.update(rng, 1, 4)
    lat.multilevel(Rng(ctx, 1), 1, 1, 2, 1, 1, 4)  # warm-up: graph capture, allocations
    torch.cuda.synchronize()
    ml, t_ml = [], 0.0
    for k in range(configs):
        for _ in range(gap):
            lat.update(rng, 1, 4)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        c = lat.multilevel(Rng(ctx, 7000 + k), n4, 1, n2, 1, 1, 4)
        t_ml += time.perf_counter() - t0
        ml.append(c.real)
    ml = np.asarray(ml)
    sl = []
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < t_ml:
        lat.update(rng, 1, 4)
        sl.append(lat.poly_corr(True).real)
    t_sl = time.perf_counter() - t0
    sl = np.asarray(sl)
    m_ml, e_ml = jackknife_bins(ml, len(ml))
    m_sl, e_sl = jackknife_bins(sl, 20)
    return {"lattice": "24^3x32", "beta": beta, "n4": n4, "n2": n2, "configs": configs, "gap_sweeps": gap,
            "therm": therm, "multilevel_seconds": t_ml, "single_level_seconds": t_sl,
            "single_level_measurements": len(sl), "C_ml": m_ml.tolist(), "err_ml": e_ml.tolist(),
            "C_sl": m_sl.tolist(), "err_sl": e_sl.tolist()}


def table(res: dict) -> str:
    lines = ["| r | C(r) multilevel | error | C(r) single-level | error | error ratio (single / multi) |",
             "|---|---|---|---|---|---|"]
    for r in range(len(res["C_ml"])):
        em, es = res["err_ml"][r], res["err_sl"][r]
        lines.append(f"| {r + 1} | {res['C_ml'][r]:.4e} | {em:.2e} | {res['C_sl'][r]:.4e} | {es:.2e} | "
                     f"{es / em:.3g} |")
    return "\n".join(lines)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", type=int, default=12)
    ap.add_argument("--gap", type=int, default=20)
    ap.add_argument("--therm", type=int, default=500)
    ap.add_argument("--n4", type=int, default=100)
    ap.add_argument("--n2", type=int, default=200)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None, help="print the table of a saved result instead of running")
    args = ap.parse_args(argv)
    if args.report:
        res = json.loads(Path(args.report).read_text())
    else:
        res = run(args.configs, args.gap, args.therm, args.n4, args.n2)
        if args.out:
            Path(args.out).write_text(json.dumps(res, indent=1))
    print(f"multilevel: {res['configs']} configurations in {res['multilevel_seconds']:.1f} s; single-level: "
          f"{res['single_level_measurements']} measurements in {res['single_level_seconds']:.1f} s")
    print(table(res))


if __name__ == "__main__":
    main()
