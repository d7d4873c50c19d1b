"""Long-run statistical parity on the target lattices (test infrastructure).

The measured workload is 1 Metropolis + 4 overrelaxation passes per sweep
with the spatial and temporal plaquettes and the Polyakov loop after every
sweep (the reference driver's loop, u1.cpp:118-128).  Each configuration
runs three Markov chains:

* ours: this library (Philox stream, float2 links, FP64 sums) through
  u1_update_measure;
* reference CUDA: the reference's own UpdateLattice / Plaquette / Polyakov
  loop (src/update.cu:449-456, src/plaquette.cu:222-228,
  src/polyakov.cu:169-174; FP64 angles, cuRAND MRG32k3a) built in place into
  oracle/_ref and started from the same configuration as ours;
* FP64 oracle: oracle/u1_oracle.cpp on the host (Philox, FP64).  A 32^4
  sweep costs about a second of host time, so this arm is shorter: either
  started from our configuration after thermalisation (`gpu` runs it beside
  the GPU arms), or as an independent chain from the same start with its own
  thermalisation (`oracle-chain`, host only, no GPU needed).

Observables: Re P_SS, Re P_ST (the reference's mean of 1 - e^{i theta_P}
over spatial-spatial and spatial-temporal plaquettes) and |L|.  Each mean
carries two errors, a binned jackknife and the Gamma-method error
sqrt(2 tau_int var / n) (U. Wolff, Comput. Phys. Commun. 156 (2004) 143);
the larger is used.  The oracle's series is too short to window its own
tau_int reliably, so its Gamma error uses the larger of its own tau_int and
that of our 5000-sweep series (the same update algorithm and observable).

    python -m tests.target_parity gpu --out DIR [--sweeps 5000 --therm 500
                                                  --oracle-sweeps 200 --oracle-drop 40]
    python -m tests.target_parity oracle-chain --out DIR --config K [--therm 500
                                                                   --oracle-sweeps 1000]
    python -m tests.target_parity report --out DIR

`gpu` runs every configuration's GPU arms on cuda:0 and starts each oracle
arm as a separate host process (`oracle-one`) while the next
configuration's GPU arms run; `report` prints the markdown summary.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

# The target configurations: 32^4 at beta 0.9, 1.0, 1.1 and the anisotropic
# 24^3 x 48 lattice with xi = 2 and beta_s = 1 (reference arguments beta = 2,
# aniso = 2: beta_s = beta / xi, beta_t = beta * xi).  The confined-phase
# chains start hot; the Coulomb-phase ones start cold, because a hot start
# there can trap a chain in a metastable state with a defect for thousands of
# sweeps (each chain in a different one).
CONFIGS = [
    dict(name="32^4 beta=0.9", dims=4, N=(32, 32, 32, 32), beta=0.9, aniso=1.0, start="hot"),
    dict(name="32^4 beta=1.0", dims=4, N=(32, 32, 32, 32), beta=1.0, aniso=1.0, start="hot"),
    dict(name="32^4 beta=1.1", dims=4, N=(32, 32, 32, 32), beta=1.1, aniso=1.0, start="cold"),
    dict(name="24^3x48 beta=2 xi=2", dims=4, N=(24, 24, 24, 48), beta=2.0, aniso=2.0, start="cold"),
]
OBS = ("Re P_SS", "Re P_ST", "|L|")


def observables(raw: np.ndarray) -> np.ndarray:
    """(n, 6) rows of (SS re, im, ST re, im, L re, im) -> (n, 3) observables."""
    raw = np.asarray(raw, dtype=np.float64)
    return np.stack([raw[:, 0], raw[:, 2], np.hypot(raw[:, 4], raw[:, 5])], axis=1)


def jackknife(x: np.ndarray, nbins: int = 20) -> tuple[float, float]:
    """Mean and jackknife error over nbins consecutive bins."""
    x = np.asarray(x, dtype=np.float64)
    b = x[: len(x) // nbins * nbins].reshape(nbins, -1).mean(axis=1)
    loo = (b.sum() - b) / (nbins - 1)
    return float(x.mean()), float(np.sqrt((nbins - 1) / nbins * np.sum((loo - loo.mean()) ** 2)))


def tau_int(x: np.ndarray, S: float = 1.5) -> float:
    """Integrated autocorrelation time with Wolff's automatic window (the
    reference's calculateCorTime, src/actime.cpp:19-145, restated)."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    d = x - x.mean()
    f = np.fft.rfft(d, 2 * n)
    G = np.fft.irfft(f * np.conj(f))[:n] / (n - np.arange(n))
    if G[0] <= 0.0:
        return 0.5
    W, acc = n // 2, 0.0
    for t in range(1, n // 2):
        acc += G[t] / G[0]
        tau = S / math.log((acc + 1.0) / acc) if acc > 0 else 1e-16
        if math.exp(-t / tau) - tau / math.sqrt(t * n) < 0:
            W = t
            break
    C0 = G[0] + 2 * G[1:W + 1].sum()
    Gc = G + C0 / n
    return float(max(0.5, 0.5 + Gc[1:W + 1].sum() / Gc[0]))


def summarize(series: np.ndarray, nbins: int = 20, tau_floor: dict | None = None) -> dict:
    """Per observable: mean, jackknife error, tau_int, Gamma error, error
    used.  tau_floor: lower bounds of tau_int per observable (from a longer
    series of the same algorithm)."""
    out = {}
    for k, name in enumerate(OBS):
        x = series[:, k]
        m, ej = jackknife(x, nbins)
        t = max(tau_int(x), (tau_floor or {}).get(name, 0.0))
        eg = float(np.sqrt(2 * t * x.var(ddof=1) / len(x)))
        out[name] = dict(mean=m, err_jk=ej, tau_int=t, err_gamma=eg, err=max(ej, eg), n=len(x),
                         bin=len(x) // nbins)
    return out


def pulls(a: dict, b: dict) -> dict:
    """(mean_a - mean_b) / combined error, per observable."""
    return {k: (a[k]["mean"] - b[k]["mean"]) / math.hypot(a[k]["err"], b[k]["err"]) for k in OBS}


# --------------------------------------------------------------- GPU arms
def run_ours(ctx, cfg: dict, sweeps: int, therm: int, seed: int = 77):
    """Our chain: the start configuration (FP64 angles), the configuration
    after `therm` sweeps, and the (therm + sweeps, 6) measurement rows."""
    import torch

    from latticeu1_b200 import Lattice, Rng
    lat = Lattice(ctx, cfg["dims"], cfg["N"], cfg["beta"], cfg["aniso"])
    rng = Rng(ctx, seed)
    if cfg["start"] == "hot":
        lat.hot_start(rng)
    else:
        lat.cold_start()
    th0 = lat.export_angles()
    out = torch.zeros((therm + sweeps, 6), dtype=torch.float64, device=f"cuda:{ctx.device}")
    for s in range(therm):
        lat.update_measure(rng, 1, 4, out[s].data_ptr())
    th_therm = lat.export_angles()
    for s in range(therm, therm + sweeps):
        lat.update_measure(rng, 1, 4, out[s].data_ptr())
    torch.cuda.synchronize()
    return th0, th_therm, out.cpu().numpy()


def run_reference_cuda(cfg: dict, th0: np.ndarray, nsweeps: int, seed: int = 1234) -> np.ndarray:
    """The reference's own CUDA chain from th0: (nsweeps, 6) rows."""
    from oracle import ref_gpu
    N = list(cfg["N"]) + [0] * (4 - len(cfg["N"]))
    inp = dict(dims=cfg["dims"], N=np.array(N), beta=cfg["beta"], aniso=cfg["aniso"], lat=th0, metrop=1, ovrn=4,
               sweeps=nsweeps, seed=seed)
    return ref_gpu.run("chain", inp, timeout=3600.0)["obs"]


# --------------------------------------------------------------- host arm
def run_oracle(cfg: dict, th_start: np.ndarray, sweeps: int, seed: int = 4242) -> np.ndarray:
    """The FP64 oracle's chain (Philox) from th_start: (sweeps, 6) rows."""
    from oracle.oracle import Oracle
    o = Oracle(cfg["dims"], cfg["N"], cfg["beta"], cfg["aniso"])
    th = np.array(th_start, dtype=np.float64)
    rows, pass_ = [], 10 ** 6
    for _ in range(sweeps):
        pass_ = o.update_philox(th, seed, pass_, 1, 4)
        ss, st = o.plaquette(th)
        lp = o.polyakov(th)
        rows.append((ss.real, ss.imag, st.real, st.imag, lp.real, lp.imag))
    return np.asarray(rows)


def _oracle_chain(args) -> None:
    """An independent FP64 oracle chain: the configuration's start (the hot
    start is Philox with our seed, bit-identical to ours), `therm` sweeps,
    then `oracle_sweeps` measured sweeps; every sweep's row is kept."""
    from oracle.oracle import Oracle
    cfg = CONFIGS[args.config]
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    o = Oracle(cfg["dims"], cfg["N"], cfg["beta"], cfg["aniso"])
    th = o.hot_start(77) if cfg["start"] == "hot" else np.zeros(o_nlinks(cfg))
    t0 = time.perf_counter()
    pass_ = 10 ** 6
    for _ in range(args.therm):
        pass_ = o.update_philox(th, 5151, pass_, 1, 4)
    rows = run_oracle(cfg, th, args.oracle_sweeps, seed=5151 + 1)
    np.save(out / f"oracle_{args.config}.npy", rows)
    with open(out / f"oracle_{args.config}.json", "w") as f:
        json.dump({"seconds": time.perf_counter() - t0, "threads": int(os.environ.get("OMP_NUM_THREADS", 0)) or
                   os.cpu_count(), "therm": args.therm, "independent": True}, f)


def o_nlinks(cfg: dict) -> int:
    return int(np.prod([n for n in cfg["N"] if n > 0])) * cfg["dims"]


def _oracle_one(args) -> None:
    cfg = CONFIGS[args.config]
    out = Path(args.out)
    th = np.load(out / f"start_{args.config}.npy")
    t0 = time.perf_counter()
    rows = run_oracle(cfg, th, args.oracle_sweeps)
    np.save(out / f"oracle_{args.config}.npy", rows)
    with open(out / f"oracle_{args.config}.json", "w") as f:
        json.dump({"seconds": time.perf_counter() - t0, "threads": os.cpu_count()}, f)


def _gpu(args) -> None:
    from latticeu1_b200 import Context
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    ctx = Context(0)
    procs = []
    for k, cfg in enumerate(CONFIGS):
        if args.only is not None and k not in args.only:
            continue
        t0 = time.perf_counter()
        th0, th_therm, ours = run_ours(ctx, cfg, args.sweeps, args.therm)
        t1 = time.perf_counter()
        np.save(out / f"start_{k}.npy", th_therm)
        if args.oracle_sweeps > 0:
            procs.append(subprocess.Popen([sys.executable, "-m", "tests.target_parity", "oracle-one", "--out",
                                           str(out), "--config", str(k), "--oracle-sweeps",
                                           str(args.oracle_sweeps)], cwd=str(ROOT)))
        ref = run_reference_cuda(cfg, th0, args.therm + args.sweeps)
        t2 = time.perf_counter()
        np.save(out / f"ours_{k}.npy", ours)
        np.save(out / f"ref_{k}.npy", ref)
        with open(out / f"gpu_{k}.json", "w") as f:
            json.dump({"therm": args.therm, "sweeps": args.sweeps, "ours_s": t1 - t0, "ref_s": t2 - t1,
                       "oracle_drop": args.oracle_drop}, f)
        print(f"{cfg['name']}: ours {t1 - t0:.1f} s, reference CUDA {t2 - t1:.1f} s", flush=True)
    rc = 0
    for p in procs:
        rc |= p.wait()
    if rc:
        raise SystemExit(f"an oracle arm failed (rc {rc})")
    for k in range(len(CONFIGS)):
        if (out / f"start_{k}.npy").exists():
            os.remove(out / f"start_{k}.npy")


def analyse(out: Path, k: int, oracle_dir: str | None = None) -> dict | None:
    """Summaries and pulls of configuration k from the files in `out`."""
    if not (out / f"ours_{k}.npy").exists():
        return None
    meta = json.load(open(out / f"gpu_{k}.json"))
    therm = meta["therm"]
    res = {"config": CONFIGS[k], "meta": meta}
    ours = observables(np.load(out / f"ours_{k}.npy")[therm:])
    ref = observables(np.load(out / f"ref_{k}.npy")[therm:])
    res["ours"], res["ref"] = summarize(ours), summarize(ref)
    res["pull_ref"] = pulls(res["ours"], res["ref"])
    floor = {o: res["ours"][o]["tau_int"] for o in OBS}
    # the short oracle arm started from our thermalised configuration (`gpu`)
    # and the independent oracle chain with its own thermalisation (`oracle-chain`)
    for tag, d in (("oracle", out), ("oracle_chain", Path(oracle_dir) if oracle_dir else None)):
        if d is None or not (d / f"oracle_{k}.npy").exists():
            continue
        ometa = json.load(open(d / f"oracle_{k}.json"))
        if (tag == "oracle") == bool(ometa.get("independent")):
            continue
        drop = 0 if ometa.get("independent") else meta["oracle_drop"]
        orc = observables(np.load(d / f"oracle_{k}.npy")[drop:])
        res[tag] = summarize(orc, nbins=10, tau_floor=floor)
        res["pull_" + tag] = pulls(res["ours"], res[tag])
        res[tag + "_meta"] = ometa
    return res


def _fmt(s: dict) -> str:
    return f"{s['mean']:.6f}({s['err'] * 1e6:.0f})"


def _report(args) -> None:
    out = Path(args.out)
    rows = [r for r in (analyse(out, k, args.oracle_dir) for k in range(len(CONFIGS))) if r is not None]
    print("| configuration | arm | sweeps used | " + " | ".join(OBS) + " | tau_int (P_SS, P_ST, |L|) |")
    print("|---|---|---|" + "---|" * len(OBS) + "---|")
    for r in rows:
        for arm, label in (("ours", "ours"), ("ref", "reference CUDA"), ("oracle", "FP64 oracle (from ours)"),
                           ("oracle_chain", "FP64 oracle (own chain)")):
            if arm not in r:
                continue
            s = r[arm]
            taus = ", ".join(f"{s[o]['tau_int']:.1f}" for o in OBS)
            print(f"| {r['config']['name']} | {label} | {s[OBS[0]]['n']} | " +
                  " | ".join(_fmt(s[o]) for o in OBS) + f" | {taus} |")
    print()
    print("Pulls (ours - other) / combined error:")
    print()
    print("| configuration | vs | " + " | ".join(OBS) + " |")
    print("|---|---|" + "---|" * len(OBS))
    allp = []
    for r in rows:
        for key, label in (("pull_ref", "reference CUDA"), ("pull_oracle", "FP64 oracle (from ours)"),
                           ("pull_oracle_chain", "FP64 oracle (own chain)")):
            if key in r:
                allp += list(r[key].values())
                print(f"| {r['config']['name']} | {label} | " + " | ".join(f"{r[key][o]:+.2f}" for o in OBS) + " |")
    allp = np.asarray(allp)
    print()
    print(f"{len(allp)} pulls: {np.sum(np.abs(allp) <= 1)} within 1 sigma, {np.sum(np.abs(allp) <= 2)} within 2, "
          f"max |pull| {np.abs(allp).max():.2f}, chi^2/dof = {np.sum(allp ** 2):.1f}/{len(allp)}")
    if args.json:
        with open(args.json, "w") as f:
            json.dump(rows, f, indent=1)


def main(argv=None) -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["gpu", "oracle-one", "oracle-chain", "report"])
    ap.add_argument("--out", required=True)
    ap.add_argument("--sweeps", type=int, default=5000)
    ap.add_argument("--therm", type=int, default=500)
    ap.add_argument("--oracle-sweeps", type=int, default=200)
    ap.add_argument("--oracle-drop", type=int, default=40)
    ap.add_argument("--config", type=int, default=0)
    ap.add_argument("--only", type=int, nargs="*", default=None)
    ap.add_argument("--json", default=None)
    ap.add_argument("--oracle-dir", default=None, help="report: take the oracle arms from this directory")
    args = ap.parse_args(argv)
    {"gpu": _gpu, "oracle-one": _oracle_one, "oracle-chain": _oracle_chain, "report": _report}[args.mode](args)


if __name__ == "__main__":
    main()
