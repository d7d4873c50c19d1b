#!/usr/bin/env python
"""Throughput of the U(1) Monte Carlo hot path: link-updates/s at 32^4.

Workload (one step): one sweep of 1 Metropolis + 4 overrelaxation passes over a
32^4 lattice at beta = 1.0 (hot start) with the plaquette (spatial/temporal) +
Polyakov-loop measurement of the new configuration (taken from the sweep's
last pass), FP64 reductions.  One chain per GPU (independent chains, no
data-path collective: weak scaling).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--geom Nx,Ny,Nz,Nt | --L L] [--beta B] [--aniso XI]
                  [--workload update32|batched|multilevel]

`value` is device time (CUDA events on the lattice's stream, L2 flushed
between steps), `e2e` runs the same step through the C ABI with host buffers:
the configuration is imported from pinned host memory (FP64 angles, the
reference layout), swept, measured, and exported back every step.
`--impl reference` times the reference's own FP64 CPU update
(oracle/_ref/libu1ref.so, all host threads) on the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

L_DEFAULT = 32
BETA = 1.0
METROP, OVRN = 1, 4
DIMS = 4
METRIC = "link-updates/s at 32^4 (1 Metropolis + 4 OR per sweep)"
UNIT = "link-updates/s"
CLOCK_WINDOW_S = 1.5
HBM_WARM_S = 0.5  # minimum warm-up of each lattice beyond L2
E2E_CHAINS = 3  # chains in flight in the end-to-end leg


def algorithmic_bytes_per_link_update(d: int) -> int:
    """Per (parity, mu) phase: read+write the V/2 updated links, read the V/2
    opposite-parity mu links and all V(d-1) nu != mu links, 8 B per link:
    8Vd + 4V bytes for V/2 link updates = 16d + 8 B per link update."""
    return 16 * d + 8


def metric_for(N) -> str:
    return METRIC if tuple(N) == (32, 32, 32, 32) else METRIC.replace("32^4", geom_name(N))


def geom_name(N) -> str:
    return f"{N[0]}^4" if len(set(N)) == 1 else "x".join(str(n) for n in N)


def workload_config(N, beta: float = BETA, aniso: float = 1.0, delta: float = 0.0, nhits: int = 1) -> dict:
    name = geom_name(N)
    prop = "" if (delta == 0.0 and nhits == 1) else f" Metropolis delta={delta:.6g} nhits={nhits}"
    cfg = {
        "workload": f"U(1) Wilson 4D {name} beta={beta}" + (f" aniso={aniso}" if aniso != 1.0 else "") + prop +
                    " hot start; step = 1 Metropolis + 4 OR sweep + plaquette(SS/ST)+Polyakov measurement "
                    "taken from the sweep's last pass",
        "lattice": name, "beta": beta, "metrop": METROP, "ovrn": OVRN,
        "links": "float2 (cos,sin) even/odd SoA, 8 B/link",
        "l2": "flushed between timed steps (512 MiB device write)",
        "rng": "Philox4x32-10 keyed by (seed, site, mu, pass)",
    }
    if aniso != 1.0:
        cfg["aniso"] = aniso
    if prop:
        cfg["metropolis"] = {"delta": delta, "nhits": nhits}
    return cfg


def volume(N) -> int:
    return int(N[0]) * int(N[1]) * int(N[2]) * int(N[3])


def link_updates_per_step(N) -> int:
    return volume(N) * DIMS * (METROP + OVRN)


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: str):
        self.gpu = gpu
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def measured_peak() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


# update kernel of each variant (u1_lattice_set_variant)
KERNEL_OF_VARIANT = {1: "k_update_pair", 2: "k_update_pair_free", 3: "k_update", 4: "k_sweep_wave",
                     5: "k_update_quad"}


def ncu_batch_traffic_per_link_sweep(group_mb: int, lanes: int) -> tuple[float | None, str]:
    """DRAM bytes per link and sweep of the grouped batch from the committed
    ncu summary, and a note; None when there is no summary or it was measured
    on another layout (group size, lanes)."""
    p = ROOT / "profiles" / "k_batch_update_512chains.md"
    if not p.exists():
        return None, "no committed ncu summary"
    fields = {}
    for line in p.read_text().splitlines():
        if ":" in line and line.split(":", 1)[0] in ("dram_bytes_per_link_sweep", "layout_group_mb", "layout_lanes"):
            k, v = line.split(":", 1)
            fields[k] = float(v.split()[0])
    if "dram_bytes_per_link_sweep" not in fields:
        return None, "no committed ncu summary"
    if (fields.get("layout_group_mb"), fields.get("layout_lanes", 1.0)) != (float(group_mb), float(lanes)):
        return None, (f"the committed ncu summary was made with {fields.get('layout_group_mb'):.0f} MiB groups on "
                      f"{fields.get('layout_lanes', 1.0):.0f} lane(s); this run uses {group_mb} MiB on {lanes}")
    return fields["dram_bytes_per_link_sweep"], "ncu, profiles/k_batch_update_512chains.md"


# Sources the update kernels compile from: a committed ncu figure counts only
# while their digest matches the one recorded beside it.
UPDATE_KERNEL_SOURCES = ("u1_update.cuh", "u1_geom.cuh", "u1_cplx.cuh", "u1_philox.h")


def update_kernel_digest() -> str:
    import hashlib
    h = hashlib.sha256()
    for name in UPDATE_KERNEL_SOURCES:
        h.update((ROOT / "latticeu1_b200" / "csrc" / name).read_bytes())
    return h.hexdigest()[:16]


def ncu_traffic_per_launch(N, kernel: str, profiles: Path | None = None) -> tuple[float | None, str]:
    """DRAM bytes per launch of `kernel` from the committed ncu summary for
    this geometry, and a note; None when there is no summary for this
    geometry and kernel or it was made from other kernel sources."""
    p = (profiles or ROOT / "profiles") / f"k_update_{geom_name(N).replace('^4', 'x4')}_traffic.txt"
    if not p.exists():
        return None, f"no committed ncu summary for {geom_name(N)}"
    fields = {k.strip(): v.strip() for k, v in (line.split(":", 1) for line in p.read_text().splitlines()
                                                if ":" in line and not line.startswith("#"))}
    if fields.get("kernel") != kernel or "dram_bytes_per_launch" not in fields:
        return None, f"the committed ncu summary is for {fields.get('kernel')}, not {kernel}"
    if fields.get("source_digest") != update_kernel_digest():
        return None, "the committed ncu summary was made from other update-kernel sources (stale)"
    return float(fields["dram_bytes_per_launch"].split()[0]), f"ncu, profiles/{p.name}"


# ------------------------------------------------------------------ CPU baselines
def cpu_reference_rate(N, beta: float, aniso: float, budget_s: float, min_sweeps: int = 1) -> dict:
    """The reference's own FP64 CPU metropolis + overrelaxation (oracle/_ref),
    OpenMP over all host threads, on the bench geometry; bounded by budget_s.
    Falls back to the oracle port (oracle/u1_oracle.cpp) if _ref is absent."""
    import numpy as np
    from oracle.oracle import Oracle, Ref
    threads = os.cpu_count() or 1
    lat = np.random.default_rng(1).uniform(0, 2 * np.pi, volume(N) * 4)
    if Ref.available():
        ref = Ref(4, tuple(N), beta, aniso, METROP, OVRN)
        ref.seed_cpu(threads, 1234)
        kind = "reference"

        def sweep():
            ref.metropolis(lat)
            for _ in range(OVRN):
                ref.overrelax(lat)
    else:
        o = Oracle(4, tuple(N), beta, aniso)
        kind = "port"
        state = {"p": 0}

        def sweep():
            state["p"] = o.update_philox(lat, 1234, state["p"], METROP, OVRN)
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    n = 0
    t0 = time.perf_counter()
    while True:
        sweep()
        n += 1
        el = time.perf_counter() - t0
        if n >= min_sweeps and el >= budget_s:
            break
        if el + el / n > 3 * budget_s:
            break
    rate = n * link_updates_per_step(N) / el
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{n} full sweeps (1 Metropolis + 4 OR) of the {geom_name(N)} lattice, {el:.1f} s, FP64"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    N, beta, aniso = geometry(args)
    import numpy as np
    from oracle.oracle import Oracle, Ref
    threads = os.cpu_count() or 1
    lat = np.random.default_rng(1).uniform(0, 2 * np.pi, volume(N) * 4)
    if Ref.available():
        ref = Ref(4, tuple(N), beta, aniso, METROP, OVRN)
        ref.seed_cpu(threads, 1234)
        kind = "reference"

        def step():
            ref.metropolis(lat)
            for _ in range(OVRN):
                ref.overrelax(lat)
            ref.plaquette(lat)
            ref.polyakov(lat)
    else:
        o = Oracle(4, tuple(N), beta, aniso)
        kind = "port"
        st = {"p": 0}

        def step():
            st["p"] = o.update_philox(lat, 1234, st["p"], METROP, OVRN)
            o.plaquette(lat)
            o.polyakov(lat)
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    el = time.perf_counter() - t0
    rate = args.steps * link_updates_per_step(N) / el
    line = {
        "impl": "reference", "metric": metric_for(N), "value": rate, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(N, beta, aniso),
        "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{args.steps} timed full sweeps of {geom_name(N)} (1 Met + 4 OR) + CPU "
                                   "plaquette and Polyakov, FP64, OpenMP"},
        "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ our arm
def hbm_resident_line(ctx, L: int, steps: int, warmup: int, flush, peak: float, gpu: str) -> dict:
    """The measured step (1 Metropolis + 4 OR + measurement) on an L^4
    lattice larger than L2, tuned as the headline lattice: device time per
    step (CUDA events, L2 flushed between steps), link-updates/s and the
    update kernel's algorithmic bandwidth against the measured HBM peak.
    Warm-up runs for at least HBM_WARM_S of steps (clock ramp after the
    lighter work before it); the clocks are sampled over the timed steps and
    CLOCK_WINDOW_S more of the same step."""
    import torch

    from latticeu1_b200 import Lattice, Rng
    N = (L,) * 4
    lat = Lattice(ctx, DIMS, N, BETA)
    stream = torch.cuda.Stream()
    lat.set_stream(stream.cuda_stream)
    rng = Rng(ctx, 4321)
    obs = torch.zeros(6, dtype=torch.float64, device="cuda")
    with torch.cuda.stream(stream):
        lat.hot_start(rng)
        t0, n = time.perf_counter(), 0
        while n < warmup or time.perf_counter() - t0 < HBM_WARM_S:
            flush.zero_()
            lat.update_measure(rng, METROP, OVRN, obs.data_ptr())
            n += 1
            if n % 20 == 0:
                stream.synchronize()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
        clocks = ClockSampler(gpu)
        clocks.start()
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(stream)
            lat.update_measure(rng, METROP, OVRN, obs.data_ptr())
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        while time.perf_counter() - t1 < CLOCK_WINDOW_S:
            for _ in range(10):
                flush.zero_()
                lat.update_measure(rng, METROP, OVRN, obs.data_ptr())
            stream.synchronize()
        clk = clocks.stop()
    ms = sum(e[0].elapsed_time(e[1]) for e in ev) / steps
    launches = 2 * DIMS * (METROP + OVRN)
    alg = algorithmic_bytes_per_link_update(DIMS) * volume(N) // 2
    achieved = alg / (ms * 1e-3 / launches) / 1e9
    line = {"lattice": geom_name(N), "link_bytes": lat.nlinks * 8, "ms_per_step": ms,
            "value": link_updates_per_step(N) / (ms * 1e-3), "unit": UNIT, "achieved_gbs": achieved,
            "frac": achieved / peak, "update_variant": Lattice.VARIANTS.get(lat.variant, str(lat.variant)),
            "update_block": lat.block, "steps": steps, "warmup_steps": n, "clocks": clk}
    lat.close()
    rng.close()
    return line


def pcie_both_gbs(nbytes: int, reps: int = 10) -> float:
    """Pinned host <-> device copy bandwidth per direction with both
    directions busy at once (one H2D and one D2H of `nbytes` on two streams),
    in GB/s: the ceiling of the end-to-end leg, which moves one
    configuration each way per step."""
    import torch
    n = nbytes // 8
    h = [torch.empty(n, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    d = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def both():
        with torch.cuda.stream(s1):
            d[0].copy_(h[0], non_blocking=True)
        with torch.cuda.stream(s2):
            h[1].copy_(d[1], non_blocking=True)

    both()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        both()
    torch.cuda.synchronize()
    return nbytes * reps / (time.perf_counter() - t0) / 1e9


def e2e_rate(ctx, lat, rng, stream, N, beta, aniso, args, rank, world):
    """End-to-end rate through the C ABI with host buffers (see the comment
    below); returns (link-updates/s, steps, observables finite)."""
    import torch

    from latticeu1_b200 import Lattice, Rng, replicas
    lu = link_updates_per_step(N)
    # e2e: C ABI with host buffers.  Three chains in flight (triple
    # buffering: host-to-device copy, sweep, device-to-host copy), each on
    # its own stream with its FP64 configuration in pinned host memory; every
    # step takes one chain through import (H2D), the measured sweep, the D2H
    # read of its 6 observables and the export of its configuration (D2H), so
    # one chain's host-to-device copy overlaps another's sweep and a third's
    # device-to-host copy (PCIe is full duplex).  Each chain's configuration
    # makes the round trip through host memory every time it steps.
    lats, rngs, streams = [lat], [rng], [stream]
    for c in range(1, E2E_CHAINS):
        lc = Lattice(ctx, DIMS, N, beta, aniso)
        lc.set_metropolis(args.delta, args.nhits)
        lc.set_variant(lat.variant)
        lc.set_block(lat.block)
        sc = torch.cuda.Stream()
        lc.set_stream(sc.cuda_stream)
        rc_ = Rng(ctx, 1234)
        rc_.set_chain(replicas.chain_id(c * world + rank))
        lc.hot_start(rc_)
        lats.append(lc)
        rngs.append(rc_)
        streams.append(sc)
    hosts = [torch.empty(lat.nlinks, dtype=torch.float64, pin_memory=True) for _ in range(E2E_CHAINS)]
    obs_dev = torch.zeros((E2E_CHAINS, 6), dtype=torch.float64, device="cuda")
    obs_host = torch.zeros((E2E_CHAINS, 6), dtype=torch.float64, pin_memory=True)
    for lc, h in zip(lats, hosts):
        lc.export_angles(h)

    def e2e_step(k):
        c = k % E2E_CHAINS
        lats[c].import_angles_async(hosts[c])
        lats[c].update_measure(rngs[c], METROP, OVRN, obs_dev[c].data_ptr())
        with torch.cuda.stream(streams[c]):
            obs_host[c].copy_(obs_dev[c], non_blocking=True)  # D2H of the step's observables
        lats[c].export_angles_async(hosts[c])

    for k in range(2 * E2E_CHAINS):
        e2e_step(k)
    for lc in lats:
        lc.synchronize()
    e2e_steps = E2E_CHAINS * max(2, min(args.steps, 15))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        e2e_step(k)
    for lc in lats:
        lc.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_value = world * e2e_steps * lu / replicas.max_over_ranks(e2e_s)
    e2e_obs_ok = bool(torch.isfinite(obs_host).all())
    for lc, rc_ in zip(lats[1:], rngs[1:]):
        lc.close()
        rc_.close()
    return e2e_value, e2e_steps, e2e_obs_ok


def run_ours(args) -> None:
    import numpy as np
    import torch

    from latticeu1_b200 import replicas
    rank, world, local = replicas.world()
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    from latticeu1_b200 import Context, Lattice, Rng, launch_count

    N, beta, aniso = geometry(args)
    ctx = Context(local)
    lat = Lattice(ctx, DIMS, N, beta, aniso)
    lat.set_metropolis(args.delta, args.nhits)
    if args.variant:  # otherwise the tuner chooses at the first update
        lat.set_variant(args.variant)
        lat.set_block(args.block)
    stream = torch.cuda.Stream()
    lat.set_stream(stream.cuda_stream)
    rng = Rng(ctx, 1234)
    rng.set_chain(replicas.chain_id(rank))  # independent replica per rank
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    obs = torch.zeros((args.steps + args.warmup, 6), dtype=torch.float64, device="cuda")
    lu = link_updates_per_step(N)

    with torch.cuda.stream(stream):
        lat.hot_start(rng)
        for w in range(args.warmup):
            flush.zero_()
            lat.update_measure(rng, METROP, OVRN, obs[w].data_ptr())
        stream.synchronize()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        props = torch.cuda.get_device_properties(local)
        uuid = str(getattr(props, "uuid", ""))
        clocks = ClockSampler(("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or str(local)))
        clocks.start()
        n0 = launch_count()
        t_wall = time.perf_counter()
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            lat.update_measure(rng, METROP, OVRN, obs[args.warmup + k].data_ptr())
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t_wall = time.perf_counter() - t_wall
        launches = launch_count() - n0
        # The timed region lasts only tens of ms, shorter than nvidia-smi's
        # 200 ms sampling period: keep the same step running (untimed) for
        # CLOCK_WINDOW_S so the sampler sees this load.
        t1 = time.perf_counter()
        while time.perf_counter() - t1 < CLOCK_WINDOW_S:
            for _ in range(20):
                lat.update_measure(rng, METROP, OVRN, obs[0].data_ptr())
            stream.synchronize()
        clk = clocks.stop()
        if clk is not None:
            clk["window"] = f"timed region + {CLOCK_WINDOW_S:.1f} s of the same step"
        # the same sweep without the measurement (not the headline; it shows what the measurement costs)
        ev2 = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)]
        lat.update(rng, METROP, OVRN)
        for k in range(args.steps):
            flush.zero_()
            ev2[k][0].record(stream)
            lat.update(rng, METROP, OVRN)
            ev2[k][1].record(stream)
        torch.cuda.synchronize()
        sweep_only_ms = sum(e[0].elapsed_time(e[1]) for e in ev2) / args.steps
    step_ms = sum(e[0].elapsed_time(e[1]) for e in ev)
    upd_ms = step_ms  # the measurement runs inside the sweep's last phase
    step_ms_max = replicas.max_over_ranks(step_ms)
    value = world * args.steps * lu / (step_ms_max * 1e-3)

    if args.no_e2e:
        e2e_value, e2e_steps, e2e_obs_ok = None, 0, None
    else:
        e2e_value, e2e_steps, e2e_obs_ok = e2e_rate(ctx, lat, rng, stream, N, beta, aniso, args, rank, world)
    bytes_cfg = lat.nlinks * 8
    pcie_gbs = None if e2e_value is None else pcie_both_gbs(bytes_cfg)

    ob = obs[args.warmup:].cpu().numpy()
    per_chain = replicas.gather_observables([float(ob[:, 0].mean()), float(ob[:, 2].mean())])
    if rank == 0:
        peak, peak_kind = measured_peak()
        upd_launches = 2 * DIMS * (METROP + OVRN)  # the last one also measures
        avg_launch_s = upd_ms * 1e-3 / (args.steps * upd_launches)
        alg_bytes = algorithmic_bytes_per_link_update(DIMS) * volume(N) // 2
        achieved = alg_bytes / avg_launch_s / 1e9
        traffic, traffic_note = ncu_traffic_per_launch(N, KERNEL_OF_VARIANT.get(lat.variant, "k_update"))
        l2_bytes = torch.cuda.get_device_properties(local).L2_cache_size
        resident = bytes_cfg < l2_bytes  # float2 links: 8 B each, as the FP64 angles
        line = {
            "metric": metric_for(N), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(N, beta, aniso, args.delta, args.nhits),
            "roofline": {"bound": "hbm",
                         "kernel": KERNEL_OF_VARIANT.get(lat.variant, "k_update") +
                                   " (one (parity,mu) phase; step average)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_note,
                         "dram_frac": (traffic / alg_bytes) if traffic else None,
                         "residency": (f"L2: the {bytes_cfg / 2 ** 20:.1f} MiB of links stay in the "
                                       f"{l2_bytes / 2 ** 20:.0f} MiB L2 across a sweep's phases, so `frac` is "
                                       "algorithmic bytes over the HBM peak while DRAM moves only `dram_frac` "
                                       "of them; `hbm_resident` measures lattices beyond L2")
                         if resident else "HBM: the links exceed L2",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "avg_launch_us": avg_launch_s * 1e6},
            "e2e": None if e2e_value is None else {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_cfg,
                    "d2h_bytes_per_step": bytes_cfg + 48, "steps": e2e_steps, "chains_in_flight": E2E_CHAINS,
                    "observables_finite": e2e_obs_ok,
                    # each step moves one configuration each way: at most one step per
                    # bytes_cfg / (per-direction bandwidth with both directions busy)
                    "roofline": {"bound": "pcie", "pcie_gbs_per_direction": pcie_gbs,
                                 "bound_value": world * lu * pcie_gbs * 1e9 / bytes_cfg,
                                 "frac": e2e_value / (world * lu * pcie_gbs * 1e9 / bytes_cfg)},
                    "path": "per step, one of three chains (own stream, own pinned host FP64 configuration): "
                            "u1_lattice_import_angles_async + u1_update_measure + D2H of the 6 observables + "
                            "u1_lattice_export_angles_async; host wall clock from a synchronised start to "
                            "u1_lattice_synchronize of every chain"},
            "gpu_launches": int(launches),
            "update_variant": Lattice.VARIANTS.get(lat.variant, str(lat.variant)),
            "update_block": lat.block,
            "clocks": clk,
            "wall_s_timed_region": t_wall,
            "update_ms_per_step": upd_ms / args.steps,
            "sweep_only_ms_per_step": sweep_only_ms,
            "observables": {"plaq_ss_re": float(ob[:, 0].mean()), "plaq_st_re": float(ob[:, 2].mean()),
                            "abs_L": float(np.abs(ob[:, 4] + 1j * ob[:, 5]).mean()),
                            "per_chain_plaq_ss_st": per_chain},
        }
        if world == 1 and args.hbm_check and args.delta == 0.0 and args.nhits == 1:
            gpu_id = ("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or str(local))
            hb = [hbm_resident_line(ctx, L, max(10, min(args.steps, 20)), max(10, args.warmup), flush, peak, gpu_id)
                  for L in args.hbm_check]
            line["hbm_resident"] = {"lattices": hb, "note": "the same measured step on lattices beyond the "
                                                            "126 MB L2, each tuned on its first update"}
        if world == 1 and not args.no_cpu_baseline and args.delta == 0.0 and args.nhits == 1:
            # the reference's CPU update has only the whole-circle single-hit proposal
            line["cpu_baseline"] = cpu_reference_rate(N, beta, aniso, args.cpu_budget)
        print(json.dumps(line), flush=True)
    lat.close()
    rng.close()
    if dist:
        dist.destroy_process_group()


def run_multilevel(args) -> None:
    """Multilevel Polyakov correlator, 24^3 x 32 at beta = 0.95, level-2
    slabs of thickness 2 and level-4 slabs of 4, 1 Metropolis + 4 OR per
    sub-update, analytic multihit on temporal links.  A step is one level-4
    iteration (k4 = 1 update + n2 level-2 sub-updates + T4 accumulation);
    the value is level-2 sub-updates per second.  The full configuration
    (n4 = 100, n2 = 200) is timed by extrapolating the per-step time; the
    single-level multihit estimator (Poly2) is timed beside it."""
    import torch

    from latticeu1_b200 import Context, Lattice, Rng
    ctx = Context(0)
    lat = Lattice(ctx, 4, (24, 24, 24, 32), 0.95)
    if args.variant:  # otherwise the tuner chooses at the first update
        lat.set_variant(args.variant)
        lat.set_block(args.block)
    rng = Rng(ctx, 1234)
    lat.hot_start(rng)
    for _ in range(50):
        lat.update(rng, METROP, OVRN)
    n2 = args.n2
    lat.multilevel(rng, 1, 1, 2, 1, METROP, OVRN)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    c_ml = lat.multilevel(rng, args.steps, 1, n2, 1, METROP, OVRN)
    el = time.perf_counter() - t0
    sub = args.steps * n2
    t1 = time.perf_counter()
    sl = []
    while time.perf_counter() - t1 < el:
        lat.update(rng, METROP, OVRN)
        sl.append(lat.poly_corr(True).real)
    import numpy as np
    sl = np.asarray(sl)
    nb = 20 if len(sl) >= 40 else max(2, len(sl) // 2)
    bins = sl[: len(sl) // nb * nb].reshape(nb, -1, sl.shape[1]).mean(axis=1)
    loo = (bins.sum(axis=0) - bins) / (nb - 1)
    sl_err = np.sqrt((nb - 1) / nb * ((loo - loo.mean(axis=0)) ** 2).sum(axis=0))
    line = {"metric": "multilevel level-2 sub-updates/s (24^3x32, beta=0.95)", "value": sub / el,
            "unit": "sub-updates/s", "n_gpus": 1, "steps": args.steps, "warmup": 1,
            "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "dtype": "f32+f64 accum",
            "data": "synthetic", "config": {"workload": "MultiLevel(n4=steps, k4=1, n2, k2=1, metrop=1, ovrn=4)",
                                           "lattice": "24^3x32", "beta": 0.95, "n2": n2},
            "full_config_seconds_n4_100_n2_200": el / sub * 100 * 200,
            "update_variant": Lattice.VARIANTS.get(lat.variant, str(lat.variant)), "update_block": lat.block,
            "C_r_multilevel": [float(c.real) for c in c_ml],
            "single_level_equal_time": {
                "measurements": len(sl), "C_r_mean": [float(v) for v in sl.mean(axis=0)],
                "C_r_err": [float(v) for v in sl_err],
                "note": "Poly2(multihit) after every sweep for the multilevel call's wall time, 20-bin "
                        "jackknife; multilevel errors over configurations: tests/multilevel_compare.py"}}
    print(json.dumps(line), flush=True)


def batched_geoms(seed: int = 20240):
    """512 chains: 256 x 16^4, 128 x 12^4, 128 x 16^3x32, beta ~ U[0.8, 1.2]
    from a seeded generator."""
    import numpy as np
    r = np.random.default_rng(seed)
    shapes = [(16, 16, 16, 16)] * 256 + [(12, 12, 12, 12)] * 128 + [(16, 16, 16, 32)] * 128
    return [(4, s, float(b)) for s, b in zip(shapes, r.uniform(0.8, 1.2, len(shapes)))]


def run_batched(args) -> None:
    """Config: 512 independent chains advanced together (one launch per
    (parity, mu) phase for all of them, whole sweep + per-chain measurement
    captured in one CUDA graph), after u1_batch_tune has chosen the
    chain-group size and each group's kernel and block size.  A step is one sweep (1 Metropolis + 4 OR)
    of every chain plus its plaquette/Polyakov measurement.  The comparator
    advances the same chains one by one (one lattice object per chain, its
    own graph-captured sweep), as a caller of the single-lattice API would."""
    import numpy as np
    import torch

    from latticeu1_b200 import Batch, Context, Lattice, Rng, launch_count
    ctx = Context(0)
    geoms = batched_geoms()
    stream = torch.cuda.Stream()
    b = Batch(ctx, geoms, seed=1234)
    b.set_stream(stream.cuda_stream)
    t_tune = time.perf_counter()
    group_mb = b.tune()  # group size and per-group kernel / block size (cached in $U1_RESOURCE_PATH if set)
    t_tune = time.perf_counter() - t_tune
    layout = b.layout()
    links = b.total_links
    lu = links * (METROP + OVRN)
    flush = torch.empty(512 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    with torch.cuda.stream(stream):
        b.hot_start()
        for _ in range(args.warmup):
            b.update(METROP, OVRN, measure=True)
            b.update(METROP, OVRN, measure=False)
        stream.synchronize()

        def timed(measure: bool, steps: int) -> float:
            ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(steps)]
            for k in range(steps):
                flush.zero_()
                ev[k][0].record(stream)
                b.update(METROP, OVRN, measure=measure)
                ev[k][1].record(stream)
            torch.cuda.synchronize()
            return sum(e[0].elapsed_time(e[1]) for e in ev)

        n0 = launch_count()
        step_ms = timed(True, args.steps)
        launches = launch_count() - n0
        upd_ms = timed(False, args.steps)
        obs = b.results_raw()
    value = args.steps * lu / (step_ms * 1e-3)
    phases = 2 * DIMS * (METROP + OVRN)
    avg_launch_s = upd_ms * 1e-3 / (args.steps * phases)
    alg_bytes = algorithmic_bytes_per_link_update(DIMS) * links // (2 * DIMS)
    achieved = alg_bytes / avg_launch_s / 1e9
    peak, peak_kind = measured_peak()
    per_link, traffic_note = ncu_batch_traffic_per_link_sweep(group_mb, b.lanes)
    traffic = per_link * links / phases if per_link is not None else None

    # comparator: the same chains one at a time through the single-lattice API
    nseq = len(geoms)
    lats, rngs = [], []
    for c, (d, N, beta) in enumerate(geoms[:nseq]):
        lat = Lattice(ctx, d, N, beta)
        lat.set_stream(stream.cuda_stream)
        lat.set_variant(1)
        rng = Rng(ctx, 1234)
        rng.set_chain(c)
        lats.append(lat)
        rngs.append(rng)
    out = torch.zeros((nseq, 6), dtype=torch.float64, device="cuda")
    with torch.cuda.stream(stream):
        for lat, rng in zip(lats, rngs):
            lat.hot_start(rng)
            lat.update_measure(rng, METROP, OVRN, out[0].data_ptr())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        seq_steps = max(1, min(args.steps, 5))
        e0.record(stream)
        for _ in range(seq_steps):
            for k, (lat, rng) in enumerate(zip(lats, rngs)):
                lat.update_measure(rng, METROP, OVRN, out[k].data_ptr())
        e1.record(stream)
        torch.cuda.synchronize()
        seq_ms = e0.elapsed_time(e1)
    seq_value = seq_steps * lu / (seq_ms * 1e-3)
    for lat in lats:
        lat.close()
    absL = np.abs(obs[:, 4] + 1j * obs[:, 5])
    line = {
        "metric": "link-updates/s, 512-chain batch (1 Metropolis + 4 OR per sweep, per-chain measurement)",
        "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "batched: 256x16^4 + 128x12^4 + 128x16^3x32 chains, beta~U[0.8,1.2] "
                               "(seeded), hot starts, 1 Met + 4 OR sweep + per-chain plaquette/Polyakov",
                   "chains": len(geoms), "links": links, "bytes": links * 8,
                   "l2": "flushed between timed steps (512 MiB device write)"},
        "roofline": {"bound": "hbm", "kernel": "k_batch_update (one (parity,mu) phase over all chains)",
                     "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_note,
                     "algorithmic_bytes_per_launch": alg_bytes,
                     "avg_launch_us": avg_launch_s * 1e6},
        "update_only_ms_per_step": upd_ms / args.steps,
        "tuned": {"group_mb": group_mb, "lanes": b.lanes, "groups": len(layout), "seconds": t_tune,
                  "kernels": {f"{Batch.VARIANTS.get(v, v)}@{t}": sum(1 for g in layout if (g[2], g[3]) == (v, t))
                              for v, t in sorted({(g[2], g[3]) for g in layout})}},
        "gpu_launches": int(launches),
        "one_by_one": {"value": seq_value, "unit": UNIT, "steps": seq_steps,
                       "path": "one Lattice per chain, graph-captured u1_update_measure each, same stream"},
        "speedup_vs_one_by_one": value / seq_value,
        "observables": {"plaq_st_re_mean": float(obs[:, 2].mean()), "absL_mean": float(absL.mean())},
    }
    print(json.dumps(line), flush=True)
    b.close()


def run_kernels(args) -> None:
    """The library's other kernels, one line of evidence each: every entry is
    one public call, timed with CUDA events over args.steps calls after
    args.warmup untimed ones (synchronous calls include their small result
    copies), with its algorithmic bytes (each input and output array once)
    and the fraction of the measured HBM bandwidth that implies.  32^4 at
    beta = 1 unless stated; the ncu summary of the same command gives each
    kernel's own duration and DRAM bytes."""
    import numpy as np
    import torch

    from latticeu1_b200 import Context, Lattice, Rng, launch_count
    from latticeu1_b200.action import WilsonAction
    from latticeu1_b200.lattice import convert_order
    ctx = Context(0)
    stream = torch.cuda.Stream()
    peak, peak_kind = measured_peak()
    N = (32, 32, 32, 32)
    V = volume(N)
    lat = Lattice(ctx, 4, N, 1.0)
    lat.set_stream(stream.cuda_stream)
    rng = Rng(ctx, 77)
    Vs, R = V // N[3], N[0] // 2
    nl = lat.nlinks
    rows = []

    def timed(name, kernels, fn, alg_bytes, note=""):
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            ts = []
            for _ in range(args.steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                fn()
                e1.record(stream)
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1) * 1e3)
        us = float(np.median(ts))
        gbs = alg_bytes / (us * 1e-6) / 1e9
        rows.append({"call": name, "kernels": kernels, "us_median": us, "algorithmic_bytes": int(alg_bytes),
                     "achieved_gbs": gbs, "frac_of_peak": gbs / peak, **({"note": note} if note else {})})

    n0 = launch_count()
    lat.hot_start(rng)
    timed("u1_hot_start", "k_hot_start", lambda: lat.hot_start(rng), 8 * nl, "writes every link")
    for _ in range(20):
        lat.update(rng, 1, 4)
    timed("u1_measure (plaquette + Polyakov)", "k_measure", lambda: lat.measure(), 8 * nl,
          "reads every link once; 48 B result copy")
    timed("u1_poly_corr(multihit=0)", "k_poly_field<4,0>, k_poly_corr", lambda: lat.poly_corr(False),
          8 * V + 16 * Vs, "temporal links, then the P field")
    timed("u1_poly_corr(multihit=1)", "k_poly_field<4,1>, k_poly_corr", lambda: lat.poly_corr(True),
          8 * nl + 16 * Vs, "every link (staples of the temporal links), then the P field")
    th = torch.empty(nl, dtype=torch.float64, device="cuda")
    timed("u1_lattice_export_angles (device FP64)", "k_export_angles", lambda: lat.export_angles(th), 16 * nl)
    timed("u1_lattice_import_angles (device FP64)", "k_import_angles", lambda: lat.import_angles(th), 16 * nl)
    timed("u1_convert_order (EO -> NO, FP64)", "k_convert_order<1>", lambda: convert_order(th, 4, N, True),
          16 * nl)
    timed("u1_plaquette_fields (space-time)", "k_plaquette_fields<1>", lambda: lat.plaquette_fields(True),
          8 * nl + 96 * V, "reads every link, writes 6 complex FP64 per site")
    S4 = WilsonAction(4, N, 1.0)
    t4 = th.to(torch.float32).reshape(1, -1)
    timed("u1_wilson_action (4D 32^4, float32, batch 1)", "k_action<4,float>, k_action_finish",
          lambda: S4(t4), 4 * nl)
    t4g = t4.clone().requires_grad_(True)
    timed("u1_wilson_action + u1_wilson_action_grad (4D 32^4)", "k_action, k_action_grad<4,float>",
          lambda: S4(t4g).sum().backward(), 4 * nl * 3, "action reads theta; adjoint reads theta, writes grad")
    L2d, B2d = 32, 1024
    S2 = WilsonAction(2, (L2d, 0, 0, L2d), 6.0)
    t2 = torch.rand((B2d, 2 * L2d * L2d), device="cuda") * 6.2831853
    timed("u1_wilson_action (2D 32^2, float32, batch 1024)", "k_action<2,float>, k_action_finish",
          lambda: S2(t2), 4 * t2.numel())
    launches = launch_count() - n0
    line = {"metric": "per-call device time and algorithmic bandwidth of the non-update kernels",
            "value": None, "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "data": "synthetic", "dtype": "f32/f64",
            "config": {"workload": "kernels: one public call per entry, 32^4 beta = 1 after 20 sweeps unless stated"},
            "peak_gbs": peak, "peak_kind": peak_kind, "gpu_launches": int(launches), "entries": rows}
    print(json.dumps(line), flush=True)
    lat.close()


def geometry(args):
    """(N, beta, aniso) of the update workload: --geom Nx,Ny,Nz,Nt or --L for L^4."""
    if args.geom:
        N = tuple(int(v) for v in args.geom.split(","))
        if len(N) != 4:
            raise SystemExit("--geom needs four extents Nx,Ny,Nz,Nt")
    else:
        N = (args.L,) * 4
    return N, args.beta, args.aniso


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--L", type=int, default=L_DEFAULT, help="L^4 lattice (update workload)")
    ap.add_argument("--geom", type=str, default=None, help="Nx,Ny,Nz,Nt instead of --L (update workload)")
    ap.add_argument("--beta", type=float, default=BETA)
    ap.add_argument("--aniso", type=float, default=1.0)
    ap.add_argument("--delta", type=float, default=0.0,
                    help="Metropolis proposal half-width (0: the reference's whole-circle proposal)")
    ap.add_argument("--nhits", type=int, default=1, help="Metropolis hits per link and pass")
    ap.add_argument("--variant", type=int, default=0,
                    help="update kernel variant (0: tuned; 1 pair32, 2 pair, 3 single, 4 wave, 5 quad)")
    ap.add_argument("--block", type=int, default=256, help="threads per block with --variant")
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU baseline sampling")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--hbm-check", type=lambda v: [int(x) for x in v.split(",") if x], default=[48, 64],
                    help="L^4 lattices beyond L2 timed beside the headline (empty: none)")
    ap.add_argument("--workload", choices=["update32", "multilevel", "batched", "kernels"], default="update32")
    ap.add_argument("--n2", type=int, default=200, help="level-2 sub-updates per step (multilevel)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "multilevel":
        run_multilevel(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "kernels":
        run_kernels(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
