"""bench.py's host-side plumbing, without a GPU: the algorithmic-bytes model,
the workload naming and the DRAM-traffic figures it reads from the committed
ncu summaries (each tied to the kernel it was measured on)."""
import importlib.util
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_algorithmic_bytes_model():
    b = _bench()
    # read+write the updated link, the opposite-parity mu link and all (d-1) nu links of both parities
    assert [b.algorithmic_bytes_per_link_update(d) for d in (2, 3, 4)] == [40, 56, 72]
    N = (32, 32, 32, 32)
    assert b.volume(N) == 32 ** 4
    assert b.link_updates_per_step(N) == 32 ** 4 * 4 * 5  # 1 Metropolis + 4 OR passes


def test_workload_names():
    b = _bench()
    assert "32^4" in b.metric_for((32, 32, 32, 32))
    assert "24x24x24x48" in b.metric_for((24, 24, 24, 48))
    cfg = b.workload_config((32, 32, 32, 32))
    assert cfg["lattice"] == "32^4" and "metropolis" not in cfg
    cfg = b.workload_config((32, 32, 32, 32), delta=1.5, nhits=3)
    assert cfg["metropolis"] == {"delta": 1.5, "nhits": 3}


def test_traffic_figures_follow_the_profiled_kernel(tmp_path):
    b = _bench()
    quad, note = b.ncu_traffic_per_launch((32, 32, 32, 32), "k_update_quad")
    # the committed figure counts only while it was measured on the current kernel sources
    assert quad is None or 0 < quad < 37.75e6, note  # L2-resident: far below the algorithmic bytes
    assert b.ncu_traffic_per_launch((32, 32, 32, 32), "k_update_pair")[0] is None
    assert b.ncu_traffic_per_launch((40, 40, 40, 40), "k_update_quad")[0] is None
    f = tmp_path / "k_update_32x4_traffic.txt"
    f.write_text(f"# test\nkernel: k_update_quad\nsource_digest: {b.update_kernel_digest()}\n"
                 "dram_bytes_per_launch: 12345\n")
    assert b.ncu_traffic_per_launch((32, 32, 32, 32), "k_update_quad", tmp_path)[0] == 12345
    assert b.ncu_traffic_per_launch((32, 32, 32, 32), "k_update_pair", tmp_path)[0] is None
    f.write_text("kernel: k_update_quad\nsource_digest: 0000000000000000\ndram_bytes_per_launch: 12345\n")
    value, note = b.ncu_traffic_per_launch((32, 32, 32, 32), "k_update_quad", tmp_path)
    assert value is None and "stale" in note
    per_link, note = b.ncu_batch_traffic_per_link_sweep(32, 2)  # the layout the summary was made with
    assert per_link is not None and 0 < per_link < 72 * 5, note
    per_link, note = b.ncu_batch_traffic_per_link_sweep(64, 1)
    assert per_link is None and "32 MiB" in note
    assert b.KERNEL_OF_VARIANT[5] == "k_update_quad" and b.KERNEL_OF_VARIANT[1] == "k_update_pair"


def test_reference_arm_line():
    """`bench.py --impl reference` (the reference's own FP64 CPU code when
    oracle/_ref is built, else the oracle port) prints one JSON line with
    the contract's keys, on the host only."""
    import json
    import subprocess
    import sys
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--L", "8", "--steps", "2",
                        "--warmup", "3"], cwd=str(ROOT), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert "8^4" in line["metric"]
