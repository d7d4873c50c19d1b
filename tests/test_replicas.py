"""Multi-rank host logic of the replica (independent chain) layout, run as
world_size-2 gloo process groups on the CPU: distinct Philox chains per
rank, max-over-ranks timing, and the gather of per-chain observables.
The per-rank chains are evolved with the FP64 oracle (the Philox counter
layout is shared with the kernels), so this needs no GPU."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank), OMP_NUM_THREADS="1")
    import datetime

    from latticeu1_b200 import replicas
    from oracle.oracle import Oracle
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    r, w, lr = replicas.world()
    assert (r, w, lr) == (rank, world, rank)
    chain = replicas.chain_id(r)
    o = Oracle(4, (4, 4, 4, 4), 1.0)
    lat = o.hot_start(99, 0, chain)
    p = 1
    for _ in range(2):
        p = o.update_philox(lat, 99, p, 1, 2, chain)
    ss, st = o.plaquette(lat)
    t_max = replicas.max_over_ranks(1.0 + rank)
    gathered = replicas.gather_observables([float(chain), ss.real, st.real])
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), lat=lat, t_max=t_max, gathered=np.array(gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas_gloo(tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    r0, r1 = np.load(tmp_path / "rank0.npz"), np.load(tmp_path / "rank1.npz")
    assert float(r0["t_max"]) == float(r1["t_max"]) == 2.0
    np.testing.assert_array_equal(r0["gathered"], r1["gathered"])
    g = r0["gathered"]
    assert g.shape == (2, 3) and list(g[:, 0]) == [0.0, 1.0]
    # chains differ (independent streams), and each equals a single-process rerun of its chain
    assert not np.allclose(r0["lat"], r1["lat"])
    from oracle.oracle import Oracle
    o = Oracle(4, (4, 4, 4, 4), 1.0)
    lat = o.hot_start(99, 0, 1)
    p = 1
    for _ in range(2):
        p = o.update_philox(lat, 99, p, 1, 2, 1)
    np.testing.assert_array_equal(lat, r1["lat"])


def test_chain_id_range():
    from latticeu1_b200 import replicas
    assert replicas.chain_id(3, 4, 2) == 14
    with pytest.raises(ValueError):
        replicas.chain_id(70000)
