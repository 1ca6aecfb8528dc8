"""Host side of the serving form, on the CPU: the seeded request stream, its
packing caps, replica partitioning across ranks (gloo, world size 2) and the
C ABI refusing to start a server without a device."""
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from kapsel3_b200 import _native as N
from kapsel3_b200.serve import max_packable, partition, serving_workload


def test_workload_is_seeded_and_capped():
    a = serving_workload(n_runs=40, sides=(32, 64), np_max=300, nsteps=5, seed=3)
    b = serving_workload(n_runs=40, sides=(32, 64), np_max=300, nsteps=5, seed=3)
    ra, rb = a["requests"], b["requests"]
    assert [r.arrival_s for r in ra] == [r.arrival_s for r in rb]
    assert all(np.array_equal(x.particles, y.particles) for x, y in zip(ra, rb))
    assert a["np_cap"][32] < 300 and a["np_cap"][32] >= 10
    gaps = np.diff([0.0] + [r.arrival_s for r in ra])
    assert np.all(gaps > 0)
    for r in ra:
        side = r.cfg.shape[0]
        assert side in (32, 64) and 1 <= r.cfg.n_particles <= a["np_cap"][side]
        x = r.particles[:, :3]
        assert np.all((x >= 0) & (x < side))
        d = x[:, None, :] - x[None, :, :]
        d -= np.rint(d / side) * side
        dist2 = (d ** 2).sum(-1) + np.eye(len(x)) * 1e9
        assert np.sqrt(dist2.min()) > 1.05 * 8.0


def test_packing_cap_below_excluded_volume_limit():
    n = max_packable(32, a=4.0, seed=0, tries=2000)
    # 300 spheres of diameter 8.4 cannot fit in 32^3; random sequential
    # addition saturates far below
    assert 10 <= n < 80


def _rank_main(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    reqs = list(range(23))
    mine = partition(reqs, rank, world)
    import torch
    t = torch.tensor([len(mine)], dtype=torch.int64)
    gathered = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(gathered, t)
    ids = [None] * world
    dist.all_gather_object(ids, mine)
    if rank == 0:
        flat = sorted(i for part in ids for i in part)
        out.put((flat, [int(g) for g in gathered]))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_partition_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    flat, counts = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert flat == list(range(23)) and counts == [12, 11]


def test_server_refuses_without_device():
    L = N.lib()
    n = __import__("ctypes").c_int()
    L.spm_device_count(n)
    if n.value > 0:
        pytest.skip("a device is visible")
    from kapsel3_b200.serve import Server
    with pytest.raises(N.SpmError, match="status 5"):
        Server()
