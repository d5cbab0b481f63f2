"""CPU tests of the multi-GPU partitioning, including world-size-2 gloo ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from neural_wavelet_prt_demo_b200 import sharding


@pytest.mark.parametrize("height,world", [(1080, 1), (1080, 2), (1080, 8), (7, 3), (0, 4), (5, 8)])
def test_row_bands_tile_the_frame(height, world):
    bands = [sharding.row_band(height, r, world) for r in range(world)]
    assert bands[0][0] == 0 and bands[-1][1] == height
    for (a0, a1), (b0, b1) in zip(bands, bands[1:]):
        assert a1 == b0
    sizes = [e - b for b, e in bands]
    assert max(sizes) - min(sizes) <= 1


def test_request_assignment_is_a_balanced_partition():
    import random
    rnd = random.Random(0)
    res = [(256, 256), (512, 512), (1280, 720), (1920, 1080), (2560, 1440)]
    costs = [sharding.request_cost(*rnd.choice(res), rnd.choice([64, 128, 300])) for _ in range(200)]
    for world in (1, 2, 4, 8):
        plan = sharding.assign_requests(costs, world)
        flat = sorted(i for lst in plan for i in lst)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in lst) for lst in plan]
        assert max(loads) <= sum(costs) / world + max(costs)   # LPT bound
        assert plan == sharding.assign_requests(costs, world)   # deterministic


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = sharding.assign_requests(costs, world)[rank]
        band = sharding.row_band(1080, rank, world)
        # each rank reports the "elapsed time" of its own share; the max must come back everywhere
        t = float(sum(costs[i] for i in mine)) / 1e6
        tmax = sharding.max_over_ranks(t)
        q.put((rank, mine, band, t, tmax))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_cover_all_work_and_agree_on_the_max():
    world, costs = 2, [5, 9, 1, 7, 3, 3, 8]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert sorted(i for r in res for i in r[1]) == list(range(len(costs)))
    assert res[0][2] == (0, 540) and res[1][2] == (540, 1080)
    tmax = max(r[3] for r in res)
    assert all(r[4] == tmax for r in res)
