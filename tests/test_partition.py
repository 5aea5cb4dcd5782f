"""Config-4 systems split across ranks with no data-path collective: every rank
computes the same LPT partition; run as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from lima_b200.partition import lpt_partition, step_cost


def test_lpt_partition_properties():
    costs = [step_cost(n) for n in (30000, 1500, 9000, 12000, 2500, 28000, 4000, 7000)]
    parts = lpt_partition(costs, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / 3 + max(costs)   # LPT bound
    assert lpt_partition(costs, 3) == parts             # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = lpt_partition(costs, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    out[rank] = gathered
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_a_disjoint_cover():
    from lima_b200 import systems
    sys_sizes = [s for s in (1500, 2900, 30000, 11000, 6100, 1800, 25000)]
    costs = [step_cost(n) for n in sys_sizes]
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, costs, out), nprocs=world, start_method="spawn")
    views = [out[r] for r in range(world)]
    assert views[0] == views[1]
    parts = views[0]
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    assert not set(parts[0]) & set(parts[1])


def _c4_rank_main(rank, world, port, out):
    import hashlib

    from lima_b200 import systems
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    specs = systems.batch_specs(6, lo=1500, hi=3000)
    costs = [step_cost(sp[1], int(-(-sp[4] // 0.12)) ** 3) for sp in specs]
    mine = lpt_partition(costs, world)[rank]
    digests = {}
    for i in mine:                 # each rank generates only its own systems
        s = systems.batch_system(specs[i])
        digests[i] = (s.n, hashlib.sha256(s.pos.tobytes() + s.charge.tobytes()).hexdigest())
    gathered = [None] * world
    dist.all_gather_object(gathered, digests)
    out[rank] = gathered
    dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_c4_batch_split_over_two_gloo_ranks_matches_one_process():
    """The multi-rank batch: each rank partitions the same specs, generates only
    its share, and the union over ranks is exactly the batch one process makes
    (same systems, bit for bit), with no system on two ranks."""
    import hashlib

    from lima_b200 import systems
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_c4_rank_main, args=(world, port, out), nprocs=world, start_method="spawn")
    views = [out[r] for r in range(world)]
    assert views[0] == views[1]
    per_rank = views[0]
    assert not set(per_rank[0]) & set(per_rank[1])
    merged = {**per_rank[0], **per_rank[1]}
    whole = systems.batch_systems(6, lo=1500, hi=3000)
    assert sorted(merged) == list(range(len(whole)))
    for i, s in enumerate(whole):
        assert merged[i] == (s.n, hashlib.sha256(s.pos.tobytes() + s.charge.tobytes()).hexdigest())
