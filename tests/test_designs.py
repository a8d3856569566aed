"""Many designs over the ranks of a job (eplace_b200/designs.py), on CPU: the
bin-count estimate equals the reference's choice on the golden designs, the
cost partition deals every design exactly once and balances the ranks, and
over gloo with world size 2 the per-rank results reach rank 0 in design
order, equal to a single-process run.  The placement callback here is a
stand-in computed on the host; the GPU one (designs.engine_batch) is
ep_run_batch, covered by the GPU tests of the batch runner."""
import datetime
import os
import random
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
from eplace_b200 import designs, synth  # noqa: E402
from tests.helpers import golden_netlist, load_golden  # noqa: E402


@pytest.mark.parametrize("name", ["stdcell_2k", "mixed_5k", "ref_smoke"])
def test_reference_bins_match_the_reference(name):
    g = load_golden(name)
    assert designs.reference_bins(golden_netlist(g)) == int(g["info_bins_x"]) == int(g["info_bins_y"])


def test_cost_grows_with_pins_and_bins():
    small, big = synth.standard_cell(2_000, seed=1), synth.standard_cell(20_000, seed=1)
    assert designs.design_cost(big) > designs.design_cost(small) > small.num_pins


@pytest.mark.parametrize("world", [1, 2, 3, 5, 8])
def test_partition_deals_each_design_once_and_balances(world):
    rng = random.Random(world)
    costs = [rng.uniform(1.0, 100.0) for _ in range(37)]
    share = designs.partition(costs, world)
    assert len(share) == world
    assert sorted(i for s in share for i in s) == list(range(len(costs)))
    loads = [sum(costs[i] for i in s) for s in share]
    assert max(loads) <= sum(costs) / world + max(costs)
    assert share == designs.partition(costs, world)  # deterministic
    assert all(s == sorted(s) for s in share)


def test_partition_longest_first_example():
    # 7, 5, 4, 3, 1 over 2 ranks: 7 -> r0 (7), 5 -> r1 (5), 4 -> r1 (9),
    # 3 -> r0 (10), 1 -> r1 (10)
    assert designs.partition([3, 7, 1, 5, 4], 2) == [[0, 1], [2, 3, 4]]


def _fake_place(netlists):
    return [dict(name=nl.name, pins=int(nl.num_pins), nets=int(nl.num_nets)) for nl in netlists]


def _batch():
    return [synth.standard_cell(n, seed=s) for n, s in ((300, 1), (1200, 2), (500, 3), (2000, 4), (800, 5))]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        out = designs.place_designs(_batch(), _fake_place, rank=rank, world=world, dist=dist)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def test_place_designs_gathers_to_rank0_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got[1] is None
    single = designs.place_designs(_batch(), _fake_place)
    assert got[0] == [single[i] for i in range(len(single))]
    assert [r["name"] for r in got[0]] == [nl.name for nl in _batch()]


def test_place_designs_local_share():
    nls = _batch()
    costs = [designs.design_cost(nl) for nl in nls]
    share = designs.partition(costs, 2)
    for rank in range(2):
        local = designs.place_designs(nls, _fake_place, rank=rank, world=2)
        assert sorted(local) == share[rank]
