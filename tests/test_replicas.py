"""Replica parallelism host logic (mpsw/replicas.py) on CPU with the gloo backend, world size 2:
shards cover every member exactly once, the job time is the slowest rank's, and gathered
members come back in member order on every rank."""
import socket

import pytest

torch = pytest.importorskip('torch')
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from mpsw import replicas  # noqa: E402


@pytest.mark.parametrize('total', [0, 1, 7, 64])
@pytest.mark.parametrize('world', [1, 2, 3, 8])
def test_shards_cover_members_once(total, world):
    seen = []
    for r in range(world):
        s, c = replicas.shard(total, r, world)
        seen.extend(range(s, s + c))
    assert seen == list(range(total))
    sizes = [replicas.shard(total, r, world)[1] for r in range(world)]
    assert max(sizes) - min(sizes) <= 1


def test_bad_shard_request_raises():
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def test_single_process_is_identity():
    x = torch.arange(6.0).reshape(2, 3)
    assert replicas.max_over_ranks(3.5) == 3.5
    assert torch.equal(replicas.gather_members(x, 3), x)
    assert replicas.rank_world() == (0, 1)


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, total, q):
    try:
        dist.init_process_group('gloo', init_method='tcp://127.0.0.1:%d' % port, rank=rank,
                                world_size=world)
        start, count = replicas.shard(total, rank, world)
        # member j of the job holds the column [j, 100 + j]
        local = torch.stack([torch.arange(start, start + count, dtype=torch.float64),
                             100 + torch.arange(start, start + count, dtype=torch.float64)])
        full = replicas.gather_members(local, total)
        slowest = replicas.max_over_ranks(10.0 + rank)
        q.put((rank, full.tolist(), slowest, replicas.member_seed(1, rank)))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, 'error', repr(e), None))


@pytest.mark.parametrize('total', [5, 8])
def test_two_ranks_gloo(total):
    world = 2
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, total, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    for _ in range(world):
        r, full, slowest, seed = q.get(timeout=120)
        assert full != 'error', slowest
        res[r] = (full, slowest, seed)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [[float(j) for j in range(total)], [100.0 + j for j in range(total)]]
    for r in range(world):
        assert res[r][0] == expect
        assert res[r][1] == 11.0
    assert res[0][2] != res[1][2]


def test_bench_spawns_one_process_per_rank(capfd):
    """bench.py --gpus N without a launcher starts N rank processes with the launcher's
    environment; here they run a gloo probe and the job maximum reaches rank 0."""
    import json
    import os
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    rc = bench.spawn_ranks(2, script=os.path.join(root, 'tests', 'rank_probe.py'), argv=[])
    assert rc == 0
    line = [x for x in capfd.readouterr().out.splitlines() if x.startswith('{')][-1]
    assert json.loads(line) == {'world': 2, 'max': 2.0, 'local_rank': 0}
