"""
The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1), each in its own process. The path
shards frames (each rank correlates its own batches with its own copy of the reference spectra) and
has no data-path collective; what crosses ranks is the barrier and the maximum of the ranks' times.
"""

import datetime
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        starts = bench.shard_starts(rank, world, 301, 16, 30)
        everyone = [None] * world
        dist.all_gather_object(everyone, starts)
        slowest = bench.max_over_ranks(10.0 * (rank + 1), dist, 'cpu')
        dist.barrier()
        q.put((rank, everyone, slowest))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in range(2):
            rank, everyone, slowest = q.get(timeout=120)
            results[rank] = (everyone, slowest)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert sorted(results) == [0, 1]
    for rank in (0, 1):
        everyone, slowest = results[rank]
        assert slowest == 20.0   # the maximum over the ranks, on every rank
        a, b = everyone
        nb = (301 - 1) // 16   # 18 batches: each rank takes 9 before the video wraps around
        assert not set(a[:nb // 2]) & set(b[:nb // 2])
        assert sorted(a[:nb // 2] + b[:nb // 2]) == [1 + 16 * i for i in range(nb)]
        assert all(1 <= s <= 301 - 16 for s in a + b)


def test_shard_starts_one_rank_and_errors():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.shard_starts(0, 1, 49, 16, 5) == [1, 17, 33, 1, 17]
    assert bench.max_over_ranks(3.5, None, 'cpu') == 3.5
    with pytest.raises(ValueError):
        bench.shard_starts(0, 1, 10, 16, 1)


def test_bench_launches_its_own_ranks():
    """bench.py --gpus 2 without a launcher starts two ranks itself (torch.distributed.run, gloo here
    without a GPU); both ran, took disjoint batches, and the line reports n_gpus 2."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ('RANK', 'WORLD_SIZE', 'LOCAL_RANK', 'MASTER_ADDR', 'MASTER_PORT')}
    env['CUDA_VISIBLE_DEVICES'] = ''
    r = subprocess.run([sys.executable, os.path.join(root, 'bench.py'), '--gpus', '2', '--workload', 'launch-check',
                        '--steps', '3'], capture_output=True, text=True, timeout=240, env=env, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([ln for ln in r.stdout.splitlines() if ln.startswith('{')][-1])
    assert line['n_gpus'] == 2
    assert sorted(x['rank'] for x in line['ranks']) == [0, 1]
    assert len({x['first_batch'] for x in line['ranks']}) == 2
