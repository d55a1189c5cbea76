"""The multi-rank host logic of bench.py on the CPU: two gloo ranks
(127.0.0.1), no GPU.  Column sharding of one Jacobian (contiguous blocks,
padded all-gather, assembly into J) and the max-over-ranks timing reduction
that every multi-GPU number goes through."""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, nn, q):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = np.arange(nn * nn, dtype=np.float64).reshape(nn, nn) * 0.5 - 3.0  # J[row][col]
        blocks = bench.column_blocks(nn, world)
        c0, c1 = blocks[rank]
        nb = max(b - a for a, b in blocks)
        local = torch.zeros(nb * nn, dtype=torch.float64)
        local[:(c1 - c0) * nn] = torch.from_numpy(np.ascontiguousarray(A[:, c0:c1].T).ravel())
        J = bench.gather_columns(local, nn, blocks, world).numpy()
        worst = bench.max_over_ranks(world, float(rank) + 0.25)
        q.put((rank, bool(np.array_equal(J, A)), worst, blocks))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nn", [7, 96])
def test_column_sharding_two_gloo_ranks(nn):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, nn, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ok, worst, blocks in res:
        assert ok, rank
        assert worst == 1.25
        assert blocks[0][0] == 0 and blocks[-1][1] == nn
        assert abs((blocks[0][1] - blocks[0][0]) - (blocks[1][1] - blocks[1][0])) <= 1


def test_column_blocks_cover_every_column():
    sys.path.insert(0, str(REPO))
    import bench

    for nn in [96, 384, 768]:
        for world in [1, 2, 3, 8]:
            b = bench.column_blocks(nn, world)
            assert len(b) == world and b[0][0] == 0 and b[-1][1] == nn
            assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))


def test_bench_launches_its_own_ranks_dry_run():
    """`bench.py --gpus 2` with no outer launcher starts two ranks itself
    (torch.distributed.run, 127.0.0.1); with --dry-run they run the column
    partition, the all-gather and the max-over-ranks reduction on gloo, and
    rank 0 alone prints one line with n_gpus = 2."""
    import json
    import subprocess

    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--gpus", "2", "--dry-run", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=300, env=env, cwd=str(REPO))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout
    line = lines[0]
    assert line["dry_run"] and line["n_gpus"] == 2 and line["gather_ok"]
    assert line["blocks"] == [[0, 384], [384, 768]] and line["max_over_ranks"] == 2.0
    assert line["config"]["parallelism"] == "2 independent solves, one per GPU"
