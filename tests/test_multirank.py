"""bench.py's multi-rank host logic on CPU (no GPU): the timed region's
max over ranks (and the sum and minimum the batched and served forms use)
on a 2-rank gloo group, the served form's request placement (the same in
every rank without an exchange), and the reference arm's non-zero ranks,
which leave without work or output. The plain path runs as independent
replicas per rank, so these reductions are its only collectives."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks(1.5 + rank, dist)
        none = bench.max_over_ranks(0.25, None)
        tot = bench._sum_over_ranks(10.0 + rank, dist)
        lowest = -bench.max_over_ranks(-(3.0 + rank), dist)
        # the served form's placement of one request stream: every rank
        # derives the same owner for every request, without an exchange
        owner = bench.place_requests([5, 1, 1, 7, 2, 2, 9, 1], world)
        mine = [r for r in range(8) if owner[r] == rank]
        every = [None] * world
        dist.all_gather_object(every, owner.tolist())
        with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
            f.write(f"{got} {none} {tot} {lowest} {int(every[0] == every[1])} {len(mine)}")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    counts = 0
    for r in range(world):
        got, none, tot, lowest, same, mine = (float(x) for x in open(tmp_path / f"r{r}.txt").read().split())
        assert got == 2.5 and none == 0.25 and tot == 21.0 and lowest == 3.0 and same == 1
        counts += mine
    assert counts == 8


@pytest.mark.parametrize("rank", [1, 3])
def test_reference_arm_other_ranks_exit_quietly(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="4", LOCAL_RANK=str(rank),
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "4"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
