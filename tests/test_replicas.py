"""Multi-GPU replicas, host side, on CPU with two gloo ranks: both ranks agree on
the mesh assignment, every mesh is taken exactly once, the reported time is the
slowest rank's, and a rank that fails makes the other's next collective end
with an error instead of waiting for good."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, out_path, fail_rank):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from pamo_b200 import replicas

    w, r = replicas.init("gloo", timeout_s=10.0)
    mine = replicas.my_share(sizes, r, w)
    local = 1.0 + r  # this rank's "time"
    try:
        if r == fail_rank:
            raise RuntimeError("rank failed before the reduction")
        worst = replicas.max_over_ranks([local, float(len(mine))])
        result = f"ok {r} {worst[0]} {','.join(map(str, mine))}"
    except RuntimeError as e:
        result = f"err {r} {type(e).__name__}"
    with open(f"{out_path}.{r}", "w") as f:
        f.write(result)
    if r == fail_rank:
        os._exit(0)  # leaves without the collective
    try:
        dist.destroy_process_group()
    except Exception:
        pass


def _run(world, sizes, tmp_path, fail_rank=-1):
    import torch.multiprocessing as mp

    port = _free_port()
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, port, sizes, out, fail_rank), nprocs=world, join=True,
                       start_method="spawn")
    return [open(f"{out}.{r}").read().split() for r in range(world)]


def test_assignment_is_balanced_and_complete():
    from pamo_b200 import replicas

    sizes = [500_000, 5_000, 120_000, 80_000, 2_000_000, 7_000, 64_000, 300_000]
    owner = replicas.assign_by_footprint(sizes, 3)
    loads = [sum(s for s, o in zip(sizes, owner) if o == r) for r in range(3)]
    assert sorted(i for r in range(3) for i in replicas.my_share(sizes, r, 3)) == list(range(len(sizes)))
    assert max(loads) == 2_000_000  # the biggest mesh alone on one rank
    assert replicas.assign_by_footprint(sizes, 3) == owner  # deterministic


def test_two_gloo_ranks_agree_and_take_the_max(tmp_path):
    sizes = [10, 40, 30, 20, 50]
    res = _run(2, sizes, tmp_path)
    assert all(r[0] == "ok" for r in res)
    assert all(float(r[2]) == 2.0 for r in res)  # max over ranks of 1 + rank
    taken = sorted(int(i) for r in res for i in r[3].split(","))
    assert taken == list(range(len(sizes)))


@pytest.mark.timeout(120)
def test_failed_rank_is_detected_by_the_other(tmp_path):
    res = _run(2, [1, 2, 3], tmp_path, fail_rank=1)
    assert res[1][0] == "err"
    assert res[0][0] == "err"  # the reduction ended with an error, not a hang
