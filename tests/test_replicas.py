"""The multi-GPU plumbing of bench.py (independent replicas) on CPU: two gloo ranks join
over 127.0.0.1, meet at the barrier, and the whole-job rate is the units of both ranks over
the slower rank's time; a rank that never joins makes the other's init end with an error
inside the short timeout instead of waiting for good."""
import json
import os
import socket

import pytest

from conftest import load_package

lt = load_package()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir, seconds, units):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from lenstool_hpc_b200 import replicas
    assert replicas.env() == (rank, rank, world)
    assert replicas.init("gloo", timeout_s=30.0) == world
    replicas.barrier()
    rate, tmax, total = replicas.throughput(units[rank], seconds[rank])
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"rate": rate, "tmax": tmax, "total": total}, f)
    replicas.finalize()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    seconds, units = [0.5, 2.0], [1000.0, 3000.0]
    mp.spawn(_rank, args=(2, port, str(tmp_path), seconds, units), nprocs=2, join=True)
    for r in range(2):
        res = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert res["tmax"] == 2.0 and res["total"] == 4000.0 and res["rate"] == 2000.0


def _lonely(port, q):
    os.environ.update(RANK="0", LOCAL_RANK="0", WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from lenstool_hpc_b200 import replicas
    try:
        replicas.init("gloo", timeout_s=3.0)
        q.put("joined")
    except Exception as ex:  # the peer never came: the rendezvous times out
        q.put(type(ex).__name__)


def test_missing_rank_times_out():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_lonely, args=(_free_port(), q))
    p.start()
    p.join(120)
    alive = p.is_alive()
    if alive:
        p.kill()
    assert not alive, "a rank whose peer never joined kept waiting"
    assert q.get(timeout=5) != "joined"


def test_single_process_needs_no_group():
    from lenstool_hpc_b200 import replicas
    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    assert replicas.init("gloo") == 1
    assert replicas.throughput(10.0, 2.0) == (5.0, 2.0, 10.0)
