"""Column sharding across ranks (gloo, world_size 2, CPU): each rank solves its column range
with the oracle and the emergent-flux planes are all-gathered; the result equals one solve of
the whole block.  A rank that exits before the collective makes the other rank's collective
fail within the process-group timeout (failure detected on the host)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, mode, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    from oracle import pyoracle
    from ocotillo_b200 import shard, workloads
    rho, T, dz = workloads.agn_block(3, 3, 24, seed=5)
    wa = workloads.log_wavelengths(5, 2000.0, 20000.0)

    def solve(r, t):
        o = pyoracle.solve_block(r, t, wa, dz, form=pyoracle.FORM_STABLE, backend="glibc", want=("V",))
        return {"Vtop": o["V"][..., -1], "Vbot": o["V"][..., 0]}

    try:
        if mode == "exit" and rank == 1:
            q.put((rank, "exited"))
            q.close()
            q.join_thread()  # flush the message before leaving
            os._exit(0)  # leaves before the collective
        res = shard.solve_sharded(solve, rho, T, rank, world)
        q.put((rank, res))
    except Exception as ex:  # the surviving rank's collective fails
        q.put((rank, f"error: {type(ex).__name__}"))
    finally:
        if mode != "exit":
            dist.destroy_process_group()


def _run(world, mode):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=90) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return out


def test_column_range_partitions():
    from ocotillo_b200.shard import column_range
    for ncol in (1, 7, 64, 65537):
        for world in (1, 2, 3, 8):
            rs = [column_range(ncol, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == ncol
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(c1 - c0 for c0, c1 in rs) - min(c1 - c0 for c0, c1 in rs) <= 1
    with pytest.raises(ValueError):
        column_range(10, 2, 2)


def test_more_ranks_than_columns_refused_before_any_collective():
    """A rank without columns could not join the gather with a plane of the right height, so
    every rank refuses (no process group needed: nothing collective has started)."""
    from ocotillo_b200.shard import solve_sharded
    rho = np.ones((1, 3, 8))

    def solve(r, t):
        raise AssertionError("must not be reached")

    for rank in range(4):
        with pytest.raises(ValueError, match="3 columns"):
            solve_sharded(solve, rho, rho, rank, 4)


def test_sharded_solve_matches_single_solve():
    from oracle import pyoracle
    from ocotillo_b200 import workloads
    out = _run(2, "ok")
    rho, T, dz = workloads.agn_block(3, 3, 24, seed=5)
    wa = workloads.log_wavelengths(5, 2000.0, 20000.0)
    ref = pyoracle.solve_block(rho, T, wa, dz, form=pyoracle.FORM_STABLE, backend="glibc", want=("V",))
    for rank in (0, 1):
        assert np.array_equal(out[rank]["Vtop"], ref["V"][..., -1])
        assert np.array_equal(out[rank]["Vbot"], ref["V"][..., 0])


def test_rank_leaving_is_detected():
    out = _run(2, "exit")
    assert out[1] == "exited"
    assert isinstance(out[0], str) and out[0].startswith("error")
