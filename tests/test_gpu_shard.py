"""The engine across ranks: two processes (gloo process group) share the one GPU, each runs the
real Engine on its contiguous column range (shard.column_range, the reference's procx x procy
split of flux_feautrier.f90:132-133), and the emergent-flux planes are all-gathered
(shard.solve_sharded).  Each rank's kernels are independent of the other's (no kernel waits on
another rank), so sharing one device is safe.  The gathered planes must equal one solve of the
whole block, bit for bit, in the plain and in the mixed form."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _block():
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(5, 7, 96, seed=13)
    return rho, T, dz, workloads.log_wavelengths(40)


def _worker(rank, world, port, form, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    try:
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from ocotillo_b200 import Engine, shard
        rho, T, dz, wa = _block()
        eng = Engine(0)
        eng.set_wavelengths(wa)

        def solve(r, t):
            return eng.solve_block(r, t, dz, form=form, want=("Vtop", "Vbot"), allow_zero_pivot=True)

        res = shard.solve_sharded(solve, rho, T, rank, world)
        eng.close()
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, res))
    except Exception as ex:
        q.put((rank, f"error: {type(ex).__name__}: {ex}"))


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_two_ranks_share_the_gpu_and_gather_the_planes(form):
    import multiprocessing as mp
    from ocotillo_b200 import Engine
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, form, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=300) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    rho, T, dz, wa = _block()
    eng = Engine(0)
    eng.set_wavelengths(wa)
    ref = eng.solve_block(rho, T, dz, form=form, want=("Vtop", "Vbot"), allow_zero_pivot=True)
    eng.close()
    for rank in (0, 1):
        assert not isinstance(out[rank], str), out[rank]
        for k in ("Vtop", "Vbot"):
            a, b = out[rank][k], ref[k]
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (rank, k)
