"""bench.py's multi-rank plumbing on the CPU: the arguments of a `--gpus 2` launch, the
max-over-ranks reduction of the timed region through a real two-rank process group (gloo),
the whole-job rate from the slowest rank's time, and the shape of the printed line."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2, timeout=datetime.timedelta(seconds=30))
    import bench
    ms = 100.0 + 50.0 * rank  # rank 1 is the slower one
    got = bench.max_over_ranks(ms, 2, dist, "cpu")
    dist.destroy_process_group()
    q.put((rank, got))


def test_parse_gpus_two():
    import bench
    a = bench.parse(["--gpus", "2", "--steps", "4", "--warmup", "3"])
    assert (a.gpus, a.steps, a.warmup, a.impl, a.form) == (2, 4, 3, "ours", "plain")


def test_max_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
    assert out == {0: 150.0, 1: 150.0}


def test_whole_job_rate_and_single_rank():
    import bench
    assert bench.max_over_ranks(7.0, 1) == 7.0
    # two ranks of 1e9 points per step each, 4 steps, slowest rank 2 s
    assert bench.whole_job_rate(2, 1e9, 4, 2000.0) == pytest.approx(4e9)


def test_contract_line_for_two_ranks():
    import bench

    class G:
        zero_pivot, CH = False, 8192

    a = bench.parse(["--gpus", "2", "--steps", "4", "--warmup", "3"])
    m = {"value": 4e9, "total_ms": 2000.0, "step_ms": [500.0] * 4, "launches": 64, "clocks": {"sm_mhz": 1965}}
    line = bench.contract_line(a, 2, m, G(), {"bound": "hbm"}, {"value": 1.0}, None)
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "clocks", "gpu_launches", "roofline", "e2e", "cpu_baseline"):
        assert k in line, k
    assert line["n_gpus"] == 2 and line["scaling"] == "weak" and line["ms_per_step"] == 500.0
    assert line["config"]["chunk_columns"] == 8192 and "2 rank" in line["config"]["parallelism"]
