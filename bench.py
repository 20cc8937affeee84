#!/usr/bin/env python3
"""Throughput of the B200 engine in mesh*lambda points per second.

Workload (one step = one pass of the hot path over the whole grid): the 'plain FP64 non-grey
AGN grid' -- nx = ny = 256 columns, nz = 512, nw = 256 log-spaced wavelengths from 100 A to
10 um, Gaussian density (rho0 = 1e-9 g/cm^3, H = 1.496e14 cm, floor 1e-24) times a seeded
lognormal perturbation (0.3 dex) per cell, T = max(6.1e4 K exp(-z^2/2 sigma_T^2), 2000 K),
fully_ionized_T = 2e4 K.  Seeded synthetic inputs stand in for a snapshot.

  value  device-resident throughput: inputs in HBM, the full grid solved in column chunks,
         every U (with ghosts), kappa and V of every chunk written to HBM (rotating chunk
         buffers; 206 GB of outputs per step do not fit at once) plus the emergent planes.
  e2e    the same metric through the host-array C-ABI call (oco_solve_block) a Fortran or
         Python caller makes: pinned host inputs copied in, every output copied back to
         pinned host memory, per step one batch of columns.
  --impl reference   the reference's CPU algorithm (the C restatement of the Fortran loop,
         glibc math) on all host cores, on a bounded sample of the same workload.

Run: python bench.py [--gpus N] [--steps K] [--warmup W] [--form plain|stable|mixed]
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="plain", choices=["plain", "stable", "mixed"])
    ap.add_argument("--layout", default="reference", choices=["reference", "lambda"])
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=512)
    ap.add_argument("--nw", type=int, default=256)
    ap.add_argument("--chunk-cols", type=int, default=8192)
    ap.add_argument("--e2e-cols", type=int, default=2048)
    ap.add_argument("--cpu-cols", type=int, default=1024, help="columns in the CPU-baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


# ---- clocks during the timed region ---------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = sorted(float(r[1]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


# ---- CPU baseline: the oracle (C restatement of the reference loop, glibc math) -----------
def _cpu_worker(args):
    rho, T, wa, dz = args
    from oracle import pyoracle
    t0 = time.perf_counter()
    pyoracle.solve_block(rho, T, wa, dz, backend="glibc", want=("U", "kappa", "V"))
    return time.perf_counter() - t0


def cpu_baseline(rho, T, wa, dz, ncols, procs):
    """Times the oracle on `ncols` columns (all z, all lambda) split over `procs` spawned
    processes.  Returns (points/s, seconds, points)."""
    import multiprocessing as mp
    nx, ny, nz = rho.shape
    flat_r = rho.reshape(-1, nz)[:ncols]
    flat_t = T.reshape(-1, nz)[:ncols]
    parts = np.array_split(np.arange(ncols), procs)
    jobs = [(flat_r[p].reshape(len(p), 1, nz), flat_t[p].reshape(len(p), 1, nz), wa, dz) for p in parts if len(p)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(len(jobs)) as pool:
        pool.map(_cpu_worker, [(j[0][:1], j[1][:1], j[2], j[3]) for j in jobs])  # warm-up (import, build)
        t0 = time.perf_counter()
        pool.map(_cpu_worker, jobs)
        dt = time.perf_counter() - t0
    pts = ncols * nz * len(wa)
    return pts / dt, dt, pts


def run_reference(a):
    """--impl reference: the reference's algorithm on the host cores (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from ocotillo_b200 import workloads
    rho, T, dz = workloads.agn_block(a.nx, a.ny, a.nz, seed=2)
    wa = workloads.log_wavelengths(a.nw)
    procs = os.cpu_count() or 1
    cols = max(procs, min(a.cpu_cols // 4, a.nx * a.ny))
    import multiprocessing as mp
    nz = a.nz
    flat_r, flat_t = rho.reshape(-1, nz), T.reshape(-1, nz)
    ctx = mp.get_context("spawn")
    times = []
    with ctx.Pool(procs) as pool:
        pool.map(_cpu_worker, [(flat_r[:1].reshape(1, 1, nz), flat_t[:1].reshape(1, 1, nz), wa, dz)] * procs)
        for step in range(a.warmup + a.steps):
            c0 = (step * cols) % (a.nx * a.ny - cols + 1)
            parts = np.array_split(np.arange(c0, c0 + cols), procs)
            jobs = [(flat_r[p].reshape(len(p), 1, nz), flat_t[p].reshape(len(p), 1, nz), wa, dz) for p in parts]
            t0 = time.perf_counter()
            pool.map(_cpu_worker, jobs)
            if step >= a.warmup:
                times.append(time.perf_counter() - t0)
    pts = cols * a.nz * a.nw
    v = pts * len(times) / sum(times)
    line = {"impl": "reference", "metric": "mesh*lambda points/s", "value": v, "unit": "points/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(a, "reference CPU loop"),
            "cpu_baseline": {"value": v, "unit": "points/s", "cores": procs, "kind": "port",
                             "sample": f"{cols} columns x nz={a.nz} x nw={a.nw} per step, glibc math, "
                                       f"{procs} processes"},
            "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(a, form):
    return {"workload": "plain FP64 non-grey AGN grid, 256x256 columns, nz=512, nw=256",
            "nx": a.nx, "ny": a.ny, "nz": a.nz, "nw": a.nw, "lambda": "100 A - 10 um log-spaced",
            "form": form, "l2": "inputs and outputs larger than L2 (no flush needed)"}


def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q
    f, c = math.floor(k), math.ceil(k)
    return xs[f] + (xs[c] - xs[f]) * (k - f)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    from ocotillo_b200 import Engine, workloads, LAYOUT_REFERENCE, LAYOUT_LAMBDA_FASTEST

    nx, ny, nz, nw = a.nx, a.ny, a.nz, a.nw
    ncol, mz = nx * ny, nz + 6
    rho_h, T_h, dz = workloads.agn_block(nx, ny, nz, seed=2 + rank)
    wa = workloads.log_wavelengths(nw)
    rho = torch.from_numpy(rho_h).to(dev).reshape(ncol, nz)
    T = torch.from_numpy(T_h).to(dev).reshape(ncol, nz)
    eng = Engine(local)
    eng.set_wavelengths(wa)
    eng.set_profiling(True)
    layout = LAYOUT_REFERENCE if a.layout == "reference" else LAYOUT_LAMBDA_FASTEST
    CH = min(a.chunk_cols, ncol)
    assert ncol % CH == 0, "chunk must divide the grid"
    nchunk = ncol // CH

    def mk(shape):
        return torch.empty(shape, dtype=torch.float64, device=dev)

    sets = []
    for _ in range(2):
        if layout == LAYOUT_REFERENCE:
            o = {"U": mk((nw, CH, mz)), "kappa": mk((nw, CH, nz)), "V": mk((nw, CH, nz))}
        else:
            o = {"U": mk((mz, CH, nw)), "kappa": mk((nz, CH, nw)), "V": mk((nz, CH, nw))}
        sets.append(o)
    Vtop, Vbot = mk((nchunk, nw, CH)), mk((nchunk, nw, CH))
    stream = torch.cuda.current_stream(dev)

    def step():
        for k in range(nchunk):
            o = dict(sets[k % 2])
            o["Vtop"], o["Vbot"] = Vtop[k], Vbot[k]
            r = rho[k * CH:(k + 1) * CH].reshape(CH, 1, nz)
            t = T[k * CH:(k + 1) * CH].reshape(CH, 1, nz)
            eng.solve_block_device(r, t, dz, o, form=a.form, layout=layout, stream=stream)

    zero_pivot = False

    def sync_engine():
        nonlocal zero_pivot
        try:
            eng.synchronize()
        except Exception as e:
            if getattr(e, "code", None) != -3:
                raise
            zero_pivot = True

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize(dev)
    sync_engine()
    eng.kernel_times()  # discard warm-up timings
    clocks = Clocks(local)
    clocks.start()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    launches0 = eng.kernel_launches
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    evs[0].record(stream)
    for i in range(a.steps):
        step()
        evs[i + 1].record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = eng.kernel_launches - launches0
    sync_engine()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(a.steps)]
    total_ms = evs[0].elapsed_time(evs[-1])
    solve_ms, pil_ms, nsolve = eng.kernel_times()
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    pts_step = ncol * nz * nw
    value = world * pts_step * a.steps / (total_ms / 1e3)

    # roofline of the dominant kernel (the solve): algorithmic bytes per mesh*lambda point
    # = outputs U (nz+6 per nz), kappa, V (8 B each) + per-column pillars read once (26*8 B
    # per z, shared by nw wavelengths).
    bytes_pt = 8.0 * (mz / nz) + 16.0 + 26 * 8.0 / nw
    launch_ms = solve_ms / max(nsolve, 1)
    pts_launch = pts_step * a.steps / max(nsolve, 1)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    achieved = bytes_pt * pts_launch / (launch_ms / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
            "traffic": None, "kernel": "k_solve", "launch_ms": launch_ms,
            "algorithmic_bytes_per_point": bytes_pt,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "solve_share_of_step": solve_ms / total_ms, "pillars_ms_per_step": pil_ms / a.steps}

    # ---- e2e: host arrays through oco_solve_block (pinned), one batch of columns per step
    e2e = None
    if not a.no_e2e:
        E = min(a.e2e_cols, ncol)
        pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
        rho_p = pin((ncol, nz))
        T_p = pin((ncol, nz))
        rho_p[:] = rho_h.reshape(ncol, nz)
        T_p[:] = T_h.reshape(ncol, nz)
        outs = {"U": pin((nw, E, 1, mz)), "kappa": pin((nw, E, 1, nz)), "V": pin((nw, E, 1, nz)),
                "Vtop": pin((nw, E, 1)), "Vbot": pin((nw, E, 1))}
        nb = ncol // E

        def e2e_step(i):
            c0 = (i % nb) * E
            eng.solve_block(rho_p[c0:c0 + E].reshape(E, 1, nz), T_p[c0:c0 + E].reshape(E, 1, nz), dz,
                            form=a.form, out=outs, allow_zero_pivot=True)

        for i in range(a.warmup):
            e2e_step(i)
        if world > 1:
            dist.barrier()
        lat = []
        t0 = time.perf_counter()
        for i in range(a.steps):
            s0 = time.perf_counter()
            e2e_step(i)
            lat.append(time.perf_counter() - s0)
        el = time.perf_counter() - t0
        if world > 1:
            t = torch.tensor([el], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        e2e = {"value": world * E * nz * nw * a.steps / el, "unit": "points/s",
               "h2d_bytes_per_step": 2 * E * nz * 8, "d2h_bytes_per_step": E * nw * (mz + 2 * nz + 2) * 8,
               "columns_per_step": E, "p50_ms": 1e3 * pct(lat, 0.5), "p99_ms": 1e3 * pct(lat, 0.99)}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        procs = os.cpu_count() or 1
        v, dt, pts = cpu_baseline(rho_h, T_h, wa, dz, min(a.cpu_cols, ncol), procs)
        cpu = {"value": v, "unit": "points/s", "cores": procs, "kind": "port",
               "sample": f"first {min(a.cpu_cols, ncol)} columns of the same grid, all z and lambda "
                         f"({pts:.3g} points, {dt:.1f} s wall on {procs} processes), glibc math"}

    if rank == 0:
        line = {"metric": "mesh*lambda points/s", "value": value, "unit": "points/s", "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "config": config_dict(a, a.form),
                "latency_ms": {"p50": pct(step_ms, 0.5), "p99": pct(step_ms, 0.99)},
                "zero_pivot_items": zero_pivot, "clocks": clk, "gpu_launches": int(launches),
                "roofline": roof, "e2e": e2e, "cpu_baseline": cpu}
        line["config"]["layout"] = a.layout
        line["config"]["chunk_columns"] = CH
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
