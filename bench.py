#!/usr/bin/env python3
"""Throughput of the B200 engine in mesh*lambda points per second, mixed vs plain FP64.

Workload (one step = one pass of the hot path over the whole grid): the 'plain FP64 non-grey
AGN grid' -- nx = ny = 256 columns, nz = 512, nw = 256 log-spaced wavelengths from 100 A to
10 um, Gaussian density (rho0 = 1e-9 g/cm^3, H = 1.496e14 cm, floor 1e-24) times a seeded
lognormal perturbation (0.3 dex) per cell, T = max(6.1e4 K exp(-z^2/2 sigma_T^2), 2000 K),
fully_ionized_T = 2e4 K.  Seeded synthetic inputs stand in for a snapshot.

  value   device-resident throughput of the plain FP64 form (the reference's arithmetic):
          inputs in HBM, the full grid solved in column chunks, every U (with ghosts), kappa
          and V of every chunk written to HBM (rotating chunk buffers; 206 GB of outputs per
          step do not fit at once) plus the emergent planes.
  mixed   the same step in the mixed-precision form, its ratio to `value`, and its emergent-flux
          error against the FP64 (stable) form over the whole grid.
  batch   the batching form: 8192 ragged columns (nz 64-2048, nw 32-1024) in one persistent
          launch replayed as a CUDA graph, autotuned tiling, mixed form.
  serving the serving form: a Poisson stream of jobs (nx = ny in {64..512}, nz 128-1024, nw
          64-512) through the serving loop, p50/p99 latency and throughput, mixed and plain.
  e2e     the headline metric through the host-array C-ABI call (oco_solve_block) a Fortran
          or Python caller makes: pinned host inputs copied in, every output copied back to
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

METRIC = "mesh\u00b7\u03bb points/s + p50/p99 latency: mixed vs plain FP64, 1 B200, \u22641e-4 rel"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="plain", choices=["plain", "stable", "mixed"])
    ap.add_argument("--layout", default="lambda", choices=["reference", "lambda"])
    ap.add_argument("--nx", type=int, default=256)
    ap.add_argument("--ny", type=int, default=256)
    ap.add_argument("--nz", type=int, default=512)
    ap.add_argument("--nw", type=int, default=256)
    ap.add_argument("--chunk-cols", type=int, default=8192)
    ap.add_argument("--e2e-cols", type=int, default=2048)
    ap.add_argument("--cpu-cols", type=int, default=1024, help="columns in the CPU-baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the mixed, batch and serving measurements")
    ap.add_argument("--serve-jobs", type=int, default=50, help="jobs per serving run (each rate of the sweep)")
    ap.add_argument("--batch-cols", type=int, default=8192)
    ap.add_argument("--no-c3", action="store_true", help="skip the precision-config (c3) measurement")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving (c5) measurement")
    ap.add_argument("--cpu1-cols", type=int, default=64, help="columns in the one-core CPU-baseline sample")
    return ap.parse_args(argv)


def max_over_ranks(x, world, dist=None, device=None):
    """The largest of the ranks' values of x (every rank gets it; x itself when world == 1)."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, points_per_rank_step, steps, max_ms):
    """Whole-job throughput: the points all ranks processed over the slowest rank's time."""
    return world * points_per_rank_step * steps / (max_ms / 1e3)


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
                "samples": len(rows),
                "power_w_max": max((float(r[3]) for r in rows if r[3].replace(".", "").isdigit()), default=None)}


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
    cols = min(max(procs, a.cpu_cols // 4), a.nx * a.ny)  # the sample never exceeds the grid
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
            jobs = [(flat_r[p].reshape(len(p), 1, nz), flat_t[p].reshape(len(p), 1, nz), wa, dz) for p in parts
                    if len(p)]
            t0 = time.perf_counter()
            pool.map(_cpu_worker, jobs)
            if step >= a.warmup:
                times.append(time.perf_counter() - t0)
    pts = cols * a.nz * a.nw
    v = pts * len(times) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "points/s",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(a, "plain"),  # the reference loop is the plain form's arithmetic
            "cpu_baseline": {"value": v, "unit": "points/s", "cores": procs, "kind": "port",
                             "sample": f"{cols} columns x nz={a.nz} x nw={a.nw} per step, glibc math, "
                                       f"{procs} processes"},
            "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_dict(a, form):
    return {"workload": f"plain FP64 non-grey AGN grid, {a.nx}x{a.ny} columns, nz={a.nz}, nw={a.nw}",
            "nx": a.nx, "ny": a.ny, "nz": a.nz, "nw": a.nw, "lambda": "100 A - 10 um log-spaced",
            "form": form, "l2": "inputs and outputs larger than L2 (no flush needed)"}


def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q
    f, c = math.floor(k), math.ceil(k)
    return xs[f] + (xs[c] - xs[f]) * (k - f)


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class Grid:
    """The AGN grid on the device and the chunked step over it (one pass of the hot path)."""

    def __init__(self, a, eng, dev, rank, workload="agn"):
        import torch
        from ocotillo_b200 import workloads, LAYOUT_REFERENCE, LAYOUT_LAMBDA_FASTEST
        self.a, self.eng, self.dev = a, eng, dev
        nx, ny, nz, nw = a.nx, a.ny, a.nz, a.nw
        self.ncol, self.nz, self.nw, self.mz = nx * ny, nz, nw, nz + 6
        if workload == "precision":  # rho0 log-uniform in [1e-11, 1e-7] (seed 3), generated on the device
            r, t, self.dz, self.rho0 = workloads.precision_block_device(eng, nx, ny, nz, seed=3 + rank)
            self.rho, self.T = r.reshape(self.ncol, nz), t.reshape(self.ncol, nz)
            self.rho_h = self.T_h = None
        else:
            self.rho_h, self.T_h, self.dz = workloads.agn_block(nx, ny, nz, seed=2 + rank)
            self.rho = torch.from_numpy(self.rho_h).to(dev).reshape(self.ncol, nz)
            self.T = torch.from_numpy(self.T_h).to(dev).reshape(self.ncol, nz)
        self.wa = workloads.log_wavelengths(nw)
        self.layout = LAYOUT_REFERENCE if a.layout == "reference" else LAYOUT_LAMBDA_FASTEST
        self.CH = min(a.chunk_cols, self.ncol)
        self.nchunk = -(-self.ncol // self.CH)  # the last chunk may be smaller
        mk = lambda shape: torch.empty(shape, dtype=torch.float64, device=dev)
        CH, mz = self.CH, self.mz
        self.sets = []
        for _ in range(2):
            if self.layout == LAYOUT_REFERENCE:
                o = {"U": mk((nw, CH, mz)), "kappa": mk((nw, CH, nz)), "V": mk((nw, CH, nz))}
            else:
                o = {"U": mk((mz, CH, nw)), "kappa": mk((nz, CH, nw)), "V": mk((nz, CH, nw))}
            self.sets.append(o)
        # emergent-flux planes per chunk [nw][columns of the chunk]; slots past a short last chunk
        # stay NaN, which every comparison leaves out
        self.Vtop = torch.full((self.nchunk, nw, CH), float("nan"), dtype=torch.float64, device=dev)
        self.Vbot = torch.full((self.nchunk, nw, CH), float("nan"), dtype=torch.float64, device=dev)
        self.stream = torch.cuda.current_stream(dev)
        self.zero_pivot = False

    def step(self, form, fields=True):
        for k in range(self.nchunk):
            c0 = k * self.CH
            n = min(self.CH, self.ncol - c0)
            # the chunk's arrays: the first n columns' worth of each buffer (columns are dimension
            # 1 of every one of them), contiguous
            head = lambda x: x.view(-1)[:x.numel() // self.CH * n].view(x.shape[0], n, *x.shape[2:])
            o = {key: head(v) for key, v in self.sets[k % 2].items()} if fields else {}
            o["Vtop"], o["Vbot"] = head(self.Vtop[k]), head(self.Vbot[k])
            r = self.rho[c0:c0 + n].reshape(n, 1, self.nz)
            t = self.T[c0:c0 + n].reshape(n, 1, self.nz)
            self.eng.solve_block_device(r, t, self.dz, o, form=form, layout=self.layout, stream=self.stream)

    def sync(self):
        try:
            self.eng.synchronize()
        except Exception as e:
            if getattr(e, "code", None) != -3:
                raise
            self.zero_pivot = True

    def measure(self, form, steps, warmup, world, dist=None, clocks=None):
        """Times `steps` steps of `form` (after `warmup`), CUDA events on the launching stream,
        max over ranks.  Returns a dict of the timing and the kernel accounting."""
        import torch
        for _ in range(warmup):
            self.step(form)
        torch.cuda.synchronize(self.dev)
        self.sync()
        self.eng.kernel_times()
        if clocks:
            clocks.start()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(self.dev)
        launches0 = self.eng.kernel_launches
        evs = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
        evs[0].record(self.stream)
        for i in range(steps):
            self.step(form)
            evs[i + 1].record(self.stream)
        torch.cuda.synchronize(self.dev)
        if world > 1:
            dist.barrier()
        clk = clocks.stop() if clocks else None
        launches = self.eng.kernel_launches - launches0
        self.sync()
        step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(steps)]
        total_ms = evs[0].elapsed_time(evs[-1])
        solve_ms, pil_ms, nsolve = self.eng.kernel_times()
        total_ms = max_over_ranks(total_ms, world, dist, self.dev)
        pts_step = self.ncol * self.nz * self.nw
        return {"value": whole_job_rate(world, pts_step, steps, total_ms), "total_ms": total_ms, "step_ms": step_ms,
                "launches": launches, "solve_ms": solve_ms, "pil_ms": pil_ms, "nsolve": nsolve, "clocks": clk,
                "pts_step": pts_step}

    def roofline(self, m, steps, form):
        """Roofline of the dominant kernel (the solve).  Algorithmic bytes per mesh*lambda point:
        outputs U (nz+6 per nz), kappa, V (8 B each) + the per-column records read once (shared
        by nw wavelengths).  Algorithmic flops per point: the reference's census, 97 (90
        add/mul + 7 divisions; transcendentals not counted)."""
        nz, nw = self.nz, self.nw
        rec = 26 * 8.0 if form != "mixed" else 64 * 4.0
        bytes_pt = 8.0 * (self.mz / nz) + 16.0 + rec / nw
        launch_ms = m["solve_ms"] / max(m["nsolve"], 1)
        pts_launch = m["pts_step"] * steps / max(m["nsolve"], 1)
        pk = peaks()
        hbm_peak = pk.get("hbm_gbs", 6650.0)
        achieved = bytes_pt * pts_launch / (launch_ms / 1e3) / 1e9
        flops = 97.0 * pts_launch / (launch_ms / 1e3) / 1e12
        tpp = TRAFFIC_BYTES_PER_POINT.get(form) if (self.nz, self.nw, self.layout) == (512, 256, 1) else None
        res = {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "traffic": tpp * pts_launch if tpp else None,
                "traffic_source": "ncu capture of a 1024-column launch, scaled by points" if tpp else None,
                "kernel": "k_solve_staged" if form != "mixed" else "k_solve_mixed_staged",
                "launch_ms": launch_ms, "points_per_launch": pts_launch, "algorithmic_bytes_per_point": bytes_pt,
                "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in pk else "fallback",
                "algorithmic_tflops": flops, "census_flops_per_point": 97,
                "solve_share_of_step": m["solve_ms"] / m["total_ms"], "pillars_ms_per_step": m["pil_ms"] / steps}
        fc = FP_COUNTERS["mixed" if form == "mixed" else "plain"]
        rate = pts_launch / (launch_ms / 1e3)
        res["fp64"] = {"executed_flops_per_point": fc["fp64_flops_per_point"],
                       "achieved_tflops": fc["fp64_flops_per_point"] * rate / 1e12, "peak_tflops": FP64_PEAK_TFLOPS,
                       "frac": fc["fp64_flops_per_point"] * rate / 1e12 / FP64_PEAK_TFLOPS,
                       "pipe_active": fc["fp64_pipe_active"], "peak_source": "nominal"}
        res["fp32"] = {"executed_flops_per_point": fc["fp32_flops_per_point"],
                       "achieved_tflops": fc["fp32_flops_per_point"] * rate / 1e12, "peak_tflops": FP32_PEAK_TFLOPS,
                       "frac": fc["fp32_flops_per_point"] * rate / 1e12 / FP32_PEAK_TFLOPS,
                       "fma_pipe_active": fc["fma_pipe_active"], "xu_active": fc["xu_active"], "peak_source": "nominal"}
        res["fp_counters_source"] = "ncu counters of a 1024-column launch (profiles/fp_pipes_*); rate from this run"
        return res


# The reference's published rate for this path: 0.14415 us per mesh*lambda point (its README,
# multiInTest sample, one CPU core) = 6.94e6 points/s.
PUBLISHED_POINTS_PER_S = 1e6 / 0.14415

# Executed floating-point work per mesh*lambda point of the solve kernels (ncu counters of a
# 1024-column launch of this grid: profiles/fp_pipes_k_solve_staged_k_solve_mixed_staged_agn_32x32x512x256.txt):
# FP64 flops = DADD + DMUL + 2 DFMA, FP32 flops = FADD + FMUL + 2 FFMA, and the pipes' activity.
FP_COUNTERS = {"plain": {"fp64_flops_per_point": 347.6, "fp32_flops_per_point": 12.0, "fp64_pipe_active": 0.470,
                         "fma_pipe_active": 0.096, "xu_active": 0.052},
               "mixed": {"fp64_flops_per_point": 14.1, "fp32_flops_per_point": 128.9, "fp64_pipe_active": 0.052,
                         "fma_pipe_active": 0.328, "xu_active": 0.461}}
FP64_PEAK_TFLOPS, FP32_PEAK_TFLOPS = 37.0, 75.0  # nominal B200 (no measured FP figure in MEASURED_PEAKS.json)

# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) per mesh*lambda point of the solve
# kernel, from one ncu --set full capture of a 1024-column launch of this grid (outputs 3.2 GB,
# larger than L2), scaled to a launch by its points: profiles/k_solve_staged_plain_agn_32x32x512x256.txt
# and profiles/k_solve_mixed_staged_agn_32x32x512x256.txt.
TRAFFIC_BYTES_PER_POINT = {"plain": 71.8, "mixed": 56.7}


def flux_error(g, form_a, form_b, eps=1e-7, seed=7):
    """Relative difference of the emergent-flux planes of form_a against form_b (FP64) over the
    whole grid, with the conditioning mask: s = relative change of form_b's flux when rho is
    perturbed by eps * N(0,1) relative per cell.  Items with s <= 100 eps are 'conditioned'
    (their FP64 flux is stable to 100x the perturbation); elsewhere the FP64 flux itself moves
    by more than 1e-5 under perturbations below float32 resolution of the input."""
    import torch

    def planes(form, rho=None):
        if rho is not None:
            keep, g.rho = g.rho, rho
        g.step(form, fields=False)
        g.sync()
        if rho is not None:
            g.rho = keep
        return torch.stack([g.Vtop.clone(), g.Vbot.clone()])

    rb = planes(form_b)
    gen = torch.Generator(device=g.rho.device)
    gen.manual_seed(seed)
    pert = g.rho * (1.0 + eps * torch.randn(g.rho.shape, generator=gen, device=g.rho.device, dtype=g.rho.dtype))
    rp = planes(form_b, pert)
    del pert
    g.eng.mixed_repairs()  # counts from here: the items form_a re-solves in FP64
    ra = planes(form_a)
    repaired = g.eng.mixed_repairs()
    ok = torch.isfinite(rb) & (rb != 0) & torch.isfinite(rp)
    rel = ((ra - rb).abs() / rb.abs())[ok]
    sens = ((rp - rb).abs() / rb.abs())[ok]
    cond = sens <= 100 * eps
    sub = lambda x: x.float()[torch.randperm(x.numel(), device=x.device)[:1 << 24]]
    q = lambda x, p: torch.quantile(sub(x), p).item() if x.numel() else None
    sensitive = sens > 10 * eps  # items whose FP64 flux responds to the perturbation
    backward = rel[sensitive] / sens[sensitive] * eps
    return {"reference_form": form_b, "items": int(rel.numel()),
            "repaired_items": repaired, "repaired_frac": repaired / (g.ncol * g.nw),
            "all": {"max": rel.max().item(), "p99": q(rel, 0.99), "p9999": q(rel, 0.9999),
                    "frac_above_1e-4": (rel > 1e-4).double().mean().item()},
            "conditioned": {"definition": f"FP64 flux changes by <= {100 * eps:g} under a {eps:g} relative "
                                          "random perturbation of rho",
                            "fraction_of_items": cond.double().mean().item(),
                            "max": rel[cond].max().item(), "p99": q(rel[cond], 0.99),
                            "frac_above_1e-4": (rel[cond] > 1e-4).double().mean().item()},
            "sensitive_items": {"definition": f"FP64 flux changes by > {10 * eps:g} under the perturbation",
                                "count": int(sensitive.sum()),
                                "equivalent_rho_perturbation_p50": q(backward, 0.5),
                                "equivalent_rho_perturbation_max": backward.max().item() if backward.numel() else None}}


def intensity_error(g, form_a="mixed", form_b="stable"):
    """Relative difference of the mean intensity U (every z, ghost zones included, every item)
    of form_a against form_b on a grid that fits one chunk (its fields stay on the device)."""
    import torch
    if g.nchunk != 1:
        raise ValueError("intensity_error: the grid must fit one chunk")

    def field(form):
        g.step(form, fields=True)
        g.sync()
        return g.sets[0]["U"].clone()

    ub, ua = field(form_b), field(form_a)
    ok = torch.isfinite(ub) & (ub != 0)
    rel = ((ua - ub).abs() / ub.abs())[ok]
    sub = rel.float()[torch.randperm(rel.numel(), device=rel.device)[:1 << 24]]
    res = {"reference_form": form_b, "values": int(rel.numel()), "p50": torch.quantile(sub, 0.5).item(),
           "p99": torch.quantile(sub, 0.99).item(), "max": rel.max().item(),
           "frac_above_1e-4": (rel > 1e-4).double().mean().item()}
    del ub, ua, rel, sub
    return res


def flux_error_vs_plain(g, agree=1e-8):
    """Mixed emergent flux against the reference-form (plain) FP64 flux where that flux is
    itself accurate: items whose plain and stable FP64 fluxes agree to `agree` relative.  (In
    optically thin top layers the plain form's flux is rounding noise that a random
    perturbation of rho does not move, so a perturbation mask cannot isolate it.)"""
    import torch

    def planes(form):
        g.step(form, fields=False)
        g.sync()
        return torch.stack([g.Vtop.clone(), g.Vbot.clone()])

    rp, rs, rm = planes("plain"), planes("stable"), planes("mixed")
    ok = torch.isfinite(rp) & (rp != 0) & torch.isfinite(rs) & (rs != 0)
    acc = ok & ((rp - rs).abs() <= agree * rs.abs())
    rel = ((rm - rp).abs() / rp.abs())[acc]
    sub = lambda x: x.float()[torch.randperm(x.numel(), device=x.device)[:1 << 24]]
    q = lambda x, pq: torch.quantile(sub(x), pq).item() if x.numel() else None
    return {"reference_form": "plain", "mask": f"plain and stable FP64 emergent fluxes agree to {agree:g} relative",
            "items": int(ok.sum()), "fraction_in_mask": acc.double().sum().item() / max(int(ok.sum()), 1),
            "max": rel.max().item() if rel.numel() else None, "p99": q(rel, 0.99),
            "frac_above_1e-4": (rel > 1e-4).double().mean().item() if rel.numel() else None}


def _time_batch(a, eng, dev, d, form):
    """Creates, binds and tunes a batch of `form` over workload d, then times a.steps graph
    replays (CUDA events on the launching stream).  A plain-form zero pivot is reported by
    oco_batch_wait after every item is computed; it does not stop the measurement."""
    import torch
    from ocotillo_b200 import OcoError

    def wait(b):
        try:
            b.wait()
            return False
        except OcoError as e:
            if e.code != -3:
                raise
            return True

    b = eng.batch(d["nz"], d["nw"], d["dz"], d["waves"], d["wave_off"], layout=1, form=form)
    rho = torch.from_numpy(d["rho"]).to(dev)
    T = torch.from_numpy(d["T"]).to(dev)
    out = b.alloc(dev)
    b.bind(rho, T, out)
    try:
        info = b.tune()
    except OcoError as e:
        if e.code != -3:
            raise
        info = b.info()
    for _ in range(a.warmup):
        b.run()
    zp = wait(b)
    st = torch.cuda.current_stream(dev)
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    evs[0].record(st)
    for i in range(a.steps):
        b.run(st)
        evs[i + 1].record(st)
    zp = wait(b) or zp
    ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(a.steps)]
    total = evs[0].elapsed_time(evs[-1])
    info = b.info()
    res = {"value": info["npoints"] * a.steps / (total / 1e3), "unit": "points/s", "form": form,
           "ms_per_run": total / a.steps, "p50_ms": pct(ms, 0.5), "p99_ms": pct(ms, 0.99),
           "tiling": info["tiling"], "blocks_per_sm": info["blocks_per_sm"],
           "tuning": [(c["tiling"], c["blocks_per_sm"], round(c["ms"], 3)) for c in info["candidates"]],
           "graph_replays": info["graph_launches"]}
    if form == "plain":
        res["zero_pivot_items"] = zp
    b.close()
    del out, rho, T
    torch.cuda.empty_cache()
    return res, info


def measure_batch(a, eng, dev):
    """Config 'batching form': the ragged batch in the mixed form and, on the same columns, in
    the plain FP64 form (the same persistent warp-column kernel design with FP64 records)."""
    from ocotillo_b200 import workloads
    d = workloads.ragged_batch(ncol=a.batch_cols, seed=4)
    res, info = _time_batch(a, eng, dev, d, "mixed")
    res.update({"columns": info["ncol"], "points": info["npoints"], "max_nz": info["max_nz"],
                "max_nw": info["max_nw"], "layout": "per column [z][lambda]",
                "workload": "8192 columns, nz log-uniform [64,2048], nw log-uniform [32,1024], Athena-style "
                            "rho/p (0.5 dex lognormal), T = mu m_u p/(rho k), mu=0.6, floor 2000 K (seed 4)"})
    plain, _ = _time_batch(a, eng, dev, d, "plain")
    res["plain"] = plain
    res["ratio_mixed_vs_plain"] = res["value"] / plain["value"]
    res["emergent_flux_rel_err"] = batch_flux_error(eng, dev, d)
    return res


def batch_flux_error(eng, dev, d):
    """The mixed batch's emergent fluxes against the stable FP64 batch's, every item of the batch
    (both runs store only Vtop and Vbot), with the re-solve at its current threshold."""
    import torch
    from ocotillo_b200 import OcoError
    fl, rep = {}, 0
    for form in ("stable", "mixed"):
        b = eng.batch(d["nz"], d["nw"], d["dz"], d["waves"], d["wave_off"], layout=1, form=form)
        rho = torch.from_numpy(d["rho"]).to(dev)
        T = torch.from_numpy(d["T"]).to(dev)
        out = b.bind(rho, T, b.alloc(dev, want=("Vtop", "Vbot")))
        eng.mixed_repairs()
        b.run()
        try:
            b.wait()
        except OcoError as e:
            if e.code != -3:
                raise
        rep = eng.mixed_repairs() if form == "mixed" else rep
        fl[form] = torch.stack([out["Vtop"], out["Vbot"]])
        b.close()
        del out, rho, T
    ra, rb = fl["mixed"], fl["stable"]
    ok = torch.isfinite(rb) & (rb != 0)
    rel = ((ra - rb).abs() / rb.abs())[ok].double()
    items = int(rb[0].numel())
    res = {"reference_form": "stable", "items": items, "repaired_items": int(rep), "repaired_frac": rep / items,
           "max": float(rel.max()), "p99": float(torch.quantile(rel[torch.randperm(rel.numel(), device=rel.device)[:1 << 24]].float(), 0.99)),
           "frac_above_1e-4": float((rel > 1e-4).double().mean()), "sample": "every item of the batch (Vtop and Vbot)"}
    del fl, ra, rb, rel
    torch.cuda.empty_cache()
    return res


def measure_precision_c3(a, eng, dev):
    """Config 'precision form': 512x512 columns, nz=1024, nw=512 log-spaced 100 A - 10 um, the AGN
    construction with rho0 drawn log-uniform in [1e-11, 1e-7].  Mixed and plain throughput over
    the whole grid (2048-column chunks, lambda-fastest outputs), the mixed emergent-flux error
    against the difference-form FP64 path over the whole grid, and against the reference-form
    FP64 path and the mean-intensity error on a 32x32-column draw of the same construction."""
    import copy
    import torch
    b = copy.copy(a)
    b.nx = b.ny = 512
    b.nz, b.nw, b.chunk_cols, b.layout = 1024, 512, 2048, "lambda"
    steps = max(1, min(a.steps, 2))
    g = Grid(b, eng, dev, 0, workload="precision")
    eng.set_wavelengths(g.wa)
    mm = g.measure("mixed", steps, 1, 1)
    mp = g.measure("plain", steps, 1, 1)
    rho0 = g.rho0
    g.sets = None  # the error passes store the emergent planes only
    torch.cuda.empty_cache()
    err = flux_error(g, "mixed", "stable")
    del g
    torch.cuda.empty_cache()
    s = copy.copy(b)
    s.nx = s.ny = 32
    s.chunk_cols = 1024
    gs = Grid(s, eng, dev, 0, workload="precision")
    res = {"workload": "512x512 columns, nz=1024, nw=512, rho0 = %.3g g/cm^3 (log-uniform draw, seed 3)" % rho0,
           "points": 512 * 512 * 1024 * 512, "steps": steps,
           "mixed_value": mm["value"], "plain_value": mp["value"], "ratio": mm["value"] / mp["value"],
           "mixed_ms_per_step": mm["total_ms"] / steps, "plain_ms_per_step": mp["total_ms"] / steps,
           "emergent_flux_rel_err": dict(err, sample="whole grid (2.6e8 emergent fluxes)"),
           "error_sample": "32x32 columns of the same construction, all z and lambda",
           "emergent_flux_rel_err_vs_plain": flux_error_vs_plain(gs),
           "mean_intensity_rel_err": intensity_error(gs)}
    del gs
    torch.cuda.empty_cache()
    return res


def run_stream(eng, dev, form, specs, make, pinned, window=None):
    """Runs one job stream through a fresh server.  Each job's inputs are generated on the device
    (make(k)) when it arrives and released once the server has consumed them, so only queued jobs
    hold input memory.  Open loop (window None): job k arrives at its arrival_s.  Closed loop
    (window w): a job arrives whenever fewer than w are outstanding, which keeps the server
    saturated.  Every finished job is fetched at once (emergent-flux planes into pinned host
    memory).  Per job: device latency (submit -> results complete on the device, server clock),
    fetch latency (submit -> planes in host memory) and admission wait (submit -> admitted)."""
    import torch
    from ocotillo_b200 import Server, workloads
    srv = Server(dev.index or 0, max_jobs=4, max_nz=1024, reserve_bytes=24e9)
    wr, wt, _ = workloads.job_arrays_device({"nx": 8, "ny": 8, "nz": 128, "nw": 64, "rho0": 1e-9, "seed": 1}, eng)
    jid = srv.submit(wr, wt, workloads.log_wavelengths(64), 1e16 / 127, form=form)  # warm-up
    srv.wait(jid)
    srv.fetch(jid)
    del wr, wt
    torch.cuda.synchronize(dev)
    ids = {}
    pending = list(range(len(specs)))
    outstanding = set()
    live = {}  # inputs of submitted jobs the server has not consumed yet
    done = {}
    t0 = time.monotonic()
    while pending or outstanding:
        now = time.monotonic()
        while pending and (len(outstanding) < window if window else t0 + specs[pending[0]]["arrival_s"] <= now):
            k = pending.pop(0)
            rho, T, dz = make(k)
            ids[k] = srv.submit(rho, T, workloads.log_wavelengths(specs[k]["nw"]), dz, form=form)
            live[k] = (rho, T)
            outstanding.add(k)
        for k in list(outstanding):
            st = srv.status(ids[k])
            if k in live and (st["inputs_consumed"] or st["state"] in ("done", "failed")):
                del live[k]
            if st["state"] == "done":
                sp = specs[k]
                n = sp["nw"] * sp["nx"] * sp["ny"]
                shp = (sp["nw"], sp["nx"], sp["ny"])
                srv.fetch(ids[k], out={"Vtop": pinned[0][:n].reshape(shp), "Vbot": pinned[1][:n].reshape(shp)})
                done[k] = (st, time.monotonic())
                outstanding.discard(k)
            elif st["state"] == "failed":
                raise RuntimeError(f"serving job {k} failed: {st['error']}")
        if pending and not outstanding and not window:
            time.sleep(max(0.0, min(0.002, t0 + specs[pending[0]]["arrival_s"] - time.monotonic())))
        else:
            time.sleep(0.0005)
    srv.close()
    lat, fet, adm, cls = [], [], [], {}
    first, last, pts = None, None, 0
    for k, (st, tf) in done.items():
        sp = specs[k]
        lat.append(1e3 * (st["done_s"] - st["submit_s"]))
        fet.append(1e3 * (tf - st["submit_s"]))
        adm.append(1e3 * (st["admit_s"] - st["submit_s"]))
        cls.setdefault(sp["nx"], []).append((lat[-1], fet[-1]))
        first = st["submit_s"] if first is None else min(first, st["submit_s"])
        last = tf if last is None else max(last, tf)
        pts += sp["nx"] * sp["ny"] * sp["nz"] * sp["nw"]
    return {"jobs": len(lat), "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99),
            "fetch_p50_ms": pct(fet, 0.5), "fetch_p99_ms": pct(fet, 0.99),
            "admission_wait_p99_ms": pct(adm, 0.99), "admission_wait_max_ms": max(adm),
            "throughput_points_per_s": pts / (last - first), "makespan_s": last - first,
            "per_class": {f"{n}x{n}": {"jobs": len(v), "p50_ms": pct([x[0] for x in v], 0.5),
                                       "p99_ms": pct([x[0] for x in v], 0.99),
                                       "fetch_p99_ms": pct([x[1] for x in v], 0.99)} for n, v in sorted(cls.items())}}


def measure_serving_sweep(a, eng, dev):
    """Config 'serving form': the Poisson job stream (seed 5) at rising arrival rates.  The
    saturation rate comes from the same jobs run in a closed loop that keeps 8 jobs outstanding
    (jobs / makespan); the mixed form then runs at 0.3, 0.5, 0.7 and 0.9 of its saturation rate and
    the plain FP64 form at half of its own.  Each job's inputs are generated on the device when it
    arrives (the same seed gives the same jobs at every rate; only the arrival times scale)."""
    import torch
    from ocotillo_b200 import workloads
    n = a.serve_jobs
    base = workloads.serving_stream(n, 1.0, seed=5)
    make = lambda k: workloads.job_arrays_device(base[k], eng)  # the same inputs at every rate
    maxn = max(sp["nw"] * sp["nx"] * sp["ny"] for sp in base)
    pinned = [torch.empty(maxn, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    points = int(sum(sp["nx"] * sp["ny"] * sp["nz"] * sp["nw"] for sp in base))
    res = {"jobs_per_run": n, "points_per_run": points, "max_jobs_resident": 4,
           "stream": "Poisson (seed 5); nx=ny in {64,128,256,512}, nz U[128,1024], nw U[64,512], rho0 log-uniform "
                     "[1e-11,1e-7]; outputs: emergent-flux planes, fetched into pinned host memory as each job ends",
           "latency": "p50/p99_ms: submit to results complete on the device; fetch_*: submit to planes in host memory"}
    fracs = {"mixed": (0.3, 0.5, 0.7, 0.9), "plain": (0.5,)}
    for form in ("mixed", "plain"):
        sat = run_stream(eng, dev, form, base, make, pinned, window=8)
        sat_rate = n / sat["makespan_s"]
        runs = {"saturation": dict(sat, rate_jobs_per_s=sat_rate, loop="closed, 8 jobs outstanding")}
        for f in fracs[form]:
            specs = [dict(sp, arrival_s=sp["arrival_s"] / (f * sat_rate)) for sp in base]
            runs[f"{f:g}x_saturation"] = dict(run_stream(eng, dev, form, specs, make, pinned),
                                              rate_jobs_per_s=f * sat_rate)
        res[form] = runs
    torch.cuda.empty_cache()
    mx = res["mixed"]
    res["headline"] = {"serving_saturation_jobs_per_s": mx["saturation"]["rate_jobs_per_s"],
                       "serving_rate_jobs_per_s": mx["0.7x_saturation"]["rate_jobs_per_s"],
                       "serving_p50_ms": mx["0.7x_saturation"]["p50_ms"], "serving_p99_ms": mx["0.7x_saturation"]["p99_ms"],
                       "serving_fetch_p99_ms": mx["0.7x_saturation"]["fetch_p99_ms"],
                       "serving_plain_p99_ms": res["plain"]["0.5x_saturation"]["p99_ms"]}
    return res


def _rel_inf(a, b):
    with np.errstate(all="ignore"):
        return np.nan_to_num(np.abs(a - b) / np.abs(b), nan=np.inf)


def parity_vs_glibc(eng):
    """The plain form (GPU) against the oracle built on glibc's exp/log/pow (what the gfortran
    reference calls), on 16 AGN columns x 64 wavelengths of two constructions: the benchmark
    grid's (density floor 1e-24) and the NongreyAGN deck's floor (1e-15).  The conditioning mask
    keeps the items whose U (every z) and emergent fluxes move by < 1e-14 relative when rho is
    perturbed by one ulp (glibc oracle); reported: the fraction of items in the mask, the largest
    relative difference there (U, kappa, Vtop, Vbot), whether the finite class and sign agree
    everywhere, and the fraction of bit-identical items."""
    from oracle import pyoracle
    from ocotillo_b200 import workloads
    res = {"mask": "U and emergent fluxes change < 1e-14 under a one-ulp random perturbation of rho"}
    for name, floor in (("floor_1e-24", 1e-24), ("floor_1e-15", 1e-15)):
        rho, T, dz = workloads.agn_block(4, 4, 512, seed=2, rho_floor=floor)
        wa = workloads.log_wavelengths(256)[::4]
        eng.set_wavelengths(wa)
        gpu = eng.solve_block(rho, T, dz, form="plain", allow_zero_pivot=True)
        ref = pyoracle.solve_block(rho, T, wa, dz, form=pyoracle.FORM_REFERENCE, backend="glibc")
        rp = rho * (1.0 + 2.0 ** -52 * np.random.default_rng(7).standard_normal(rho.shape))
        refp = pyoracle.solve_block(rp, T, wa, dz, form=pyoracle.FORM_REFERENCE, backend="glibc")
        s_ = np.maximum(_rel_inf(refp["U"], ref["U"]).max(-1),
                        np.maximum(_rel_inf(refp["V"][..., -1], ref["V"][..., -1]),
                                   _rel_inf(refp["V"][..., 0], ref["V"][..., 0])))
        mask = s_ < 1e-14
        d = np.maximum(np.maximum(_rel_inf(gpu["U"], ref["U"]).max(-1), _rel_inf(gpu["kappa"], ref["kappa"]).max(-1)),
                       np.maximum(_rel_inf(gpu["Vtop"], ref["V"][..., -1]), _rel_inf(gpu["Vbot"], ref["V"][..., 0])))
        cls = True
        for x, y in ((gpu["U"], ref["U"]), (gpu["kappa"], ref["kappa"]), (gpu["Vtop"], ref["V"][..., -1]),
                     (gpu["Vbot"], ref["V"][..., 0])):
            fx, fy = np.isfinite(x), np.isfinite(y)
            cls = cls and bool(np.array_equal(fx, fy) and np.array_equal(np.sign(x[fx]), np.sign(y[fy])))
        res[name] = {"items": int(d.size), "in_mask": float(mask.mean()),
                     "max_rel_in_mask": float(d[mask].max()) if mask.any() else None, "class_equal": cls,
                     "bitwise": float((d == 0).mean())}
    return res


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
    from ocotillo_b200 import Engine, workloads

    eng = Engine(local)
    g = Grid(a, eng, dev, rank)
    eng.set_wavelengths(g.wa)
    eng.set_profiling(True)
    ncol, nz, nw, mz = g.ncol, g.nz, g.nw, g.mz

    m = g.measure(a.form, a.steps, a.warmup, world, dist, Clocks(local))
    roof = g.roofline(m, a.steps, a.form)

    extra = {}
    if world == 1 and not a.no_extra:
        other = "mixed" if a.form != "mixed" else "plain"
        mm = g.measure(other, a.steps, a.warmup, world)
        plain_v, mixed_v = (m["value"], mm["value"]) if other == "mixed" else (mm["value"], m["value"])
        mixed_m = mm if other == "mixed" else m
        extra["mixed"] = {"value": mixed_v, "unit": "points/s", "ms_per_step": mixed_m["total_ms"] / a.steps,
                          "latency_ms": {"p50": pct(mixed_m["step_ms"], 0.5), "p99": pct(mixed_m["step_ms"], 0.99)},
                          "ratio_vs_plain_fp64": mixed_v / plain_v,
                          "emergent_flux_rel_err": flux_error(g, "mixed", "stable"),
                          "emergent_flux_rel_err_vs_plain": flux_error_vs_plain(g),
                          "roofline": g.roofline(mixed_m, a.steps, "mixed")}
        extra["plain_fp64_value"] = plain_v
        import copy
        sa = copy.copy(a)
        sa.nx = sa.ny = 32
        sa.chunk_cols, sa.layout = 1024, "lambda"
        gs = Grid(sa, eng, dev, rank)
        extra["mixed"]["mean_intensity_rel_err"] = dict(
            intensity_error(gs), sample="32x32 columns of the same construction (seed 2), all z and lambda")
        del gs
        torch.cuda.empty_cache()

    # ---- e2e: host arrays through oco_solve_block (pinned), one batch of columns per step
    e2e, e2e_mixed = None, None
    if not a.no_e2e:
        E = min(a.e2e_cols, ncol)
        pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()
        rho_p = pin((ncol, nz))
        T_p = pin((ncol, nz))
        rho_p[:] = g.rho_h.reshape(ncol, nz)
        T_p[:] = g.T_h.reshape(ncol, nz)
        outs = {"U": pin((nw, E, 1, mz)), "kappa": pin((nw, E, 1, nz)), "V": pin((nw, E, 1, nz)),
                "Vtop": pin((nw, E, 1)), "Vbot": pin((nw, E, 1))}
        nb = ncol // E

        def e2e_measure(form):
            def e2e_step(i):
                c0 = (i % nb) * E
                eng.solve_block(rho_p[c0:c0 + E].reshape(E, 1, nz), T_p[c0:c0 + E].reshape(E, 1, nz), g.dz,
                                form=form, out=outs, allow_zero_pivot=True)

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
            el = max_over_ranks(time.perf_counter() - t0, world, dist, dev)
            return {"value": whole_job_rate(world, E * nz * nw, a.steps, 1e3 * el), "unit": "points/s",
                    "h2d_bytes_per_step": 2 * E * nz * 8, "d2h_bytes_per_step": E * nw * (mz + 2 * nz + 2) * 8,
                    "columns_per_step": E, "form": form,
                    "outputs": "U, kappa, V, Vtop, Vbot (all, FP64, reference layout)",
                    "p50_ms": 1e3 * pct(lat, 0.5), "p99_ms": 1e3 * pct(lat, 0.99)}

        e2e = e2e_measure(a.form)
        if world == 1 and not a.no_extra:
            e2e_mixed = e2e_measure("mixed" if a.form != "mixed" else "plain")
        del outs
        # the same call returning only the emergent-flux planes (the spectra), whole grid per step
        if world == 1 and not a.no_extra:
            fl = {"Vtop": pin((nw, ncol, 1)), "Vbot": pin((nw, ncol, 1))}
            rho_all, T_all = rho_p.reshape(ncol, 1, nz), T_p.reshape(ncol, 1, nz)
            for form in (a.form, "mixed"):
                for i in range(max(1, a.warmup)):
                    eng.solve_block(rho_all, T_all, g.dz, form=form, out=fl, want=("Vtop", "Vbot"),
                                    allow_zero_pivot=True)
                lat = []
                for i in range(a.steps):
                    s0 = time.perf_counter()
                    eng.solve_block(rho_all, T_all, g.dz, form=form, out=fl, want=("Vtop", "Vbot"),
                                    allow_zero_pivot=True)
                    lat.append(time.perf_counter() - s0)
                extra[f"e2e_emergent_flux_only_{form}"] = {
                    "value": ncol * nz * nw * a.steps / sum(lat), "unit": "points/s", "form": form,
                    "h2d_bytes_per_step": 2 * ncol * nz * 8, "d2h_bytes_per_step": 2 * ncol * nw * 8,
                    "outputs": "Vtop, Vbot only (oco_solve_block with U, kappa, V NULL), whole grid per call",
                    "p50_ms": 1e3 * pct(lat, 0.5), "p99_ms": 1e3 * pct(lat, 0.99)}
            del fl
        del rho_p, T_p

    if world == 1 and not a.no_extra:
        g.sets = None
        torch.cuda.empty_cache()
        extra["batch"] = measure_batch(a, eng, dev)
        torch.cuda.empty_cache()
    if world == 1 and not a.no_extra and not a.no_serve:
        extra["serving"] = measure_serving_sweep(a, eng, dev)
        torch.cuda.empty_cache()
    if world == 1 and not a.no_extra and not a.no_c3:
        extra["precision_c3"] = measure_precision_c3(a, eng, dev)
        torch.cuda.empty_cache()

    cpu, cpu1 = None, None
    if rank == 0 and world == 1 and not a.no_cpu:
        # the CPU leg also checks the plain form against the glibc build of the oracle
        extra["parity_vs_glibc"] = parity_vs_glibc(eng)
        procs = os.cpu_count() or 1
        v, dt, pts = cpu_baseline(g.rho_h, g.T_h, g.wa, g.dz, min(a.cpu_cols, ncol), procs)
        cpu = {"value": v, "unit": "points/s", "cores": procs, "kind": "port",
               "sample": f"first {min(a.cpu_cols, ncol)} columns of the same grid, all z and lambda "
                         f"({pts:.3g} points, {dt:.1f} s wall on {procs} processes), glibc math"}
        v1, dt1, pts1 = cpu_baseline(g.rho_h, g.T_h, g.wa, g.dz, min(a.cpu1_cols, ncol), 1)
        cpu1 = {"value": v1, "unit": "points/s", "cores": 1, "kind": "port",
                "sample": f"first {min(a.cpu1_cols, ncol)} columns of the same grid, all z and lambda "
                          f"({pts1:.3g} points, {dt1:.1f} s on one process), glibc math: the serial "
                          "reference's setting (its published rate is 6.94e6 points/s on one core)"}

    if rank == 0:
        line = {"details": extra} if extra else {}
        line.update(contract_line(a, world, m, g, roof, e2e, cpu))
        if cpu1:
            line["cpu_baseline_1core"] = cpu1
        line.update(headline(extra, e2e_mixed, cpu1))
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


def contract_line(a, world, m, g, roof, e2e, cpu):
    """The keys of the one-line result every run prints (value: the plain FP64 form)."""
    line = {"metric": METRIC, "value": m["value"], "unit": "points/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": m["total_ms"] / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": m["value"] / PUBLISHED_POINTS_PER_S,
            "vs_baseline_source": "reference's published xy-loop rate, 6.94e6 mesh*lambda points/s (one CPU "
                                  "core, multiInTest sample; README.md:41-42)",
            "dtype": "f64" if a.form != "mixed" else "f32 (FP64 Saha)", "data": "synthetic",
            "config": config_dict(a, a.form),
            "latency_ms": {"p50": pct(m["step_ms"], 0.5), "p99": pct(m["step_ms"], 0.99)},
            "zero_pivot_items": g.zero_pivot, "clocks": m["clocks"], "gpu_launches": int(m["launches"]),
            "roofline": roof, "e2e": e2e, "cpu_baseline": cpu}
    line["config"]["layout"] = a.layout
    line["config"]["chunk_columns"] = g.CH
    line["config"]["parallelism"] = f"columns sharded over {world} rank(s), no exchange"
    return line


def headline(extra, e2e_mixed, cpu1):
    """Compact top-level keys, printed last: the mixed form against the plain FP64 form on each
    config, the mixed error bar, serving p99 at a named rate, the one-core CPU rate."""
    h = {}
    mx = extra.get("mixed")
    if mx:
        er = mx["emergent_flux_rel_err"]
        h.update({"mixed_value": mx["value"], "mixed_ratio": mx["ratio_vs_plain_fp64"],
                  "mixed_flux_err_max": er["all"]["max"], "mixed_flux_frac_above_1e-4": er["all"]["frac_above_1e-4"],
                  "mixed_repaired_frac": er["repaired_frac"]})
    if e2e_mixed:
        h["mixed_e2e"] = e2e_mixed["value"]
    c3 = extra.get("precision_c3")
    if c3:
        er = c3["emergent_flux_rel_err"]
        h.update({"c3_mixed_value": c3["mixed_value"], "c3_mixed_ratio": c3["ratio"], "c3_flux_err_max": er["all"]["max"],
                  "c3_flux_frac_above_1e-4": er["all"]["frac_above_1e-4"], "c3_repaired_frac": er["repaired_frac"]})
    bt = extra.get("batch")
    if bt:
        h.update({"c4_mixed_value": bt["value"], "c4_mixed_ratio": bt["ratio_mixed_vs_plain"]})
        if "emergent_flux_rel_err" in bt:
            e4 = bt["emergent_flux_rel_err"]
            h.update({"c4_flux_err_max": e4["max"], "c4_flux_frac_above_1e-4": e4["frac_above_1e-4"],
                      "c4_repaired_frac": e4["repaired_frac"]})
    sv = extra.get("serving")
    if sv and sv.get("headline"):
        h.update(sv["headline"])
    pg = extra.get("parity_vs_glibc")
    if pg:
        h["glibc_parity"] = {k: pg["floor_1e-15"][k] for k in ("in_mask", "max_rel_in_mask", "class_equal")}
    if cpu1:
        h["cpu_1core_value"] = cpu1["value"]
    return h


if __name__ == "__main__":
    main()
