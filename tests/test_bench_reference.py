"""The benchmark's reference arm (`bench.py --impl reference`: the CPU restatement of the
reference loop on the host cores) prints one JSON line with the benchmark's fields (value,
unit, CPU-baseline description, end-to-end entry), checked here on a small grid so that it
runs in seconds; and the summary of the clock samples taken during the timed region."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nx", "2", "--ny", "2",
                        "--steps", "3", "--warmup", "3"], capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "points/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 3 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["config"]["nx"] == 2 and d["config"]["ny"] == 2 and "2x2 columns" in d["config"]["workload"]
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


class _Done:
    def terminate(self):
        pass

    def wait(self):
        return 0


def _clocks_from(rows):
    sys.path.insert(0, ROOT)
    import bench
    c = bench.Clocks(0)
    c.f.write("".join(r + "\n" for r in rows))
    c.p = _Done()
    return c.stop()


def test_clock_record_summary():
    """The clock record of the timed region (nvidia-smi samples): median SM clock, max clock,
    the throttle reasons seen Active in any sample, malformed lines skipped."""
    s = _clocks_from(["0, 1965, 1965, 900.50, 0x0, Not Active, Not Active, Not Active, Not Active",
                      "0, 1900, 1965, 990.10, 0x4, Not Active, Not Active, Not Active, Active",
                      "garbage",
                      "0, 1950, 1965, [N/A], 0x0, Not Active, Not Active, Not Active, Not Active"])
    assert s["sm_mhz"] == 1950.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"] and s["power_w_max"] == 990.1
    s = _clocks_from(["0, 1500, 1965, [N/A], 0x0, Active, Not Active, Active, Not Active"])
    assert s["reasons"] == ["hw_slowdown", "sw_thermal_slowdown"] and s["power_w_max"] is None
    assert _clocks_from([])["reasons"] == ["no samples"]


def test_reference_arm_under_torchrun_two_ranks():
    """Launched as the multi-GPU bench is (torchrun, two ranks), rank 0 alone runs the reference
    arm and prints its one line; the other rank exits 0 without work."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--nx", "2", "--ny", "2", "--steps", "3", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, cwd=ROOT, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip().startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0


def test_profile_commands_parse(monkeypatch):
    """Every profile summary gives the bench command it was captured from; each must still be a
    valid bench.py command line (the chunking of its grid included)."""
    import glob
    import re
    sys.path.insert(0, ROOT)
    import bench
    found = 0
    for f in glob.glob(os.path.join(ROOT, "profiles", "*.txt")):
        text = open(f).read().replace("\\\n", " ")
        for m in re.finditer(r"python bench\.py([^\n]*)", text):
            argv = m.group(1).split()
            monkeypatch.setattr(sys, "argv", ["bench.py"] + argv)
            a = bench.parse()
            ncol = a.nx * a.ny
            assert ncol % min(a.chunk_cols, ncol) == 0, (f, argv)
            found += 1
    assert found >= 6
