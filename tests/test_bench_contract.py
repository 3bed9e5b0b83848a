"""The reference arm of bench.py (CPU only): one JSON line with the keys the
benchmark contract names, on the same metric and workload as the GPU arm,
and no output from ranks other than 0."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "1"],
                         capture_output=True, text=True, env=env, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    return [l for l in out.stdout.splitlines() if l.startswith("{")]


def test_reference_arm_json_line():
    lines = _run({})
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, ROOT)
    import bench

    assert d["impl"] == "reference" and d["metric"] == bench.METRIC
    assert d["unit"] == "GB/s" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["n_gpus"] == 1 and d["steps"] == 1 and d["warmup"] == 1
    assert d["ms_per_step"] > 0 and d["scaling"] == "weak" and d["vs_baseline"] is None
    assert d["dtype"] == "u8" and d["data"] == "synthetic"
    assert d["config"] == bench.CONFIG and "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert cb["sample"] and cb["cpu"]["nproc"] >= 1
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_are_silent():
    assert _run({"RANK": "1", "WORLD_SIZE": "2"}) == []


def test_line_traffic_model():
    """The line-traffic bound of a sweep point, by hand: 64-B rows at byte
    120 of a 128-B line touch two lines (a pack reads 256 B per row and
    writes 64), and three 32-B sectors (an unpack reads 64 packed bytes and
    writes three sectors)."""
    sys.path.insert(0, ROOT)
    import bench

    sizes, subs, starts = [256, 256, 256], [256, 256, 16], [0, 0, 30]
    rows = 256 * 256
    assert bench.line_traffic(sizes, subs, starts, 1, 0) == rows * (256 + 64)
    assert bench.line_traffic(sizes, subs, starts, 1, 1) == rows * (64 + 32 * 3)
    # a full subarray is one contiguous run per object: read and write it once
    full = bench.line_traffic(sizes, sizes, [0, 0, 0], 4, 0)
    assert full == 2 * 4 * 4 * 256 ** 3
    # every point's bound is at most the copy peak, and the contiguous ones reach it
    for label, sz, sb, st, n in bench.sweep_points():
        alg = 2 * 4 * int(np.prod(sb)) * n
        for u in (0, 1):
            t = bench.line_traffic(sz, sb, st, n, u)
            assert t >= alg, (label, u)
            if label in ("2d_i1024", "3d_i256"):
                assert t == alg


def test_launch_list_summary(tmp_path):
    """--summarize-launches reads ncu's CSV of a --launch-list run (launches
    in the order launch_list_order gives, flush and inference kernels in
    between) into per-point in-kernel times."""
    sys.path.insert(0, ROOT)
    import bench

    header = ["ID", "Process ID", "Process Name", "Host Name", "Kernel Name", "Context",
              "Stream", "Block Size", "Grid Size", "Device", "CC", "Section Name",
              "Metric Name", "Metric Unit", "Metric Value"]
    lines = [",".join(f'"{h}"' for h in header)]
    k = 0

    def add(name, ns):
        nonlocal k
        row = [str(k), "1", "python", "h", name, "1", "7", "(256, 1, 1)", "(148, 1, 1)", "0",
               "10.0", "Command line profiler metrics", "gpu__time_duration.sum", "nsecond",
               f"{ns:,}"]
        lines.append(",".join(f'"{x}"' for x in row))
        k += 1

    add("tempi::k_mlp_predict(const float *, const float *, int, float *)", 9000)
    for i, (label, direction) in enumerate(bench.launch_list_order()):
        add("(anonymous namespace)::read_all(const uint4 *, unsigned long, unsigned int *)", 80000)
        ns = {"empty": 1900, "gather": 3500, "gather_big": 1900 + 6554}.get(
            label, 3000 + 10 * i)
        gname = ("(anonymous namespace)::k_bench_gather(const char *, long long, int, "
                 "unsigned int *)")
        name = {"empty": "(anonymous namespace)::k_bench_empty()", "gather": gname,
                "gather_big": gname}.get(
            label, "void tempi::k_words<4, 1, 0>(char *, char *, tempi::Geometry)")
        add(name, ns)
    csv = tmp_path / "launches.csv"
    csv.write_text("==PROF== Connected\n" + "\n".join(lines) + "\n")
    out = tmp_path / "kernel_times.txt"
    bench.summarize_launches(str(csv), str(out))
    txt = out.read_text().splitlines()
    assert "empty kernel 1.90 us" in txt[0] and "gather 3.50 us" in txt[0]
    assert "scattered line 25.00 ps" in txt[0]
    got = dict(((l.split()[0], l.split()[1]), float(l.split()[2])) for l in txt[1:])
    assert len(got) == 2 * len(bench.sweep_points())
    order = bench.launch_list_order()
    per = len(order) // bench.LAUNCH_LIST_REPS
    i = order.index(("2d_i1", "pack"))
    assert got[("2d_i1", "pack")] == (3000 + 10 * (i + per)) / 1e3  # the median of three
