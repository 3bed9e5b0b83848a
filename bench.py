"""Benchmark of the interposed MPI_Pack/MPI_Unpack path on B200.

Workload (the strided sweep): MPI_Type_create_subarray of a row-major array
of MPI_FLOAT, 2-D 1024x1024 (inner extent 1..1024 elements, 1024 rows,
incount 16) and 3-D 256^3 (inner extent 1..256, 256x256 outer, incount 4),
starts drawn from a seed, random bytes.  One step = MPI_Pack then MPI_Unpack
of every sweep point through the interposed entry points (the plain per-call
path, device-resident buffers).  Metric: algorithmic GB/s = 2 x packed bytes
per pack or unpack (every described byte read once and written once),
summed over the step, divided by the step's device time.

Also reported on the same GPU in the same run:
  roofline   the dominant kernel (largest time share), timed alone with CUDA
             events on the stream it runs on, against the measured HBM copy
             bandwidth
  halo       26-region halo of a 256^3 grid of doubles (radius 2): 26 plain
             MPI_Pack calls vs one batched launch vs one CUDA-graph replay,
             plus the mixed batch of 8 grids
  e2e        the same sweep with host-resident data through MPI_Pack /
             MPI_Unpack on pinned host buffers (the kernels read and write
             host memory over the link); `e2e.staged` is the alternative that
             copies every source span host->device, packs, copies the packed
             bytes back, and the reverse for the unpack
  sendrecv   self-sends of strided device objects (4 KiB - 1 GiB)
             by DEVICE, ONE_SHOT and STAGED, and what the learned model, the
             restated perf-table model and the fixed rules pick
  dispatch   a held-out sample (seed never trained on) of random layouts:
             total-time regret of the learned kernel-configuration choice
             and of the fixed rules against exhaustive measurement
  vector_1024x64  the 1024 x 64 B vector (stride 512) through the interposer
             on host buffers (the library's host pack) and on device buffers
  type_commit  MPI_Type_commit cost: one shape committed repeatedly, and
             fresh shapes (one cost-model inference each)
  cpu_baseline  the oracle's C type-map walker (a port of what the underlying
             MPI's host MPI_Pack does) on one host core, on a bounded sample

--impl reference times that C walker with every host core on the same
workload (the reference's path for host buffers is the library's MPI_Pack).

Defaults: 50 warm-up steps, then 50 timed steps.  In a fresh process the
first ~30 steps run about 6 % slower than every later one, so a warm-up of a
few steps would time that transient instead of the steady state.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0
FLUSH_BYTES = 512 << 20  # > 126 MB L2

SWEEP_2D_INNER = (1, 2, 4, 8, 16, 64, 256, 1024)
SWEEP_3D_INNER = (1, 2, 4, 8, 16, 64, 256)
INCOUNT_2D, INCOUNT_3D = 16, 4


def sweep_points(seed=2026):
    """(label, sizes, subsizes, starts, incount) of the strided sweep."""
    rng = np.random.default_rng(seed)
    pts = []
    for c in SWEEP_2D_INNER:
        sc = int(rng.integers(0, 1024 - c + 1))
        pts.append((f"2d_i{c}", [1024, 1024], [1024, c], [0, sc], INCOUNT_2D))
    for c in SWEEP_3D_INNER:
        sc = int(rng.integers(0, 256 - c + 1))
        pts.append((f"3d_i{c}", [256, 256, 256], [256, 256, c], [0, 0, sc], INCOUNT_3D))
    return pts


def traffic_from_profiles(label, direction="pack"):
    """Per-launch DRAM bytes of a sweep point's kernel from the committed ncu
    summary (profiles/traffic.txt), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        f = line.split()
        if len(f) == 3 and not line.startswith("#") and f[0] == label and f[1] == direction:
            return int(f[2])
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p:
            time.sleep(0.2)
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 6:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for n, v in zip(names, f[2:6]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# reference arm and CPU baseline: the oracle's C walker (host cores)
# ---------------------------------------------------------------------------


def _oracle_points(pts, incount_cap=None):
    from oracle import types as T
    from oracle import walker as W

    out = []
    for label, sizes, subs, starts, incount in pts:
        o = T.subarray(sizes, subs, starts, T.ORDER_C, T.FLOAT)
        n = incount if incount_cap is None else min(incount, incount_cap)
        out.append((label, W.Walker(o), o, n))
    return out


def cpu_walk_step(items, bufs, nthreads):
    nbytes = 0
    for (label, w, o, n), (src, packed, dst) in zip(items, bufs):
        w.pack_into(src, n, packed, nthreads=nthreads)
        w.unpack(packed, dst, n, nthreads=nthreads)
        nbytes += 4 * o.size * n
    return nbytes


def cpu_buffers(items, seed=7):
    bufs = []
    rng = np.random.default_rng(seed)
    for label, w, o, n in items:
        src = rng.integers(0, 256, o.extent * n, dtype=np.uint8)
        bufs.append((src, np.empty(o.size * n, np.uint8), np.empty_like(src)))
    return bufs


def cpu_model():
    """The host CPU's model name and logical core count."""
    name = "unknown"
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    name = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": name, "nproc": os.cpu_count()}


def cpu_baseline(budget_s=12.0):
    """Single-core C walker on the sweep with incount 1 per point, repeated
    for about `budget_s` seconds (at least 20 passes); the rate of the median
    pass."""
    items = _oracle_points(sweep_points(), incount_cap=1)
    bufs = cpu_buffers(items)
    cpu_walk_step(items, bufs, 1)  # warm
    t0 = time.perf_counter()
    times, nbytes = [], 0
    while time.perf_counter() - t0 < budget_s or len(times) < 20:
        a = time.perf_counter()
        nbytes = cpu_walk_step(items, bufs, 1)
        times.append(time.perf_counter() - a)
    dt = time.perf_counter() - t0
    med = statistics.median(times)
    return {"value": round(nbytes / med / 1e9, 3), "unit": "GB/s", "cores": 1, "kind": "port",
            "sample": f"median of {len(times)} passes over the {len(items)} sweep points at "
                      f"incount 1 ({dt:.1f} s), pack + unpack, oracle/typemap.c single thread",
            "cpu": cpu_model()}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    nthreads = len(os.sched_getaffinity(0)) or 1
    items = _oracle_points(sweep_points())
    bufs = cpu_buffers(items)
    for _ in range(args.warmup):
        cpu_walk_step(items, bufs, nthreads)
    times, nbytes = [], 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        nbytes = cpu_walk_step(items, bufs, nthreads)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = nbytes * args.steps / total / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": CONFIG,
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": nthreads,
                         "kind": "port",
                         "sample": "every sweep point at full incount per step, pack + unpack, "
                                   "oracle/typemap.c on all host threads",
                         "cpu": cpu_model()},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


METRIC = "MPI_Pack+MPI_Unpack algorithmic GB/s over the strided subarray sweep"
CONFIG = {
    "workload": "strided sweep: float subarrays of 1024^2 (inner 1..1024, 1024 rows, incount 16) "
                "and 256^3 (inner 1..256, 256x256, incount 4), seeded starts, plain per-call path",
    "points": len(SWEEP_2D_INNER) + len(SWEEP_3D_INNER),
    "l2": "flushed (512 MiB write) before every timed step",
    "parallelism": "replicas",
}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------


class GpuSweep:
    def __init__(self, torch, mpi, dev):
        self.torch = torch
        self.pts = []
        gen = torch.Generator(device="cpu").manual_seed(11)
        # one source / destination array per shape, incount objects each
        self.src2 = torch.randint(0, 256, (INCOUNT_2D * 1024 * 1024 * 4,), dtype=torch.uint8,
                                  generator=gen).to(dev)
        self.dst2 = torch.zeros_like(self.src2)
        self.src3 = torch.randint(0, 256, (INCOUNT_3D * 256 ** 3 * 4,), dtype=torch.uint8,
                                  generator=gen).to(dev)
        self.dst3 = torch.zeros_like(self.src3)
        maxp = 0
        for label, sizes, subs, starts, incount in sweep_points():
            t = mpi.Type_create_subarray(sizes, subs, starts, mpi.ORDER_C, mpi.FLOAT)
            assert mpi.Type_commit(t) == 0
            size = mpi.Type_size(t)
            src, dst = (self.src2, self.dst2) if len(sizes) == 2 else (self.src3, self.dst3)
            self.pts.append(dict(label=label, t=t, size=size, incount=incount, src=src, dst=dst,
                                 sizes=sizes, subs=subs, starts=starts))
            maxp = max(maxp, size * incount)
        self.packed = torch.zeros(maxp, dtype=torch.uint8, device=dev)
        self.flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)
        self.alg_bytes = sum(4 * p["size"] * p["incount"] for p in self.pts)

    def flush_l2(self, stream):
        """Write, then read back, a buffer larger than L2 (clean lines)."""
        driver().tempi_bench_flush(self.flush.data_ptr(), self.flush.numel(),
                                   stream.cuda_stream)

    def ops(self):
        """One step: MPI_Pack then MPI_Unpack of every sweep point."""
        out = []
        cap = self.packed.numel()
        for p in self.pts:
            out.append(BenchOp(0, p["t"], p["src"].data_ptr(), self.packed.data_ptr(),
                               p["incount"], 0, cap, 0))
            out.append(BenchOp(1, p["t"], p["dst"].data_ptr(), self.packed.data_ptr(),
                               p["incount"], 0, cap, 0))
        return out

    def step(self, mpi):
        packed = self.packed.data_ptr()
        cap = self.packed.numel()
        for p in self.pts:
            err, pos = mpi.Pack(p["src"].data_ptr(), p["incount"], p["t"], packed, cap, 0)
            if err:
                raise RuntimeError(f"MPI_Pack {p['label']}: {err}")
            err, _ = mpi.Unpack(packed, cap, p["dst"].data_ptr(), p["incount"], p["t"], 0)
            if err:
                raise RuntimeError(f"MPI_Unpack {p['label']}: {err}")


def time_events(torch, stream, fn, reps, flush=None):
    """Average device time (ms) of fn() on `stream`, L2 flushed before each."""
    ts = []
    for _ in range(reps):
        if flush is not None:
            flush()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return sum(ts) / len(ts)


def learned_configs(lib, d, n):
    """The kernel configurations MPI_Pack and MPI_Unpack run for `n` objects
    of `d` on device buffers (the learned dispatch's picks), as tempi_config
    structures (None: the fixed rules)."""
    from tempi_b200 import _lib

    pc, uc, mi = ctypes.c_int(-1), ctypes.c_int(-1), ctypes.c_int(0)
    _lib.check(lib.tempi_dispatch_choose(ctypes.byref(d), n, 0, 0, 0, ctypes.byref(pc),
                                         ctypes.byref(uc), ctypes.byref(mi), None, None))
    out = []
    for k in (pc.value, uc.value):
        out.append(_lib.Config(*_lib.CANDIDATE_CONFIGS[k]) if k >= 0 else None)
    return out


def line_traffic(sizes, subs, starts, incount, unpack, elem=4, line=128, sector=32):
    """DRAM bytes a pack (or unpack) of `incount` C-order subarray objects
    cannot avoid, a lower bound: a pack reads every 128-B line its rows
    touch (ncu shows L2 fetching whole lines for rows scattered this far
    apart) and writes the packed bytes; an unpack reads the packed bytes and
    writes every 32-B sector its rows touch (the reads that merge partial
    sectors are not counted).  Dimensions whose subarray spans the full
    extent merge into longer runs.  Every run starts at the same offset
    modulo 128 (the sweep's row pitches and extents are multiples of 128 B,
    and buffers are 128-B aligned)."""
    nd = len(sizes)
    k = nd - 1
    run = subs[k] * elem
    off = (starts[k] * elem) % line if subs[k] != sizes[k] else 0
    while k > 0 and subs[k] == sizes[k]:
        run *= subs[k - 1]
        k -= 1
    runs = incount * int(np.prod(subs[:k])) if k > 0 else incount
    packed = runs * run
    if not unpack:
        return runs * line * (-(-(off + run) // line)) + packed
    so = off % sector
    return packed + runs * sector * (-(-(so + run) // sector))


def empty_kernel_events(torch, sw, stream, reps=20):
    """Median CUDA-event time (ms) of one empty kernel launched the way the
    per-point kernels are timed (L2 flushed first): the fixed cost of a
    timed launch on this GPU."""
    ts = []
    for _ in range(reps):
        sw.flush_l2(stream)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        driver().tempi_bench_empty(stream.cuda_stream)
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def kernel_table(torch, sw, stream, lib, reps=5):
    """Per point: the pack and the unpack kernel that MPI_Pack / MPI_Unpack
    run (the learned dispatch's picks), each launched alone through
    tempi_pack/tempi_unpack with the L2 flushed first, CUDA events around
    the launch (`call`: the event pair and the launch's own fixed cost
    included); the line-traffic bound of the layout; and, where the committed
    launch list (profiles/kernel_times.txt) has the point, ncu's in-kernel
    duration."""
    from tempi_b200 import _lib, mpi

    rows = []
    s = stream.cuda_stream
    ktimes = kernel_times_from_profiles()
    for p in sw.pts:
        err, d = mpi.describe(p["t"])
        assert err == 0
        n = p["incount"]
        cp, cu = learned_configs(lib, d, n)
        pk = lambda: _lib.check(lib.tempi_pack(ctypes.byref(d), p["src"].data_ptr(), n,
                                               sw.packed.data_ptr(),
                                               ctypes.byref(cp) if cp else None, s))
        up = lambda: _lib.check(lib.tempi_unpack(ctypes.byref(d), sw.packed.data_ptr(), n,
                                                 p["dst"].data_ptr(),
                                                 ctypes.byref(cu) if cu else None, s))
        pk()
        kname = lib.tempi_last_kernel().decode()
        up()
        uname = lib.tempi_last_kernel().decode()
        t_pack = time_events(torch, stream, pk, reps, lambda: sw.flush_l2(stream))
        t_unpack = time_events(torch, stream, up, reps, lambda: sw.flush_l2(stream))
        alg = 2 * p["size"] * n
        tr = [line_traffic(p["sizes"], p["subs"], p["starts"], n, u) for u in (0, 1)]
        row = dict(label=p["label"], packed_bytes=p["size"] * n, kernel=kname, ukernel=uname,
                   pack_ms=t_pack, unpack_ms=t_unpack,
                   pack_gbs=alg / t_pack / 1e6, unpack_gbs=alg / t_unpack / 1e6,
                   line_bound=[alg / t for t in tr], traffic=tr)  # fractions of the peak
        for direction in ("pack", "unpack"):
            us = ktimes.get((p["label"], direction))
            if us:
                row[direction + "_kernel_us"] = us
        rows.append(row)
    return rows


def point_bound(empty_us, gather_us, traffic, peak):
    """Least in-kernel time (us) of a launch that moves `traffic` DRAM
    bytes: a launch's fixed cost (an empty kernel) plus the traffic at the
    copy peak, and never less than a kernel that reads one scattered line
    per thread and stores it (one DRAM round trip)."""
    return max(empty_us + traffic / peak / 1e3, gather_us)


def sweep_row(r, peak):
    """The bench line's entry for one sweep point."""
    out = {"p": r["label"], "k": r["kernel"], "ku": r["ukernel"],
           "pack_gbs": round(r["pack_gbs"], 1), "unpack_gbs": round(r["unpack_gbs"], 1),
           "line_bound": [round(x, 3) for x in r["line_bound"]]}
    empty, gather, _ = KERNEL_FLOORS_US
    kg, ob = [], []
    for u, direction in enumerate(("pack", "unpack")):
        us = r.get(direction + "_kernel_us")
        if us:
            kg.append(round(2 * r["packed_bytes"] / us / 1e3, 1))
            if empty is not None and gather is not None:
                ob.append(round(point_bound(empty, gather, r["traffic"][u], peak) / us, 3))
    if len(kg) == 2:
        out["kernel_gbs"] = kg
        out["kernel_frac"] = [round(x / peak, 3) for x in kg]
    if len(ob) == 2:
        out["of_bound"] = ob
    return out


# in-kernel times of the empty kernel, the one-load gather and one scattered
# line in the committed launch list (ncu)
KERNEL_FLOORS_US = [None, None, None]


def dominant_back_to_back(torch, sw, stream, lib, label, k=10, reps=5):
    """Median over `reps` of (time of `k` back-to-back launches of the
    point's pack kernel between one event pair) / k, in ms."""
    from tempi_b200 import _lib, mpi

    p = next(q for q in sw.pts if q["label"] == label)
    err, d = mpi.describe(p["t"])
    assert err == 0
    n = p["incount"]
    cp, _ = learned_configs(lib, d, n)
    s = stream.cuda_stream

    def pk():
        _lib.check(lib.tempi_pack(ctypes.byref(d), p["src"].data_ptr(), n, sw.packed.data_ptr(),
                                  ctypes.byref(cp) if cp else None, s))

    ts = []
    for _ in range(reps):
        sw.flush_l2(stream)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            pk()
        b.record(stream)
        b.synchronize()
        ts.append(a.elapsed_time(b) / k)
    return statistics.median(ts)


def kernel_times_from_profiles():
    """(point, direction) -> ncu in-kernel microseconds of the kernel the
    interposer runs, from the committed launch-list summary."""
    path = os.path.join(ROOT, "profiles", "kernel_times.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            f = line.split()
            if line.startswith("#") and "empty kernel" in line:
                KERNEL_FLOORS_US[0] = float(line.split("empty kernel")[1].split()[0])
                if "gather" in line:
                    KERNEL_FLOORS_US[1] = float(line.split("gather")[1].split()[0])
                if "scattered line" in line:
                    KERNEL_FLOORS_US[2] = float(line.split("scattered line")[1].split()[0]) / 1e6
            elif len(f) >= 3 and not line.startswith("#"):
                out[(f[0], f[1])] = float(f[2])
    return out


def halo_bench(torch, sw, stream, reps=20):
    """The 256^3-double radius-2 halo (26 regions) and the mixed batch of 8
    grids, seeded data: plain per-region MPI_Pack / MPI_Unpack calls against
    one batched launch, one CUDA-graph replay and one call of the
    allocation-free entry point, the L2 flushed before each timed pass.
    `bit_exact`: the batched, graph and allocation-free outputs equal the
    plain path's, byte for byte (compared on the device)."""
    from tempi_b200 import _lib, halo

    flush = lambda: sw.flush_l2(stream)
    s = stream.cuda_stream
    gen = torch.Generator(device="cuda")
    gen.manual_seed(256)
    g = halo.Grid((256, 256, 256), 2)
    data = torch.randint(0, 256, (g.nbytes,), dtype=torch.uint8, device="cuda", generator=gen)
    p_plain = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    p_batch, p_graph = torch.zeros_like(p_plain), torch.zeros_like(p_plain)
    torch.cuda.synchronize()

    def plain_ops(grid, dptr, pptr, unpack=False):
        ops, pos = [], 0
        for d in halo.directions():
            t = grid.recv[tuple(-x for x in d)] if unpack else grid.send[d]
            ops.append(BenchOp(int(unpack), t, dptr, pptr, 1, pos, grid.packed_bytes, 0))
            pos += grid.region_bytes[d]
        return ops

    ops = plain_ops(g, data.data_ptr(), p_plain.data_ptr())
    run_ops(ops, 3)
    t_plain = statistics.median(run_ops(ops, reps, sw.flush))
    b = halo.HaloBatch([g], [data.data_ptr()], [p_batch.data_ptr()])
    for _ in range(3):
        b.launch(s)
    t_batch = time_events(torch, stream, lambda: b.launch(s), reps, flush)
    bg = halo.HaloBatch([g], [data.data_ptr()], [p_graph.data_ptr()])
    bg.capture(s)
    for _ in range(3):
        bg.replay(s)
    t_graph_default = time_events(torch, stream, lambda: bg.replay(s), reps, flush)
    cfg_default = bg.config()
    # the autotuner on this batch (its choices then hold for every batch of
    # the same regions, the unpack's below included once tuned)
    bg.tune(s, 5)
    bg.capture(s)
    for _ in range(3):
        bg.replay(s)
    t_graph = time_events(torch, stream, lambda: bg.replay(s), reps, flush)
    cfg_tuned = bg.config()
    # the allocation-free entry point: the same regions through the
    # library's fixed device table (fill kernels + the batch kernel, no
    # cudaMalloc and no host-to-device copy)
    p_static = torch.zeros_like(p_plain)
    regs = halo.regions([g], [data.data_ptr()], [p_static.data_ptr()])
    arr = (_lib.Region * len(regs))(*regs)
    lib = _lib.tempi()

    def run_static():
        _lib.check(lib.tempi_batch_run_static(arr, len(regs), 0, s), "tempi_batch_run_static")

    for _ in range(3):
        run_static()
    t_static = time_events(torch, stream, run_static, reps, flush)
    torch.cuda.synchronize()
    pack_exact = bool(torch.equal(p_plain, p_batch) and torch.equal(p_plain, p_graph))
    static_exact = bool(torch.equal(p_plain, p_static))
    b.close()
    bg.close()
    del p_static

    # unpack into the ghost cells: the packed bytes land in the ghost region
    # opposite their direction, three copies of the grid, one per method
    grids = [data.clone() for _ in range(3)]
    uops = plain_ops(g, grids[0].data_ptr(), p_plain.data_ptr(), unpack=True)
    run_ops(uops, 3)
    t_uplain = statistics.median(run_ops(uops, reps, sw.flush))
    ub = halo.HaloBatch([g], [grids[1].data_ptr()], [p_plain.data_ptr()], unpack=True)
    for _ in range(3):
        ub.launch(s)
    t_ubatch = time_events(torch, stream, lambda: ub.launch(s), reps, flush)
    ug = halo.HaloBatch([g], [grids[2].data_ptr()], [p_plain.data_ptr()], unpack=True)
    ug.tune(s, 5)
    ug.capture(s)
    for _ in range(3):
        ug.replay(s)
    t_ugraph = time_events(torch, stream, lambda: ug.replay(s), reps, flush)
    torch.cuda.synchronize()
    unpack_exact = bool(torch.equal(grids[0], grids[1]) and torch.equal(grids[0], grids[2])
                        and not torch.equal(grids[0], data))
    ub.close()
    ug.close()
    del grids

    # mixed batch of 8 grids
    grids_m = [halo.Grid(interior, r) for interior, r in halo.mixed_shapes()]
    datas = [torch.randint(0, 256, (gg.nbytes,), dtype=torch.uint8, device="cuda", generator=gen)
             for gg in grids_m]
    pk_plain = [torch.zeros(gg.packed_bytes, dtype=torch.uint8, device="cuda") for gg in grids_m]
    pk_graph = [torch.zeros_like(x) for x in pk_plain]
    mb = halo.HaloBatch(grids_m, [d.data_ptr() for d in datas], [p.data_ptr() for p in pk_graph])
    mb.tune(s, 5)
    mb.capture(s)
    for _ in range(3):
        mb.replay(s)
    t_mixed = time_events(torch, stream, lambda: mb.replay(s), reps, flush)
    mixed_ops = []
    for gg, dd, pp in zip(grids_m, datas, pk_plain):
        mixed_ops += plain_ops(gg, dd.data_ptr(), pp.data_ptr())
    run_ops(mixed_ops, 2)
    t_mixed_plain = statistics.median(run_ops(mixed_ops, 5, sw.flush))
    torch.cuda.synchronize()
    mixed_exact = all(torch.equal(x, y) for x, y in zip(pk_plain, pk_graph))
    mb.close()
    del datas, pk_plain, pk_graph
    mixed_bytes = int(sum(gg.packed_bytes for gg in grids_m))
    return {
        "grid": "256^3 doubles, radius 2, 26 regions, 6390272 B packed, seeded data",
        "timing": "median of %d passes, L2 flushed before each, CUDA events" % reps,
        "plain_us": round(1e3 * t_plain, 2), "batched_us": round(1e3 * t_batch, 2),
        "graph_us": round(1e3 * t_graph, 2),
        "graph_untuned_us": round(1e3 * t_graph_default, 2),
        "static_us": round(1e3 * t_static, 2),
        "tuned": {"threads": cfg_tuned[0], "ctas_per_sm": cfg_tuned[1],
                  "passes_per_class": {str(k): v for k, v in cfg_tuned[2].items()}},
        "untuned": {"threads": cfg_default[0], "ctas_per_sm": cfg_default[1],
                    "passes_per_class": {str(k): v for k, v in cfg_default[2].items()}},
        "class": "8 * log2(vector width) + min(7, log2(words per row))",
        "speedup_graph_vs_plain": round(t_plain / t_graph, 2),
        "graph_gbs": round(2 * g.packed_bytes / t_graph / 1e6, 1),
        "unpack_plain_us": round(1e3 * t_uplain, 2), "unpack_batched_us": round(1e3 * t_ubatch, 2),
        "unpack_graph_us": round(1e3 * t_ugraph, 2),
        "unpack_speedup_graph_vs_plain": round(t_uplain / t_ugraph, 2),
        "bit_exact": pack_exact and unpack_exact and mixed_exact and static_exact,
        "bit_exact_parts": {"pack": pack_exact, "unpack": unpack_exact, "mixed8": mixed_exact,
                            "static": static_exact},
        "mixed8_regions": 26 * len(grids_m), "mixed8_bytes": mixed_bytes,
        "mixed8_graph_us": round(1e3 * t_mixed, 2),
        "mixed8_plain_us": round(1e3 * t_mixed_plain, 2),
        "mixed8_speedup_graph_vs_plain": round(t_mixed_plain / t_mixed, 2),
    }


def _tempi_stream():
    from tempi_b200 import _lib

    return _lib.tempi().tempi_stream()


class BenchOp(ctypes.Structure):
    """``tempi_bench_op`` of tempi_b200/csrc/bench/driver.cu."""

    _fields_ = [("unpack", ctypes.c_int), ("datatype", ctypes.c_int),
                ("typed", ctypes.c_void_p), ("packed", ctypes.c_void_p),
                ("incount", ctypes.c_int), ("position", ctypes.c_int),
                ("capacity", ctypes.c_int), ("reserved", ctypes.c_int)]


_driver = None


def halo_exchange_bench(torch, stream, reps=20):
    """Periodic halo exchange of a 256^3-double grid (radius 2) with
    itself, the reference's bench_halo_exchange at world size 1: its
    sequence (26 MPI_Pack, MPI_Neighbor_alltoallv of the packed bytes, 26
    MPI_Unpack), one interposed MPI_Neighbor_alltoallw (the fused kernel),
    and the fused kernel replayed from a CUDA graph.  All three must leave
    the same grid."""
    from tempi_b200 import halo

    g = halo.Grid((256, 256, 256), 2)
    sg = halo.SelfGraph(g)
    n = len(sg.sendtypes)
    base = torch.randint(0, 256, (g.nbytes,), dtype=torch.uint8, device="cuda")
    grids = [base.clone() for _ in range(3)]
    # tune the fused exchange first: the interposed MPI_Neighbor_alltoallw
    # below takes the same choices (same copy pairs, same signature)
    xt = halo.HaloExchange([g], [grids[2].data_ptr()])
    xt.tune(stream.cuda_stream, 5)
    xt.close()
    sendbuf = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    recvbuf = torch.zeros_like(sendbuf)
    ints = lambda v: (ctypes.c_int * n)(*v)
    st, rt, cnt, dsp = ints(sg.sendtypes), ints(sg.recvtypes), ints(sg.counts), ints(sg.displs)
    out = (ctypes.c_float * reps)()
    res = {"grid": "256^3 doubles, radius 2, periodic, one rank: 26 self-edges",
           "bytes_exchanged": g.packed_bytes}
    torch.cuda.synchronize()
    for mode, key, gbuf in ((0, "pack_alltoallv_unpack_us", grids[0]),
                            (1, "neighbor_alltoallw_us", grids[1])):
        err = driver().tempi_bench_halo(mode, n, st, rt, cnt, dsp, gbuf.data_ptr(),
                                        sendbuf.data_ptr(), recvbuf.data_ptr(),
                                        g.packed_bytes, sg.comm, reps, out)
        if err:
            raise RuntimeError(f"halo exchange mode {mode} failed: {err}")
        res[key] = round(1e3 * sorted(out)[reps // 2], 2)  # median
    x = halo.HaloExchange([g], [grids[2].data_ptr()])
    s = stream.cuda_stream
    x.capture(s)
    for _ in range(reps):
        x.replay(s)
    res["fused_graph_us"] = round(1e3 * time_events(torch, stream, lambda: x.replay(s), reps), 2)
    x.close()
    sg.close()
    torch.cuda.synchronize()
    # an exchange only writes ghost cells from interior cells, so repeating
    # it changes nothing: however often each method ran, the grids agree
    res["same_grid"] = bool(torch.equal(grids[0], grids[1]) and torch.equal(grids[0], grids[2]))
    res["speedup_alltoallw_vs_reference_sequence"] = round(
        res["pack_alltoallv_unpack_us"] / res["neighbor_alltoallw_us"], 2)
    res["speedup_graph_vs_reference_sequence"] = round(
        res["pack_alltoallv_unpack_us"] / res["fused_graph_us"], 2)
    return res


def driver():
    """The C benchmark driver (MPI call loops run from C)."""
    global _driver
    if _driver is None:
        from tempi_b200 import _lib

        _lib.tempi()
        _driver = ctypes.CDLL(os.path.join(ROOT, "tempi_b200", "csrc", "libtempi_bench.so"))
        _driver.tempi_bench_flush.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        _driver.tempi_bench_empty.argtypes = [ctypes.c_void_p]
        _driver.tempi_bench_gather.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int,
                                               ctypes.c_void_p, ctypes.c_void_p]
        sz = ctypes.c_size_t
        _driver.tempi_bench_copy2d.argtypes = [ctypes.c_void_p, sz, ctypes.c_void_p, sz, sz, sz,
                                               ctypes.c_int, ctypes.c_void_p]
        _driver.tempi_bench_mpi_ops.argtypes = [
            ctypes.POINTER(BenchOp), ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_size_t, ctypes.POINTER(ctypes.c_float)]
        _driver.tempi_bench_call_overhead.argtypes = [
            ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        ip = ctypes.POINTER(ctypes.c_int)
        _driver.tempi_bench_halo.argtypes = [
            ctypes.c_int, ctypes.c_int, ip, ip, ip, ip, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            ctypes.POINTER(ctypes.c_float)]
    return _driver


def run_ops(ops, iters, flush=None):
    """Device ms of each of `iters` passes over `ops` (C loop)."""
    arr = (BenchOp * len(ops))(*ops)
    out = (ctypes.c_float * max(iters, 1))()
    fp, fb = (flush.data_ptr(), flush.numel()) if flush is not None else (None, 0)
    err = driver().tempi_bench_mpi_ops(arr, len(ops), iters, fp, fb, out)
    if err:
        from tempi_b200 import _lib

        raise RuntimeError(f"MPI call failed in the benchmark loop: {err} {_lib.last_error()}")
    return list(out)[:iters]


def e2e_bench(torch, sw, mpi, steps, warmup):
    """Host-resident data: H2D copy of each source span, MPI_Pack, D2H of the
    packed bytes, H2D of packed bytes, MPI_Unpack, D2H of the object span."""
    tstream = torch.cuda.ExternalStream(_tempi_stream())
    host = {}
    for p in sw.pts:
        span = p["src"].numel()
        if id(p["src"]) not in host:
            host[id(p["src"])] = (torch.empty(span, dtype=torch.uint8).pin_memory(),
                                  torch.empty(span, dtype=torch.uint8).pin_memory())
            host[id(p["src"])][0].copy_(p["src"].cpu())
    hpacked = torch.empty(sw.packed.numel(), dtype=torch.uint8).pin_memory()
    h2d = d2h = 0

    def step():
        nonlocal h2d, d2h
        h2d = d2h = 0
        cap = sw.packed.numel()
        for p in sw.pts:
            hs, hd = host[id(p["src"])]
            n = p["size"] * p["incount"]
            with torch.cuda.stream(tstream):
                p["src"].copy_(hs, non_blocking=True)
            err, _ = mpi.Pack(p["src"].data_ptr(), p["incount"], p["t"], sw.packed.data_ptr(), cap)
            assert err == 0
            with torch.cuda.stream(tstream):
                hpacked[:n].copy_(sw.packed[:n], non_blocking=True)
                sw.packed[:n].copy_(hpacked[:n], non_blocking=True)
            err, _ = mpi.Unpack(sw.packed.data_ptr(), cap, p["dst"].data_ptr(), p["incount"], p["t"])
            assert err == 0
            with torch.cuda.stream(tstream):
                hd.copy_(p["dst"], non_blocking=True)
            h2d += hs.numel() + n
            d2h += n + hd.numel()

    for _ in range(warmup):
        step()
    ms = time_events(torch, tstream, step, steps)
    return {"value": round(sw.alg_bytes / ms / 1e6, 3), "unit": "GB/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(ms, 3)}


def e2e_zero_copy(torch, sw, steps, warmup):
    """Host-resident data through MPI_Pack/MPI_Unpack with pinned host
    buffers (device-accessible, so the kernels read and write host memory
    directly over the link): typed source -> packed (host) -> typed
    destination (host).  Link bytes counted are the described bytes each
    kernel reads from or writes to host memory."""
    from tempi_b200 import _lib

    host = {}
    for p in sw.pts:
        key = id(p["src"])
        if key not in host:
            hs = torch.empty(p["src"].numel(), dtype=torch.uint8).pin_memory()
            hs.copy_(p["src"].cpu())
            host[key] = (hs, torch.empty_like(hs).pin_memory())
    hp = torch.empty(sw.packed.numel(), dtype=torch.uint8).pin_memory()
    ops, nbytes = [], 0
    for p in sw.pts:
        hs, hd = host[id(p["src"])]
        n = p["size"] * p["incount"]
        ops.append(BenchOp(0, p["t"], hs.data_ptr(), hp.data_ptr(), p["incount"], 0, hp.numel(), 0))
        ops.append(BenchOp(1, p["t"], hd.data_ptr(), hp.data_ptr(), p["incount"], 0, hp.numel(), 0))
        nbytes += n
    launches0 = _lib.tempi().tempi_kernel_launches()
    dma0 = _lib.counter("host_link_copies")
    run_ops(ops, warmup)
    ms = sum(run_ops(ops, steps)) / steps
    # per point: its MPI_Pack + MPI_Unpack pair alone, against the link: the
    # packed bytes cross it once each way per call (typed rows in and packed
    # bytes out, then back), both directions at once
    link = host_link_both_ways(torch)
    points = []
    for i, p in enumerate(sw.pts):
        n = p["size"] * p["incount"]
        t = statistics.median(run_ops(ops[2 * i: 2 * i + 2], max(3, steps // 5)))
        bound_ms = 2 * n / (link * 1e6)
        points.append({"p": p["label"], "ms": round(t, 4), "gbs": round(4 * n / t / 1e6, 2),
                       "link_bound_ms": round(bound_ms, 4), "of_link_bound": round(bound_ms / t, 3)})
    # every call ran a pack or unpack kernel, or (a contiguous run between the
    # two host buffers) the copy-engine pipeline; the first call per buffer
    # kind also runs the cost model's inference kernel
    kernels = _lib.tempi().tempi_kernel_launches() - launches0
    dma = _lib.counter("host_link_copies") - dma0
    assert kernels + dma >= len(ops) * (steps + warmup)
    return {"value": round(sw.alg_bytes / ms / 1e6, 3), "unit": "GB/s",
            "h2d_bytes_per_step": int(2 * nbytes), "d2h_bytes_per_step": int(2 * nbytes),
            "ms_per_step": round(ms, 3),
            "kernel_calls_per_step": round((kernels) / (steps + warmup), 1),
            "link_gbs_each_way": round(link, 1),
            "points": points,
            "copy_engine_calls_per_step": round(dma / (steps + warmup), 1),
            "how": "MPI_Pack/MPI_Unpack on pinned host buffers: strided objects by kernels "
                   "that read and write host memory directly; objects of 8 MiB or more that "
                   "are one contiguous run, and unpacks of rows of 128 B or more of one "
                   "strided dimension, by the copy-engine pipeline (link bytes = described "
                   "bytes)"}


def host_link_both_ways(torch, nbytes=256 << 20, reps=5):
    """GB/s per direction of the copy engines moving `nbytes` host->device
    and device->host at the same time (pinned host memory): the link's
    rate when both directions are busy, as they are in a pack or unpack
    between two host buffers."""
    ha = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    hb = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    da = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    db = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    ts = []
    for _ in range(reps + 1):
        torch.cuda.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(s1)
        s2.wait_event(a)
        with torch.cuda.stream(s1):
            da.copy_(ha, non_blocking=True)
        with torch.cuda.stream(s2):
            hb.copy_(db, non_blocking=True)
        c = torch.cuda.Event()
        c.record(s2)
        s1.wait_event(c)
        b.record(s1)
        b.synchronize()
        ts.append(a.elapsed_time(b))
    del ha, hb, da, db
    return nbytes / statistics.median(ts[1:]) / 1e6


def sendrecv_bench(torch, mpi, reps=20):
    """Self-sends (MPI_Isend + MPI_Irecv + MPI_Wait x2) of strided device
    objects by each method, and what each policy picks.  Every repetition
    times one round trip per policy, the policies in an order rotated by one
    each repetition (so no policy always runs first or last), each on a
    freshly committed type after one untimed round trip; medians per policy.
    For the ONE_SHOT method, the rate of its pack kernel writing the packed
    bytes into mapped pinned host memory, against a kernel's contiguous
    write rate into pinned host memory measured in the same run."""
    import time as _t

    from tempi_b200 import _lib

    lib = _lib.tempi()
    objs = [  # (label, constructor, count)
        ("2d_byte_b4_4KiB", lambda: mpi.Type_vector(1024, 4, 16, mpi.BYTE), 1),
        ("2d_byte_b64_1MiB", lambda: mpi.Type_vector(16384, 64, 256, mpi.BYTE), 1),
        ("3d_float_i4_1MiB", lambda: mpi.Type_create_subarray(
            [64, 64, 64], [64, 64, 16], [0, 0, 8], mpi.ORDER_C, mpi.FLOAT), 1),
        ("3d_float_i64_16MiB", lambda: mpi.Type_create_subarray(
            [256, 256, 256], [256, 256, 64], [0, 0, 67], mpi.ORDER_C, mpi.FLOAT), 1),
        ("2d_byte_b4096_64MiB", lambda: mpi.Type_vector(16384, 4096, 8192, mpi.BYTE), 1),
        ("2d_byte_b4096_1GiB", lambda: mpi.Type_vector(262144, 4096, 8192, mpi.BYTE), 1),
    ]
    knobs = {"DEVICE": "TEMPI_DATATYPE_DEVICE", "ONE_SHOT": "TEMPI_DATATYPE_ONESHOT",
             "STAGED": "TEMPI_DATATYPE_STAGED"}
    policies = [("DEVICE", (knobs["DEVICE"], None)), ("ONE_SHOT", (knobs["ONE_SHOT"], None)),
                ("STAGED", (knobs["STAGED"], None)), ("learned", (None, "learned")),
                ("table", (None, "table")), ("fixed", (None, "heuristic"))]

    def set_env(method_var=None, dispatch=None):
        for v in knobs.values():
            os.environ.pop(v, None)
        os.environ.pop("TEMPI_DISPATCH", None)
        if method_var:
            os.environ[method_var] = ""
        if dispatch:
            os.environ["TEMPI_DISPATCH"] = dispatch
        lib.tempi_reload_env()

    def round_trip(t, count, src, dst):
        e1, rr = mpi.Irecv(dst.data_ptr(), count, t, tag=5)
        e2, rs = mpi.Isend(src.data_ptr(), count, t, tag=5)
        assert (e1, e2) == (0, 0), _lib.last_error()
        assert mpi.Wait(rr)[0] == 0 and mpi.Wait(rs)[0] == 0, _lib.last_error()

    host_write = host_write_gbs(torch, lib)
    rows = []
    for label, make, count in objs:
        t0 = make()
        lbext = mpi.Type_get_extent(t0)[1]
        size = int(mpi.Type_size(t0)) * count
        src = torch.randint(0, 256, (lbext * count,), dtype=torch.uint8, device="cuda")
        dst = torch.zeros_like(src)
        n_reps = reps if size < (256 << 20) else max(3, reps // 4)
        times = {name: [] for name, _ in policies}
        chosen = {}
        for rep in range(n_reps):
            k = rep % len(policies)
            for name, (var, disp) in policies[k:] + policies[:k]:
                set_env(var, disp)
                t = make()  # a fresh type: no cached choice carries over
                assert mpi.Type_commit(t) == 0
                round_trip(t, count, src, dst)  # untimed: the policy's choice, warm slabs
                counts0 = {m: _lib.counter("send_" + m) for m in ("device", "oneshot", "staged")}
                torch.cuda.synchronize()
                t1 = _t.perf_counter()
                round_trip(t, count, src, dst)
                times[name].append(1e6 * (_t.perf_counter() - t1))
                after = {m: _lib.counter("send_" + m) for m in ("device", "oneshot", "staged")}
                chosen[name] = [m for m in after if after[m] != counts0[m]]
                mpi.Type_free(t)
        set_env()
        med = {name: statistics.median(v) for name, v in times.items()}
        best = min(med[m] for m in ("DEVICE", "ONE_SHOT", "STAGED"))
        row = {"object": label, "bytes": size, "reps": n_reps,
               **{k + "_us": round(v, 1) for k, v in med.items()},
               "best": min(("DEVICE", "ONE_SHOT", "STAGED"), key=lambda m: med[m]),
               "learned_pick": chosen.get("learned"), "table_pick": chosen.get("table"),
               "learned_regret": round(med["learned"] / best - 1, 4),
               "table_regret": round(med["table"] / best - 1, 4),
               "fixed_regret": round(med["fixed"] / best - 1, 4)}
        os_ = oneshot_pack_gbs(torch, lib, mpi, make(), count, src)
        if os_ is not None:
            row["oneshot_pack_gbs"] = round(os_, 2)
            row["oneshot_pack_of_host_write"] = round(os_ / host_write, 3)
        rows.append(row)
        del src, dst
    tot = {p: sum(r[p + "_us"] for r in rows) for p in ("learned", "table", "fixed")}
    best_tot = sum(min(r[m + "_us"] for m in ("DEVICE", "ONE_SHOT", "STAGED")) for r in rows)
    return {"objects": rows, "host_write_gbs": round(host_write, 2),
            "timing": "host wall clock per round trip, median over repetitions with the "
                      "policy order rotated each repetition",
            "total_regret": {p: round(v / best_tot - 1, 4) for p, v in tot.items()}}


def host_write_gbs(torch, lib, nbytes=256 << 20, reps=5):
    """GB/s of a kernel writing pinned host memory: tempi_pack of a
    contiguous 256 MiB type from device memory into a pinned host buffer."""
    from tempi_b200 import _lib

    d = _lib.Desc.make(0, nbytes, nbytes, [], [])
    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    cfg = _lib.Config(1, 16, 256, 0, 0, 0)
    s = torch.cuda.Stream()
    fn = lambda: _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), 1, dst.data_ptr(),
                                           ctypes.byref(cfg), s.cuda_stream))
    fn()
    ms = time_events(torch, s, fn, reps)
    del src, dst
    return nbytes / ms / 1e6


def oneshot_pack_gbs(torch, lib, mpi, t, count, src, reps=5):
    """GB/s (packed bytes per second) of the pack a ONE_SHOT send runs: the
    kernel the interposer picks for a pinned host packed buffer, writing
    into mapped pinned host memory."""
    from tempi_b200 import _lib

    assert mpi.Type_commit(t) == 0
    err, d = mpi.describe(t)
    if err:
        mpi.Type_free(t)
        return None
    n = d.size * count
    host = torch.empty(n, dtype=torch.uint8).pin_memory()
    pc, uc, mi = ctypes.c_int(-1), ctypes.c_int(-1), ctypes.c_int(0)
    _lib.check(lib.tempi_dispatch_choose(ctypes.byref(d), count, 0, 1, 0, ctypes.byref(pc),
                                         ctypes.byref(uc), ctypes.byref(mi), None, None))
    cfg = _lib.Config(*_lib.CANDIDATE_CONFIGS[pc.value]) if pc.value >= 0 else None
    s = torch.cuda.Stream()
    fn = lambda: _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), count,
                                           host.data_ptr(), ctypes.byref(cfg) if cfg else None,
                                           s.cuda_stream))
    fn()
    ms = time_events(torch, s, fn, reps)
    mpi.Type_free(t)
    del host
    return n / ms / 1e6


def dispatch_sample(torch, n=200, seed=777):
    """Held-out sample for the learned kernel-configuration choice: fresh
    random layouts (a seed the model never saw), every eligible candidate
    timed, the learned pick and the fixed rules against the best.  Every
    layout is measured twice: the second measurement shows how often the
    first one's own fastest candidate stays within 5 % of the fastest when
    timed again (the noise ceiling of the within-5 % figure), and the learned
    pick is also scored on the mean of the two measurements (the
    `_two_measurements` figures), which halves the variance of each
    candidate's time.  The `deployed_` figures score what MPI_Type_commit
    actually runs: the model's pick where the ensemble's spread is within
    TEMPI_DISPATCH_SPREAD, else a measurement's fastest candidate."""
    from tempi_b200 import _lib
    from tempi_b200 import dispatch_train as DT

    lib = _lib.tempi()
    rng = np.random.default_rng(seed)
    times = (ctypes.c_float * DT.N_MEAS)()
    times2 = (ctypes.c_float * DT.N_MEAS)()
    learned, fixed, best, where, rep_best, rep_self = [], [], [], [], [], []
    learned_m, best_m, deployed, untrusted, sweep_lim = [], [], [], [], []
    spr = (ctypes.c_float * DT.N_OUT)()
    # the library's TEMPI_DISPATCH_SPREAD (default 0.5 in log2): above it,
    # MPI_Type_commit measures the candidates instead of trusting the model
    limit = float(os.environ.get("TEMPI_DISPATCH_SPREAD", "0.5"))
    t0 = time.time()
    while len(best) < n and time.time() - t0 < 90:
        d, incount, th, ph = DT.random_layout(rng)
        if DT.span_of(d, incount) > (2 << 30) or (th and DT.span_of(d, incount) > (16 << 20)):
            continue
        size = d.size * incount
        reps = 64 if size < (1 << 20) else 16 if size < (64 << 20) else 4
        _lib.check(lib.tempi_measure(ctypes.byref(d), incount, int(th), int(ph), 1, reps, times))
        _lib.check(lib.tempi_measure(ctypes.byref(d), incount, int(th), int(ph), 1, reps, times2))
        pc, uc, mi = ctypes.c_int(-1), ctypes.c_int(-1), ctypes.c_int(0)
        if lib.tempi_dispatch_choose(ctypes.byref(d), incount, int(th), int(ph), 0,
                                     ctypes.byref(pc), ctypes.byref(uc), ctypes.byref(mi),
                                     None, spr):
            return {"error": _lib.last_error()}
        t = np.frombuffer(times, np.float32)
        t2 = np.frombuffer(times2, np.float32)
        tp, tu = t[DT.PACK:DT.PACK + DT.N_CFG], t[DT.UNPACK:DT.UNPACK + DT.N_CFG]
        tp2, tu2 = t2[DT.PACK:DT.PACK + DT.N_CFG], t2[DT.UNPACK:DT.UNPACK + DT.N_CFG]
        best.append(float(np.nanmin(tp) + np.nanmin(tu)))
        learned.append(float(tp[pc.value] + tu[uc.value]))
        fixed.append(float(t[DT.FIXED_PACK] + t[DT.FIXED_UNPACK]))
        # the first measurement's own picks, timed again
        rep_self.append(float(tp2[int(np.nanargmin(tp))] + tu2[int(np.nanargmin(tu))]))
        rep_best.append(float(np.nanmin(tp2) + np.nanmin(tu2)))
        # both measurements averaged: each candidate's time with half the
        # variance of one measurement
        mp, mu = (tp + tp2) / 2, (tu + tu2) / 2
        best_m.append(float(np.nanmin(mp) + np.nanmin(mu)))
        learned_m.append(float(mp[pc.value] + mu[uc.value]))
        # the deployed policy: the model's pick where the ensemble agrees,
        # else a measurement's fastest (the first one here), scored on the
        # second measurement against its own fastest
        tr_p = spr[DT.PACK + pc.value] <= limit
        tr_u = spr[DT.UNPACK + uc.value] <= limit
        dp = pc.value if tr_p else int(np.nanargmin(tp))
        du = uc.value if tr_u else int(np.nanargmin(tu))
        deployed.append(float(tp2[dp] + tu2[du]))
        untrusted.append(not (tr_p and tr_u))
        # for other spread limits: the spreads of both picks and the
        # second measurement's times of the model's and the measured picks
        sweep_lim.append((spr[DT.PACK + pc.value], spr[DT.UNPACK + uc.value],
                          float(tp2[pc.value]), float(tp2[int(np.nanargmin(tp))]),
                          float(tu2[uc.value]), float(tu2[int(np.nanargmin(tu))])))
        where.append((d.as_dict(), incount, bool(th), bool(ph), pc.value, uc.value))
    L, F, B = map(np.array, (learned, fixed, best))
    RS, RB = np.array(rep_self), np.array(rep_best)
    LM, BM = np.array(learned_m), np.array(best_m)
    DP = np.array(deployed)
    by_limit = {}
    for lim in (0.1, 0.2, 0.3, 0.5, 1.0):
        d = np.array([(a if sa <= lim else b) + (c if su <= lim else e)
                      for sa, su, a, b, c, e in sweep_lim])
        meas = np.mean([not (sa <= lim and su <= lim) for sa, su, *_ in sweep_lim])
        by_limit[str(lim)] = {"within_5pct": round(float(np.mean(d <= 1.05 * RB)), 3),
                              "total_regret": round(float(d.sum() / RB.sum() - 1), 4),
                              "measured_fraction": round(float(meas), 3)}
    worst = [{"us_learned": round(float(L[i]), 1), "us_best": round(float(B[i]), 1),
              "layout": where[i][0], "incount": where[i][1], "typed_host": where[i][2],
              "packed_host": where[i][3], "picks": where[i][4:]}
             for i in np.argsort(-(L - B))[:3]]
    return {"layouts": len(B), "seed": seed, "seconds": round(time.time() - t0, 1),
            "learned_total_regret": round(float(L.sum() / B.sum() - 1), 4),
            "fixed_rules_total_regret": round(float(F.sum() / B.sum() - 1), 4),
            "learned_within_5pct": round(float(np.mean(L <= 1.05 * B)), 3),
            "learned_mean_regret": round(float(np.mean(L / B - 1)), 4),
            "learned_within_5pct_two_measurements": round(float(np.mean(LM <= 1.05 * BM)), 3),
            "learned_total_regret_two_measurements": round(float(LM.sum() / BM.sum() - 1), 4),
            "deployed_within_5pct": round(float(np.mean(DP <= 1.05 * RB)), 3),
            "deployed_total_regret": round(float(DP.sum() / RB.sum() - 1), 4),
            "deployed_measured_fraction": round(float(np.mean(untrusted)), 3),
            "deployed_by_spread_limit": by_limit,
            "exhaustive_repeat_within_5pct": round(float(np.mean(RS <= 1.05 * RB)), 3),
            "exhaustive_repeat_total_regret": round(float(RS.sum() / RB.sum() - 1), 4),
            "exhaustive_total_us": round(float(B.sum()), 1),
            "reps": "64 back-to-back launches per candidate under 1 MiB, 16 under 64 MiB, else 4",
            "largest_losses": worst}


def vector_1024x64_bench(torch, mpi, reps=200):
    """MPI_Type_vector(1024, 64, 512, MPI_BYTE), incount 1, 512 KiB
    of seeded random bytes.  With host buffers the interposed MPI_Pack hands
    the call to the underlying library (its host pack, as the reference does,
    src/pack.cpp:51-55); the same type on device buffers runs the kernel.
    Both are checked byte for byte against each other and timed per call."""
    t = mpi.Type_vector(1024, 64, 512, mpi.BYTE)
    assert mpi.Type_commit(t) == 0
    src = np.random.default_rng(0).integers(0, 256, 512 * 1024, dtype=np.uint8)
    out = np.zeros(65536, np.uint8)
    back = np.full_like(src, 0xAA)
    dsrc = torch.from_numpy(src).cuda()
    dout = torch.zeros(65536, dtype=torch.uint8, device="cuda")
    dback = torch.full_like(dsrc, 0xAA)
    torch.cuda.synchronize()

    def run(a, b, c):
        e1, _ = mpi.Pack(a, 1, t, b, 65536)
        e2, _ = mpi.Unpack(b, 65536, c, 1, t)
        assert (e1, e2) == (0, 0)

    res = {}
    for name, (a, b, c) in (("host_library", (src.ctypes.data, out.ctypes.data, back.ctypes.data)),
                            ("device_kernel", (dsrc.data_ptr(), dout.data_ptr(), dback.data_ptr()))):
        run(a, b, c)
        t0 = time.perf_counter()
        for _ in range(reps):
            run(a, b, c)
        us = 1e6 * (time.perf_counter() - t0) / reps
        res[name] = {"pack_plus_unpack_us": round(us, 2),
                     "gbs": round(2 * 2 * 65536 / us / 1e3, 3)}
    same = out.tobytes() == dout.cpu().numpy().tobytes()
    gaps = bool((back.reshape(1024, 512)[:1023, 64:] == 0xAA).all())
    mpi.Type_free(t)
    return dict(res, packed_bytes=65536, host_equals_device=same, gaps_untouched=gaps,
                timing="host wall clock per MPI_Pack+MPI_Unpack pair, 200 pairs")


def type_commit_bench(mpi, reps=200):
    """MPI_Type_commit + MPI_Type_free through the interposer, as the
    reference's bin/bench_type_commit.cpp times them: a 3-D subarray committed
    again and again (the learned dispatch's choice is reused), and `reps`
    subarrays of distinct shapes (each one inference of the cost model)."""
    import time as _t

    def timed(make):
        t = make()
        a = _t.perf_counter()
        assert mpi.Type_commit(t) == 0
        b = _t.perf_counter()
        mpi.Type_free(t)
        return b - a

    same = [timed(lambda: mpi.Type_create_subarray([256, 256, 256], [256, 256, 16], [0, 0, 3],
                                                  mpi.ORDER_C, mpi.FLOAT))
            for _ in range(reps)]
    fresh = [timed(lambda i=i: mpi.Type_create_subarray([256, 256, 256],
                                                       [256, 1 + i % 255, 3 + i // 255],
                                                       [0, 0, 0], mpi.ORDER_C, mpi.FLOAT))
             for i in range(reps)]
    return {"repeated_shape_commit_us": round(1e6 * float(np.median(same)), 2),
            "new_shape_commit_us": round(1e6 * float(np.median(fresh)), 2),
            "reps": reps, "timing": "host wall clock, median"}


def call_overhead_bench(torch, mpi, n=2000):
    """Where the time of a synchronous call goes: host wall clock per call of
    MPI_Pack of a tiny type on device buffers (16 objects of 1024 rows of 4 B,
    4 KiB apart: the 2d_i1 sweep point's shape) beside an empty kernel launch
    + cudaStreamSynchronize, the launch alone, an idle synchronise and the two
    pointer-attribute queries the interposer makes, all from C."""
    t = mpi.Type_vector(1024, 1, 1024, mpi.FLOAT)
    assert mpi.Type_commit(t) == 0
    typed = torch.zeros(16 * 1024 * 1024 * 4 + 4096, dtype=torch.uint8, device="cuda")
    packed = torch.zeros(1 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    us = (ctypes.c_double * 5)()
    err = driver().tempi_bench_call_overhead(t, typed.data_ptr(), packed.data_ptr(), 16,
                                             1 << 20, n, us)
    mpi.Type_free(t)
    if err:
        return {"error": err}
    names = ("mpi_pack_us", "empty_launch_sync_us", "launch_only_us", "idle_sync_us",
             "pointer_attributes_x2_us")
    out = {k: round(v, 3) for k, v in zip(names, us)}
    out["beyond_round_trip_us"] = round(us[0] - us[1], 3)
    out["timing"] = (f"host wall clock, median of 5 batches of {n} calls; beyond_round_trip_us "
                     "= MPI_Pack minus the empty launch + synchronise round trip: the pack "
                     "kernel's own work beyond an empty kernel's (about 1.8 us in-kernel for "
                     "this shape) plus the library's host work")
    return out


def reduce_max(value, dist, device=None):
    """Max over ranks of a per-rank time (replicas: one process per GPU)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([float(value)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args):
    import torch

    from tempi_b200 import _lib, mpi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    assert mpi.Init() == 0
    lib = _lib.tempi()
    dev = torch.device("cuda", local)
    sw = GpuSweep(torch, mpi, dev)
    tstream = torch.cuda.ExternalStream(_tempi_stream())
    torch.cuda.synchronize()
    ops = sw.ops()
    run_ops(ops, args.warmup, sw.flush)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    launches0 = lib.tempi_kernel_launches()
    barrier()
    with Clocks(local) as clk:
        times = run_ops(ops, args.steps, sw.flush)
    barrier()
    launches = lib.tempi_kernel_launches() - launches0
    if launches < len(ops) * args.steps:
        raise RuntimeError(f"only {launches} TEMPI kernel launches in the timed region: "
                           "the MPI calls did not reach the interposer's GPU path")
    ms = reduce_max(sum(times) / len(times), dist, dev)
    value = world * sw.alg_bytes / ms / 1e6  # GB/s over all replicas

    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": round(value, 3), "unit": "GB/s",
                              "ms_per_step": round(ms, 4), "gpu_launches": int(launches),
                              "note": "--no-extras run (launch-list capture)"}))
        return
    side = torch.cuda.Stream()
    table = kernel_table(torch, sw, side, lib)
    empty_ms = empty_kernel_events(torch, sw, side)
    total_t = sum(r["pack_ms"] + r["unpack_ms"] for r in table)
    top = max(table, key=lambda r: r["pack_ms"])
    peak, peak_kind = measured_peaks()
    # the dominant kernel again, launched back to back between one event
    # pair: its inputs (typed and packed) are larger than the L2, so every
    # launch streams from DRAM, and the event pair's own cost is spread over
    # the launches
    top_ms = dominant_back_to_back(torch, sw, side, lib, top["label"])
    achieved = 2 * top["packed_bytes"] / top_ms / 1e6
    # the single-GPU characterisations run at N = 1 only: they would keep
    # the other ranks waiting at the final barrier
    solo = rank == 0 and world == 1
    halo_res = halo_bench(torch, sw, side) if solo else None
    if halo_res is not None:
        halo_res["exchange"] = halo_exchange_bench(torch, side)
    # end to end: every rank at once, the whole job's rate from the slowest
    # rank's time (replicas: each rank moves its own copy of the workload)
    barrier()
    e2e_staged = e2e_bench(torch, sw, mpi, max(1, args.steps // 2), 1)
    barrier()
    e2e_zc = e2e_zero_copy(torch, sw, max(1, args.steps // 2), 1)
    barrier()
    for part in (e2e_staged, e2e_zc):
        part["ms_per_step"] = round(reduce_max(part["ms_per_step"], dist, dev), 3)
        part["value"] = round(world * sw.alg_bytes / part["ms_per_step"] / 1e6, 3)
        part["h2d_bytes_per_step"] *= world
        part["d2h_bytes_per_step"] *= world
    e2e = dict(e2e_zc, staged=e2e_staged)
    send_res = sendrecv_bench(torch, mpi) if solo and not args.no_sendrecv else None
    c1_res = vector_1024x64_bench(torch, mpi) if solo else None
    commit_res = type_commit_bench(mpi) if solo else None
    overhead_res = call_overhead_bench(torch, mpi) if solo else None
    disp_res = dispatch_sample(torch) if solo and not args.no_sendrecv else None
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic", "config": CONFIG,
        "roofline": {
            "bound": "hbm", "kernel": f"{top['label']} pack ({top['kernel']})",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": peak_kind,
            "traffic": traffic_from_profiles(top["label"]),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/traffic.txt",
            "share_of_kernel_time": round(top["pack_ms"] / total_t, 3),
            "alg_bytes_per_launch": 2 * top["packed_bytes"],
            "launch_us": round(1e3 * top_ms, 2),
            "timing": "10 back-to-back launches between one CUDA event pair on the launching "
                      "stream (inputs 512 MiB, larger than L2), median of 5",
        },
        "clocks": clk.summary(),
        "gpu_launches": int(launches),
        "e2e": e2e,
        "halo": halo_res,
        "vector_1024x64": c1_res,
        "type_commit": commit_res,
        "call_overhead": overhead_res,
        "sendrecv": send_res,
        "dispatch": disp_res,
        "sweep": [sweep_row(r, peak) for r in table],
        "sweep_notes": {
            "pack_gbs/unpack_gbs": "one launch of the kernel MPI_Pack/MPI_Unpack runs (the "
                                   "learned pick), L2 flushed first, CUDA events around it: "
                                   "includes the event pair and the launch's fixed cost",
            "empty_kernel_us": round(1e3 * empty_ms, 2),
            "kernel_gbs": "ncu in-kernel duration of the same launch (profiles/kernel_times.txt)",
            "line_bound": "fraction of the copy peak the layout's unavoidable DRAM traffic "
                          "allows (lines read by a pack, sectors written and merged by an unpack)",
            "of_bound": "least in-kernel time (the larger of: empty kernel + line traffic at "
                        "the peak; a one-load gather of scattered lines) / measured in-kernel "
                        "time",
        },
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_budget)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


LAUNCH_LIST_REPS = 3
GATHER_ROWS, GATHER_STRIDE = 16384, 4096
BIG_GATHER_ROWS, BIG_GATHER_STRIDE = 262144, 1024


def launch_list_order():
    """The launches of --launch-list, in order: an empty kernel, then each
    sweep point's pack and unpack kernel, LAUNCH_LIST_REPS times over."""
    order = []
    for _ in range(LAUNCH_LIST_REPS):
        order += [("empty", "-"), ("gather", "-"), ("gather_big", "-")]
        for label, *_ in sweep_points():
            order += [(label, "pack"), (label, "unpack")]
    return order


def run_launch_list(args):
    """For an ncu launch list (gpu__time_duration, one pass): the kernel
    MPI_Pack / MPI_Unpack run for every sweep point at its benchmark
    incount, one launch at a time with the L2 flushed before each, after an
    empty kernel; see --summarize-launches."""
    import torch

    from tempi_b200 import _lib, mpi

    assert mpi.Init() == 0
    lib = _lib.tempi()
    sw = GpuSweep(torch, mpi, torch.device("cuda", 0))
    stream = torch.cuda.Stream()
    s = stream.cuda_stream
    plans = {}
    for p in sw.pts:  # every cost-model inference happens here, before the list
        err, d = mpi.describe(p["t"])
        assert err == 0
        plans[p["label"]] = (p, d, learned_configs(lib, d, p["incount"]))
    torch.cuda.synchronize()
    names = []
    for label, direction in launch_list_order():
        sw.flush_l2(stream)
        if label == "empty":
            assert driver().tempi_bench_empty(s) == 0
            names.append("empty")
        elif label == "gather":  # one scattered line per thread: 16,384 rows 4 KiB apart
            assert GATHER_ROWS * GATHER_STRIDE <= sw.src2.numel()
            assert driver().tempi_bench_gather(sw.src2.data_ptr(), GATHER_STRIDE, GATHER_ROWS,
                                               sw.packed.data_ptr(), s) == 0
            names.append("gather")
        elif label == "gather_big":  # 262,144 rows 1 KiB apart: the scattered-line rate
            assert BIG_GATHER_ROWS * BIG_GATHER_STRIDE <= sw.src3.numel()
            assert 4 * BIG_GATHER_ROWS <= sw.packed.numel()
            assert driver().tempi_bench_gather(sw.src3.data_ptr(), BIG_GATHER_STRIDE,
                                               BIG_GATHER_ROWS, sw.packed.data_ptr(), s) == 0
            names.append("gather_big")
        else:
            p, d, (cp, cu) = plans[label]
            n = p["incount"]
            if direction == "pack":
                _lib.check(lib.tempi_pack(ctypes.byref(d), p["src"].data_ptr(), n,
                                          sw.packed.data_ptr(), ctypes.byref(cp) if cp else None, s))
            else:
                _lib.check(lib.tempi_unpack(ctypes.byref(d), sw.packed.data_ptr(), n,
                                            p["dst"].data_ptr(), ctypes.byref(cu) if cu else None, s))
            names.append(lib.tempi_last_kernel().decode())
        stream.synchronize()
    print(json.dumps({"launch_list": len(names), "kernels": names[:3 + 2 * len(sw.pts)]}))


def summarize_launches(path, out_txt=None):
    """Per sweep point and direction, the median in-kernel time of the
    kernels --launch-list ran, from ncu's CSV (gpu__time_duration.sum),
    against the measured copy peak and the point's line-traffic bound.
    Prints a markdown table; writes `out_txt` (point direction us) when
    given."""
    import csv

    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hi]
    ki, vi, ui = h.index("Kernel Name"), h.index("Metric Value"), h.index("Metric Unit")
    seq = []
    for r in rows[hi + 1:]:
        if len(r) <= vi or r[h.index("Metric Name")] != "gpu__time_duration.sum":
            continue
        name = r[ki]
        if "read_all" in name or "k_mlp" in name or "Fill" in name or "fill" in name:
            continue
        v = float(r[vi].replace(",", ""))
        scale = {"nsecond": 1e-3, "usecond": 1.0, "msecond": 1e3}.get(r[ui], 1e-3)
        seq.append((name, v * scale))
    order = launch_list_order()
    if len(seq) != len(order):
        raise SystemExit(f"{len(seq)} kernels in the CSV, {len(order)} expected")
    by = {}
    for (label, direction), (name, us) in zip(order, seq):
        by.setdefault((label, direction), []).append((name, us))
    peak, kind = measured_peaks()
    pts = {p[0]: p for p in sweep_points()}
    empty = statistics.median(us for _, us in by[("empty", "-")])
    gather = statistics.median(us for _, us in by[("gather", "-")])
    line_us = (statistics.median(us for _, us in by[("gather_big", "-")]) - empty) / BIG_GATHER_ROWS
    lines = ["| point | dir | kernel | packed | in-kernel us | GB/s | of peak | line bound us "
             "| bound us | of that bound |", "|" + "---|" * 10]
    txt = [f"# point direction in_kernel_us  (ncu gpu__time_duration.sum, median of "
           f"{LAUNCH_LIST_REPS}; empty kernel {empty:.2f} us; one-load gather {gather:.2f} us; "
           f"scattered line {1e6 * line_us:.2f} ps)"]
    for label, sizes, subs, starts, n in sweep_points():
        size = 4 * int(np.prod(subs)) * n
        for u, direction in enumerate(("pack", "unpack")):
            ks = by[(label, direction)]
            us = statistics.median(x for _, x in ks)
            kname = ks[0][0].split("(")[0].replace("void ", "").replace("tempi::", "")
            tr = line_traffic(sizes, subs, starts, n, u)
            lb = tr / peak / 1e3
            gbs = 2 * size / us / 1e3
            bound = point_bound(empty, gather, tr, peak)
            lines.append(f"| {label} | {direction} | `{kname}` | {size / 2**20:.3g} MiB | "
                         f"{us:.2f} | {gbs:.0f} | {gbs / peak:.3f} | {lb:.2f} | "
                         f"{bound:.2f} | {bound / us:.2f} |")
            txt.append(f"{label} {direction} {us:.3f}")
    print(f"empty kernel: {empty:.2f} us, one-load gather of {GATHER_ROWS} rows: {gather:.2f} us, "
          f"one scattered line {1e6 * line_us:.2f} ps (gather of {BIG_GATHER_ROWS} rows) "
          f"in-kernel (medians); peak {peak} GB/s ({kind})")
    print("\n".join(lines))
    if out_txt:
        with open(out_txt, "w") as f:
            f.write("\n".join(txt) + "\n")


def run_profile(args):
    """A small case for ncu: one sweep point's pack (or unpack) kernel, the
    one the learned dispatch picks, launched --profile-reps times through
    tempi_pack/tempi_unpack."""
    import torch

    from tempi_b200 import _lib, mpi

    assert mpi.Init() == 0
    lib = _lib.tempi()
    pt = [p for p in sweep_points() if p[0] == args.profile_point]
    if not pt:
        raise SystemExit(f"unknown point {args.profile_point}")
    label, sizes, subs, starts, _ = pt[0]
    t = mpi.Type_create_subarray(sizes, subs, starts, mpi.ORDER_C, mpi.FLOAT)
    assert mpi.Type_commit(t) == 0
    err, d = mpi.describe(t)
    assert err == 0
    n = args.profile_incount
    src = torch.randint(0, 256, (d.extent * n,), dtype=torch.uint8, device="cuda")
    dst = torch.zeros_like(src)
    packed = torch.zeros(d.size * n, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    cp, cu = learned_configs(lib, d, n)  # the kernels MPI_Pack / MPI_Unpack run
    for _ in range(args.profile_reps):
        if args.profile_unpack:
            _lib.check(lib.tempi_unpack(ctypes.byref(d), packed.data_ptr(), n, dst.data_ptr(),
                                        ctypes.byref(cu) if cu else None, None))
        else:
            _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), n, packed.data_ptr(),
                                      ctypes.byref(cp) if cp else None, None))
    torch.cuda.synchronize()
    print(json.dumps({"profile_point": label, "incount": n, "packed_bytes": d.size * n,
                      "kernel": lib.tempi_last_kernel().decode(),
                      "device_bytes": int(src.numel() * 2 + packed.numel())}))


def run_profile_halo(args):
    """A small case for ncu: the batched pack of the 256^3-double, radius-2
    halo (26 regions, one launch), launched --profile-reps times."""
    import torch

    from tempi_b200 import halo, mpi

    assert mpi.Init() == 0
    g = halo.Grid((256, 256, 256), 2)
    data = torch.randint(0, 256, (g.nbytes,), dtype=torch.uint8, device="cuda")
    packed = torch.zeros(g.packed_bytes, dtype=torch.uint8, device="cuda")
    b = halo.HaloBatch([g], [data.data_ptr()], [packed.data_ptr()], unpack=args.profile_unpack)
    torch.cuda.synchronize()
    for _ in range(args.profile_reps):
        b.launch()
    torch.cuda.synchronize()
    b.close()
    print(json.dumps({"profile": "halo 256^3 doubles r=2", "regions": 26,
                      "packed_bytes": g.packed_bytes, "device_bytes": g.nbytes + g.packed_bytes,
                      "unpack": bool(args.profile_unpack)}))


def run_profile_exchange(args):
    """A small case for ncu: the fused periodic halo exchange of the
    256^3-double, radius-2 grid (26 copy pairs, one launch), launched
    --profile-reps times."""
    import torch

    from tempi_b200 import halo, mpi

    assert mpi.Init() == 0
    g = halo.Grid((256, 256, 256), 2)
    data = torch.randint(0, 256, (g.nbytes,), dtype=torch.uint8, device="cuda")
    x = halo.HaloExchange([g], [data.data_ptr()])
    torch.cuda.synchronize()
    for _ in range(args.profile_reps):
        x.launch()
    torch.cuda.synchronize()
    x.close()
    print(json.dumps({"profile": "periodic halo exchange 256^3 doubles r=2", "pairs": 26,
                      "bytes_copied": g.packed_bytes, "device_bytes": g.nbytes}))


def run_host_link(args):
    """Host-link rates on this machine: the copy engines one way and both
    ways, the word kernel reading, writing and copying pinned host memory,
    and the copy-engine pipeline MPI_Pack uses for contiguous runs between
    two pinned host buffers (256 MiB each)."""
    import torch

    from tempi_b200 import _lib, mpi

    assert mpi.Init() == 0
    lib = _lib.tempi()
    n = 256 << 20
    ha = torch.randint(0, 256, (n,), dtype=torch.uint8).pin_memory()
    hb = torch.empty(n, dtype=torch.uint8).pin_memory()
    da = torch.empty(n, dtype=torch.uint8, device="cuda")
    db = torch.empty(n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.ExternalStream(_tempi_stream())
    s2 = torch.cuda.Stream()
    reps = max(3, args.profile_reps)

    def gbs(fn, nbytes):
        fn()
        torch.cuda.synchronize()
        return round(nbytes / time_events(torch, st, fn, reps) / 1e6, 1)

    def h2d():
        with torch.cuda.stream(st):
            da.copy_(ha, non_blocking=True)

    def d2h():
        with torch.cuda.stream(st):
            hb.copy_(db, non_blocking=True)

    def both():
        e0 = torch.cuda.Event()
        e0.record(st)
        s2.wait_event(e0)
        with torch.cuda.stream(st):
            da.copy_(ha, non_blocking=True)
        with torch.cuda.stream(s2):
            hb.copy_(db, non_blocking=True)
        e1 = torch.cuda.Event()
        e1.record(s2)
        st.wait_event(e1)

    t = mpi.Type_contiguous(n, mpi.BYTE)
    assert mpi.Type_commit(t) == 0
    err, d = mpi.describe(t)
    assert err == 0

    def kernel(src, dst):
        return lambda: _lib.check(lib.tempi_pack(ctypes.byref(d), src.data_ptr(), 1,
                                                 dst.data_ptr(), None, st.cuda_stream))

    def pipeline():
        err, _ = mpi.Pack(ha.data_ptr(), 1, t, hb.data_ptr(), n)
        assert err == 0

    out = {
        "copy_engine_h2d": gbs(h2d, n), "copy_engine_d2h": gbs(d2h, n),
        "copy_engines_both_ways_each": round(gbs(both, 2 * n) / 2, 1),
        "kernel_reads_host": gbs(kernel(ha, da), n),
        "kernel_writes_host": gbs(kernel(da, hb), n),
        "kernel_host_to_host_each_way": gbs(kernel(ha, hb), n),
    }
    dma0 = _lib.counter("host_link_copies")
    out["mpi_pack_host_to_host_each_way"] = gbs(pipeline, n)
    out["mpi_pack_used_copy_engines"] = _lib.counter("host_link_copies") > dma0
    assert torch.equal(ha, hb)

    # rows of one strided dimension: a lone 2-D copy each way, and MPI_Pack /
    # MPI_Unpack host -> host by the copy-engine pipeline and by the kernels
    rows_out = []
    saved = os.environ.get("TEMPI_HOST_LINK")
    for width, pitch, off in ((64, 1024, 0), (64, 1024, 120), (256, 1024, 28),
                              (1024, 4096, 116)):
        nrows = (16 << 20) // width
        assert off + (nrows - 1) * pitch + width <= n
        src = ha.data_ptr() + off

        def g2d():
            _lib_check2d(driver().tempi_bench_copy2d(da.data_ptr(), width, src, pitch, width,
                                                     nrows, 0, st.cuda_stream))

        def s2d():
            _lib_check2d(driver().tempi_bench_copy2d(hb.data_ptr() + off, pitch, da.data_ptr(),
                                                     width, width, nrows, 1, st.cuda_stream))

        ty = mpi.Type_create_hvector(nrows, width, pitch, mpi.BYTE)
        assert mpi.Type_commit(ty) == 0
        row = {"row_bytes": width, "pitch": pitch, "offset": off, "rows": nrows,
               "copy2d_gather_h2d": gbs(g2d, width * nrows),
               "copy2d_scatter_d2h": gbs(s2d, width * nrows)}
        for path in ("copy_engines", "kernels"):
            if path == "kernels":
                os.environ["TEMPI_HOST_LINK"] = "kernel"
            else:
                os.environ.pop("TEMPI_HOST_LINK", None)
            lib.tempi_reload_env()

            def pk():
                err, _ = mpi.Pack(src, 1, ty, hb.data_ptr(), n)
                assert err == 0

            def up():
                err, _ = mpi.Unpack(hb.data_ptr(), n, db_host_ptr + off, 1, ty)
                assert err == 0

            db_host_ptr = ha.data_ptr()  # unpack back into the source span: same bytes
            row[f"mpi_pack_{path}"] = gbs(pk, width * nrows)
            row[f"mpi_unpack_{path}"] = gbs(up, width * nrows)
            os.environ.pop("TEMPI_HOST_LINK", None)
            if saved is not None:
                os.environ["TEMPI_HOST_LINK"] = saved
            lib.tempi_reload_env()
        mpi.Type_free(ty)
        rows_out.append(row)
    print(json.dumps({"host_link_gbs_per_direction": out, "bytes": n,
                      "strided_rows_gbs_per_direction": rows_out}))


def _lib_check2d(rc):
    if rc:
        raise RuntimeError("cudaMemcpy2DAsync failed")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # defaults: the first ~30 steps of a fresh process run about 6 % slower
    # than the steady state (a transient of the driver or GPU, not of this
    # library's caches), so the default warm-up outlasts it
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sendrecv", action="store_true",
                    help="skip the self-send and dispatch-regret sections")
    ap.add_argument("--no-extras", action="store_true",
                    help="time the sweep only (for launch-list captures)")
    ap.add_argument("--profile-point", default=None,
                    help="run only this sweep point's pack kernel (for ncu)")
    ap.add_argument("--profile-incount", type=int, default=2)
    ap.add_argument("--profile-reps", type=int, default=3)
    ap.add_argument("--profile-unpack", action="store_true")
    ap.add_argument("--profile-halo", action="store_true",
                    help="run only the batched halo kernel (for ncu)")
    ap.add_argument("--host-link", action="store_true",
                    help="measure the host-link rates and exit")
    ap.add_argument("--profile-exchange", action="store_true",
                    help="run only the fused halo-exchange kernel (for ncu)")
    ap.add_argument("--launch-list", action="store_true",
                    help="each sweep point's kernels once per pass, L2 flushed (for an ncu "
                         "launch list)")
    ap.add_argument("--summarize-launches", default=None, metavar="CSV",
                    help="per-point in-kernel times from the ncu CSV of --launch-list")
    ap.add_argument("--out", default=None, help="with --summarize-launches: a table file")
    args = ap.parse_args()
    if args.summarize_launches:
        summarize_launches(args.summarize_launches, args.out)
    elif args.launch_list:
        run_launch_list(args)
    elif args.host_link:
        run_host_link(args)
    elif args.profile_exchange:
        run_profile_exchange(args)
    elif args.profile_halo:
        run_profile_halo(args)
    elif args.profile_point:
        run_profile(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
