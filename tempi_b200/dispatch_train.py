"""Measure, train and evaluate the learned dispatch on this machine.

The reference measures tables of pack, unpack and transfer times once per
machine (bin/measure_system.cpp -> $TEMPI_CACHE_DIR/perf.json) and
interpolates them to choose a send method.  This tool does the learned
equivalent:

1. draws random strided layouts (ndims 1-3, block 1 B - 64 KiB log-uniform,
   strides = inner extent x U[1,16] rounded to an alignment in
   {1,2,4,8,16}, totals 1 KiB - 256 MiB log-uniform, typed and packed
   buffers in device or mapped pinned host memory) and times every
   candidate on each with tempi_measure: a pack and an unpack with each of
   ten kernel configurations and with the fixed rules, and -- on a
   subset -- the three transfer methods;
2. trains the cost model (a 5-member FP32 MLP ensemble, 12 -> 64 -> 64 -> 23)
   on the GPU with tempi_mlp_train;
3. measures the reference's table model on this machine (pack/unpack
   tables over 2^(2i+6) bytes x 2^j-byte blocks at a 512-byte stride,
   self-send ping-pong and host-copy tables), the comparison policy;
4. evaluates on held-out layouts: prediction error, and the time regret of
   the learned choice, the table model and the fixed rules against
   exhaustive search;
5. writes the model and tables (read by MPI_Init from TEMPI_CACHE_DIR or
   tempi_b200/models/) and a JSON report.

    python -m tempi_b200.dispatch_train --types 50000 --heldout 5000 \\
        --budget-s 900 --out /tmp/dispatch
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np

from . import _lib, mpi

HERE = os.path.dirname(os.path.abspath(__file__))
MODELS = os.path.join(HERE, "models")
MODEL_FILE = "tempi_b200_dispatch.bin"
TABLE_FILE = "tempi_b200_table.bin"
N_CFG, N_METH = 10, 3
PACK, UNPACK, METH = 0, N_CFG, 2 * N_CFG      # model output offsets
N_OUT = 2 * N_CFG + N_METH                    # 23
FIXED_PACK, FIXED_UNPACK = N_OUT, N_OUT + 1   # measured after the outputs
N_MEAS = N_OUT + 2                            # 25
P = (12 * 64 + 64) + (64 * 64 + 64) + (64 * N_OUT + N_OUT)


def round_up(x, a):
    return ((x + a - 1) // a) * a


def random_layout(rng):
    """One layout of the benchmark's dispatch config: (desc, incount,
    typed_host, packed_host)."""
    nd = int(rng.integers(1, 4))
    a = [1, 2, 4, 8, 16][int(rng.integers(0, 5))]
    block = max(1, int(math.exp(rng.uniform(0, math.log(65536)))))
    total = int(math.exp(rng.uniform(math.log(1024), math.log(256 << 20))))
    typed_host = bool(rng.uniform() < 0.2)
    packed_host = bool(rng.uniform() < 0.2)
    if typed_host or packed_host:
        total = min(total, 4 << 20)  # host-link traffic: keep it bounded
    incount = 1 if rng.uniform() < 0.7 else int(rng.integers(2, 17))
    start = a * int(rng.integers(0, 4))
    counts, strides = [], []
    if nd == 1:
        block = max(1, total // incount)
    else:
        rows = max(1, total // (block * incount))
        if nd == 2:
            cs = [rows]
        else:
            c1 = max(1, int(math.exp(rng.uniform(0, math.log(rows)))))
            cs = [c1, max(1, rows // c1)]
        inner = block
        for c in cs:
            s = round_up(max(inner, int(inner * rng.uniform(1, 16))), a)
            counts.append(c)
            strides.append(s)
            inner = c * s
    hi = start + block + sum((c - 1) * s for c, s in zip(counts, strides))
    extent = round_up(hi, a)
    desc = _lib.Desc.make(start, extent, block, counts, strides)
    return desc, incount, typed_host, packed_host


def span_of(desc, incount):
    hi = desc.start + desc.block + desc.extent * (incount - 1)
    for k in range(desc.ndims):
        hi += (desc.counts[k] - 1) * desc.strides[k]
    return hi


# back-to-back launches per candidate for objects under 1 MiB, under 64 MiB,
# and larger (their mean is the label)
REPS = (12, 6, 2)


def measure_dataset(n, budget_s, seed, method_every=8, log=print):
    lib = _lib.tempi()
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 12), np.float32)
    T = np.full((n, N_MEAS), np.nan, np.float32)
    meta = np.zeros((n, 4), np.int64)  # incount, typed_host, packed_host, block
    t0 = time.time()
    done = 0
    f = (ctypes.c_float * 12)()
    times = (ctypes.c_float * N_MEAS)()
    while done < n and time.time() - t0 < budget_s:
        d, incount, th, ph = random_layout(rng)
        span = span_of(d, incount)
        if span > (2 << 30) or (th and span > (16 << 20)):
            continue
        size = d.size * incount
        # transfers by all three methods on every 8th device layout up to
        # 64 MiB (host-staged transfers of larger objects take too long)
        methods = done % method_every == 0 and not th and not ph and size <= (64 << 20)
        what = 1 | (2 if methods else 0)
        reps = REPS[0] if size < (1 << 20) else REPS[1] if size < (64 << 20) else REPS[2]
        err = lib.tempi_measure(ctypes.byref(d), incount, int(th), int(ph), what, reps, times)
        if err:
            raise RuntimeError(f"tempi_measure failed: {_lib.last_error()}")
        lib.tempi_features(ctypes.byref(d), incount, int(th), int(ph), f)
        X[done] = np.frombuffer(f, np.float32)
        T[done] = np.frombuffer(times, np.float32)
        meta[done] = (incount, th, ph, d.block)
        done += 1
        if done % 2000 == 0:
            log(f"  measured {done} layouts in {time.time() - t0:.0f} s")
    return X[:done], T[:done], meta[:done], time.time() - t0


def train(X, Y, M, members=5, epochs=None, lr=2e-3, seed=1234, log=print):
    import torch

    lib = _lib.tempi()
    n = len(X)
    if epochs is None:  # about 40k mini-batch steps
        epochs = int(min(400, max(20, round(40000 * 64 / max(n, 1)))))
    params = torch.zeros(members * P, dtype=torch.float32, device="cuda")
    _lib.check(lib.tempi_mlp_init(ctypes.c_void_p(params.data_ptr()), members, seed))
    dx = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    dy = torch.from_numpy(np.ascontiguousarray(Y)).cuda()
    dm = torch.from_numpy(np.ascontiguousarray(M)).cuda()
    losses = torch.zeros(members * epochs, dtype=torch.float32, device="cuda")
    t0 = time.time()
    _lib.check(lib.tempi_mlp_train(
        ctypes.c_void_p(params.data_ptr()), members, ctypes.c_void_p(dx.data_ptr()),
        ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(dm.data_ptr()), n, epochs, 64,
        ctypes.c_float(lr), seed, ctypes.c_void_p(losses.data_ptr()), None))
    torch.cuda.synchronize()
    dt = time.time() - t0
    l = losses.cpu().numpy().reshape(members, epochs)
    log(f"  trained {members} members x {epochs} epochs on {n} rows in {dt:.1f} s; "
        f"loss {l[:, 0].mean():.3f} -> {l[:, -1].mean():.3f}")
    return params, l, dt, epochs


def predict(params, members, X):
    import torch

    lib = _lib.tempi()
    dx = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    out = torch.zeros(members * len(X) * N_OUT, dtype=torch.float32, device="cuda")
    _lib.check(lib.tempi_mlp_predict(ctypes.c_void_p(params.data_ptr()), members,
                                     ctypes.c_void_p(dx.data_ptr()), len(X),
                                     ctypes.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(members, len(X), N_OUT)


def write_model(path, params_np, members, y_mean, y_std, gpu):
    with open(path, "wb") as fh:
        fh.write(b"TMLPv001")
        fh.write(np.array([12, 64, N_OUT, members], np.int32).tobytes())
        fh.write(np.asarray(y_mean, np.float32).tobytes())
        fh.write(np.asarray(y_std, np.float32).tobytes())
        fh.write(np.asarray(params_np, np.float32).tobytes())


def measure_tables(log=print):
    """The reference's table model, measured with this library's kernels
    and transfers on this machine (microseconds)."""
    import torch

    lib = _lib.tempi()
    times = (ctypes.c_float * N_MEAS)()
    NI, NJ = 10, 10
    tabs = {k: np.zeros((NI, NJ)) for k in ("pack_dev", "unpack_dev", "pack_host", "unpack_host")}
    for i in range(NI):
        nbytes = 1 << (2 * i + 6)
        for j in range(NJ):
            block = 1 << j
            count = max(1, nbytes // block)
            d = _lib.Desc.make(0, count * 512, block, [count], [512])
            for ph, key in ((0, "dev"), (1, "host")):
                _lib.check(lib.tempi_measure(ctypes.byref(d), 1, 0, ph, 1, 3, times))
                tabs["pack_" + key][i, j] = float(times[FIXED_PACK])
                tabs["unpack_" + key][i, j] = float(times[FIXED_UNPACK])
    # self-send ping-pong of contiguous bytes, device and host buffers, and
    # copies between device and pinned host memory (the reference's d2h/h2d
    # tables, measure_system.cu)
    N1 = 28
    pp_dev, pp_host = np.zeros(N1), np.zeros(N1)
    d2h, h2d = np.zeros(N1), np.zeros(N1)
    dbuf = torch.zeros(1 << (N1 - 1), dtype=torch.uint8, device="cuda")
    dbuf2 = torch.zeros_like(dbuf)
    hbuf = np.zeros(1 << (N1 - 1), np.uint8)
    hbuf2 = np.zeros_like(hbuf)
    pinned = torch.zeros(1 << (N1 - 1), dtype=torch.uint8).pin_memory()
    for i in range(N1):
        n = 1 << i
        for arr, dst, src in ((d2h, pinned, dbuf), (h2d, dbuf2, pinned)):
            reps = 5 if n < (1 << 20) else 2
            dst[:n].copy_(src[:n])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(reps):
                dst[:n].copy_(src[:n])
                torch.cuda.synchronize()
            arr[i] = 1e6 * (time.perf_counter() - t0) / reps
        for arr, (a, b) in ((pp_dev, (dbuf.data_ptr(), dbuf2.data_ptr())),
                            (pp_host, (hbuf.ctypes.data, hbuf2.ctypes.data))):
            reps = 5 if n < (1 << 20) else 2
            mpi.Send(a, n, mpi.BYTE, tag=91)
            mpi.Recv(b, n, mpi.BYTE, tag=91)
            t0 = time.perf_counter()
            for _ in range(reps):
                mpi.Send(a, n, mpi.BYTE, tag=91)
                mpi.Recv(b, n, mpi.BYTE, tag=91)
            arr[i] = 1e6 * (time.perf_counter() - t0) / reps
    log("  measured the table model's tables")
    return tabs, pp_dev, pp_host, d2h, h2d


def write_tables(path, tabs, pp_dev, pp_host, d2h, h2d):
    with open(path, "wb") as fh:
        fh.write(b"TTABv001")
        NI, NJ = tabs["pack_dev"].shape
        fh.write(np.array([len(pp_dev), NI, NJ], np.int32).tobytes())
        for a in (pp_dev, pp_host, d2h, h2d):
            fh.write(np.asarray(a, np.float64).tobytes())
        for k in ("pack_dev", "unpack_dev", "pack_host", "unpack_host"):
            fh.write(np.asarray(tabs[k], np.float64).tobytes())


def regret(chosen, best):
    chosen, best = np.asarray(chosen), np.asarray(best)
    return {
        "total_time_regret": float(chosen.sum() / best.sum() - 1),
        "mean_regret": float(np.mean(chosen / best - 1)),
        "within_5pct": float(np.mean(chosen <= 1.05 * best)),
    }


def evaluate(params, members, y_mean, y_std, X, T, meta, spread_limit=0.5):
    pred = predict(params, members, X) * y_std + y_mean  # log2 us
    mean, spread = pred.mean(0), pred.std(0)
    rows = np.arange(len(X))
    rep = {}
    # kernel configurations: measured (finite) entries are exactly the
    # eligible candidates, which is all the dispatcher chooses among; a pack
    # and an unpack are chosen separately
    elig = np.isfinite(T[:, PACK:PACK + N_CFG]) & np.isfinite(T[:, UNPACK:UNPACK + N_CFG])
    ok = elig.any(1) & np.isfinite(T[:, FIXED_PACK]) & np.isfinite(T[:, FIXED_UNPACK])
    E, n_ok = elig[ok], int(ok.sum())
    r = np.arange(n_ok)
    tp, tu = T[ok, PACK:PACK + N_CFG], T[ok, UNPACK:UNPACK + N_CFG]
    mp, mu = mean[ok, PACK:PACK + N_CFG], mean[ok, UNPACK:UNPACK + N_CFG]
    sp_p, sp_u = spread[ok, PACK:PACK + N_CFG], spread[ok, UNPACK:UNPACK + N_CFG]
    best_p = np.where(E, tp, np.inf).min(1)
    best_u = np.where(E, tu, np.inf).min(1)
    best_cfg = best_p + best_u
    cp = np.where(E, mp, np.inf).argmin(1)
    cu = np.where(E, mu, np.inf).argmin(1)
    t_learned = tp[r, cp] + tu[r, cu]
    fb_p, fb_u = sp_p[r, cp] > spread_limit, sp_u[r, cu] > spread_limit
    t_fallback = np.where(fb_p, best_p, tp[r, cp]) + np.where(fb_u, best_u, tu[r, cu])
    # one configuration for both directions, as a single prediction would pick
    cj = np.where(E, 2.0 ** mp + 2.0 ** mu, np.inf).argmin(1)
    t_joint = tp[r, cj] + tu[r, cj]
    fixed = T[ok, FIXED_PACK] + T[ok, FIXED_UNPACK]
    rep["configs"] = {
        "layouts": n_ok,
        "learned": regret(t_learned, best_cfg),
        "learned_with_fallback": regret(t_fallback, best_cfg),
        "fallback_rate": float(np.mean(fb_p | fb_u)),
        "learned_one_config_for_both": regret(t_joint, best_cfg),
        "fixed_rules": regret(fixed, best_cfg),
        "exhaustive_total_us": float(best_cfg.sum()),
        "learned_total_us": float(t_learned.sum()),
        "fixed_rules_total_us": float(fixed.sum()),
    }
    host = (meta[ok, 1] > 0) | (meta[ok, 2] > 0)
    if host.any():
        rep["configs"]["host_buffers"] = {
            "layouts": int(host.sum()),
            "learned": regret(t_learned[host], best_cfg[host]),
            "learned_one_config_for_both": regret(t_joint[host], best_cfg[host]),
            "fixed_rules": regret(fixed[host], best_cfg[host]),
        }
    y = np.log2(T[:, :N_OUT])
    obs = np.isfinite(y)
    err = np.abs(mean - np.where(obs, y, 0))[obs]
    rep["prediction"] = {
        "mae_log2": float(err.mean()), "median_abs_rel_err": float(np.median(2 ** err - 1)),
        "p90_abs_rel_err": float(np.percentile(2 ** err - 1, 90)),
    }
    # transfer methods
    okm = np.isfinite(T[:, METH:METH + N_METH]).all(1)
    if okm.any():
        tm = T[okm, METH:METH + N_METH]
        best_m = tm.min(1)
        lm = mean[okm, METH:METH + N_METH].argmin(1)
        rep["methods"] = {
            "layouts": int(okm.sum()),
            "learned": regret(tm[np.arange(len(tm)), lm], best_m),
            "fixed_rules_device": regret(tm[:, 0], best_m),
            "exhaustive_choice_share": {n: float(np.mean(tm.argmin(1) == k))
                                        for k, n in enumerate(("DEVICE", "ONE_SHOT", "STAGED"))},
        }
    return rep, mean


def table_regret(X_rows_desc, T, okm_rows):
    """Regret of the restated table model on the method rows."""
    lib = _lib.tempi()
    chosen = []
    for d, incount in X_rows_desc:
        mi, pc, uc = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
        _lib.check(lib.tempi_dispatch_choose(ctypes.byref(d), incount, 0, 0, 1,
                                             ctypes.byref(pc), ctypes.byref(uc),
                                             ctypes.byref(mi), None, None))
        chosen.append(mi.value - 1)
    tm = T[okm_rows, METH:METH + N_METH]
    best = tm.min(1)
    return regret(tm[np.arange(len(tm)), np.array(chosen)], best), chosen


def main(argv=None):
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--types", type=int, default=50000)
    ap.add_argument("--heldout", type=int, default=5000)
    ap.add_argument("--budget-s", type=float, default=900)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--members", type=int, default=5)
    ap.add_argument("--epochs", type=int, default=None)
    ap.add_argument("--out", default=None)
    ap.add_argument("--reps", default=None,
                    help="launches per candidate under 1 MiB,64 MiB,above (default 12,6,2)")
    ap.add_argument("--dataset", default=None,
                    help="train on a dispatch_dataset.npz saved by an earlier run instead of "
                         "measuring (same --seed and --types)")
    ap.add_argument("--no-install", action="store_true",
                    help="do not write tempi_b200/models/")
    args = ap.parse_args(argv)
    global REPS
    if args.reps:
        REPS = tuple(int(x) for x in args.reps.split(","))
        assert len(REPS) == 3 and min(REPS) >= 1
    out = args.out or os.path.join(os.environ.get("TEMPI_CACHE_DIR", "."), "dispatch")
    os.makedirs(out, exist_ok=True)
    assert mpi.Init() == 0
    gpu = torch.cuda.get_device_name(0)
    print(f"measuring up to {args.types} layouts on {gpu} (budget {args.budget_s:.0f} s)")
    if args.dataset:
        z = np.load(args.dataset)
        X, T, meta, t_meas = z["X"], z["T"], z["meta"], 0.0
    else:
        X, T, meta, t_meas = measure_dataset(args.types, args.budget_s, args.seed)
    n = len(X)
    h = min(args.heldout, n // 10)
    # regenerate the held-out descriptors for the table policy
    rng = np.random.default_rng(args.seed)
    descs = []
    while len(descs) < n:
        d, incount, th, ph = random_layout(rng)
        span = span_of(d, incount)
        if span > (2 << 30) or (th and span > (16 << 20)):
            continue
        descs.append((d, incount))
    Y = np.log2(T[:, :N_OUT])
    M = np.isfinite(Y).astype(np.float32)
    tr = slice(0, n - h)
    y_mean = np.array([np.nanmean(Y[tr, j]) if M[tr, j].any() else 0.0 for j in range(N_OUT)], np.float32)
    y_std = np.array([max(np.nanstd(Y[tr, j]), 1e-3) if M[tr, j].any() else 1.0 for j in range(N_OUT)], np.float32)
    Yn = np.where(M > 0, (Y - y_mean) / y_std, 0).astype(np.float32)
    params, losses, t_train, epochs = train(X[tr], Yn[tr], M[tr], args.members, args.epochs)
    ho = slice(n - h, n)
    report, _ = evaluate(params, args.members, y_mean, y_std, X[ho], T[ho], meta[ho])
    # the table model on the same held-out method rows
    tabs, pp_dev, pp_host, d2h, h2d = measure_tables()
    tpath = os.path.join(out, TABLE_FILE)
    write_tables(tpath, tabs, pp_dev, pp_host, d2h, h2d)
    _lib.check(_lib.tempi().tempi_dispatch_load(None, tpath.encode()))
    okm = np.isfinite(T[ho, METH:METH + N_METH]).all(1)
    if okm.any():
        ho_descs = [descs[n - h + i] for i in np.nonzero(okm)[0]]
        report["methods"]["table_model"], _ = table_regret(ho_descs, T[ho], okm)
    mpath = os.path.join(out, MODEL_FILE)
    params_np = params.cpu().numpy()
    write_model(mpath, params_np, args.members, y_mean, y_std, gpu)
    if not args.no_install:
        os.makedirs(MODELS, exist_ok=True)
        write_model(os.path.join(MODELS, MODEL_FILE), params_np, args.members, y_mean, y_std, gpu)
        write_tables(os.path.join(MODELS, TABLE_FILE), tabs, pp_dev, pp_host, d2h, h2d)
    report.update({
        "gpu": gpu, "layouts_measured": n, "train_rows": n - h, "heldout_rows": h,
        "method_rows": int(np.isfinite(T[:, METH]).sum()),
        "measure_s": round(t_meas, 1), "train_s": round(t_train, 2), "epochs": epochs,
        "members": args.members, "loss_first_epoch": float(losses[:, 0].mean()),
        "loss_last_epoch": float(losses[:, -1].mean()),
        "seed": args.seed, "reps": list(REPS),
    })
    with open(os.path.join(out, "dispatch_report.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    np.savez_compressed(os.path.join(out, "dispatch_dataset.npz"), X=X, T=T, meta=meta)
    print(json.dumps(report, indent=1))


if __name__ == "__main__":
    main()
