"""Benchmark suite for the configurations beside the headline SpMV.

    python -m hbdia_b200.suite small       # 27-point 64^3: launch-bound; separate launches vs one CUDA graph
    python -m hbdia_b200.suite precision   # banded n = 8M, FP64 / FP32 / BF16-scaled value storage
    python -m hbdia_b200.suite spmm        # 7-point Laplacian 128^3, k in {4, 16, 32}, FP64 and FP32 storage
    python -m hbdia_b200.suite cg          # SPD 27-point 128^3: mixed-precision vs plain FP64 CG
    python -m hbdia_b200.suite batched     # 64 stencils of edge U[16,96]: separate launches vs one batched launch
    python -m hbdia_b200.suite serve       # 32 resident matrices, Poisson arrivals: batched server vs plain FP64
    python -m hbdia_b200.suite convert --grid 256   # host vs GPU converter, COO -> device layout
    python -m hbdia_b200.suite partition   # 256^3 cut into 2/4/8 row partitions: per-rank SpMV and halo
    python -m hbdia_b200.suite spmv --grid 128 --storage 1 --kernel pipe   # one kernel on the
                                           # headline workload's shape (what the profiles capture)

Each measurement prints one JSON line.  Times are CUDA-event device times on
a dedicated stream after warm-up; inputs exceed L2 unless stated.  Accuracy
is the maximum over rows of |y - y_fp64| / sum_j |a_ij x_j| against the FP64
SpMV of the same matrix (this library's, which tests/ pin bit for bit to the
oracle).
"""
from __future__ import annotations

import argparse
import json
import sys

import numpy as np

PEAK_NOTE = "fraction of the measured HBM copy bandwidth (MEASURED_PEAKS.json)"


def _peak():
    import os
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"])
    except Exception:
        return 6650.0


def _time(fn, stream, reps=20, warmup=3):
    import torch
    for _ in range(warmup):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def _scaled_err(y, yref, rows, cols, vals, x):
    scale = np.zeros(len(y))
    np.add.at(scale, rows, np.abs(vals * x[cols]))
    return float(np.max(np.abs(y - yref) / np.maximum(scale, np.finfo(float).tiny)))


def precision(args):
    import torch
    import hbdia_b200 as hb
    n = args.n
    offs = [0, 1, -1, 2, -2, 64, -64, 4096, -4096]
    rows, cols, vals = hb.generate_banded(n, offs, 0.5, 1.5, 0.3, 0.002, 2)
    x = hb.fill_uniform(n, -1.0, 1.0, 2)
    xt = torch.from_numpy(x).cuda()
    stream = torch.cuda.Stream()
    yref = None
    base_rate = None
    for name, st in (("fp64", hb.STORE_NATIVE), ("fp32", hb.STORE_F32), ("bf16_scaled", hb.STORE_BF16_SCALED),
                     ("fp32_quad_interleaved", hb.STORE_F32_QUAD), ("bf16_scaled_quad_interleaved", hb.STORE_BF16_QUAD)):
        m = hb.HBDIA(rows, cols, vals, n, n)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(st)
        yt = torch.zeros(n, dtype=torch.float64, device="cuda")
        ms = _time(lambda: hb.spmv_device(m, xt.data_ptr(), yt.data_ptr(), stream.cuda_stream), stream)
        m.synchronize()
        y = yt.cpu().numpy()
        if yref is None:
            yref = y
            base_rate = 1e3 / ms
        err = _scaled_err(y, yref, rows, cols, vals, x)
        b = m.bytesPerSpmv()
        print(json.dumps({"suite": "precision", "workload": f"banded n={n} offsets {offs}, drop 0.3, 0.2% scattered",
                          "storage": name, "accumulate": "fp64", "ms_per_spmv": ms, "spmv_per_s": 1e3 / ms,
                          "speedup_vs_fp64": (1e3 / ms) / base_rate, "bytes_per_spmv": b,
                          "gbs": b / (ms / 1e3) / 1e9, "frac_of_peak": b / (ms / 1e3) / 1e9 / _peak(),
                          "max_scaled_err_vs_fp64": err, "nnz": int(len(vals))}), flush=True)
        del m


def spmm(args):
    import torch
    import hbdia_b200 as hb
    g = args.grid
    n = g ** 3
    rows, cols, vals = hb.generate_stencil7(g, g, g, 6.0, -1.0)
    stream = torch.cuda.Stream()
    for stname, st in (("fp64", hb.STORE_NATIVE), ("fp32", hb.STORE_F32)):
        m = hb.HBDIA(rows, cols, vals, n, n)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(st)
        info = m.info()
        vbytes = info.numSlots * (8 if st == hb.STORE_NATIVE else 4) + 4 * info.totalOffsets + 4 * (info.numBlocks + 1)
        x1 = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, n)).cuda()
        y1 = torch.zeros(n, dtype=torch.float64, device="cuda")
        ms1 = _time(lambda: hb.spmv_device(m, x1.data_ptr(), y1.data_ptr(), stream.cuda_stream), stream)
        if stname == "fp64":
            ms_plain = ms1
        for k in (4, 16, 32):
            X = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (n, k))).cuda().contiguous()
            Y = torch.zeros((n, k), dtype=torch.float64, device="cuda")
            tune = m.autotune(X.data_ptr(), Y.data_ptr(), k=k, stream=stream.cuda_stream)
            ms = _time(lambda: hb.spmm_device(m, X.data_ptr(), k, Y.data_ptr(), k, k, stream.cuda_stream), stream)
            Xc = X.t().contiguous()  # column-major: each right-hand side contiguous
            Yc = torch.zeros((k, n), dtype=torch.float64, device="cuda")
            msc = _time(lambda: hb.spmm_device_colmajor(m, Xc.data_ptr(), n, Yc.data_ptr(), n, k, stream.cuda_stream),
                        stream)
            # separate vectors (one allocation each): the vector-list form
            xs = [torch.from_numpy(np.random.default_rng(3 + j).uniform(-1, 1, n)).cuda() for j in range(k)]
            ys = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(k)]
            xp, yp = [t.data_ptr() for t in xs], [t.data_ptr() for t in ys]
            msl = _time(lambda: hb.spmv_list_device(m, xp, yp, stream.cuda_stream), stream)
            m.synchronize()
            b = vbytes + k * 16 * n
            for layout, t, tile in (("row-major (autotuned tile)", ms, tune.spmmTile), ("column-major (default tile)", msc, 4),
                                    ("vector list (default tile)", msl, 4)):
                print(json.dumps({"suite": "spmm", "workload": f"7-point Laplacian {g}^3 (centre 6, -1)",
                                  "storage": stname, "k": k, "layout": layout, "rhs_tile": tile, "ms": t,
                                  "ms_k_spmv": k * ms1, "speedup_vs_k_spmv": k * ms1 / t,
                                  "spmv_per_s_vs_plain_fp64_spmv": k * ms_plain / t,
                                  "bytes": b, "gbs": b / (t / 1e3) / 1e9,
                                  "frac_of_peak": b / (t / 1e3) / 1e9 / _peak()}), flush=True)
        del m


def small(args):
    """Config 1: the 27-point stencil on 64^3 (centre 26, neighbours -1) with
    0.5 % extras U(0.1, 1) (seed 0), blockWidth 32, threshold 2, x_i = i + 1.
    One SpMV is ~61 MB, so a lone launch is launch-bound: timed as separate
    launches on a stream and as 100 SpMVs replayed from one CUDA graph, and
    through the host entry points (one call per SpMV; pipelined)."""
    import time
    import torch
    import hbdia_b200 as hb
    g = args.grid if args.grid != 128 else 64
    n = g ** 3
    rows, cols, vals = hb.generate_stencil27(g, g, g, 26.0, -1.0, 0.005, 0.1, 1.0, 0)
    m = hb.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    b = m.bytesPerSpmv()
    x = torch.arange(1, n + 1, dtype=torch.float64, device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    ms_launch = _time(lambda: hb.spmv_device(m, x.data_ptr(), y.data_ptr(), sp), stream, reps=200)
    reps = 100
    gr = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        hb.spmv_device(m, x.data_ptr(), y.data_ptr(), sp)  # warm outside capture
        torch.cuda.synchronize()
        with torch.cuda.graph(gr, stream=stream):
            for _ in range(reps):
                hb.spmv_device(m, x.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    with torch.cuda.stream(stream):
        ms_graph = _time(gr.replay, stream, reps=10) / reps
    xh = torch.arange(1, n + 1, dtype=torch.float64).pin_memory().numpy()
    yh = [torch.zeros(n, dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
    hb.spmv_host(m, xh, yh[0])
    t = time.perf_counter()
    for _ in range(50):
        hb.spmv_host(m, xh, yh[0])
    ms_host = 1e3 * (time.perf_counter() - t) / 50
    hb.spmv_host_many(m, [xh] * 3, yh)
    t = time.perf_counter()
    hb.spmv_host_many(m, [xh] * 60, [yh[j % 3] for j in range(60)])
    ms_many = 1e3 * (time.perf_counter() - t) / 60
    for name, ms in (("device, separate launches", ms_launch), ("device, 100 SpMVs in one CUDA graph", ms_graph),
                     ("host buffers, hbdia_spmv_host per SpMV", ms_host),
                     ("host buffers, hbdia_spmv_host_many (pipelined)", ms_many)):
        print(json.dumps({"suite": "small", "workload": f"27-point stencil {g}^3 + 0.5% extras, x_i = i + 1",
                          "path": name, "ms_per_spmv": ms, "bytes_per_spmv": b, "gbs": b / (ms / 1e3) / 1e9,
                          "frac_of_peak": b / (ms / 1e3) / 1e9 / _peak()}), flush=True)


def cg(args):
    import torch
    import hbdia_b200 as hb
    g = args.grid
    n = g ** 3
    rows, cols, vals = hb.generate_stencil27_spd(g, g, g, 1e-3, 7)
    b = hb.fill_uniform(n, -1.0, 1.0, 11)
    bt = torch.from_numpy(b).cuda()
    m = hb.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2)
    for name, st in (("mixed: fp32-storage iterations, fp64 reliable updates", hb.STORE_F32),
                     ("mixed: fp32 quad-interleaved iterations, fp64 reliable updates", hb.STORE_F32_QUAD),
                     ("plain fp64 CG", hb.STORE_NATIVE)):
        xt = torch.zeros(n, dtype=torch.float64, device="cuda")
        hb.cg_solve(m, bt.data_ptr(), xt.data_ptr(), tol=1e-10, iter_storage=st)  # warm
        xt.zero_()
        torch.cuda.synchronize()
        r = hb.cg_solve(m, bt.data_ptr(), xt.data_ptr(), tol=1e-10, iter_storage=st)
        x = xt.cpu().numpy()
        ax = np.zeros(n)
        np.add.at(ax, rows, vals * x[cols])
        host_res = float(np.linalg.norm(b - ax) / np.linalg.norm(b))
        print(json.dumps({"suite": "cg", "workload": f"SPD symmetrised 27-point stencil {g}^3, b ~ U(-1,1)",
                          "method": name, "fp64_residual_updates": r.updates,
                          "iterations": r.iterations, "seconds": r.seconds,
                          "ms_per_iteration": 1e3 * r.seconds / max(1, r.iterations),
                          "rel_residual": r.relResidual, "rel_residual_host_check": host_res,
                          "converged": bool(r.converged)}), flush=True)


def batched(args):
    """64 27-point stencils of edge U[16, 96] (numpy default_rng(4)), matrix i
    with 0.5 % off-pattern extras (seed 100 + i) and x ~ U(-1, 1) (seed
    200 + i).  Timed on one stream: 64 single-matrix launches, the same
    launches replayed from one CUDA graph, and the batch (hbdia_batch_*)
    with its concurrent and queue schedules, then autotuned."""
    import torch
    import hbdia_b200 as hb
    edges = np.random.default_rng(4).integers(16, 97, args.count)
    mats, xs, ys = [], [], []
    for i, e in enumerate(edges.tolist()):
        r, c, v = hb.generate_stencil27(e, e, e, extra_fraction=0.005, seed=100 + i)
        n = e ** 3
        m = hb.HBDIA(r, c, v, n, n)
        m.convertToHBDIAFormat(32, 2, upload=False)
        m.prepareForGPU(args.storage)
        mats.append(m)
        xs.append(torch.from_numpy(hb.fill_uniform(n, -1.0, 1.0, 200 + i)).cuda())
        ys.append(torch.zeros(n, dtype=torch.float64, device="cuda"))
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    total_bytes = sum(m.bytesPerSpmv() for m in mats)
    rows = int(sum(int(e) ** 3 for e in edges))
    peak = _peak()

    def report(name, ms, extra=None):
        d = {"suite": "batched", "workload": f"{len(mats)} 27-point stencils, edge U[16,96] seed 4, "
             f"0.5% extras, {rows} rows", "storage": ["fp64", "fp32", "bf16_scaled"][args.storage],
             "method": name, "ms_per_batch": ms, "spmv_per_s": len(mats) * 1e3 / ms,
             "bytes_per_batch": total_bytes, "gbs": total_bytes / (ms / 1e3) / 1e9,
             "frac_of_peak": total_bytes / (ms / 1e3) / 1e9 / peak}
        if extra:
            d.update(extra)
        print(json.dumps(d), flush=True)

    def separate():
        for m, x, y in zip(mats, xs, ys):
            hb.spmv_device(m, x.data_ptr(), y.data_ptr(), sp)

    report("64 single-matrix launches", _time(separate, stream))
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(stream):
        separate()  # warm (per-device kernel attributes set outside capture)
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=stream):
            for m, x, y in zip(mats, xs, ys):
                hb.spmv_device(m, x.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
    with torch.cuda.stream(stream):  # replay() launches on the current stream
        report("64 single-matrix launches in one CUDA graph", _time(g.replay, stream))
    ref = [y.clone() for y in ys]
    for y in ys:
        y.zero_()
    b = hb.Batch(mats)
    b.bind([x.data_ptr() for x in xs], [y.data_ptr() for y in ys])
    report("batch, concurrent schedule (graph, 16 streams)", _time(lambda: b.run(sp), stream))
    b.set_config(hb.BATCH_QUEUE)
    report("batch, queue schedule (one persistent launch, graph)", _time(lambda: b.run(sp), stream))
    ms_tune, ncand = b.autotune(sp)
    c = b.config()
    ms = _time(lambda: b.run(sp), stream)
    torch.cuda.synchronize()
    same = all(torch.equal(a.view(torch.int64), y.view(torch.int64)) for a, y in zip(ref, ys))
    report("batch, autotuned", ms,
           {"config": {"schedule": ["concurrent", "queue"][c.schedule], "streams": c.streams,
                       "threads": c.threadsPerBlock, "tiles_per_grab": c.tilesPerGrab, "graph": c.useGraph},
            "candidates": ncand, "bit_identical_to_single": same})


def _serve_run(hb, srv, ids, mats_n, kinds, mids, xbuf, ybuf, rate, seed):
    """Submits the request list (kinds[i] on matrix mids[i]) -- all at once
    (rate None: closed loop, the server paused until all are queued) or with
    Poisson arrivals at `rate` requests/s -- and collects them.  Returns
    (wall seconds from first submit to last completion, latencies in seconds,
    SpMV batch widths, worst submit lag behind the arrival schedule)."""
    import threading
    import time
    n_req = len(kinds)
    tickets = [None] * n_req
    ready = threading.Semaphore(0)
    lag = [0.0]

    seq = np.zeros(n_req, np.int64)  # each request's number on its matrix: picks its buffers
    cnt = {}
    for i, m in enumerate(mids):
        seq[i] = cnt.get(m, 0)
        cnt[m] = seq[i] + 1

    def submit_all():
        arrivals = np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, n_req)) if rate else None
        t0 = time.perf_counter()
        for i in range(n_req):
            if arrivals is not None:
                while True:
                    d = arrivals[i] - (time.perf_counter() - t0)
                    if d <= 0:
                        break
                    if d > 2e-4:
                        time.sleep(d - 1e-4)
                lag[0] = max(lag[0], (time.perf_counter() - t0) - arrivals[i])
            m = mids[i]
            x, y = xbuf[m][seq[i] % len(xbuf[m])], ybuf[m][seq[i] % len(ybuf[m])]
            if isinstance(x, np.ndarray):
                tickets[i] = srv.submit(ids[m], kinds[i], x, y)
            else:  # CUDA tensors: a device request
                tickets[i] = srv.submit_device(ids[m], kinds[i], x, y)
            ready.release()

    if rate is None:
        srv.pause(True)
    th = threading.Thread(target=submit_all)
    th.start()
    if rate is None:
        th.join()
        srv.pause(False)
    lat, widths, first, last = [], [], None, 0.0
    for i in range(n_req):
        ready.acquire()
        info = srv.wait(tickets[i])
        if info.status != 0:
            raise RuntimeError(f"request {i} failed with status {info.status}")
        lat.append(info.finished - info.submitted)
        if kinds[i] == hb.REQ_SPMV:
            widths.append(info.batchRhs)
        first = info.submitted if first is None else min(first, info.submitted)
        last = max(last, info.finished)
    th.join()
    return last - first, np.array(lat), np.array(widths), lag[0]


def _latency_summary(hb, kinds, lat, widths):
    is_cg = kinds == hb.REQ_CG
    pct = lambda a, q: 1e3 * float(np.percentile(a, q)) if len(a) else None  # noqa: E731
    return {"p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
            "spmv_p50_ms": pct(lat[~is_cg], 50), "spmv_p99_ms": pct(lat[~is_cg], 99),
            "cg_p50_ms": pct(lat[is_cg], 50), "cg_p99_ms": pct(lat[is_cg], 99),
            "mean_spmv_batch": float(widths.mean()) if len(widths) else None}


def serve_workload(hb, matrices=32, edge_min=32, edge_max=160, seed=5):
    """Config 5's matrices: SPD 27-point stencils of edge U[edge_min,
    edge_max] (numpy default_rng(seed)), each with 0.5 % symmetric
    off-pattern entries (seed 50 + i), converted on the host (blockWidth 32,
    threshold 2)."""
    edges = np.random.default_rng(seed).integers(edge_min, edge_max + 1, matrices)
    mats, ns = [], []
    for i, e in enumerate(edges.tolist()):
        r, c, v = hb.generate_stencil27_spd(e, e, e, 1e-3, 50 + i, extra_fraction=0.005)
        n = e ** 3
        m = hb.HBDIA(r, c, v, n, n)
        del r, c, v
        m.convertToHBDIAFormat(32, 2, upload=False)
        mats.append(m)
        ns.append(n)
    return mats, ns, edges


def served_comparison(requests=10000, capacity_requests=3000, load=0.7, cg_fraction=0.2, matrices=32,
                      edge_min=32, edge_max=160, log=None, served_options=None):
    """Config 5 measured as one comparison, for the benchmark line.

    Workload: serve_workload's 32 resident matrices (150 GB admission cap);
    requests 80 % SpMV / 20 % CG (CG to ||b - A y|| / ||b|| <= 1e-10 on the
    FP64 residual), matrix uniform (default_rng(6)), x / b and y in device
    memory.  Two servers:
      * served: continuous batching of SpMVs into SpMMs, FP32-stored values
        (FP64 accumulation), CG iterating on the FP32 values with FP64
        reliable updates, 4 concurrent solves (served_options override the
        server's defaults, e.g. cgMaxGroup for lockstep CG groups);
      * plain: FP64 values, one request per launch, FP64 CG, one solver.
    Each server's capacity is its closed-loop rate (capacity_requests queued,
    then released); then each takes `requests` Poisson arrivals at `load` x
    its own capacity, and reports the completed rate and p50 / p99 latency
    (completion - submission).  The SpMV-only capacity of both (same
    matrices, no CG) is reported beside it."""
    import time
    import torch
    import hbdia_b200 as hb
    t_start = time.time()
    mats, ns, edges = serve_workload(hb, matrices, edge_min, edge_max)
    rng = np.random.default_rng(6)
    mids = rng.integers(0, len(mats), requests)
    kinds = np.where(rng.random(requests) < cg_fraction, hb.REQ_CG, hb.REQ_SPMV)
    xbuf = [[torch.from_numpy(rng.uniform(-1, 1, n)).cuda() for _ in range(2)] for n in ns]
    ybuf = [[torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(40)] for n in ns]
    servers = {
        "served": hb.Server(**(served_options or {})),
        "plain": hb.Server(batching=0, spmvStorage=hb.STORE_NATIVE, cgIterStorage=hb.STORE_NATIVE,
                           cgWorkers=1, cgMaxGroup=1),
    }
    ids = {k: [s.add_matrix(m) for m in mats] for k, s in servers.items()}
    del mats
    if log:
        log(f"[serve] {len(ns)} matrices, {sum(ns)} rows resident in {time.time() - t_start:.1f}s")
    out = {"workload": f"{len(ns)} SPD 27-point stencils, edge U[{edge_min},{edge_max}] seed 5 "
                       f"(min {int(edges.min())}, max {int(edges.max())}), 0.5% symmetric extras, {int(sum(ns))} rows; "
                       f"{requests} Poisson requests, {cg_fraction:.0%} CG to 1e-10, device vectors",
           "servers": {"served": "continuous batching of the SpMV requests of a matrix into one SpMM; FP32-stored "
                                 "values with FP64 accumulation; CG on the FP32 values with FP64 reliable "
                                 "updates, 4 concurrent solves",
                       "plain": "FP64 values, one request per launch, FP64 CG, one solve at a time"}}
    spmv_only = np.full(capacity_requests, hb.REQ_SPMV)
    for name, srv in servers.items():
        w_k = np.array([hb.REQ_SPMV] * len(ns) + [hb.REQ_CG] * min(4, len(ns)))
        w_m = np.concatenate([np.arange(len(ns)), np.arange(min(4, len(ns)))])
        _serve_run(hb, srv, ids[name], ns, w_k, w_m, xbuf, ybuf, None, 0)  # warm-up
        c0 = srv.stats()
        wall, _, _, _ = _serve_run(hb, srv, ids[name], ns, kinds[:capacity_requests], mids[:capacity_requests],
                                   xbuf, ybuf, None, 0)
        c1 = srv.stats()
        cap = capacity_requests / wall
        wall_s, _, wid_s, _ = _serve_run(hb, srv, ids[name], ns, spmv_only, mids[:capacity_requests], xbuf, ybuf,
                                         None, 0)
        g0 = srv.stats()
        rate = load * cap
        wall, lat, widths, lag = _serve_run(hb, srv, ids[name], ns, kinds, mids, xbuf, ybuf, rate, 7)
        g1 = srv.stats()
        thr = requests / wall
        out[name] = dict(capacity_req_s=cap, offered_req_s=rate, throughput_req_s=thr,
                         saturated=bool(thr < 0.97 * rate), **_latency_summary(hb, kinds, lat, widths),
                         spmv_only_capacity_req_s=capacity_requests / wall_s,
                         spmv_only_mean_batch=float(wid_s.mean()), max_submit_lag_ms=1e3 * lag,
                         mean_cg_group=(g1.cgRequests - g0.cgRequests) / max(1, g1.cgGroups - g0.cgGroups),
                         capacity_mean_cg_group=(c1.cgRequests - c0.cgRequests) / max(1, c1.cgGroups - c0.cgGroups),
                         device_bytes=int(srv.stats().deviceBytes))
        if log:
            log(f"[serve] {name}: capacity {cap:.1f} req/s, {thr:.1f} req/s at {rate:.1f} offered, "
                f"p50 {out[name]['p50_ms']:.2f} ms p99 {out[name]['p99_ms']:.2f} ms")
    for s in servers.values():
        s.close()
    out["capacity_ratio"] = out["served"]["capacity_req_s"] / out["plain"]["capacity_req_s"]
    out["spmv_only_capacity_ratio"] = (out["served"]["spmv_only_capacity_req_s"] /
                                       out["plain"]["spmv_only_capacity_req_s"])
    out["load"] = load
    out["memory_budget_bytes"] = 150 * 10 ** 9
    out["seconds"] = time.time() - t_start
    return out


def serve(args):
    """Config 5: resident matrices, Poisson arrivals, continuous batching.

    32 SPD 27-point stencils of edge U[32, 160] (numpy default_rng(5)), each
    with 0.5 % symmetric off-pattern entries (seed 50 + i), resident in a
    server with a 150 GB admission budget.  Requests: 80 % SpMV, 20 % CG
    (to ||b - A y|| / ||b|| <= 1e-10), matrix uniform (default_rng(6)), x / b
    from a pool of pinned host vectors per matrix (--device: device vectors,
    served in place).  Two servers:
      * batched: continuous batching, FP32-stored values (FP64 accumulation),
        mixed-precision CG (FP32 inner, FP64 refinement), 4 CG solvers;
      * plain: FP64 values, one request per launch, plain FP64 CG, 1 solver.
    (--serial-too adds the batched server with two batches per matrix in flight.)
    Each is first driven closed-loop (all requests queued, then released) to
    measure its capacity; then every server takes the same open-loop Poisson
    arrivals at each of --loads x the batched server's capacity, and reports
    its completed rate beside the offered one (below it: saturated, the queue
    grows over the run) with p50 / p99 latency = completion - submission on
    the server's clock.  Output buffers are picked per request on its matrix
    (results are checked by the tests, not here)."""
    import torch
    import hbdia_b200 as hb
    edges = np.random.default_rng(5).integers(args.edge_min, args.edge_max + 1, args.matrices)
    mats, ns = [], []
    for i, e in enumerate(edges.tolist()):
        r, c, v = hb.generate_stencil27_spd(e, e, e, 1e-3, 50 + i, extra_fraction=0.005)
        n = e ** 3
        m = hb.HBDIA(r, c, v, n, n)
        del r, c, v
        m.convertToHBDIAFormat(32, 2, upload=False)
        mats.append(m)
        ns.append(n)
    rng = np.random.default_rng(6)
    n_req = args.requests
    mids = rng.integers(0, len(mats), n_req)
    kinds = np.where(rng.random(n_req) < args.cg_fraction, hb.REQ_CG, hb.REQ_SPMV)
    pins = []

    def pinned(n, fill):
        t = torch.empty(n, dtype=torch.float64).pin_memory()
        a = t.numpy()
        a[:] = fill(n)
        pins.append(t)
        return a

    if args.device:  # one output per request of a batch: no two writers of one y
        xbuf = [[torch.from_numpy(rng.uniform(-1, 1, n)).cuda() for _ in range(2)] for n in ns]
        ybuf = [[torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(40)] for n in ns]
    else:
        xbuf = [[pinned(n, lambda k: rng.uniform(-1, 1, k)) for _ in range(2)] for n in ns]
        ybuf = [[pinned(n, np.zeros) for _ in range(8)] for n in ns]
    servers = {
        "batched": hb.Server(),
        "plain": hb.Server(batching=0, spmvStorage=hb.STORE_NATIVE, cgIterStorage=hb.STORE_NATIVE,
                           cgWorkers=1, cgMaxGroup=1),
    }
    if args.serial_too:
        servers["batched, 2 batches in flight"] = hb.Server(maxInFlight=2)
    ids = {k: [s.add_matrix(m) for m in mats] for k, s in servers.items()}
    del mats
    rows = int(sum(ns))
    results = {}
    for name, srv in servers.items():
        # warm-up: every matrix once, both kinds
        w_k = np.array([hb.REQ_SPMV] * len(ns) + [hb.REQ_CG] * min(4, len(ns)))
        w_m = np.concatenate([np.arange(len(ns)), np.arange(min(4, len(ns)))])
        _serve_run(hb, srv, ids[name], ns, w_k, w_m, xbuf, ybuf, None, 0)
        wall, lat, widths, _ = _serve_run(hb, srv, ids[name], ns, kinds, mids, xbuf, ybuf, None, 0)
        results[name] = {"capacity_req_s": n_req / wall}
    cap = results["batched"]["capacity_req_s"]
    for load in [float(v) for v in args.loads.split(",")]:
        rate = load * cap
        for name, srv in servers.items():
            wall, lat, widths, lag = _serve_run(hb, srv, ids[name], ns, kinds, mids, xbuf, ybuf, rate, 7)
            st = srv.stats()
            is_cg = kinds == hb.REQ_CG
            thr = n_req / wall
            print(json.dumps({
                "suite": "serve", "server": name, "vectors": "device" if args.device else "pinned host",
                "arrivals": f"Poisson at {rate:.1f} req/s ({load:g} x the batched server's capacity)",
                "workload": f"{len(ns)} SPD 27-point stencils, edge U[{args.edge_min},{args.edge_max}] seed 5, 0.5% "
                            f"symmetric extras, {rows} rows; {n_req} requests, {args.cg_fraction:.0%} CG",
                "offered_req_s": rate, "capacity_req_s": results[name]["capacity_req_s"], "throughput_req_s": thr,
                "saturated": bool(thr < 0.97 * rate),
                "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                "spmv_p50_ms": 1e3 * float(np.percentile(lat[~is_cg], 50)) if (~is_cg).any() else None,
                "spmv_p99_ms": 1e3 * float(np.percentile(lat[~is_cg], 99)) if (~is_cg).any() else None,
                "cg_p50_ms": 1e3 * float(np.percentile(lat[is_cg], 50)) if is_cg.any() else None,
                "cg_p99_ms": 1e3 * float(np.percentile(lat[is_cg], 99)) if is_cg.any() else None,
                "mean_spmv_batch": float(widths.mean()) if len(widths) else None,
                "max_submit_lag_ms": 1e3 * lag, "device_bytes": int(st.deviceBytes),
                "memory_budget_bytes": int(srv.options.memoryBudget)}), flush=True)
    for s in servers.values():
        s.close()


def partition(args):
    """Row-partitioned SpMV, measured part by part on one GPU: the bench
    workload (27-point stencil {grid}^3, 1 % extras, blockWidth 32, threshold 2)
    cut into P row partitions (P = 2, 4, 8), each with its own x-window plan.
    Per rank: the window SpMV (CUDA events), the halo it receives from the
    other ranks (bytes) and the time of the halo-copy kernel that unpacks it
    (the sender's pack copies the same segments).  The step of a P-GPU run is
    then modelled -- not measured, one GPU here -- as the slowest rank's pack +
    unpack + transfer at the measured 770 GB/s per direction per GPU of NVLink
    5 + SpMV, against the whole matrix's SpMV on one GPU."""
    import torch
    import hbdia_b200 as hb
    from hbdia_b200.distributed import _HaloPlan
    g = args.grid if args.grid != 128 else 256
    n = g ** 3
    r, c, v = hb.generate_stencil27(g, g, g, 26.0, -1.0, 0.01, 0.1, 1.0, 1)
    x = torch.from_numpy(hb.fill_uniform(n, -1.0, 1.0, 1)).cuda()
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    whole = hb.HBDIA(r, c, v, n, n)
    whole.convertToHBDIAFormat(32, 2)
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    ms_whole = _time(lambda: hb.spmv_device(whole, x.data_ptr(), y.data_ptr(), sp), stream)
    del whole
    glob = hb.HBDIA(r, c, v, n, n)
    link_gbs = 770.0
    for P in (2, 4, 8):
        ranks = []
        for p in range(P):
            m = glob.partition(P, p)
            m.convertToHBDIAFormat(32, 2)
            w0, wl = m.window()
            win = x[w0:w0 + wl].clone()
            yl = torch.zeros(m.getNumRows(), dtype=torch.float64, device="cuda")
            ms = _time(lambda: hb.spmv_device(m, win.data_ptr(), yl.data_ptr(), sp), stream)
            meta = m.getPartialMatrixMetadata()
            segs = [(s0, e0) for q, rs in enumerate(meta["processDataRanges"]) if q != p for s0, e0 in rs]
            total = sum(e0 - s0 for s0, e0 in segs)
            ms_unpack = 0.0
            if total:
                off = np.cumsum([0] + [e0 - s0 for s0, e0 in segs])[:-1]
                buf = torch.empty(total, dtype=torch.float64, device="cuda")
                unpack = _HaloPlan(off, [s0 - w0 for s0, _ in segs], [e0 - s0 for s0, e0 in segs], total, wl, 8,
                                   torch.device("cuda"))
                with torch.cuda.stream(stream):
                    ms_unpack = _time(lambda: unpack(buf, win), stream)
            ranks.append({"rank": p, "rows": m.getNumRows(), "spmv_ms": ms, "halo_bytes": 8 * total,
                          "halo_segments": len(segs), "unpack_ms": ms_unpack,
                          "window_rows": wl, "spmv_gbs": m.bytesPerSpmv() / ms / 1e6})
            del m, win, yl
        step = max(rk["spmv_ms"] + 2 * rk["unpack_ms"] + rk["halo_bytes"] / (link_gbs * 1e6) for rk in ranks)
        print(json.dumps({"suite": "partition", "workload": f"27-point stencil {g}^3 + 1% extras, bw 32, thr 2",
                          "ranks": P, "whole_matrix_spmv_ms": ms_whole,
                          "max_rank_spmv_ms": max(rk["spmv_ms"] for rk in ranks),
                          "max_halo_bytes": max(rk["halo_bytes"] for rk in ranks),
                          "max_halo_segments": max(rk["halo_segments"] for rk in ranks),
                          "max_unpack_ms": max(rk["unpack_ms"] for rk in ranks),
                          "modelled_step_ms": step, "modelled_speedup": ms_whole / step,
                          "per_rank": ranks}), flush=True)


def convert(args):
    """convertToHBDIAFormat + prepareForGPU on the host (OpenMP, all cores)
    against the GPU converter, on the bench workload (27-point stencil
    256^3, 1 % extras, blockWidth 32, threshold 2); wall-clock seconds from
    the COO arrays to a device layout ready for SpMV."""
    import os
    import time
    import torch
    import hbdia_b200 as hb
    g = args.grid
    n = g ** 3
    r, c, v = hb.generate_stencil27(g, g, g, extra_fraction=0.01, seed=1)
    for name in ("host", "gpu", "gpu"):  # the second GPU run is warm
        m = hb.HBDIA(r, c, v, n, n)
        torch.cuda.synchronize()
        t = time.perf_counter()
        if name == "host":
            m.convertToHBDIAFormat(32, 2)
        else:
            m.convertOnDevice(32, 2)
        m.synchronize()
        dt = time.perf_counter() - t
        print(json.dumps({"suite": "convert", "workload": f"27-point stencil {g}^3 + 1% extras, blockWidth 32, threshold 2",
                          "converter": name, "seconds": dt, "nnz": int(len(v)), "host_threads": os.cpu_count(),
                          "device_bytes": int(m.info().deviceBytes)}), flush=True)
        del m


def spmv(args):
    """The headline workload's shape at --grid (27-point stencil, centre 26,
    neighbours -1, 1 % extras U(0.1, 1) seed 1, blockWidth 32, threshold 2,
    x ~ U(-1, 1) seed 1) with --storage value storage and --kernel: --reps
    SpMVs after 3 warm-up ones, each timed with CUDA events.  With --rhs K > 1
    the same matrix's column-major SpMM of K right-hand sides (X[:, 0] = that
    x, column j ~ U(-1, 1) seed 1 + j; --tile RHS per pass, 0 = default)
    instead; its algorithmic bytes count the values, offsets and COO entries
    once and x, y and the COO x gathers per right-hand side.  The profiles
    capture its launches."""
    import torch
    import hbdia_b200 as hb
    g = args.grid
    n = g ** 3
    rows, cols, vals = hb.generate_stencil27(g, g, g, 26.0, -1.0, 0.01, 0.1, 1.0, 1)
    m = hb.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(32, 2, upload=False)
    m.prepareForGPU(args.storage)
    kern = {"auto": hb.KERNEL_AUTO, "pipe": hb.KERNEL_PIPE, "quad": hb.KERNEL_QUAD, "staged": hb.KERNEL_STAGED,
            "warp": hb.KERNEL_WARP, "rowwise": hb.KERNEL_ROWWISE}[args.kernel]
    m.setKernel(kern)
    x = torch.from_numpy(hb.fill_uniform(n, -1.0, 1.0, 1)).cuda()
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    if args.rhs > 1:
        k = args.rhs
        X = torch.stack([x] + [torch.from_numpy(hb.fill_uniform(n, -1.0, 1.0, 1 + j)).cuda()
                               for j in range(1, k)])  # (k, n): column j contiguous
        Y = torch.zeros((k, n), dtype=torch.float64, device="cuda")
        m.setTuning(hb.TUNE_SPMM_TILE, args.tile)
        ms = _time(lambda: hb.spmm_device_colmajor(m, X.data_ptr(), n, Y.data_ptr(), n, k, stream.cuda_stream),
                   stream, reps=args.reps)
        m.synchronize()
        info = m.info()
        b = m.bytesPerSpmv() + (k - 1) * (16 * n + 8 * info.numCoo)
        print(json.dumps({"suite": "spmm", "workload": f"27-point stencil {g}^3 + 1% extras, column-major",
                          "storage": args.storage, "k": k, "tile": args.tile, "ms": ms, "bytes": b,
                          "gbs": b / (ms / 1e3) / 1e9, "frac_of_peak": b / (ms / 1e3) / 1e9 / _peak()}), flush=True)
        return
    ms = _time(lambda: hb.spmv_device(m, x.data_ptr(), y.data_ptr(), stream.cuda_stream), stream, reps=args.reps)
    m.synchronize()
    b = m.bytesPerSpmv()
    print(json.dumps({"suite": "spmv", "workload": f"27-point stencil {g}^3 + 1% extras", "storage": args.storage,
                      "kernel": args.kernel, "selected": m.selectedKernel(x.data_ptr()), "ms": ms, "bytes": b,
                      "gbs": b / (ms / 1e3) / 1e9, "frac_of_peak": b / (ms / 1e3) / 1e9 / _peak()}), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["precision", "spmm", "cg", "batched", "serve", "convert", "small", "partition",
                                     "spmv"])
    ap.add_argument("--requests", type=int, default=10000)
    ap.add_argument("--matrices", type=int, default=32)
    ap.add_argument("--edge-min", type=int, default=32)
    ap.add_argument("--edge-max", type=int, default=160)
    ap.add_argument("--cg-fraction", type=float, default=0.2)
    ap.add_argument("--loads", default="0.25,0.5,0.7,0.9", help="serve: offered rates, x batched capacity")
    ap.add_argument("--serial-too", action="store_true", help="serve: also the batched server, 1 step in flight")
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--storage", type=int, default=0)
    ap.add_argument("--n", type=int, default=8 * 1024 * 1024)
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--device", action="store_true", help="serve: request vectors in device memory")
    ap.add_argument("--kernel", default="auto", choices=["auto", "pipe", "quad", "staged", "warp", "rowwise"])
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--rhs", type=int, default=1, help="spmv: right-hand sides (> 1: column-major SpMM)")
    ap.add_argument("--tile", type=int, default=0, help="spmv --rhs: right-hand sides per pass (0: default)")
    args = ap.parse_args(argv)
    import torch
    torch.cuda.set_device(0)
    {"precision": precision, "spmm": spmm, "cg": cg, "batched": batched, "serve": serve,
     "convert": convert, "small": small, "partition": partition, "spmv": spmv}[args.what](args)
    return 0


if __name__ == "__main__":
    sys.exit(main())
