#!/usr/bin/env python
"""HBDIA SpMV benchmark (one JSON line on rank 0).

Workload (one GPU): the 27-point stencil on a 256^3 grid (16,777,216 rows,
449,455,096 stencil entries; centre 26.0, neighbours -1.0) plus 1% extra
off-pattern entries with values U(0.1, 1.0) that land in the COO remainder
(seed 1), converted with blockWidth 32 / threshold 2; x ~ U(-1, 1) (seed 1).
A step is one SpMV y = A x.  Inputs are larger than L2 (3.6 GB of values),
so no flush is needed between steps.

value       algorithmic HBM bytes of one SpMV x SpMVs per second (all ranks),
            device-timed with CUDA events, inputs resident in HBM
e2e         the same metric through the C ABI on pinned host buffers, every step
            copying its x host->device and its y device->host: the pipelined
            hbdia_spmv_host_many (one step's upload beside another's download),
            with one hbdia_spmv_host call per step reported beside it
roofline    the fused kernel's achieved algorithmic GB/s over the measured HBM
            copy bandwidth (MEASURED_PEAKS.json)
cpu_baseline the reference's own OpenMP COO SpMV (cpu_coo_spmv_kernel) on the
            same matrix, all host threads, bounded sample
parity      the timed SpMV's y against the reference's cpu_coo_spmv_kernel
            (1e-12 scaled) and the oracle's restated HBDIA SpMV (bit for bit)
served      the serving comparison on 32 resident SPD stencils (edge U[32,160]):
            80 % SpMV / 20 % CG requests, capacity of the served form (FP32
            storage, continuous batching, CG with FP64 reliable updates) and of
            the plain FP64 one-request-per-launch form, then 10,000 Poisson
            requests at 0.7 x each one's capacity with p50 / p99 latency

Multi-GPU (torchrun): replicas only -- every rank holds its own copy of the
matrix and runs its own SpMVs; there is no data-path collective.

--impl reference runs the reference's CPU implementation of the path (its
OpenMP COO SpMV compiled from its sources into oracle/_ref) on this host's
cores, on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(nx=256, ny=256, nz=256, center=26.0, neighbor=-1.0, extra_fraction=0.01,
                extra_lo=0.1, extra_hi=1.0, extra_seed=1, x_seed=1, block_width=32, threshold=2)
METRIC = "SpMV HBM GB/s"
UNIT = "GB/s"
KERNEL_NAMES = {1: "spmv_rowwise<double,double>", 2: "spmv_bw32<double,double>",
                3: "spmv_bw32_xs<double,double> (x window staged by bulk copies)",
                4: "spmv_bw32_pipe<double,double> (persistent, pipelined)",
                5: "spmv_bw32_quad<double,double> (4 blocks per warp)"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """Per-launch DRAM bytes of the SpMV kernel from the committed ncu summary
    (line 'traffic_bytes_per_launch: N')."""
    p = os.path.join(ROOT, "profiles", "spmv_bw32_pipe_fp64_stencil27_256cube.md")
    try:
        with open(p) as f:
            for line in f:
                if line.strip().startswith("traffic_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].strip().split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    def __init__(self, device_index: int, period_s: float = 0.005):
        self.idx, self.period = device_index, period_s
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._t = None
        self._nv = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # no NVML: report nothing rather than guess
            self._nv = None
            log("clock sampling unavailable:", e)
            return self
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _sample(self):
        nv = self._nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwSlowdown", 0x8),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwThermalSlowdown", 0x40),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonSwThermalSlowdown", 0x20),
            "sw_power_cap": getattr(nv, "nvmlClocksThrottleReasonSwPowerCap", 0x4),
            "hw_power_brake_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwPowerBrakeSlowdown", 0x80),
        }
        try:
            self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
            r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
            for k, bit in names.items():
                if r & bit:
                    self.reasons.add(k)
        except Exception:
            pass

    def _run(self):
        while not self._stop.is_set():
            self._sample()
            self._stop.wait(self.period)

    def __exit__(self, *exc):
        # one more sample while the GPU is still warm from the region: the
        # thread competes with the launch loop for the interpreter and may
        # have taken few
        if self._nv is not None:
            self._sample()
        self._stop.set()
        if self._t:
            self._t.join(timeout=2)
        return False

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                "samples": len(self.samples)}


def reduce_max(value: float, dist, device) -> float:
    """Max over ranks of a per-rank time (identity on one rank)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gbs(bytes_per_step: int, steps: int, world: int, max_ms: float) -> float:
    """Whole-job GB/s: every rank ran `steps` SpMVs of `bytes_per_step`; the
    job took the slowest rank's time."""
    return bytes_per_step * steps * world / (max_ms / 1e3) / 1e9


def build_workload(hb, torch, device):
    w = WORKLOAD
    n = w["nx"] * w["ny"] * w["nz"]
    t0 = time.time()
    rows, cols, vals = hb.generate_stencil27(w["nx"], w["ny"], w["nz"], w["center"], w["neighbor"],
                                             w["extra_fraction"], w["extra_lo"], w["extra_hi"], w["extra_seed"])
    t1 = time.time()
    m = hb.HBDIA(rows, cols, vals, n, n)
    m.convertToHBDIAFormat(w["block_width"], w["threshold"])
    t2 = time.time()
    x = hb.fill_uniform(n, -1.0, 1.0, w["x_seed"])
    log(f"[bench] generate {t1 - t0:.1f}s convert+upload {t2 - t1:.1f}s nnz {len(vals)}")
    return m, rows, cols, vals, x, n


def cpu_reference_throughput(rows, cols, vals, n, x, bytes_per_spmv, budget_s, steps=None):
    """The reference's cpu_coo_spmv_kernel (OpenMP, all threads) on the whole
    matrix in row-sorted COO (kind "reference"), or the oracle's scalar port
    on a row range when oracle/_ref is absent (kind "port")."""
    import oracle
    if oracle.Reference.available():
        ref = oracle.Reference()
        coo = ref.cpu_coo(rows, cols, vals)
        y = np.zeros(n)
        coo.spmv(x, n, y)  # warm-up
        times = []
        t_end = time.time() + budget_s
        while (steps is None and (not times or time.time() < t_end)) or (steps is not None and len(times) < steps):
            t = time.perf_counter()
            coo.spmv(x, n, y)
            times.append(time.perf_counter() - t)
        med = statistics.median(times)
        return dict(value=bytes_per_spmv / med / 1e9, unit=UNIT, cores=ref.omp_max_threads(), kind="reference",
                    sample=f"whole {WORKLOAD['nx']}^3 matrix ({len(vals)} COO entries), {len(times)} SpMVs, median",
                    spmv_per_s=1.0 / med, ms_per_spmv=med * 1e3), y
    orc = oracle.Restated()
    # scalar port on the first rows (about 1/64 of the matrix), scaled by entries
    cut = int(np.searchsorted(rows, n // 64))
    y = np.zeros(n)
    t = time.perf_counter()
    orc.coo_spmv(rows[:cut], cols[:cut], vals[:cut], x, n, y)
    dt = (time.perf_counter() - t) * len(vals) / max(cut, 1)
    return dict(value=bytes_per_spmv / dt / 1e9, unit=UNIT, cores=1, kind="port",
                sample=f"rows 0..{n // 64} ({cut} entries) of the 256^3 matrix, scaled by entries",
                spmv_per_s=1.0 / dt, ms_per_spmv=dt * 1e3), None


def parity_report(rows, cols, vals, n, x, y_gpu, y_ref_coo, full_oracle=True):
    """The GPU y of the timed SpMV against (1) the reference's own
    cpu_coo_spmv_kernel over the whole matrix in row-sorted COO (a different
    summation order: bounded by 1e-12 * sum_j |a_ij x_j| per row), and (2) the
    oracle's restated HBDIA SpMV on its own conversion (same order: bit for
    bit).  Outside every timed region."""
    out = {"tolerance": "|y - y_ref| <= 1e-12 * sum_j |a_ij x_j| per row"}
    absrow = np.bincount(rows, weights=np.abs(vals * x[cols]), minlength=n)
    scale = np.maximum(absrow, np.finfo(np.float64).tiny)
    if y_ref_coo is not None:
        err = np.abs(y_gpu - y_ref_coo) / scale
        out["reference_cpu_coo"] = {
            "oracle": "the reference's cpu_coo_spmv_kernel (oracle/_ref), whole matrix in row-sorted COO",
            "max_scaled_err": float(err.max()), "bitexact_frac": float(np.mean(y_gpu == y_ref_coo)),
            "pass": bool(err.max() <= 1e-12)}
    if full_oracle:
        import oracle
        t = time.time()
        om = oracle.Restated().convert(rows, cols, vals, n, n, WORKLOAD["block_width"], WORKLOAD["threshold"])
        y_orc = om.spmv(x)
        del om
        same = y_gpu.view(np.uint64) == y_orc.view(np.uint64)
        out["oracle_hbdia"] = {
            "oracle": "oracle/hbdia_oracle.c: convertToHBDIAFormat + hbdiaSpMV restated, same operation order",
            "bitexact_frac": float(np.mean(same)), "max_scaled_err": float((np.abs(y_gpu - y_orc) / scale).max()),
            "pass": bool(same.all()), "seconds": time.time() - t}
    out["pass"] = all(v["pass"] for v in out.values() if isinstance(v, dict))
    return out


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    # Everything here is the reference's code (oracle/_ref) or the oracle's
    # restatement (oracle/hbdia_oracle.c): the product library is not loaded.
    import oracle
    w = WORKLOAD
    n = w["nx"] * w["ny"] * w["nz"]
    orc = oracle.Restated()
    rows, cols, vals = orc.workload_stencil27(w["nx"], w["ny"], w["nz"], w["center"], w["neighbor"],
                                              w["extra_fraction"], w["extra_lo"], w["extra_hi"], w["extra_seed"])
    x = orc.fill_uniform(n, -1.0, 1.0, w["x_seed"])
    L = orc.convert(rows, cols, vals, n, n, w["block_width"], w["threshold"]).layout()
    bytes_per_spmv = bytes_model(n, len(L.data), len(L.offsets), L.num_blocks, len(L.coo_row))
    del L
    if not oracle.Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhbdia_ref.so was not built"}))
        return 0
    ref = oracle.Reference()
    coo = ref.cpu_coo(rows, cols, vals)
    y = np.zeros(n)
    t = time.perf_counter()
    coo.spmv(x, n, y)
    t_full = time.perf_counter() - t
    # each step: the reference's COO SpMV over a contiguous row range sized so
    # the whole run stays within about a minute
    target = max(0.002, 60.0 / max(1, args.steps + args.warmup))
    frac = min(1.0, target / t_full)
    r1 = max(1, int(n * frac))
    cut = int(np.searchsorted(rows, r1))
    sub = ref.cpu_coo(rows[:cut], cols[:cut], vals[:cut])
    ysub = np.zeros(r1)
    for _ in range(args.warmup):
        sub.spmv(x, r1, ysub)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        sub.spmv(x, r1, ysub)
        times.append(time.perf_counter() - t)
    total = sum(times)
    sample_frac = cut / len(vals)
    value = bytes_per_spmv * sample_frac * args.steps / total / 1e9
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": dict(workload_config(), parallelism="replicas1"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.omp_max_threads(), "kind": "reference",
                         "sample": f"rows 0..{r1} of the 256^3 matrix ({cut} of {len(vals)} entries) per step; "
                                   f"value scaled to whole-matrix SpMV bytes by entries"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "full_matrix_ms": t_full * 1e3,
    }
    print(json.dumps(out))
    return 0


def bytes_model(n, slots, total_offsets, num_blocks, num_coo):
    """Algorithmic bytes of one plain-FP64 SpMV over the HBDIA layout (bw 32
    kernel): values 8*slots + offsets 4*totalOffsets + block pointers
    4*(numBlocks+1) + x read once 8n + y written once 8n + COO (row, col, value)
    16*nCoo + one x gather per COO entry 8*nCoo + COO tile pointers 4*(n/32+1)."""
    b = 8 * slots + 4 * total_offsets + 4 * (num_blocks + 1) + 16 * n + 24 * num_coo
    if num_coo:
        b += 4 * ((n + 31) // 32 + 1)
    return b


def hbm_bytes_model(i):
    return bytes_model(i.numRows, i.numSlots, i.totalOffsets, i.numBlocks, i.numCoo)


def workload_config():
    w = WORKLOAD
    return {"workload": f"27-point stencil {w['nx']}^3 + 1% COO extras, FP64, blockWidth 32, threshold 2",
            "rows": w["nx"] * w["ny"] * w["nz"], "block_width": w["block_width"], "threshold": w["threshold"],
            "extra_fraction": w["extra_fraction"], "seeds": {"extras": w["extra_seed"], "x": w["x_seed"]},
            "l2": "inputs larger than L2 (3.6 GB of values, 134 MB x); no flush"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="hbdia", choices=["hbdia", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the full-size parity check against the oracles")
    ap.add_argument("--no-serve", action="store_true", help="skip the served comparison (config 5)")
    ap.add_argument("--serve-requests", type=int, default=10000, help="Poisson requests per server (config 5)")
    ap.add_argument("--unroll", type=int, default=0, choices=[0, 9, 27],
                    help="offsets in flight per lane in the staged kernel (0: default)")
    ap.add_argument("--kernel", default=None, choices=["pipe", "quad", "staged", "warp", "rowwise"],
                    help="force one SpMV kernel (default: the library's choice)")
    ap.add_argument("--size", type=int, default=256,
                    help="grid edge of the stencil workload (256 is the benchmark; smaller sizes for profiling)")
    args = ap.parse_args()
    if args.size != 256:
        WORKLOAD.update(nx=args.size, ny=args.size, nz=args.size)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import hbdia_b200 as hb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    hb.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    m, rows, cols, vals, x, n = build_workload(hb, torch, local)
    info = m.info()
    bytes_per_spmv = hbm_bytes_model(info)
    assert bytes_per_spmv == info.bytesPerSpmv, (bytes_per_spmv, info.bytesPerSpmv)
    if args.kernel:
        m.setKernel({"pipe": hb.KERNEL_PIPE, "quad": hb.KERNEL_QUAD, "staged": hb.KERNEL_STAGED, "warp": hb.KERNEL_WARP,
                     "rowwise": hb.KERNEL_ROWWISE}[args.kernel])
    if args.unroll:
        m.setTuning(hb.TUNE_UNROLL, args.unroll)
    xt = torch.from_numpy(x).cuda()
    kernel_used = m.selectedKernel(xt.data_ptr())
    yt = torch.zeros(n, dtype=torch.float64, device="cuda")
    # a dedicated stream: the kernels and every timing event live on it
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    sp = stream.cuda_stream

    for _ in range(args.warmup):
        hb.spmv_device(m, xt.data_ptr(), yt.data_ptr(), sp)
    torch.cuda.synchronize()

    # timed region: K SpMVs, one event pair around each launch (the kernel's
    # own duration for the roofline) and one around all of them
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    t_all0, t_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_all0.record(stream)
        for k in range(args.steps):
            evs[k][0].record(stream)
            hb.spmv_device(m, xt.data_ptr(), yt.data_ptr(), sp)
            evs[k][1].record(stream)
        t_all1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = t_all0.elapsed_time(t_all1)
    launch_ms = [a.elapsed_time(b) for a, b in evs]
    m.synchronize()  # raises if a bounded device-side wait ran out
    total_ms = reduce_max(total_ms, dist, "cuda")
    value = aggregate_gbs(bytes_per_spmv, args.steps, world, total_ms)
    avg_launch_ms = sum(launch_ms) / len(launch_ms)
    achieved = bytes_per_spmv / (avg_launch_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()

    # end to end through the C ABI with pinned host buffers.  (1) one call per
    # step (hbdia_spmv_host: x in, SpMV, y out, synchronize); (2) the
    # pipelined form (hbdia_spmv_host_many over the same steps: every step
    # still copies its own x in and its y out, but one step's upload runs
    # beside another's download).  Both calls are synchronous: wall time
    # around them, max over ranks.
    xh = torch.from_numpy(x).pin_memory()
    yh = torch.zeros(n, dtype=torch.float64).pin_memory()
    xh_np, yh_np = xh.numpy(), yh.numpy()
    hb.spmv_host(m, xh_np, yh_np)  # warm (allocates the scratch buffers)
    ms = torch.cuda.ExternalStream(m.getBDIAStream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    e0.record(ms)
    for _ in range(args.e2e_steps):
        hb.spmv_host(m, xh_np, yh_np)
    e1.record(ms)
    e1.synchronize()
    single_ms = reduce_max(e0.elapsed_time(e1), dist, "cuda")
    single_value = aggregate_gbs(bytes_per_spmv, args.e2e_steps, world, single_ms)
    ok = bool(np.array_equal(yh_np.view(np.uint64), yt.cpu().numpy().view(np.uint64)))
    ypin = [torch.zeros(n, dtype=torch.float64).pin_memory() for _ in range(3)]
    ys = [t.numpy() for t in ypin]
    hb.spmv_host_many(m, [xh_np] * 3, ys)  # warm (allocates the pipeline's staging pairs)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    hb.spmv_host_many(m, [xh_np] * args.e2e_steps, [ys[j % 3] for j in range(args.e2e_steps)])
    e2e_ms = reduce_max(1e3 * (time.perf_counter() - t0), dist, "cuda")
    e2e_value = aggregate_gbs(bytes_per_spmv, args.e2e_steps, world, e2e_ms)
    # the e2e results must be the device result
    ref_y = yt.cpu().numpy().view(np.uint64)
    ok = ok and all(np.array_equal(y.view(np.uint64), ref_y) for y in ys)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, y_ref = cpu_reference_throughput(rows, cols, vals, n, x, bytes_per_spmv, args.cpu_budget)
        if not args.no_parity:
            parity = parity_report(rows, cols, vals, n, x, yt.cpu().numpy(), y_ref)

    served = None
    if rank == 0 and world == 1 and not args.no_serve:
        from hbdia_b200 import suite
        del m  # the headline matrix's device layout is not needed any more
        torch.cuda.empty_cache()
        served = suite.served_comparison(requests=args.serve_requests,
                                         capacity_requests=min(3000, args.serve_requests), log=log)

    if rank == 0:
        cs = clk.summary()
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(), parallelism=f"replicas{world}"),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic(), "peak_source": peak_kind,
                         "traffic_source": "ncu dram__bytes_read+write of one 128^3 launch of the same kernel, "
                                           "scaled to 256^3 by the byte model (profiles/)",
                         "kernel": KERNEL_NAMES[kernel_used], "bytes_per_launch": bytes_per_spmv,
                         "avg_launch_ms": avg_launch_ms},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
                    "steps": args.e2e_steps, "ms_per_step": e2e_ms / args.e2e_steps, "matches_device": ok,
                    "api": "hbdia_spmv_host_many (3-deep pipeline, pinned host x / y)",
                    "single_call": {"api": "hbdia_spmv_host per step", "value": single_value,
                                    "ms_per_step": single_ms / args.e2e_steps}},
            "cpu_baseline": cpu,
            "parity": parity,
            "served": served,
            "gpu_launches": args.steps,
            "clocks": cs,
            "spmv_per_s": 1e3 * args.steps * world / total_ms,
            "gflops": 2.0 * info.numNonZeros * args.steps * world / (total_ms / 1e3) / 1e9,
        }
        print(json.dumps(out))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
