#!/usr/bin/env python
"""Benchmark: KIFMM3d evaluate() throughput on one B200 (and N replicas).

Workload (the configuration the metric is quoted on): Laplace single layer,
N = 1,048,576 points (50% on a sphere of radius 0.49 about the box centre,
50% in 8 Gaussian clusters, sigma 0.02), sources = targets, densities N(0,1),
np = 6, ptsMax = 64, seeded synthetic data.  One step = one evaluate() of one
right-hand side with the tree, lists and operators resident (the reference's
-do_2nd_eval semantics).  value = targets / s of the device-timed step;
e2e = the same metric through fmmg_evaluate() with pinned host buffers, the
H2D copy of the densities and the D2H copy of the values inside the timing.

--gpus N (under torchrun): every rank holds a replica of the tree and
evaluates its own right-hand side (multi-RHS sharding, weak scaling, no
collective on the data path); the step time is the max over ranks.

--impl reference: the CPU restatement of the reference evaluate() (oracle/),
timed on the host cores with all threads, on the same 1,048,576-point workload
(one evaluate per step, tree and operators prebuilt).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "fmm-g_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "Laplace 1M-pt points/s, mixed vs FP64 GPU at rel err\u22641e-5; adjoint/fwd time"
UNIT = "points/s"
WORKLOAD = "laplace_s_1M_sphere_clusters_np6_ptsmax64"
CHECK_TARGETS = 4096
WORKLOADS = ("laplace_1m", "stokes_dl_ellipsoids_1m", "laplace_adjoint_4m", "navier_np8_2m")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--precision", default="all", choices=["fp64", "all"])
    ap.add_argument("--k", type=int, default=8, help="right-hand sides of the multi-RHS mixed form")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--only", default=None, choices=["fp64", "mixed1", "mixedk"],
                    help="time one form only (profiling runs); the headline then comes from it")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint timing")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--workload", default="laplace_1m", choices=list(WORKLOADS),
                    help="laplace_1m: the headline line (the default); the others print one line for the other "
                         "configurations at their stated sizes")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi samples of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def oracle_rate(n, nthreads, reps=1):
    """Oracle (CPU restatement of the reference evaluate) points/s on the
    n-point benchmark workload."""
    import oracle as O
    import workloads as W
    cfg = W.config2(n)
    src, den = cfg["src"], cfg["den"]
    o = O.Oracle(111, np_=6, pts_max=64, nthreads=nthreads)
    o.setup(src, src, src)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        o.evaluate(den)
        times.append(time.perf_counter() - t0)
    return n / float(np.median(times)), times


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    import oracle as O
    import workloads as W
    cfg = W.config2(args.n)  # the benchmark workload itself, full size
    n = args.n
    src, den = cfg["src"], cfg["den"]
    o = O.Oracle(111, np_=6, pts_max=64, nthreads=nthreads)
    o.setup(src, src, src)
    for _ in range(args.warmup):
        o.evaluate(den)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.evaluate(den)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    v = n / dt
    sample = "the full %d-point workload, one evaluate per step, tree and operators prebuilt" % n
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "points": n, "kernel": "laplace_s_u", "np": 6, "pts_max": 64,
                   "k_rhs_per_gpu": 1, "precision": "fp64", "parallelism": "host threads x%d" % nthreads},
        "cpu_baseline": dict({"value": v, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample},
                             **host_cpu()),
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


_PEAKS = {}


def host_cpu():
    """The host CPU model and the threads this process may use."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count() or 1}


def measure_peak(torch, kind):
    """cuBLAS GEMM 8192^3 best of 3 (TFLOP/s) in FP64 or FP32 (TF32 off): the
    roof for the CUDA-core kernels, which MEASURED_PEAKS.json does not hold.
    Measured once per process."""
    if kind in _PEAKS:
        return _PEAKS[kind]
    torch.backends.cuda.matmul.allow_tf32 = False
    dt = torch.float64 if kind == "fp64" else torch.float32
    a = torch.randn(8192, 8192, dtype=dt, device="cuda")
    b = torch.randn(8192, 8192, dtype=dt, device="cuda")
    best = 1e30
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    _PEAKS[kind] = 2 * 8192 ** 3 / (best * 1e-3) / 1e12
    return _PEAKS[kind]


def stage_rooflines(f, kern, torch, k, precision):
    """Every stage of one step against the roof that bounds it: the pair sums
    and GEMMs in FLOP/s of the FP32 (FP64) pipe, the spectral transforms in
    bytes/s of HBM, with the pair rate of the pair sums."""
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    work = f.algorithmic_work(k=k, precision="fp64" if precision == "fp64" else "fp32")
    out = {}
    for name, ms in kern.items():
        w = work.get(name)
        if w is None or ms <= 0:
            continue
        t = ms * 1e-3
        if w["bound"] == "hbm":
            ach = w["bytes"] / t / 1e9
            out[name] = {"ms": ms, "bound": "hbm", "achieved": ach, "unit": "GB/s", "frac": ach / hbm_peak}
        else:
            peak = measure_peak(torch, w["bound"])
            ach = w["flops"] / t / 1e12
            out[name] = {"ms": ms, "bound": w["bound"], "achieved": ach, "unit": "TFLOP/s", "frac": ach / peak}
            if w.get("pairs"):
                out[name]["pairs_per_s"] = k * w["pairs"] / t
    return out


def time_form(f, torch, stream, den_dev, out_dev, n, k, prec, steps, warmup, flush, barrier=None):
    """Device time per step of one evaluate form, replayed as a CUDA graph
    (eager first call, captured second call, replays after); then one eager
    step with per-kernel events for the breakdown (not part of the timing).
    With several ranks, barrier() brackets the timed steps."""
    f.set_timing(False)
    f.set_graph(True)
    for _ in range(max(warmup, 3)):
        f.evaluate_device(den_dev, out_dev, k, prec)
    torch.cuda.synchronize()
    graph_active, graph_note = f.graph_state()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if barrier:
        barrier()
    torch.cuda.synchronize()
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        f.evaluate_device(den_dev, out_dev, k, prec)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    if barrier:
        barrier()
    launches = f.launch_count() * steps
    ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    f.set_graph(False)
    f.set_timing(True)
    flush.zero_()
    f.evaluate_device(den_dev, out_dev, k, prec)
    kern = f.kernel_times()
    stage = f.stage_times()
    f.set_timing(False)
    return ms, kern, stage, launches, {"graph": graph_active, "note": graph_note}


def time_adjoint(f, torch, stream, den_dev, out_dev, n, steps, warmup, flush):
    """FP64 transposed FMM (d/d density of <w, A sigma>) and the Laplace
    target-position gradient, device time per step, with w = the first values."""
    w = out_dev[0].contiguous()
    g = torch.empty(n, dtype=torch.float64, device="cuda")
    gt = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    res = {}
    f.set_timing(False)  # no host synchronisation inside the timed calls
    for key, call in (("ms_per_step", lambda: f.adjoint_device(None, w, g, None)),
                      ("target_grad_ms_per_step", lambda: f.adjoint_device(den_dev[0], w, None, gt))):
        for _ in range(max(warmup, 3)):
            call()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for i in range(steps):
            flush.zero_()
            ev[i][0].record(stream)
            call()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        res[key] = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    res["launches"] = f.launch_count()
    return res


def run_ours(args):
    import torch
    import fmmg
    import fmmg_dist as FD
    import workloads as W
    ws, rank, local = dist_env()
    dist = ws > 1
    if dist:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    stream = torch.cuda.Stream()  # one stream for the flush, the events and every library kernel
    torch.cuda.set_stream(stream)
    cfg = W.config2(args.n)
    src = cfg["src"]
    n = args.n
    K = args.k
    rng = np.random.default_rng(W.SEED + 2 + 1000 * rank)
    dens = np.stack([cfg["den"] if (rank == 0 and r == 0) else rng.normal(size=n) for r in range(K)])
    t0 = time.perf_counter()
    f = fmmg.FMM3d(111, np_=6, pts_max=64, device=dev, stream=stream.cuda_stream)
    f.setup(src)
    setup_s = time.perf_counter() - t0
    info = f.info()
    den = torch.from_numpy(dens).to("cuda")
    out = torch.zeros(K, n, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2
    idx = np.random.default_rng(W.SEED + 99).choice(n, CHECK_TARGETS, replace=False)
    forms = [("fp64", fmmg.PREC_FP64, 1), ("mixed", fmmg.PREC_MIXED, 1), ("mixed", fmmg.PREC_MIXED, K)]
    if args.precision == "fp64":
        forms = forms[:1]
    if args.only:
        forms = [forms[["fp64", "mixed1", "mixedk"].index(args.only)]]
    elif K > 1 and args.precision != "fp64":
        forms.append(("fp64", fmmg.PREC_FP64, K))  # the FP64 form at equal k
    results = []
    if dist:
        tdist.barrier()
    clocks = ClockSampler(dev if not os.environ.get("CUDA_VISIBLE_DEVICES") else
                          os.environ["CUDA_VISIBLE_DEVICES"].split(",")[dev])
    clocks.start()
    for name, prec, k in forms:
        tuned = None
        if not args.no_autotune:  # launch shapes for this (kernel, np, k, precision), timed on this GPU
            _, tuned = f.autotune(den, out, k, prec, reps=2)
        ms, kern, stage, launches, graph = time_form(f, torch, stream, den, out, n, k, prec, args.steps, args.warmup,
                                                     flush, barrier=tdist.barrier if dist else None)
        if dist:
            ms = FD.max_over_ranks(ms, device="cuda")
        # every right-hand side of the block against the dense sum; the form's
        # error is the worst of them
        vals = out[:k].cpu().numpy()
        checks = [f.check(dens[r], vals[r], idx) for r in range(k)]
        rel = max(c[0] for c in checks)
        mx = max(c[1] for c in checks)
        results.append(dict(precision=name, k=k, ms_per_step=ms, points_per_s=n * k * ws / (ms * 1e-3),
                            rel_err_vs_dense=rel, rel_err_per_rhs=[c[0] for c in checks],
                            max_abs_err_vs_dense=mx, kernel_ms=kern,
                            stage_ms=stage, launches=launches, cuda_graph=graph, tuning=tuned))
    adj = {} if args.no_adjoint else time_adjoint(f, torch, stream, den, out, n, args.steps, args.warmup, flush)
    if dist and adj:
        adj["ms_per_step"] = FD.max_over_ranks(adj["ms_per_step"], device="cuda")
        adj["target_grad_ms_per_step"] = FD.max_over_ranks(adj["target_grad_ms_per_step"], device="cuda")
    clk = clocks.stop()
    fp64 = next((r for r in results if r["precision"] == "fp64" and r["k"] == 1), None)
    fp64_ms = [r["ms_per_step"] for r in results if r["precision"] == "fp64" and r["k"] == 1]
    if adj and fp64_ms:
        adj["ratio_vs_fp64_forward"] = adj["ms_per_step"] / fp64_ms[0]
    ok = [r for r in results if r["rel_err_vs_dense"] <= 1e-5]
    head = max(ok, key=lambda r: r["points_per_s"]) if ok else (fp64 or results[0])
    prec_h = fmmg.PREC_FP64 if head["precision"] == "fp64" else fmmg.PREC_MIXED
    kh = head["k"]
    # end to end through fmmg_evaluate_host: pinned host densities in, pinned values out
    hin = torch.from_numpy(dens[:kh].copy()).pin_memory()
    hout = torch.zeros(kh, n, dtype=torch.float64).pin_memory()
    f.evaluate_host_k(hin.data_ptr(), hout.data_ptr(), kh, prec_h)
    e2e_ms = []
    for _ in range(args.steps):
        s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        s_.record(stream)
        f.evaluate_host_k(hin.data_ptr(), hout.data_ptr(), kh, prec_h)
        e_.record(stream)
        e_.synchronize()
        e2e_ms.append(s_.elapsed_time(e_))
    e2e = float(np.mean(e2e_ms))
    if dist:
        e2e = FD.max_over_ranks(e2e, device="cuda")
        tdist.barrier()
    if rank == 0:
        roof = roofline(f, head["kernel_ms"], torch, kh, head["precision"])
        # the same handle set up again (what a caller with moving points pays
        # per evaluation): after every timed and reported use of the handle
        try:  # median of three repeated setups (one-off host stalls are not the setup's cost)
            ts = []
            for _ in range(3):
                t0 = time.perf_counter()
                f.setup(src)
                ts.append(time.perf_counter() - t0)
            setup_again_s = float(np.median(ts))
        except fmmg.FmmgError as e:  # reported, never at the cost of the line
            setup_again_s = None
            print("setup again failed: %s" % e, file=sys.stderr)
        cpu = None
        if not args.no_cpu_baseline and not dist:
            nthr = os.cpu_count() or 1
            rate, times = oracle_rate(n, nthr)
            cpu = dict({"value": rate, "unit": UNIT, "cores": nthr, "kind": "port",
                        "sample": "the full %d-point workload, one evaluate on %d host threads (one MPI rank, "
                                  "OpenMP), tree/operators prebuilt, %.1f s" % (n, nthr, times[0])}, **host_cpu())
        line = {
            "metric": METRIC, "value": head["points_per_s"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec_h == fmmg.PREC_FP64 else "f32+f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "points": n, "kernel": "laplace_s_u", "np": 6, "pts_max": 64,
                       "k_rhs_per_gpu": kh, "precision": head["precision"],
                       "parallelism": "rhs-replicas x%d" % ws,
                       "l2": "256 MB written between steps; per-step working set > L2",
                       "nodes": info["nodes"], "leaves": info["leaves"], "max_depth": info["max_depth"]},
            "e2e": {"value": n * kh * ws / (e2e * 1e-3), "unit": UNIT, "h2d_bytes_per_step": 8 * n * kh,
                    "d2h_bytes_per_step": 8 * n * kh},
            "gpu_launches": head["launches"],
            "rel_err_vs_dense": head["rel_err_vs_dense"], "check_targets": CHECK_TARGETS,
            "rel_err_checked": "worst of every right-hand side of the block, at the same sampled targets",
            "fp64_points_per_s": fp64["points_per_s"] if fp64 else None,
            "speedup_vs_fp64": head["points_per_s"] / fp64["points_per_s"] if fp64 else None,
            "speedups": speedups(results),
            "stage_roofline": stage_rooflines(f, head["kernel_ms"], torch, kh, head["precision"]),
            "forms": results, "adjoint": adj, "setup_s": setup_s, "setup_again_s": setup_again_s,
            "roofline": roof, "clocks": clk,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line))
    f.close()
    if dist:
        tdist.destroy_process_group()


# DRAM traffic of the dominant kernels from one ncu capture each (dram__bytes_read.sum +
# dram__bytes_write.sum) on the 262,144-point case of this workload, with the
# algorithmic bytes of that launch; a full launch's traffic is scaled by the
# algorithmic bytes (the units processed).  Summaries under profiles/.
TRAFFIC = {
    ("m2l_had", "mixed", 8): {"dram_bytes": 859.948800e6 + 571.790592e6, "algorithmic_bytes": 1209899328,
                               "profile": "profiles/k_m2l_had_o4_laplace_sphere_clusters_262k_np6_k8.md"},
    ("m2l_had", "fp64", 1): {"dram_bytes": 253.321472e6 + 175.060480e6, "algorithmic_bytes": 424424448,
                              "profile": "profiles/k_m2l_had_pq_fp64_laplace_sphere_clusters_262k_np6.md"},
}


def roofline(f, kern, torch, k, precision):
    """Roofline of the dominant kernel class of the headline step."""
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    top = max((name for name in kern if name not in ("prep", "scatter")), key=lambda name: kern[name])
    t = kern[top] * 1e-3
    w = f.algorithmic_work(k=k, precision="fp64" if precision == "fp64" else "fp32").get(top)
    out = {"kernel": top, "avg_ms": kern[top], "k_rhs": k}
    if w is None:
        out.update({"bound": None, "achieved": None, "peak": None, "unit": None, "frac": None, "traffic": None})
        return out
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    if w["bound"] == "hbm":
        ach = w["bytes"] / t / 1e9
        out.update({"bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s", "frac": ach / hbm_peak,
                    "peak_source": "of measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks
                    else "of fallback 6650 GB/s", "algorithmic_bytes": w["bytes"]})
    else:
        fp = w["bound"]
        peak = measure_peak(torch, fp)
        ach = w["flops"] / t / 1e12
        out.update({"bound": fp, "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                    "peak_source": "of measured in bench.py: cuBLAS %s GEMM 8192^3, best of 3 (CUDA cores; "
                                   "MEASURED_PEAKS.json holds HBM and BF16 only)" % fp,
                    "algorithmic_flops": w["flops"], "pairs": w.get("pairs")})
        if "bytes" in w:
            out["hbm"] = {"algorithmic_bytes": w["bytes"], "achieved_gbs": w["bytes"] / t / 1e9,
                          "peak_gbs": hbm_peak, "frac": w["bytes"] / t / 1e9 / hbm_peak}
    tr = TRAFFIC.get((top, "fp64" if precision == "fp64" else "mixed", k))
    if tr and "bytes" in w:
        out["traffic"] = tr["dram_bytes"] / tr["algorithmic_bytes"] * w["bytes"]
        out["traffic_source"] = "ncu on the 262,144-point case, scaled by algorithmic bytes; " + tr["profile"]
    else:
        out["traffic"] = None
    return out


def speedups(results):
    """points/s ratios of the mixed form to the FP64 form: the headline block
    of k against FP64 at k = 1, at equal k, and k = 1 against k = 1."""
    pts = {(r["precision"], r["k"]): r["points_per_s"] for r in results}
    out = {}
    for (p, k), v in pts.items():
        if p != "mixed":
            continue
        if ("fp64", 1) in pts:
            out["mixed_k%d_vs_fp64_k1" % k] = v / pts[("fp64", 1)]
        if k > 1 and ("fp64", k) in pts:
            out["mixed_k%d_vs_fp64_k%d" % (k, k)] = v / pts[("fp64", k)]
    return out


def time_calls(torch, stream, call, steps, warmup, flush):
    """Mean device time (CUDA events on the launching stream) of call() over
    steps calls, after warmup untimed calls, with L2 flushed before each."""
    for _ in range(warmup):
        call()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        flush.zero_()
        ev[i][0].record(stream)
        call()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    return float(np.mean([a.elapsed_time(b) for a, b in ev]))


def dense_laplace_grads(src, den, w, chunk=1024):
    """FP64 dense sums on the GPU for the Laplace single layer, sources = targets
    = src ([n, 3]), right-hand sides den and weights w ([k, n]): per right-hand
    side the density gradient of <w, phi> (K^T w) and the target-position
    gradient w(t) grad_t phi(t) (r = 0 pairs add nothing, as the kernel)."""
    import torch
    x = torch.from_numpy(src).cuda()
    sig = torch.from_numpy(den).cuda()
    ww = torch.from_numpy(w).cuda()
    k, n = sig.shape
    gden = torch.zeros(k, n, dtype=torch.float64, device="cuda")
    gpos = torch.zeros(k, n, 3, dtype=torch.float64, device="cuda")
    c = 1.0 / (4.0 * np.pi)
    for t0 in range(0, n, chunk):
        d = x[t0:t0 + chunk, None, :] - x[None, :, :]  # [c, n, 3]
        r2 = (d * d).sum(-1)
        bad = r2 < 1e-16
        ir = torch.where(bad, torch.zeros_like(r2), r2.clamp_min(1e-300).rsqrt())
        K = c * ir                                 # K(t, s)
        gden += ww[:, t0:t0 + chunk] @ K           # sum_t w(t) K(t, s)
        G = -c * (ir ** 3)[..., None] * d          # grad_t K(t, s)
        gpos[:, t0:t0 + chunk, :] = torch.einsum("tsd,ks->ktd", G, sig) * ww[:, t0:t0 + chunk, None]
    return gden.cpu().numpy(), gpos.cpu().numpy()


def run_workload(args):
    """The other configurations at their stated sizes, one JSON line each:
    stokes_dl_ellipsoids_1m -- Stokes double layer, 1,048,576 points on 64
      ellipsoids, np=6, the mixed form on 8 right-hand sides;
    navier_np8_2m -- Navier single layer, 2,097,152 points (uniform + shell),
      np=8, the mixed form on 32 right-hand sides, autotuned, graph replays;
    laplace_adjoint_4m -- Laplace single layer, 4,194,304 uniform points, np=6,
      16 right-hand sides: forward and adjoint (density and target-position
      gradients of <w, phi>) times at the same precision and k, central
      differences (h = 1e-4) at 64 random target coordinates, and the dense FP64
      gradients on a 32,768-point subset problem."""
    import torch
    import fmmg
    import workloads as W
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    line = {"workload": args.workload, "unit": UNIT, "data": "synthetic", "steps": args.steps, "warmup": args.warmup,
            "l2": "256 MB written between timed steps"}
    clocks = ClockSampler(0)
    if args.workload in ("stokes_dl_ellipsoids_1m", "navier_np8_2m"):
        cfg = W.config3() if args.workload.startswith("stokes") else W.config5()
        n, k = cfg["src"].shape[0], cfg["den"].shape[0]
        t0 = time.perf_counter()
        f = fmmg.FMM3d(cfg["kernel"], np_=cfg["np"], pts_max=cfg["pts_max"], coefs=cfg.get("coefs", (1.0, 0.25)),
                       device=0, stream=stream.cuda_stream)
        f.setup(cfg["src"], cfg["nrm"])
        setup_s = time.perf_counter() - t0
        den = torch.from_numpy(np.ascontiguousarray(cfg["den"])).cuda()
        out = torch.zeros(k, n * f.td, dtype=torch.float64, device="cuda")
        idx = np.random.default_rng(W.SEED + 99).choice(n, CHECK_TARGETS, replace=False)
        clocks.start()
        tuned = None
        if not args.no_autotune:
            _, tuned = f.autotune(den, out, k, fmmg.PREC_MIXED, reps=1)
        ms, kern, stage, launches, graph = time_form(f, torch, stream, den, out, n, k, fmmg.PREC_MIXED, args.steps,
                                                     args.warmup, flush)
        vals = out.cpu().numpy()
        errs = [f.check(cfg["den"][r], vals[r], idx)[0] for r in range(k)]
        ms64, _, _, _, _ = time_form(f, torch, stream, den[:1].contiguous(), out[:1], n, 1, fmmg.PREC_FP64,
                                     max(2, args.steps // 4), 3, flush)
        err64 = f.check(cfg["den"][0], out[0].cpu().numpy(), idx)[0]
        line.update({"metric": "points/s (targets x right-hand sides / device time)", "points": n, "k_rhs": k,
                     "kernel": cfg["kernel"], "np": cfg["np"], "value": n * k / (ms * 1e-3), "ms_per_step": ms,
                     "dtype": "f32+f64", "rel_err_vs_dense_max": max(errs), "rel_err_vs_dense_per_rhs": errs,
                     "check_targets": CHECK_TARGETS, "fp64_k1": {"ms": ms64, "points_per_s": n / (ms64 * 1e-3),
                                                                 "rel_err_vs_dense": err64},
                     "kernel_ms": kern, "launches": launches, "cuda_graph": graph, "tuning": tuned,
                     "setup_s": setup_s})
    else:  # laplace_adjoint_4m
        cfg = W.config4()
        src, D = cfg["src"], cfg["den"]
        n, k = src.shape[0], D.shape[0]
        rng = np.random.default_rng(W.SEED + 40)
        w = rng.normal(size=(k, n))
        f = fmmg.FMM3d(111, np_=6, pts_max=64, device=0, stream=stream.cuda_stream)
        f.setup(src)
        den = torch.from_numpy(D).cuda()
        wd = torch.from_numpy(w).cuda()
        out = torch.zeros(k, n, dtype=torch.float64, device="cuda")
        g = torch.empty(k, n, dtype=torch.float64, device="cuda")
        gt = torch.empty(k, n, 3, dtype=torch.float64, device="cuda")
        clocks.start()
        ms_fwd, _, _, _, _ = time_form(f, torch, stream, den, out, n, k, fmmg.PREC_FP64, args.steps, args.warmup, flush)
        ms_mix, _, _, _, _ = time_form(f, torch, stream, den, out, n, k, fmmg.PREC_MIXED, args.steps, args.warmup,
                                       flush)
        res = {}
        for key, call in (("adjoint_ms", lambda: f.adjoint_device(None, wd, g, None, k=k)),
                          ("target_grad_ms", lambda: f.adjoint_device(den, wd, None, gt, k=k))):
            res[key] = time_calls(torch, stream, call, max(2, args.steps // 4), 3, flush)
        # the same gradients through torch.autograd (fmm_apply forward + backward)
        import fmmg_torch
        den_t = den.clone().requires_grad_(True)
        trg_t = torch.from_numpy(src).cuda().requires_grad_(True)

        def autograd_step():
            phi = fmmg_torch.fmm_apply(f, den_t, trg_t, fmmg.PREC_FP64)
            (phi.view(k, n) * wd).sum().backward()

        res["autograd_step_ms"] = time_calls(torch, stream, autograd_step, 2, 1, flush)
        den_t.grad = trg_t.grad = None
        autograd_step()
        gsum = gt.sum(0).cpu().numpy()
        autograd_vs_device = {
            "target_grad_rel_l2": float(np.linalg.norm(trg_t.grad.cpu().numpy() - gsum) / np.linalg.norm(gsum)),
            "density_grad_rel_l2": float(torch.linalg.norm(den_t.grad - g) / torch.linalg.norm(g))}
        # central differences of <w_0, phi_0> in 64 random target coordinates: one
        # handle whose targets are the 128 displaced positions (sources fixed)
        h = 1e-4
        pick = rng.choice(n, 64, replace=False)
        dims = rng.integers(0, 3, 64)
        moved = np.repeat(src[pick], 2, axis=0)
        moved[0::2, :][np.arange(64), dims] += h
        moved[1::2, :][np.arange(64), dims] -= h
        fd_h = fmmg.FMM3d(111, np_=6, pts_max=64, device=0, stream=stream.cuda_stream)
        fd_h.setup(src, None, moved)
        phi = fd_h.evaluate(D[0]).ravel()
        fd = w[0, pick] * (phi[0::2] - phi[1::2]) / (2 * h)
        adj = gt[0].cpu().numpy()[pick, dims]
        fd_err = float(np.linalg.norm(fd - adj) / np.linalg.norm(adj))
        fd_h.close()
        # the dense FP64 gradients on a 32,768-point subset problem
        m = 32768
        sub = fmmg.FMM3d(111, np_=6, pts_max=64, device=0, stream=stream.cuda_stream)
        sub.setup(src[:m])
        gs, gts = sub.adjoint(w[:, :m], D[:, :m], target_grad=True, k=k)
        dg, dgt = dense_laplace_grads(src[:m], D[:, :m], w[:, :m])
        sub.close()
        line.update({"metric": "adjoint time / forward time (same precision and k)", "points": n, "k_rhs": k,
                     "kernel": 111, "np": 6, "dtype": "f64",
                     "forward_fp64_ms": ms_fwd, "forward_mixed_ms": ms_mix, "adjoint_fp64_ms": res["adjoint_ms"],
                     "target_grad_fp64_ms": res["target_grad_ms"], "autograd_step_ms": res["autograd_step_ms"],
                     "autograd_vs_device": autograd_vs_device,
                     "value": res["adjoint_ms"] / ms_fwd, "target_grad_vs_forward": res["target_grad_ms"] / ms_fwd,
                     "central_differences": {"h": h, "coordinates": 64, "rel_l2_vs_adjoint": fd_err},
                     "dense_subset": {"points": m, "density_grad_rel_l2": float(np.linalg.norm(gs.reshape(k, m) - dg)
                                                                                 / np.linalg.norm(dg)),
                                      "target_grad_rel_l2": float(np.linalg.norm(gts - dgt) / np.linalg.norm(dgt))}})
    line["clocks"] = clocks.stop()
    print(json.dumps(line))
    f.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload != "laplace_1m":
        run_workload(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
