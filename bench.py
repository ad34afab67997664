"""P3M steps/s on one B200 (or N replicas): FP32-mixed vs FP64 plain.

Workload (the headline configuration): method 1 (P3M ik, c2c, interlaced),
1,000,000 particles uniform in a box of side 100 (density 1), +-1 charges
alternating, mesh 128^3, cao 7, rcut 3.5, alpha 0.9, mc 1.  One step = one
force evaluation (Calculate_forces, common.c:268-327): real-space pairs,
charge assignment, FFTs, convolution, back-interpolation, f = f_k + f_r.
The influence function is computed once per alpha outside the timed region,
as the reference's own timer does (main.c:382-386).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one process per GPU): independent replicas of the
workload, no collective on the data path ("replicas only"); the timed region
is bracketed by barriers and the time is the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "p3m-standalone_b200"))

WORKLOAD = dict(workload="p3m-ik-i 1M particles, box 100, mesh 128^3, cao 7, rcut 3.5, alpha 0.9",
                method=1, n=1_000_000, box=100.0, mesh=128, cao=7, mc=1, rcut=3.5, alpha=0.9,
                system_type=0, seed=12345)
# The headline's parameters on 20,000 particles at density 1: small enough
# for the reference's own full step (its O(N^2) Realteil included) to be
# timed on the host instead of extrapolated, so both arms report one
# measured, same-configuration step time beside the headline.
SAME_CONFIG = dict(workload="p3m-ik-i 20,000 particles at density 1 (box 27.14), mesh 128^3, cao 7, rcut 3.5, "
                            "alpha 0.9", method=1, n=20000, box=20000 ** (1.0 / 3.0), mesh=128, cao=7, mc=1,
                   rcut=3.5, alpha=0.9, system_type=0, seed=12345)
METRIC = "P3M steps/s at 1e-4 RMS force error: FP32-mixed vs FP64 plain, same B200"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def _env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [v.strip() for v in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return dict(sm_mhz=statistics.median(sm), sm_max_mhz=smax, reasons=sorted(reasons), samples=len(sm))


# --------------------------------------------------------------- helpers

def algorithmic_bytes(method, n, mesh, s):
    """Algorithmic HBM bytes of one step: each stage reads its inputs once
    and writes its outputs once.  R = mesh bytes (2M s interlaced, M s
    otherwise), G = M s; particles 7 n s (x, y, z, q in, f out).
    ik: 7ns + 16R + G ; ad: 7ns + 8R + G."""
    M = mesh ** 3
    interlaced = method in (1, 3)
    R = (2 * M if interlaced else M) * s
    G = M * s
    if method in (0, 1, 6):
        return 7 * n * s + 16 * R + G
    return 7 * n * s + 8 * R + G


def gather_bytes(method, n, mesh, s):
    """Algorithmic bytes of the back-interpolation kernel: the ik fields
    (3R) or the ad potential (R) read once, n (x, y, z, q) in, n f out."""
    M = mesh ** 3
    R = (2 * M if method in (1, 3) else M) * s
    return (3 * R if method in (0, 1, 6) else R) + 7 * n * s


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# the sources that define each profiled kernel: a committed ncu count is
# only used while these files are byte-identical to the ones it measured
KERNEL_SOURCES = {
    "pairs_cell_kernel": ["p3mg_pairs.cu"],
    "scatter_kernel": ["p3mg_assign_impl.cuh"],
    "gather_kernel": ["p3mg_assign_impl.cuh"],
    "gather_tile_kernel": ["p3mg_gather_tile.cu"],
}


def kernel_source_digest(kernel):
    """sha256 (first 16 hex digits) of the source files of `kernel`."""
    import hashlib
    h = hashlib.sha256()
    for f in KERNEL_SOURCES[kernel]:
        with open(os.path.join(ROOT, "p3m-standalone_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def profile_counters(kernel):
    """DRAM bytes and warp instructions per launch of `kernel` at the headline
    workload from the committed ncu summary (profiles/traffic.json), or {}
    when there is none or it was captured from other sources than the
    current ones (its source_digest differs)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            d = json.load(fh).get(kernel, {})
    except Exception:
        return {}
    if d.get("source_digest") != kernel_source_digest(kernel):
        return {}
    return d


def profile_traffic(kernel):
    v = profile_counters(kernel).get("bytes_per_launch")
    return None if v is None else float(v)


# ------------------------------------------------------------- replicas

def reduce_max(v, dist=None, device="cpu"):
    """Max of v over the ranks of the process group (v itself without one).
    NCCL needs a CUDA tensor (device = the rank's GPU); gloo a CPU one."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(ms_per_step_max, world):
    """Whole-job steps/s of `world` independent replicas (one system per rank,
    no collective on the data path) whose slowest rank takes ms_per_step_max
    per step."""
    return world * 1000.0 / ms_per_step_max


# ------------------------------------------------------------- our arm

def run_ours(args, rank, world, local_rank):
    import torch
    import p3mg

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return reduce_max(v, dist, dev)

    W = WORKLOAD
    n = args.n or W["n"]
    L = W["box"] * (n / W["n"]) ** (1.0 / 3.0)
    x, y, z, q = p3mg.generate_system(W["system_type"], n, L, seed=W["seed"] + rank)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    results = {}
    clocks = None
    for prec in (p3mg.FP32_MIXED, p3mg.FP64):
        ctx = p3mg.Context(W["method"], W["mesh"], W["cao"], W["mc"], prec)
        ctx.set_system(x, y, z, q, L)
        ctx.influence(W["alpha"])
        stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
        # the step replayed as a CUDA graph (p3mg_set_graph: the first
        # warm-up step runs eagerly, the second is captured), no per-kernel
        # timing events inside the timed steps
        ctx.set_graph(True)
        for _ in range(max(args.warmup, 3)):
            ctx.compute(W["rcut"])
        torch.cuda.synchronize()
        sampler = ClockSampler(local_rank) if prec == p3mg.FP32_MIXED else None
        barrier()
        if sampler:
            sampler.start()
            time.sleep(0.3)
        l0 = ctx.launch_count()
        dev_ms = 0.0
        for _ in range(args.steps):
            flush.fill_(1.0)  # evict the previous step from L2 (untimed)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.compute(W["rcut"])
            e1.record(stream)
            e1.synchronize()
            dev_ms += e0.elapsed_time(e1)
        launches = ctx.launch_count() - l0
        barrier()
        if sampler:
            clocks = sampler.stop()
        ms = max_over_ranks(dev_ms) / args.steps
        # the split of a step over its kernels and stages (untimed for the
        # headline): timing events on, which runs the step eagerly
        ctx.enable_timing(True)
        ctx.compute(W["rcut"])
        kms = {"pairs": 0.0, "scatter": 0.0, "gather": 0.0}
        sms = {"t_c": 0.0, "t_g": 0.0, "t_f": 0.0, "t_r": 0.0}
        reps_split = max(1, min(args.steps, 5))
        for _ in range(reps_split):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            ctx.compute(W["rcut"])
            torch.cuda.synchronize()
            for k, v in ctx.kernel_times().items():
                kms[k] += v
            for k, v in ctx.stage_times().items():
                sms[k] += v
        results[prec] = dict(ms=ms, kernels={k: v / reps_split for k, v in kms.items()},
                             stages={k: v / reps_split for k, v in sms.items()}, launches=launches)
        # each kernel's own duration (untimed for the headline): the pairs
        # before the k-space chain instead of beside it, so no kernel
        # shares the SMs with another; the roofline uses these
        ctx.set_overlap(False)
        ctx.compute(W["rcut"])
        iso = {"pairs": 0.0, "scatter": 0.0, "gather": 0.0}
        reps_iso = max(1, min(args.steps, 5))
        for _ in range(reps_iso):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            ctx.compute(W["rcut"])
            torch.cuda.synchronize()
            for k, v in ctx.kernel_times().items():
                iso[k] += v
        results[prec]["kernels_isolated"] = {k: v / reps_iso for k, v in iso.items()}
        ctx.set_overlap(True)
        ctx.enable_timing(False)
        ctx.compute(W["rcut"])  # graph replays again from here (eager, then captured)
        ctx.compute(W["rcut"])

        # end to end through the public C ABI with pinned host buffers
        hx = [torch.from_numpy(a).pin_memory() for a in (x, y, z, q)]
        hf = [torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(3)]
        for _ in range(max(1, args.warmup // 2)):
            ctx.set_system_ptr(n, *[t.data_ptr() for t in hx], L)
            ctx.compute(W["rcut"])
            ctx.get_total_forces_ptr(*[t.data_ptr() for t in hf])
        barrier()
        e2e_ms = 0.0
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.set_system_ptr(n, *[t.data_ptr() for t in hx], L)
            ctx.compute(W["rcut"])
            ctx.get_total_forces_ptr(*[t.data_ptr() for t in hf])
            e1.record(stream)
            e1.synchronize()
            e2e_ms += e0.elapsed_time(e1)
        barrier()
        results[prec]["e2e_ms"] = max_over_ranks(e2e_ms) / args.steps
        results[prec]["forces"] = np.stack([t.numpy().copy() for t in hf])
        ctx.close()

    r32, r64 = results[p3mg.FP32_MIXED], results[p3mg.FP64]
    # accuracy (untimed): DeltaF of both paths against the FP64 Ewald reference
    # forces on a seeded subset of 2000 targets (Calculate_errors, error.c:21-34)
    accuracy = None
    if rank == 0 and not args.no_accuracy:
        tg = np.sort(np.random.default_rng(2024).choice(n, min(2000, n), replace=False))
        with p3mg.Context(W["method"], W["mesh"], W["cao"], W["mc"], p3mg.FP64) as ectx:
            ectx.set_system(x, y, z, q, L)
            t0 = time.perf_counter()
            ew = ectx.ewald_forces(tg)
            t_ew = time.perf_counter() - t0
        fe = ew["f"]
        def _rms(f):
            d = f[:, tg] - fe
            return float(np.sqrt(np.sum(d * d) / len(tg)))
        fr = float(np.sqrt(np.sum(fe * fe) / len(tg)))
        accuracy = {"targets": int(len(tg)), "ewald_alpha": ew["alpha"], "ewald_kmax": ew["kmax"],
                    "ewald_seconds": round(t_ew, 3), "rms_force": fr,
                    "rms_error_fp32": _rms(r32["forces"]), "rms_error_fp64": _rms(r64["forces"]),
                    "rms_fp32_vs_fp64": float(np.sqrt(np.sum((r32["forces"][:, tg] - r64["forces"][:, tg]) ** 2)
                                                     / len(tg)))}
    value = replica_throughput(r32["ms"], world)
    e2e = replica_throughput(r32["e2e_ms"], world)

    out = None
    if rank == 0:
        # dominant kernel of the FP32 step and its HBM roofline
        k = r32["kernels_isolated"]
        dom = max(k, key=k.get)
        peak, peak_kind = measured_peaks()
        s = 4
        if dom == "gather":
            abytes = gather_bytes(W["method"], n, W["mesh"], s)
        elif dom == "scatter":
            R = 2 * W["mesh"] ** 3 * s
            abytes = R + 4 * n * s
        else:
            abytes = 16 * n + 7 * n * s  # float4 cell-sorted particles in, forces out
        achieved = abytes / (k[dom] * 1e-3) / 1e9
        kernel_names = {"gather": "gather_tile_kernel", "scatter": "scatter_kernel", "pairs": "pairs_cell_kernel"}
        traffic = profile_traffic(kernel_names[dom])
        g_bytes = gather_bytes(W["method"], n, W["mesh"], s)
        g_achieved = g_bytes / (k["gather"] * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": kernel_names[dom], "achieved": round(achieved, 2), "peak": peak,
                    "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                    "algorithmic_bytes": int(abytes), "traffic": traffic}
        inst = profile_counters("pairs_cell_kernel").get("warp_instructions_per_launch")
        if dom == "pairs" and inst and n == W["n"]:
            # The pair kernel moves ~48 MB per launch and uses no tensor cores:
            # its ceiling is instruction issue (4 warp instructions per clock
            # per SM).  Achieved = the warp instructions of one launch (ncu,
            # this workload) over the live CUDA-event time of the launch.
            sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
            ipeak = 4 * 148 * sm_mhz * 1e6 / 1e9
            iach = inst / (k["pairs"] * 1e-3) / 1e9
            pairs_unique = 2.0 * math.pi / 3.0 * W["rcut"] ** 3 * n * (n / L ** 3)
            roofline = {"bound": "issue", "kernel": "pairs_cell_kernel", "achieved": round(iach, 1),
                        "peak": round(ipeak, 1), "unit": "G warp-instructions/s", "frac": round(iach / ipeak, 4),
                        "peak_source": "4 warp instructions/clock/SM x 148 SMs x sampled SM clock",
                        "traffic": traffic, "algorithmic_bytes": int(abytes),
                        "hbm_frac": round(achieved / peak, 4),
                        "pairs_per_s": round(pairs_unique / (k["pairs"] * 1e-3), 1),
                        "unique_pairs_within_rcut": int(pairs_unique),
                        "instructions_source": "profiles/traffic.json (ncu smsp__inst_executed.sum of these "
                                               "sources, digest %s)" % kernel_source_digest("pairs_cell_kernel")}
        out = {
            "metric": METRIC,
            "value": round(value, 3),
            "unit": "steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(r32["ms"], 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (mesh, FFT, pairs; f64 G_opt and geometry)",
            "data": "synthetic: seeded uniform system (system_type 0), +-1 charges alternating",
            "config": {"workload": W["workload"], "method": W["method"], "particles": n, "box": L,
                       "mesh": W["mesh"], "cao": W["cao"], "rcut": W["rcut"], "alpha": W["alpha"], "mc": W["mc"],
                       "parallelism": "replicas%d" % world if world > 1 else "single-gpu",
                       "step": "p3mg_compute replayed as a CUDA graph (p3mg_set_graph), both precisions",
                       "l2": "flushed between timed steps (256 MB write, untimed)"},
            "fp64": {"value": round(replica_throughput(r64["ms"], world), 3), "unit": "steps/s",
                     "ms_per_step": round(r64["ms"], 4),
                     "e2e_steps_per_s": round(replica_throughput(r64["e2e_ms"], world), 3)},
            "fp32_over_fp64": round(r64["ms"] / r32["ms"], 3),
            "stages_ms": {"fp32": {k2: round(v, 4) for k2, v in r32["stages"].items()},
                          "fp64": {k2: round(v, 4) for k2, v in r64["stages"].items()}},
            "kernels_ms": {"fp32": {k2: round(v, 4) for k2, v in r32["kernels"].items()},
                           "fp64": {k2: round(v, 4) for k2, v in r64["kernels"].items()},
                           "note": "CUDA events around each kernel inside the timed steps, where the pairs "
                                   "run beside the k-space chain and share the SMs with it (an untimed "
                                   "eager pass after the timed steps)"},
            "kernels_isolated_ms": {"fp32": {k2: round(v, 4) for k2, v in r32["kernels_isolated"].items()},
                                    "fp64": {k2: round(v, 4) for k2, v in r64["kernels_isolated"].items()},
                                    "note": "the same after the timed steps with the pairs run before the "
                                            "k-space chain (each kernel alone on the GPU); the rooflines "
                                            "use these"},
            "e2e": {"value": round(e2e, 3), "unit": "steps/s", "h2d_bytes_per_step": 4 * 8 * n,
                    "d2h_bytes_per_step": 3 * 8 * n},
            "roofline": roofline,
            "roofline_hbm": {"kernel": "gather_tile_kernel", "achieved": round(g_achieved, 2), "peak": peak,
                             "unit": "GB/s", "frac": round(g_achieved / peak, 4), "peak_source": peak_kind,
                             "algorithmic_bytes": int(g_bytes), "traffic": profile_traffic("gather_tile_kernel"),
                             "note": "the tile gather is bound by the shared-memory pipe (LSU wavefronts at 82 % "
                                     "of peak under ncu), not HBM"},
            "step_roofline": {"algorithmic_bytes": int(algorithmic_bytes(W["method"], n, W["mesh"], 4)),
                              "achieved_gbs": round(algorithmic_bytes(W["method"], n, W["mesh"], 4)
                                                    / (r32["ms"] * 1e-3) / 1e9, 2)},
            "accuracy": accuracy,
            "gpu_launches": int(r32["launches"]),
            "clocks": clocks,
        }
    return out, results


# ------------------------------------------------- same-config point

def same_config_ours(dev, steps=20):
    """Device time of one step (CUDA events, median of `steps`) and of one
    step end to end through the C ABI (host buffers in, total forces out)
    at SAME_CONFIG, FP32-mixed and FP64."""
    import torch
    import p3mg
    S = SAME_CONFIG
    x, y, z, q = p3mg.generate_system(S["system_type"], S["n"], S["box"], seed=S["seed"])
    out = {"workload": S["workload"]}
    for prec, tag in ((p3mg.FP32_MIXED, "fp32"), (p3mg.FP64, "fp64")):
        with p3mg.Context(S["method"], S["mesh"], S["cao"], S["mc"], prec) as ctx:
            ctx.set_system(x, y, z, q, S["box"])
            ctx.influence(S["alpha"])
            st = torch.cuda.ExternalStream(ctx.stream(), device=dev)
            ctx.set_graph(True)
            ctx.compute(S["rcut"])  # eager warm-up; the next call captures
            step = _timed(st, lambda: ctx.compute(S["rcut"]), reps=steps)
            hx = [torch.from_numpy(a).pin_memory() for a in (x, y, z, q)]
            hf = [torch.empty(S["n"], dtype=torch.float64).pin_memory() for _ in range(3)]

            def e2e():
                ctx.set_system_ptr(S["n"], *[t.data_ptr() for t in hx], S["box"])
                ctx.compute(S["rcut"])
                ctx.get_total_forces_ptr(*[t.data_ptr() for t in hf])
            e2e_ms = _timed(st, e2e, reps=steps)
        out[tag] = {"ms_per_step": round(step, 4), "steps_per_s": round(1000.0 / step, 2),
                    "e2e_ms_per_step": round(e2e_ms, 4), "e2e_steps_per_s": round(1000.0 / e2e_ms, 2)}
    return out


# ------------------------------------------------- secondary workloads

def _events(stream):
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _timed(stream, fn, reps=3):
    """Median device time (ms) of fn() bracketed by events on `stream`."""
    import torch
    fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = _events(stream)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def _smooth_even(m):
    while True:
        r = m
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1 and m % 2 == 0:
            return m
        m += 1


def secondary_workloads(dev):
    """The batched, differentiated and multi-system workloads, each timed on
    the device (median of three runs after one warm-up)."""
    import torch
    import p3mg
    out = {}

    def stream_of(ctx):
        return torch.cuda.ExternalStream(ctx.stream(), device=dev)

    # alpha sweep: the reference's example (method 7, 1000 particles, box 10,
    # mesh 16, cao 7, mc 2, rcut 3, alpha 0.1..2.5 step 0.05: 49 alphas), FP64;
    # each sweep returns the RMS force error per alpha against the Ewald forces
    x, y, z, q = p3mg.generate_system(0, 1000, 10.0, seed=12345)
    with p3mg.Context(7, 16, 7, 2, p3mg.FP64) as ctx:
        ctx.set_system(x, y, z, q, 10.0)
        st = stream_of(ctx)
        ref = ctx.ewald_forces()["f"]
        al = p3mg.alpha_range(0.1, 2.5, 0.05)
        ctx.influence(1.0)
        ctx.set_graph(True)
        step = _timed(st, lambda: ctx.compute(3.0), reps=7)
        loop = _timed(st, lambda: [(ctx.influence(a), ctx.compute(3.0)) for a in al])
        sweep = _timed(st, lambda: ctx.sweep(3.0, al, ref=ref))
        a64 = np.linspace(0.1, 2.5, 64)
        sweep64 = _timed(st, lambda: ctx.sweep(3.0, a64, ref=ref))
    out["alpha_sweep_1000"] = {
        "workload": "method 7, 1000 particles, box 10, mesh 16, cao 7, mc 2, rcut 3, FP64, "
                    "RMS error per alpha against the Ewald forces",
        "step_ms": round(step, 4), "alphas": len(al), "sweep_ms": round(sweep, 3),
        "per_alpha_loop_ms": round(loop, 3), "sweep_64_alphas_ms": round(sweep64, 3),
        "sweep_64_over_step": round(sweep64 / step, 2)}

    # the same 64-alpha sweep at the headline size (method 1, 1M, mesh 128),
    # FP32, RMS error per alpha against the FP64 P3M forces at the headline
    # alpha (host rows, uploaded inside the timed call)
    W = WORKLOAD
    x, y, z, q = p3mg.generate_system(0, W["n"], W["box"], seed=W["seed"])
    with p3mg.Context(W["method"], W["mesh"], W["cao"], W["mc"], p3mg.FP64) as ctx:
        ctx.set_system(x, y, z, q, W["box"])
        ctx.influence(W["alpha"])
        ctx.compute(W["rcut"])
        ref = ctx.get_forces()["f"]
    with p3mg.Context(W["method"], W["mesh"], W["cao"], W["mc"], p3mg.FP32_MIXED) as ctx:
        ctx.set_system(x, y, z, q, W["box"])
        st = stream_of(ctx)
        ctx.influence(W["alpha"])
        ctx.set_graph(True)
        step = _timed(st, lambda: ctx.compute(W["rcut"]), reps=5)
        a64 = np.linspace(0.6, 1.2, 64)
        sweep64 = _timed(st, lambda: ctx.sweep(W["rcut"], a64, ref=ref), reps=3)
        # every alpha evaluated (no interpolation): max_batch > 0
        exact64 = _timed(st, lambda: ctx.sweep(W["rcut"], a64, ref=ref, max_batch=64), reps=2)
    out["alpha_sweep_1m"] = {"workload": W["workload"] + ", FP32, 64 alphas 0.6..1.2, RMS error per alpha "
                                                        "against FP64 P3M forces",
                             "step_ms": round(step, 4), "sweep_64_alphas_ms": round(sweep64, 2),
                             "sweep_64_over_step": round(sweep64 / step, 2),
                             "interpolated": "10 Chebyshev nodes in 1/alpha^2 + 2 checked alphas",
                             "exact_sweep_64_alphas_ms": round(exact64, 2),
                             "exact_sweep_64_over_step": round(exact64 / step, 2)}

    # the metric's accuracy point: the headline system (1M, box 100, method 1,
    # rcut 3.5) with mesh, cao and alpha chosen by the reference's Tune search
    # (p3mg_tune, FP32 candidates timed) for a 1e-4 RMS force error estimate;
    # FP32-mixed and FP64 steps at those parameters and their RMS errors
    # against the FP64 Ewald forces on 2000 seeded targets
    x, y, z, q = p3mg.generate_system(0, W["n"], W["box"], seed=W["seed"])
    tuned = p3mg.tune(W["method"], x, y, z, q, W["box"], W["rcut"], 1e-4, precision=p3mg.FP32_MIXED)
    tg = np.sort(np.random.default_rng(2024).choice(W["n"], 2000, replace=False))
    acc = {"workload": "p3m-ik-i 1M particles, box 100, rcut 3.5, (mesh, cao, alpha) from p3mg_tune for a 1e-4 "
                       "RMS force error estimate", "tuned": tuned}
    with p3mg.Context(W["method"], tuned["mesh"], tuned["cao"], W["mc"], p3mg.FP64) as ectx:
        ectx.set_system(x, y, z, q, W["box"])
        fe = ectx.ewald_forces(tg)["f"]
    for prec, tag in ((p3mg.FP32_MIXED, "fp32"), (p3mg.FP64, "fp64")):
        with p3mg.Context(W["method"], tuned["mesh"], tuned["cao"], W["mc"], prec) as ctx:
            ctx.set_system(x, y, z, q, W["box"])
            ctx.influence(tuned["alpha"])
            st = stream_of(ctx)
            ms = _timed(st, lambda: ctx.compute(W["rcut"]), reps=5)
            f = ctx.get_forces()["f"]
        acc[tag] = {"ms_per_step": round(ms, 4), "steps_per_s": round(1000.0 / ms, 2),
                    "rms_error_vs_ewald": float(np.sqrt(np.sum((f[:, tg] - fe) ** 2) / len(tg)))}
    acc["fp32_over_fp64"] = round(acc["fp64"]["ms_per_step"] / acc["fp32"]["ms_per_step"], 3)
    out["accuracy_1e-4_1m"] = acc

    # adjoint: 50,000 separated dipoles, box 46.4, method 2, mesh 64, cao 5,
    # rcut 3, alpha 1, FP32; -dE/dx against FP64 Ewald forces on 2000 targets
    x, y, z, q = p3mg.generate_system(3, 100000, 46.4, seed=12345)
    with p3mg.Context(2, 64, 5, 1, p3mg.FP32_MIXED) as ctx:
        ctx.set_system(x, y, z, q, 46.4)
        ctx.influence(1.0)
        st = stream_of(ctx)
        fwd = _timed(st, lambda: ctx.compute(3.0))
        # device-resident like the force step (gradients stay on the GPU);
        # with the gradients copied to host arrays beside it
        bwd = _timed(st, lambda: ctx.backward_device(3.0))
        bwd_host = _timed(st, lambda: ctx.backward(3.0))
        g = ctx.backward(3.0)
        tg = np.sort(np.random.default_rng(7).choice(len(x), 2000, replace=False))
        ew = ctx.ewald_forces(tg)["f"]
        err = float(np.sqrt(np.sum((-g["dx"][:, tg] - ew) ** 2) / len(tg)))
        f = ctx.calculate_forces(3.0)["f"]
        ferr = float(np.sqrt(np.sum((f[:, tg] - ew) ** 2) / len(tg)))
    out["adjoint_dipoles_100k"] = {
        "workload": "method 2, 50000 dipoles (100000 charges), box 46.4, mesh 64, cao 5, rcut 3, alpha 1, FP32",
        "force_step_ms": round(fwd, 3), "energy_and_gradients_ms": round(bwd, 3),
        "energy_and_gradients_to_host_ms": round(bwd_host, 3),
        "energy": g["energy"]["total"], "dE_dalpha": g["dalpha"], "virial_minus_L_dE_dL": -46.4 * g["dL"],
        "rms_minus_grad_vs_ewald": err, "rms_force_vs_ewald": ferr}

    # uneven multi-system batch: 16 systems, N log-uniform in 2e3..2e6 at
    # density 1, uniform / Gaussian (sigma L/6) alternating, mesh the next
    # even 7-smooth size >= clamp(1.28 L, 32, 160), cao 7, rcut 3.5,
    # alpha 0.9, methods 1 and 3 alternating
    rng = np.random.default_rng(16)
    ns = np.sort(np.exp(rng.uniform(np.log(2e3), np.log(2e6), 16)).astype(int))
    res = {}
    for prec, tag in ((p3mg.FP32_MIXED, "fp32"), (p3mg.FP64, "fp64")):
        ctxs = []
        for k, nk in enumerate(ns):
            Lk = float(nk) ** (1.0 / 3.0)
            mk = _smooth_even(int(np.ceil(min(max(1.28 * Lk, 32), 160))))
            xs = p3mg.generate_system(0 if k % 2 == 0 else 4, int(nk), Lk, seed=1000 + k)
            c = p3mg.Context(1 if k % 2 == 0 else 3, mk, 7, 1, prec)
            c.set_system(*xs, Lk)
            c.influence(0.9)
            ctxs.append(c)
        # host clock around device-synchronised calls: the contexts run on
        # their own streams, which one stream's events would not cover
        for c in ctxs:
            c.compute(3.5)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(3):
            for c in ctxs:
                c.compute(3.5)
        torch.cuda.synchronize()
        seq = (time.perf_counter() - t0) / 3 * 1e3
        with p3mg.Batch(ctxs) as b:
            b.compute([3.5] * len(ctxs))
            b.compute([3.5] * len(ctxs))
            b.synchronize()
            t0 = time.perf_counter()
            for _ in range(3):
                b.compute([3.5] * len(ctxs))
            b.synchronize()
            bt = (time.perf_counter() - t0) / 3 * 1e3
        for c in ctxs:
            c.close()
        res[tag] = {"batch_graph_ms": round(bt, 3), "sequential_ms": round(seq, 3),
                    "systems_per_s": round(16 * 1000.0 / bt, 2)}
    out["multi_system_batch"] = {"particles": [int(v) for v in ns], "timing": "host clock, device synchronised",
                                 **res}

    # tuning grid: slab of 20,000 charges in [0.25L, 0.75L) x [0,L)^2, L 34.2,
    # method 7, mesh {32,48,64,96} x cao 3..7 x 64 alphas 0.1..2.5, FP32;
    # RMS error of every point against the FP64 Ewald forces and the estimate
    Lg = 34.2
    x, y, z, q = p3mg.generate_system(5, 20000, Lg, seed=12345)
    q2 = float(np.sum(q * q))
    al = np.linspace(0.1, 2.5, 64)
    with p3mg.Context(7, 32, 7, 1, p3mg.FP64) as ec:
        ec.set_system(x, y, z, q, Lg)
        ref = ec.ewald_forces()["f"]
    # every (mesh, cao) point one context of the same system: one
    # p3mg_sweep_grid call (real space once per alpha, k-space passes
    # concurrent); host clock around the call, which synchronises
    pts = [(mesh, cao) for mesh in (32, 48, 64, 96) for cao in range(3, 8)]
    ctxs = []
    for mesh, cao in pts:
        cg = p3mg.Context(7, mesh, cao, 1, p3mg.FP32_MIXED)
        cg.set_system(x, y, z, q, Lg)
        ctxs.append(cg)
    p3mg.sweep_grid(ctxs, 3.0, al, ref)  # warm-up: workspaces, lane tables
    torch.cuda.synchronize()
    # best of three calls: one call's host clock includes whatever else the
    # host does meanwhile (single calls ranged 24-120 ms on shared machines)
    grid_calls = []
    for _ in range(3):
        t_all = time.perf_counter()
        rms = p3mg.sweep_grid(ctxs, 3.0, al, ref)
        grid_calls.append((time.perf_counter() - t_all) * 1e3)
    grid_ms = min(grid_calls)
    for cg in ctxs:
        cg.close()
    i, k = np.unravel_index(int(np.argmin(rms)), rms.shape)
    mesh, cao = pts[i]
    est = p3mg.estimate_errors(7, mesh, cao, len(x), q2, Lg, float(al[k]), 3.0)["total"]
    best = (float(rms[i, k]), mesh, cao, float(al[k]), est)
    out["tuning_grid_slab_20k"] = {
        "points": 4 * 5 * 64, "grid_ms": round(grid_ms, 2),
        "grid_calls_ms": [round(v, 2) for v in grid_calls],
        "timing": "host clock around each of three p3mg_sweep_grid calls (each synchronises the device), the best",
        "best": {"rms_error": best[0], "mesh": best[1], "cao": best[2], "alpha": best[3], "estimate": best[4]}}
    return out


# ----------------------------------------------------------- CPU baseline

def reference_sample(n_k=20000, n_r=5000):
    """One bounded sample of the reference's own CPU code (oracle/_ref, the
    reference compiled from its sources, single-threaded) scaled to a full
    step of the workload:
      k-space: Kspace_force in the reference's timing mode (tuning=1, stage
        timers t_c/t_g/t_f, p3m-common.h:48-57) on n_k particles at the
        workload's mesh; charge and force assignment scale with N, the
        FFT/convolution stage does not;
      real space: Realteil (O(N^2) loop) on n_r particles at density 1,
        scaled by (N/n_r)^2.
    Returns (seconds per full step, description, kind)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import p3mg
    W = WORKLOAD
    N = W["n"]
    kind = "reference" if O.ref_available() else "port"
    rng = np.random.default_rng(7)
    x, y, z, q = p3mg.generate_system(0, N, W["box"], seed=W["seed"])
    sel = np.sort(rng.choice(N, n_k, replace=False))
    qq = 1.0 - 2.0 * (np.arange(n_k) % 2)
    if kind == "reference":
        r = O.ref_forces(W["method"], W["mesh"], W["cao"], W["mc"], W["alpha"], 0.0, x[sel], y[sel], z[sel], qq,
                         W["box"], tuning=True)
        tc, tg, tf = r["times"]
    else:
        t0 = time.perf_counter()
        O.kspace(W["method"], W["mesh"], W["cao"], W["mc"], W["alpha"], x[sel], y[sel], z[sel], qq, W["box"],
                 G=np.ones(W["mesh"] ** 3))
        tc, tg, tf = 0.0, 0.0, time.perf_counter() - t0
    t_k = (tc + tf) * (N / n_k) + tg
    Lr = W["box"] * (n_r / N) ** (1.0 / 3.0)
    xr, yr, zr, qr = p3mg.generate_system(0, n_r, Lr, seed=3)
    t0 = time.perf_counter()
    if kind == "reference":
        O.ref_realteil(xr, yr, zr, qr, Lr, W["rcut"], W["alpha"])
    else:
        O.realspace(xr, yr, zr, qr, Lr, W["rcut"], W["alpha"], cells=False)
    t_r = (time.perf_counter() - t0) * (N / n_r) ** 2
    desc = ("extrapolated: k-space on %d of the 1M particles (stage times t_c+t_f scaled x%d, t_g as is) + "
            "real-space N^2 loop on %d particles at density 1 scaled x%d; FFT is the oracle's DFT standing in for "
            "FFTW" % (n_k, N // n_k, n_r, (N // n_r) ** 2))
    return t_k + t_r, desc, kind, dict(t_c=tc, t_g=tg, t_f=tf, t_real_sample=t_r / (N / n_r) ** 2)


def same_config_reference():
    """One measured step of the reference's own code at SAME_CONFIG: the
    whole Calculate_forces (common.c:268-327), its timed region
    (main.c:382-386), single-threaded -- not extrapolated."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import p3mg
    S = SAME_CONFIG
    x, y, z, q = p3mg.generate_system(S["system_type"], S["n"], S["box"], seed=S["seed"])
    if O.ref_available():
        t = O.ref_step_seconds(S["method"], S["mesh"], S["cao"], S["mc"], S["alpha"], S["rcut"], x, y, z, q,
                               S["box"], reps=1)
        kind = "reference"
    else:
        t0 = time.perf_counter()
        O.forces(S["method"], S["mesh"], S["cao"], S["mc"], S["alpha"], S["rcut"], x, y, z, q, S["box"],
                 G=np.ones(S["mesh"] ** 3), cells=False)
        t = time.perf_counter() - t0
        kind = "port"
    return {"workload": S["workload"], "kind": kind, "extrapolated": False, "seconds_per_step": round(t, 4),
            "steps_per_s": 1.0 / t, "cores": 1,
            "note": "one full Calculate_forces (real space N^2 loop + k-space with the oracle's DFT for FFTW)"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    times = []
    for i in range(args.warmup + args.steps):
        t, desc, kind, parts = reference_sample()
        if i >= args.warmup:
            times.append(t)
    v = 1.0 / statistics.mean(times)
    try:
        import scipy.fft
        a = np.random.default_rng(0).standard_normal((128, 128, 128)) + 0j
        t0 = time.perf_counter()
        scipy.fft.fftn(a, workers=1)
        fft_proxy = time.perf_counter() - t0
    except Exception:
        fft_proxy = None
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 / v,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded uniform system (system_type 0), +-1 charges alternating",
        "config": {"workload": WORKLOAD["workload"], "parallelism": "cpu, 1 thread"},
        "cpu_baseline": {"value": v, "unit": "steps/s", "cores": 1, "kind": kind, "sample": desc,
                         "extrapolated": True, "last_sample_parts_s": parts,
                         "scipy_fft_128cube_1thread_s": fft_proxy, "cpu": _cpu_model()},
        "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "same_config_measured": same_config_reference(),
    }


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip() + " (nproc %d)" % os.cpu_count()
    except Exception:
        pass
    return "nproc %d" % os.cpu_count()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=0, help="particles (default: the workload's 1,000,000)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the Ewald error report")
    ap.add_argument("--no-workloads", action="store_true",
                    help="skip the sweep / adjoint / batch / tuning-grid workloads")
    args = ap.parse_args()
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    local_rank = _env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return
    out, _ = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1:
        import torch
        out["same_config_measured"] = same_config_ours(torch.device("cuda", local_rank))
        if not args.no_workloads:
            out["workloads"] = secondary_workloads(torch.device("cuda", local_rank))
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            t, desc, kind, parts = reference_sample()
            out["cpu_baseline"] = {"value": 1.0 / t, "unit": "steps/s", "cores": 1, "kind": kind, "sample": desc,
                                   "extrapolated": True, "cpu": _cpu_model()}
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
