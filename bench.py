"""Benchmark: Vext pose evaluations/s (forward + adjoint) on the full-size field.

Workload (default ``full_field``): 37 x 37 x 3.6 A layered cell (gamma
119.993), 600 seeded synthetic atoms, two-site guest 85 K / 3.685 A / bond
1.33 A, cutoff 12.8 A, 60^3 grid x 64 Fibonacci directors = 13,824,000 poses
per field.  One step = the energy, dE/d(center) and tangent dE/d(director)
of every pose (one replay of the one-system batched forward + adjoint
kernel), region lists and outputs resident in HBM.

Our arm prints one JSON line with: value (poses/s over all ranks, device time
from CUDA events, max over ranks), e2e (the public host C-ABI call
vext_field_adjoint: directors up, float32 energy + gradient down into pinned
host memory, which the kernels write over PCIe during the pair work), roofline of the fused pair kernel against the measured FP32
FFMA peak of this GPU, the forward-only field (list build + pair kernels +
epilogue, with the far kernel's roofline), the plain and tiled FP64 GPU
kernels and the error of the mixed result against FP64, the random-pose
forward+adjoint path and its error against its FP64 mode, the precision
study, the GPU String update, the drop-in mode (the reference's driver calling
this library's evaluate_reused_neighbors), the 100-field batches and 100
String paths,
clocks sampled during the timed
region, and a CPU baseline (the reference kernel compiled from its source,
driven by the restated reference driver, on a bounded sample of the field).

``--impl reference`` times that reference CPU path alone (all host cores,
rank 0 only) on the same metric.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from string_vext_b200 import ranks  # noqa: E402  (no CUDA work at import)

FLOP_FWD = 16          # algorithmic FLOP per in-cutoff (site, image) pair, forward
FLOP_FWD_ADJ = 28      # forward + adjoint
METRIC = "Vext pose evals/s at <=1e-4 K vs FP64, fwd+adjoint evals/s; % FP32 peak"
# dram__bytes_read.sum + dram__bytes_write.sum of one field_far2_kernel launch on
# full_field, from an ncu capture (--set full) of `bench.py --profile field`.
FAR_DRAM_BYTES_FULL_FIELD = 776_213_504 + 100_771_584
# the same for one forward + adjoint batch_field_kernel launch on full_field,
# from an ncu capture (--set full) of `bench.py --profile adjoint`.
ADJ_DRAM_BYTES_FULL_FIELD = 771_922_688 + 367_529_216
CPU_CENTERS_PER_CORE_S = 900.0   # reference driver throughput estimate used to size the sample


def ensure_built():
    lib = ROOT / "string_vext_b200" / "lib" / "libvext_b200.so"
    if not lib.exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "string_vext_b200" / "csrc"), "-j8"],
                       check=True)
    if not (ROOT / "oracle" / "libvext_oracle.so").exists():
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)


def workload(name):
    from string_vext_b200 import synth
    maker, size = synth.WORKLOADS[name]
    return maker(), size


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons of one GPU every 100 ms (samples
    taken before the timed region starts are dropped)."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.time() + 5.0      # sampling must be live before timing starts
            while not self.rows and time.time() < deadline and self.proc.poll() is None:
                time.sleep(0.02)
            self.rows.clear()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 4 + k and r[4 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_reference_sample(case, size, n_axes, seconds_target, processes):
    """The reference CPU path (kernel.cpp built from source when present,
    else the oracle's restatement) on a strided sample of the grid centers."""
    from oracle import oracle
    from string_vext_b200.orientation import regular_pose_grid
    library, kind, symbol = oracle.REF_KERNEL, "reference", "evaluate_reused_neighbors"
    if not library.exists():
        library, kind, symbol = oracle.LIB_PATH, "port", "oracle_reused_neighbors"
    centers, axes = regular_pose_grid(size, n_axes)
    n_sample = int(min(len(centers), max(processes * 64,
                                         CPU_CENTERS_PER_CORE_S * processes * seconds_target)))
    stride = max(1, len(centers) // n_sample)
    sample = centers[::stride][:n_sample]
    energy, wall, used, compute = oracle.reference_field_parallel(
        case, sample, axes, library=library, processes=processes, symbol=symbol)
    poses = len(sample) * n_axes
    which = ("reference driver (baseline/_ref)" if symbol == "evaluate_reused_neighbors"
             and oracle.reference_driver_class() is not None else "restated driver (oracle)")
    return {"value": poses / compute, "unit": "poses/s", "cores": used, "kind": kind,
            "sample": f"{len(sample)} of {len(centers)} grid centers (stride {stride}) x "
                      f"{n_axes} directors (forward energies only), {used} spawn processes, "
                      f"{which}; "
                      f"time = slowest worker's kd-tree query + kernel ({compute:.2f} s; "
                      f"{wall:.2f} s with process start), {cpu_model()}",
            "seconds": compute, "poses": poses}


def cpu_reference_single_core(case, size, n_axes, seconds_target):
    """The reference CPU path in its own mode (one process, one thread): the
    reference driver in this process on a strided sample of the grid
    centers; poses/s with and without the kd-tree query."""
    from oracle import oracle
    from string_vext_b200.orientation import regular_pose_grid
    library, kind, symbol = oracle.REF_KERNEL, "reference", "evaluate_reused_neighbors"
    if not library.exists():
        library, kind, symbol = oracle.LIB_PATH, "port", "oracle_reused_neighbors"
    centers, axes = regular_pose_grid(size, n_axes)
    n_sample = int(min(len(centers), max(512, CPU_CENTERS_PER_CORE_S * seconds_target)))
    stride = max(1, len(centers) // n_sample)
    sample = centers[::stride][:n_sample]
    driver, which = oracle.cpu_driver(case, library, symbol)
    t0 = time.perf_counter()
    driver.evaluate(sample, axes)
    wall = time.perf_counter() - t0
    poses = len(sample) * n_axes
    return {"value": poses / wall, "unit": "poses/s", "cores": 1, "kind": kind,
            "kernel_only": poses / driver.compute_seconds,
            "query_share": driver.query_seconds / wall,
            "sample": f"{len(sample)} of {len(centers)} grid centers (stride {stride}) x "
                      f"{n_axes} directors, one process, {which}; {wall:.2f} s, kd-tree query "
                      f"{driver.query_seconds:.2f} s, kernel {driver.compute_seconds:.2f} s, "
                      f"{cpu_model()}"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    case, size = workload(args.workload)
    cores = host_cores()
    values = []
    # each step a bounded sample: about two minutes of CPU work over the whole run
    per_step = max(0.5, min(args.cpu_seconds, 120.0 / (args.warmup + args.steps)))
    for step in range(args.warmup + args.steps):
        res = cpu_reference_sample(case, size, 64, per_step, cores)
        if step >= args.warmup:
            values.append(res)
    value = sum(r["poses"] for r in values) / sum(r["seconds"] for r in values)
    line = {"metric": METRIC, "value": value, "unit": "poses/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * statistics.mean(r["seconds"] for r in values),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": config_of(args.workload, size),
            "cpu_baseline": {"value": value, "unit": "poses/s", "cores": values[0]["cores"],
                             "kind": values[0]["kind"], "sample": values[0]["sample"]},
            "e2e": {"value": value, "unit": "poses/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def config_of(name, size):
    return {"workload": f"{name}: Vext field {size}^3 grid x 64 directors",
            "poses_per_field": size ** 3 * 64, "parallelism": "independent fields per GPU",
            "l2": "inputs larger than L2 (region lists > 126 MB per field)"}


def error_stats(mixed, exact):
    neg = exact <= 0
    diff = np.abs(mixed - exact)
    rel = diff / np.maximum(np.abs(exact), 1.0)
    return {"poses_E_le_0": int(neg.sum()), "poses_E_gt_0": int((~neg).sum()),
            "max_abs_K_E_le_0": float(diff[neg].max()) if neg.any() else None,
            "max_rel_E_gt_0": float(rel[~neg].max()) if (~neg).any() else None,
            "passed": bool((diff[neg] < 1e-4).all() and (rel[~neg] < 1e-6).all())}


def hbm_check(traffic_bytes, ms):
    """The kernel's DRAM throughput (ncu bytes / device time) against the
    measured HBM copy bandwidth in MEASURED_PEAKS.json."""
    try:
        peak = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]
        source = "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, KeyError, ValueError):
        peak, source = 6650.0, "fallback 6.65 TB/s"
    if not traffic_bytes:
        return {"achieved": None, "peak": peak, "unit": "GB/s", "peak_source": source}
    achieved = traffic_bytes / (ms * 1e-3) / 1e9
    return {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_source": source}


def timed_region(fn, steps, stream):
    """CUDA-event time (ms) of `steps` calls of fn on `stream`."""
    import torch
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def run_ours(args, rank, world, local_rank):
    import torch
    from string_vext_b200 import _lib
    from string_vext_b200.orientation import normalized_directors, regular_pose_grid
    from string_vext_b200.system import VextSystem

    torch.cuda.set_device(local_rank)
    device = torch.device("cuda", local_rank)
    case, size = workload(args.workload)
    _, axes = regular_pose_grid(size, 64)
    axes = normalized_directors(axes)
    n_axes = len(axes)
    poses = size ** 3 * n_axes
    shape = (n_axes, size, size, size)
    stream = torch.cuda.Stream(device)
    energy = torch.empty(shape, dtype=torch.float32, device=device)
    grad = torch.empty(shape + (6,), dtype=torch.float32, device=device)
    system = VextSystem(case)

    pairs, far_pairs = system.count_pairs(size, axes)
    pipes = _lib.measure_pipes()
    peak = 2.0 * max(pipes["ffma_per_s"], pipes["ffma2_fma_per_s"])   # FLOP/s, FMA = 2

    # ---- headline: forward + adjoint of every pose, one-system batched kernel
    t0 = time.perf_counter()
    system.field_adjoint_device(size, axes, energy, grad, stream=stream)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0

    def step():
        system.field_adjoint_device(size, axes, energy, grad, stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ranks.barrier()
    with ClockSampler(local_rank) as clocks:
        ms_total = timed_region(step, args.steps, stream)
    ms_total = ranks.max_over_ranks(ms_total, device)
    ms_step = ms_total / args.steps
    value = world * poses * args.steps / (ms_total * 1e-3)
    achieved = pairs * FLOP_FWD_ADJ / (ms_step * 1e-3)

    # ---- e2e through the public host entry (vext_field_adjoint): directors
    # up, float32 energy + gradient down into pinned host buffers, every call
    h_energy = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    h_grad = torch.empty(shape + (6,), dtype=torch.float32, pin_memory=True)
    lib = _lib.load()
    opt = _lib.options()

    def e2e_call():
        _lib.check(lib.vext_field_adjoint(system.handle, size, n_axes, _lib.ptr(axes),
                                          ctypes.byref(opt), _lib.ptr(h_energy),
                                          _lib.ptr(h_grad)))

    e2e_call()
    e2e_times = []
    for _ in range(max(3, min(args.steps, 10))):
        t0 = time.perf_counter()
        e2e_call()
        e2e_times.append(time.perf_counter() - t0)
    e2e_value = world * poses / statistics.median(e2e_times)
    h2d, d2h = axes.nbytes, h_energy.numel() * 4 + h_grad.numel() * 4
    del h_energy, h_grad

    extra = {}
    if rank == 0:
        extra["e2e_cold"] = e2e_cold_field(case, size, axes)
        extra.update(secondary_measurements(args, system, case, size, axes, poses, pairs,
                                            far_pairs, peak, stream, device, ms_step, energy,
                                            grad))
    ranks.barrier()
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu:
        cpu = cpu_reference_sample(case, size, n_axes, args.cpu_seconds, host_cores())
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        extra["cpu_baseline_single_core"] = cpu_reference_single_core(case, size, n_axes, 5.0)
    line = {"metric": METRIC, "value": value, "unit": "poses/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32x2+f64 (pairs < 5 A in FP64, beyond in packed FP32 with FP64-flushed "
                     "partial sums; FP64 energy refinement band; FP64 re-evaluation of poses "
                     "with a shell pair within the FP32 error of the cutoff)",
            "data": "synthetic", "config": config_of(args.workload, size),
            "step": "forward + adjoint of every pose: energy, dE/d(center), tangent dE/du; "
                    "region lists resident (built once per framework, reported as setup)",
            "e2e": {"value": e2e_value, "unit": "poses/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h,
                    "path": "vext_field_adjoint into page-locked host float32 energy + "
                            "gradient (the kernels write them over PCIe during the pair "
                            "work)"},
            "gpu_launches": args.steps * 2,
            "setup_s": setup_s,
            "roofline": {"bound": "fp32",
                         "kernel": "batch_field_kernel<adjoint> (fused FP64 near + FP32x2 far, autotuned shape)",
                         "achieved": achieved / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         "peak_source": "measured on this GPU: max(FFMA, FFMA2) FMA rate x 2 "
                                        "(vext_measure_pipes); MEASURED_PEAKS.json has no FP32 "
                                        "figure",
                         "algorithmic": f"{pairs} in-cutoff pairs x {FLOP_FWD_ADJ} FLOP "
                                        "(forward + adjoint) per field",
                         "traffic": (ADJ_DRAM_BYTES_FULL_FIELD
                                     if args.workload == "full_field" else None),
                         "traffic_unit": "bytes per launch (ncu dram__bytes_read+write)",
                         "bound_note": "non-tensor FP32 SIMT pipe: pairwise LJ is not a dense "
                                       "contraction, so neither the HBM nor the tensor-core "
                                       "roofline applies; see hbm_check",
                         "hbm_check": hbm_check(ADJ_DRAM_BYTES_FULL_FIELD
                                                if args.workload == "full_field" else None,
                                                ms_step),
                         "pipes": pipes},
            "clocks": clocks.summary(), "cpu_baseline": cpu}
    # the numbers the secondary measurements support, also inside the standard
    # keys (records that keep only those keys still carry them)
    if "e2e_cold" in extra:
        line["e2e"]["cold"] = {k: extra["e2e_cold"][k] for k in
                               ("value", "seconds", "value_tuned_afresh", "seconds_tuned_afresh")}
    vs = {k: extra[k] for k in ("speedup_fwd_adjoint_vs_fp64_tiled_fwd_adjoint",
                                "speedup_fwd_adjoint_vs_fp64_plain_fwd_adjoint",
                                "speedup_fwd_adjoint_vs_fp64_plain_forward",
                                "speedup_fwd_adjoint_vs_fp64_tiled_forward") if k in extra}
    if "error_vs_fp64" in extra:
        vs.update({f"error_{k}": extra["error_vs_fp64"][k] for k in
                   ("max_abs_K_E_le_0", "max_rel_E_gt_0", "gradient_max_rel", "passed")})
    line["roofline"]["vs_fp64"] = vs
    line.update(extra)
    print(json.dumps(line))


def e2e_cold_field(case, size, axes):
    """One-shot cost of a field: a fresh system (framework upload, type
    tables), then vext_field_adjoint into page-locked host memory -- region
    lists, the batch's autotuning, graph capture, pair work, results in host
    memory -- by the host clock from before the system exists.  Measured
    with the autotuner timing its candidates afresh (the cost of the first
    field of its size class in a process) and with the pick of the
    process-wide tuning cache (every later field of that class); the median
    of three runs of each."""
    import torch
    from string_vext_b200 import _lib
    from string_vext_b200.system import VextSystem
    n_axes = len(axes)
    shape = (n_axes, size, size, size)
    h_energy = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    h_grad = torch.empty(shape + (6,), dtype=torch.float32, pin_memory=True)
    lib = _lib.load()
    runs = {"tuned_afresh": [], "tuning_cached": []}
    for _ in range(3):   # the median of three: device-memory set-up and release vary a lot
        for label, variant in (("tuned_afresh", 2048), ("tuning_cached", 0)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            system = VextSystem(case)
            opt = _lib.options(variant=variant)
            _lib.check(lib.vext_field_adjoint(system.handle, size, n_axes, _lib.ptr(axes),
                                              ctypes.byref(opt), _lib.ptr(h_energy),
                                              _lib.ptr(h_grad)))
            runs[label].append(time.perf_counter() - t0)
            system.close()
    out = {k: float(np.median(v)) for k, v in runs.items()}
    poses = size ** 3 * n_axes
    return {"value": poses / out["tuning_cached"], "unit": "poses/s",
            "seconds": out["tuning_cached"], "seconds_tuned_afresh": out["tuned_afresh"],
            "value_tuned_afresh": poses / out["tuned_afresh"],
            "runs_s": {k: [round(x, 4) for x in v] for k, v in runs.items()},
            "h2d_bytes": axes.nbytes, "d2h_bytes": h_energy.numel() * 4 + h_grad.numel() * 4,
            "path": "fresh VextSystem -> vext_field_adjoint into page-locked host memory "
                    "(region lists, autotune pick, graph capture, pair work, results in host "
                    "memory); host clock"}


def secondary_measurements(args, system, case, size, axes, poses, pairs, far_pairs, peak,
                           stream, device, ms_adj, energy, grad):
    """Forward-only field, FP64 baselines, error against FP64, pose path and
    the 100-field batches (rank 0)."""
    import torch
    from string_vext_b200 import _lib
    n_axes = len(axes)
    shape = (n_axes, size, size, size)
    out = {}
    # forward only: per-field near/far kernels, region lists rebuilt every step
    fwd_out = torch.empty(shape, dtype=torch.float32, device=device)
    timings = []

    def fwd_step():
        system.invalidate()
        system.field_device(size, axes, fwd_out, stream=stream)
        timings.append(system.last_timings())

    for _ in range(args.warmup):
        fwd_step()
    timings.clear()
    n_fwd = max(3, min(args.steps, 10))
    fwd_ms = timed_region(fwd_step, n_fwd, stream) / n_fwd
    near_ms = statistics.mean(t["near_ms"] for t in timings)
    far_ms = statistics.mean(t["far_ms"] for t in timings)
    list_ms = statistics.mean(t["list_ms"] for t in timings)
    epi_ms = statistics.mean(t["epilogue_ms"] for t in timings)
    achieved_far = far_pairs * FLOP_FWD / (far_ms * 1e-3)
    out["forward"] = {
        "value": poses / (fwd_ms * 1e-3), "unit": "poses/s", "ms_per_field": fwd_ms,
        "step": "region-list build + near (FP64) + far (FP32x2) kernels + refinement + "
                "float32 epilogue",
        "breakdown_ms": {"list_build": list_ms, "near_pairs_fp64": near_ms,
                         "far_pairs_fp32x2": far_ms, "refine_epilogue": epi_ms},
        "roofline_far_kernel": {"kernel": "field_far2_kernel<16,8,4,6>", "bound": "fp32",
                                "achieved": achieved_far / 1e12, "peak": peak / 1e12,
                                "unit": "TFLOP/s", "frac": achieved_far / peak,
                                "algorithmic": f"{far_pairs} far in-cutoff pairs x {FLOP_FWD} FLOP",
                                "traffic": (FAR_DRAM_BYTES_FULL_FIELD
                                            if args.workload == "full_field" else None)}}
    del fwd_out
    # FP64 GPU baselines, one field per launch
    e64 = torch.empty(shape, dtype=torch.float64, device=device)
    g64 = torch.empty(shape + (6,), dtype=torch.float64, device=device)

    def plain_adj():
        system.field_adjoint_device(size, axes, None, None, e64, g64,
                                    mode=_lib.VEXT_MODE_FP64_PLAIN, stream=stream)

    plain_adj()
    plain_adj_ms = timed_region(plain_adj, 1, stream)
    fp64 = {"fp64_plain_fwd_adjoint": {"value": poses / (plain_adj_ms * 1e-3),
                                       "unit": "poses/s", "ms_per_field": plain_adj_ms}}
    for label, mode in (("fp64_tiled_forward", _lib.VEXT_MODE_FP64),
                        ("fp64_plain_forward", _lib.VEXT_MODE_FP64_PLAIN)):
        times = []
        for _ in range(2):
            system.invalidate()
            torch.cuda.synchronize()
            system.field(size, axes, mode=mode, orientation=False)
            st = system.last_stats
            times.append(st["kernel_ms"] + st["list_build_ms"] + st["epilogue_ms"])
        fp64[label] = {"value": poses / (min(times) * 1e-3), "unit": "poses/s",
                       "ms_per_field": min(times)}
    # the same tiled forward + adjoint batch kernel with every pair in FP64
    # (r_split beyond the cutoff: every list entry is near)
    from string_vext_b200.system import VextBatch
    e32 = torch.empty(shape, dtype=torch.float32, device=device)
    g32 = torch.empty(shape + (6,), dtype=torch.float32, device=device)
    tiled = VextBatch([system], size, axes, [e32], gradients=[g32], r_split=1e3)
    tiled.run(stream)
    tiled_adj_ms = timed_region(lambda: tiled.run(stream), 3, stream) / 3
    tiled.close()
    del e32, g32
    fp64["fp64_tiled_fwd_adjoint"] = {"value": poses / (tiled_adj_ms * 1e-3), "unit": "poses/s",
                                      "ms_per_field": tiled_adj_ms,
                                      "kernel": "the headline batch kernel with r_split beyond "
                                                "the cutoff (every pair in FP64)"}
    out["fp64_kernels"] = fp64
    out["speedup_fwd_adjoint_vs_fp64_tiled_fwd_adjoint"] = tiled_adj_ms / ms_adj
    out["speedup_fwd_adjoint_vs_fp64_plain_fwd_adjoint"] = plain_adj_ms / ms_adj
    out["speedup_fwd_adjoint_vs_fp64_plain_forward"] = (fp64["fp64_plain_forward"]["ms_per_field"]
                                                        / ms_adj)
    out["speedup_forward_vs_fp64_plain_forward"] = (fp64["fp64_plain_forward"]["ms_per_field"]
                                                    / fwd_ms)
    out["speedup_fwd_adjoint_vs_fp64_tiled_forward"] = (fp64["fp64_tiled_forward"]["ms_per_field"]
                                                        / ms_adj)
    # error of the headline result against the plain FP64 forward + adjoint
    e_mixed64 = torch.empty(shape, dtype=torch.float64, device=device)
    system.field_adjoint_device(size, axes, energy, grad, e_mixed64, stream=stream)
    torch.cuda.synchronize()
    exact = e64.cpu().numpy()
    err = error_stats(e_mixed64.cpu().numpy(), exact)
    gx = g64.cpu().numpy()
    gm = grad.cpu().numpy().astype(np.float64)
    grel = np.linalg.norm(gm - gx, axis=-1) / np.maximum(np.linalg.norm(gx, axis=-1), 1.0)
    err["gradient_max_rel"] = float(grel.max())
    err["gradient_median_rel"] = float(np.median(grel))
    err["reference"] = "plain FP64 kernel (IEEE division) on the same poses"
    out["error_vs_fp64"] = err
    del e64, g64, e_mixed64, exact, gx, gm, grel
    torch.cuda.empty_cache()
    system.field(size, axes, orientation=False)
    out["list_entries"] = system.last_stats["list_entries"]
    out["near_entries"] = system.last_stats["near_entries"]
    out["refined_poses_forward"] = system.last_stats["refined_poses"]
    # forward + adjoint on a random pose batch of the same framework (pose path)
    n_pose = 1 << 20
    rng = np.random.default_rng(9)
    cart = torch.tensor(rng.random((n_pose, 3)) @ case["cell"], device=device)
    q = torch.tensor(rng.normal(size=(n_pose, 4)), device=device)
    e = torch.empty(n_pose, dtype=torch.float64, device=device)
    gc = torch.empty((n_pose, 3), dtype=torch.float64, device=device)
    gq = torch.empty((n_pose, 4), dtype=torch.float64, device=device)

    def pose_step():
        system.pose_energy_grad_device(cart, q, e, gc, gq, stream=stream)

    pose_step()
    pose_ms = timed_region(pose_step, 5, stream) / 5
    out["pose_fwd_adjoint"] = {"value": n_pose / (pose_ms * 1e-3), "unit": "poses/s",
                               "poses": n_pose, "workload": "random poses (center, quaternion), "
                               "same framework", "flop_per_pair": FLOP_FWD_ADJ}
    # error of the pose path against its FP64 mode on the same poses
    e64p, gc64, gq64 = torch.empty_like(e), torch.empty_like(gc), torch.empty_like(gq)
    system.pose_energy_grad_device(cart, q, e64p, gc64, gq64, mode=_lib.VEXT_MODE_FP64,
                                   stream=stream)
    torch.cuda.synchronize()
    perr = error_stats(e.cpu().numpy(), e64p.cpu().numpy())
    for name, mixed, exact in (("center", gc, gc64), ("quaternion", gq, gq64)):
        gx, gm = exact.cpu().numpy(), mixed.cpu().numpy()
        grel = np.linalg.norm(gm - gx, axis=-1) / np.maximum(np.linalg.norm(gx, axis=-1), 1.0)
        perr[f"gradient_{name}_max_rel"] = float(grel.max())
        perr[f"gradient_{name}_median_rel"] = float(np.median(grel))
    perr["reference"] = ("the pose path's FP64 mode (every pair in FP64, correctly rounded "
                         "reciprocal) on the same poses")
    out["pose_fwd_adjoint"]["error_vs_fp64"] = perr
    del cart, q, e, gc, gq, e64p, gc64, gq64
    out["precision_study"] = precision_study(device)
    out["string_update"] = bench_string_update()
    out["dropin"] = bench_dropin(case, size, axes)
    if not args.no_batch:
        out["batch"] = bench_batch(args, size, axes, device, stream, adjoint=False)
        out["batch_fwd_adjoint"] = bench_batch(args, size, axes, device, stream, adjoint=True)
        out["string_batch_fwd_adjoint"] = bench_string_batch(device, stream)
    return out


def precision_study(device):
    """The precision study: naive FP32, FP32 compensated throughout (every pair
    beyond 1 A in packed FP32 with FP64-flushed partials, no FP64 band) and the
    default mixed field, each against the tiled FP64 oracle kernel, on
    skewed_field (28 x 31 x 24 A, alpha/beta/gamma 75/85/110, 3000 atoms,
    60^3 x 64: every pose has E > 0) and small_field (20^3 x 64: the workload
    with E <= 0 poses)."""
    from string_vext_b200 import _lib, synth
    from string_vext_b200.orientation import normalized_directors, regular_pose_grid
    from string_vext_b200.system import VextSystem
    out = {}
    for name, maker, size in (("skewed_field", synth.skewed_field, 60),
                              ("small_field", synth.small_field, 20)):
        _, axes = regular_pose_grid(size, 64)
        axes = normalized_directors(axes)
        res = {"workload": f"{name}: {size}^3 x 64"}
        with VextSystem(maker()) as system:
            exact = system.field(size, axes, mode=_lib.VEXT_MODE_FP64, energy=True,
                                 orientation=False)["energy"]
            res["fp64_oracle_ms"] = system.last_stats["kernel_ms"]
            for label, mode, opts in (
                    ("fp32_naive", _lib.VEXT_MODE_FP32_NAIVE, {}),
                    ("fp32_compensated", _lib.VEXT_MODE_MIXED,
                     {"r_split": 1.0, "band": (0.0, 0.0)}),
                    ("mixed_default", _lib.VEXT_MODE_MIXED, {})):
                got = system.field(size, axes, mode=mode, energy=True, orientation=False,
                                   **opts)["energy"]
                stats = error_stats(got, exact)
                stats["kernel_ms"] = system.last_stats["kernel_ms"]
                res[label] = stats
        out[name] = res
    return out


def bench_string_update():
    """The GPU String update on the config-4 path (small_field framework,
    64 images along c from (0.25, 0.25, 0) to (0.25, 0.25, 1), seed-3
    quaternions): 200 iterations with forces, step, end fixing,
    reparametrisation, smoothing and the convergence test (vext_string_run)."""
    from string_vext_b200 import synth
    from string_vext_b200.string_path import euler_from_quaternions, run_string
    from string_vext_b200.system import VextSystem
    case, frac, quat, _, _ = synth.string_path()
    path = np.column_stack([frac, np.mod(euler_from_quaternions(quat), 2 * np.pi)])
    with VextSystem(case) as system:
        run_string(system, path, direction=3, max_iterations=2)       # lists, scratch
        t0 = time.perf_counter()
        _, _, res = run_string(system, path, direction=3, max_iterations=200)
        wall = time.perf_counter() - t0
    return {"iterations": res["iterations"], "images": len(path), "seconds": wall,
            "ms_per_iteration": 1e3 * wall / max(res["iterations"], 1),
            "workload": "config-4 path, 64 images, 200 iterations, host wall time of "
                        "vext_string_run (graph-replayed iterations)"}


def reference_package_driver():
    """``NativeReusePotential`` of the reference package installed unchanged in
    baseline/_ref (pip --target), or None when it is not installed."""
    package = ROOT / "baseline" / "_ref"
    if not (package / "string_vext" / "native.py").exists():
        return None
    if str(package) not in sys.path:
        sys.path.append(str(package))
    from string_vext.native import NativeReusePotential
    return NativeReusePotential


def bench_dropin(case, size, axes):
    """The drop-in mode: the reference's own, unmodified driver (its package
    installed in baseline/_ref: host kd-tree query and CSR per 512-center
    batch, one process) calling this library's evaluate_reused_neighbors, on
    the strided center sample of cpu_baseline_single_core.  Poses/s with the
    host query and for the library calls alone (host buffers in and out)."""
    from string_vext_b200 import _lib
    from string_vext_b200.orientation import regular_pose_grid
    driver_class = reference_package_driver()
    if driver_class is None:
        return {"unavailable": "reference package not installed in baseline/_ref"}
    centers, _ = regular_pose_grid(size, len(axes))
    n_sample = int(min(len(centers), max(512, CPU_CENTERS_PER_CORE_S * 5.0)))
    stride = max(1, len(centers) // n_sample)
    sample = centers[::stride][:n_sample]
    pot = driver_class(case, _lib.LIB_PATH)
    pot.evaluate(sample[:512], axes)          # device buffers and context
    # three passes over the sample, the median reported (single passes on one
    # box took 0.02-1.5 s in the library calls for the same work)
    runs = []
    for _ in range(3):
        pot.query_seconds = pot.compute_seconds = 0.0
        t0 = time.perf_counter()
        pot.evaluate(sample, axes)
        runs.append((time.perf_counter() - t0, pot.query_seconds, pot.compute_seconds))
    wall, query_s, calls_s = (statistics.median(r[k] for r in runs) for k in range(3))
    poses = len(sample) * len(axes)
    return {"value": poses / wall, "unit": "poses/s",
            "library_calls_only": poses / calls_s,
            "query_share": query_s / wall,
            "library_calls_s_runs": [round(r[2], 4) for r in runs],
            "sample": f"{len(sample)} of {len(centers)} grid centers (stride {stride}) x "
                      f"{len(axes)} directors, one process, median of 3 passes; {wall:.2f} s, "
                      f"kd-tree query {query_s:.2f} s, library calls {calls_s:.2f} s",
            "path": "reference driver from baseline/_ref (kd-tree + CSR on the host) -> "
                    "evaluate_reused_neighbors of this library (FP64, bit-identical to the "
                    "reference kernel)"}


def bench_string_batch(device, stream):
    """Forward + adjoint of 100 String paths (32-96 images, one per framework x
    guest of the batched workload) in one launch (vext_pose_batch_run)."""
    import torch
    from string_vext_b200 import synth
    from string_vext_b200.system import VextPoseBatch, VextSystem
    cases = synth.batch_frameworks()
    paths = synth.string_paths_batch(cases, n_paths=len(cases))
    centers = np.concatenate([f @ np.asarray(cases[k]["cell"], dtype=float) for k, f, _ in paths])
    quats = np.concatenate([q for _, _, q in paths])
    counts = [len(f) for _, f, _ in paths]          # path p belongs to system p
    t0 = time.perf_counter()
    systems = [VextSystem(c) for c in cases]
    batch = VextPoseBatch(systems, counts)
    setup_s = time.perf_counter() - t0
    dev = dict(dtype=torch.float64, device=device)
    n = len(centers)
    c, q = torch.tensor(centers, **dev), torch.tensor(quats, **dev)
    e, gc, gq = torch.empty(n, **dev), torch.empty((n, 3), **dev), torch.empty((n, 4), **dev)

    def step():
        batch.run(c, q, e, gc, gq, stream=stream)

    for _ in range(3):
        step()
    reps = 20
    ms = timed_region(step, reps, stream) / reps
    batch.check()
    result = {"value": n / (ms * 1e-3), "unit": "poses/s", "ms_per_batch": ms, "paths": len(paths),
              "poses": n, "systems": len(systems), "setup_s": setup_s,
              "workload": "100 seeded String paths (32-96 images, random quaternions) over "
                          "50 frameworks x 2 guests, one launch per evaluation"}
    batch.close()
    for s_ in systems:
        s_.close()
    return result


def bench_batch(args, size, axes, device, stream, adjoint=False):
    """The batched workload: 50 seeded frameworks x 2 guests = 100 fields of
    size^3 x 64 in one persistent, graph-captured launch (autotuned);
    forward only, or forward + adjoint (energy and 6 gradient components)."""
    import torch
    from string_vext_b200 import synth
    from string_vext_b200.system import VextBatch, VextSystem
    t0 = time.perf_counter()
    systems = [VextSystem(c) for c in synth.batch_frameworks()]
    t_sys = time.perf_counter()
    shape = (len(axes), size, size, size)
    outs = [torch.empty(shape, dtype=torch.float32, device=device) for _ in systems]
    grads = ([torch.empty(shape + (6,), dtype=torch.float32, device=device) for _ in systems]
             if adjoint else None)
    torch.cuda.synchronize()
    t_out = time.perf_counter()
    batch = VextBatch(systems, size, axes, outs, gradients=grads)
    t_batch = time.perf_counter()
    setup_s = t_batch - t_out   # region lists, work queue, autotuning, graph capture
    info = batch.info()
    t1 = time.perf_counter()
    batch.run(stream)
    torch.cuda.synchronize()
    first_run_s = time.perf_counter() - t1
    for _ in range(max(0, args.warmup // 2 - 1)):
        batch.run(stream)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    a.record(stream)
    for _ in range(reps):
        batch.run(stream)
    b.record(stream)
    torch.cuda.synchronize()
    batch.check()
    ms = a.elapsed_time(b) / reps
    result = {"value": info["poses"] / (ms * 1e-3), "unit": "poses/s", "ms_per_batch": ms,
              "fields": len(systems), "poses": info["poses"], "work_items": info["work_items"],
              "list_gb": info["list_bytes"] / 1e9, "setup_s": setup_s,
              "setup_parts_s": {"systems": t_sys - t0, "outputs": t_out - t_sys,
                                "batch": setup_s},
              "cold": {"value": info["poses"] / (t_batch - t0 + first_run_s), "unit": "poses/s",
                       "seconds": t_batch - t0 + first_run_s,
                       "path": "systems created, region lists (one set per framework, shared "
                               "by its two guests), autotuning, graph capture and the first "
                               "replay; outputs on the device; host clock"},
              "autotuned": {"cta_shape": info["cta_shape"], "resident_ctas": info["grid"]},
              "workload": "50 seeded frameworks x 2 guests, one graph launch",
              "step": "forward + adjoint" if adjoint else "forward"}
    batch.close()
    for s_ in systems:
        s_.close()
    del outs, grads
    torch.cuda.empty_cache()
    return result


def run_profile_case(kind, batch_shape=0):
    """Short, fixed cases for ncu (no timing is reported from them)."""
    import torch
    from string_vext_b200 import synth
    from string_vext_b200.orientation import normalized_directors, regular_pose_grid
    from string_vext_b200.system import VextSystem
    case = synth.full_field()
    with VextSystem(case) as system:
        _, axes = regular_pose_grid(60, 64)
        axes = normalized_directors(axes)
        if kind == "field":
            for _ in range(2):
                system.field(60, axes, orientation=False)
        elif kind == "adjoint":
            e = torch.empty((64, 60, 60, 60), dtype=torch.float32, device="cuda")
            g = torch.empty((64, 60, 60, 60, 6), dtype=torch.float32, device="cuda")
            for _ in range(2):
                system.field_adjoint_device(60, axes, e, g, batch_shape=batch_shape)
            torch.cuda.synchronize()
        else:
            n = 1 << 20
            rng = np.random.default_rng(9)
            cart = torch.tensor(rng.random((n, 3)) @ case["cell"], device="cuda")
            q = torch.tensor(rng.normal(size=(n, 4)), device="cuda")
            e = torch.empty(n, dtype=torch.float64, device="cuda")
            gc = torch.empty((n, 3), dtype=torch.float64, device="cuda")
            gq = torch.empty((n, 4), dtype=torch.float64, device="cuda")
            for _ in range(2):
                system.pose_energy_grad_device(cart, q, e, gc, gq)
            torch.cuda.synchronize()
    print(f"profile case {kind} done")


def main():
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=30)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--workload", default="full_field",
                        choices=("full_field", "small_field", "skewed_field"))
    parser.add_argument("--cpu-seconds", type=float, default=15.0,
                        help="target length of the CPU-baseline sample")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    parser.add_argument("--no-batch", action="store_true", help="skip the 100-field batch")
    parser.add_argument("--profile", choices=("field", "adjoint", "pose"),
                        help="run one short case for an ncu capture and exit: 'field' = two "
                             "mixed full_field fields (forward), 'adjoint' = two forward + "
                             "adjoint full_field fields (the first builds, autotunes and "
                             "captures), 'pose' = two 2^20-pose forward+adjoint batches of the "
                             "same framework")
    parser.add_argument("--batch-shape", type=int, default=0,
                        help="with --profile adjoint: 1 + the index of the CTA shape to run "
                             "instead of the autotuner's pick (one launch per call, no tuning "
                             "launches)")
    args = parser.parse_args()
    ensure_built()
    if args.profile:
        run_profile_case(args.profile, args.batch_shape)
        return
    rank, world, local_rank = ranks.rank_info()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        ranks.init("nccl", local_rank)
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
