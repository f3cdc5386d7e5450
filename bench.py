"""Benchmark: Vext pose evaluations/s on the full-size field workload.

Workload (default ``full_field``): 37 x 37 x 3.6 A layered cell (gamma
119.993), 600 seeded synthetic atoms, two-site guest 85 K / 3.685 A / bond
1.33 A, cutoff 12.8 A, 60^3 grid x 64 Fibonacci directors = 13,824,000 poses
per field.  One step = one complete field: region-list build + pair kernel +
FP64 refinement + float32 epilogue, inputs resident in HBM.

Our arm prints one JSON line with: value (poses/s over all ranks, device time
from CUDA events, max over ranks), e2e (the public host C-ABI call:
system upload + field + float32 download), roofline of the pair kernel
against the measured FP32 FFMA peak of this GPU, the FP64 GPU oracle kernel's
throughput and the error of the mixed-precision result against it, the
forward+adjoint pose throughput, clocks sampled during the timed region, and
a CPU baseline (the reference kernel compiled from its source, driven by the
restated reference driver, on a bounded sample of the same field).

``--impl reference`` times that reference CPU path alone (all host cores,
rank 0 only) on the same metric.
"""
from __future__ import annotations

import argparse
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

FLOP_FWD = 16          # algorithmic FLOP per in-cutoff (site, image) pair, forward
FLOP_FWD_ADJ = 28      # forward + adjoint
METRIC = "Vext pose evals/s at <=1e-4 K vs FP64, fwd+adjoint evals/s; % FP32 peak"
# dram__bytes_read.sum + dram__bytes_write.sum of one field_far_kernel launch on
# full_field, from an ncu capture (--set full) of `bench.py --profile field`.
FAR_DRAM_BYTES_FULL_FIELD = 741_898_752 + 101_475_584
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
    """nvidia-smi clocks/throttle reasons of one GPU every 200 ms."""
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
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
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
    energy, wall, used = oracle.reference_field_parallel(case, sample, axes, library=library,
                                                         processes=processes, symbol=symbol)
    poses = len(sample) * n_axes
    return {"value": poses / wall, "unit": "poses/s", "cores": used, "kind": kind,
            "sample": f"{len(sample)} of {len(centers)} grid centers (stride {stride}) x "
                      f"{n_axes} directors, {processes} spawn processes, kd-tree query + "
                      f"kernel, {cpu_model()}",
            "seconds": wall, "poses": poses}


def run_reference(args, rank, world):
    if rank != 0:
        return
    case, size = workload(args.workload)
    cores = host_cores()
    values = []
    for step in range(args.warmup + args.steps):
        res = cpu_reference_sample(case, size, 64, args.cpu_seconds, cores)
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


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
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
    stream = torch.cuda.Stream(device)
    out = torch.empty((n_axes, size, size, size), dtype=torch.float32, device=device)
    system = VextSystem(case)

    pairs, far_pairs = system.count_pairs(size, axes)
    pipes = _lib.measure_pipes()
    peak = 2.0 * max(pipes["ffma_per_s"], pipes["ffma2_fma_per_s"])   # FLOP/s, FMA = 2

    def step():
        system.invalidate()
        system.field_device(size, axes, out, stream=stream)
        return system.last_timings()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    timings = []
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(args.steps):
            timings.append(step())
        stop.record(stream)
        torch.cuda.synchronize()
    ms_total = start.elapsed_time(stop)
    if world > 1:
        t = torch.tensor([ms_total], device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    value = world * poses * args.steps / (ms_total * 1e-3)
    near_ms = statistics.mean(t["near_ms"] for t in timings)
    far_ms = statistics.mean(t["far_ms"] for t in timings)
    list_ms = statistics.mean(t["list_ms"] for t in timings)
    epi_ms = statistics.mean(t["epilogue_ms"] for t in timings)
    achieved_far = far_pairs * FLOP_FWD / (far_ms * 1e-3)
    achieved_pairs = pairs * FLOP_FWD / ((near_ms + far_ms) * 1e-3)

    # e2e through the public host API: system upload + field + float32 download
    e2e_times = []
    h2d = d2h = 0
    for i in range(max(2, args.steps // 2) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with VextSystem(case) as sys_e2e:
            res = sys_e2e.field(size, axes)
        dt = time.perf_counter() - t0
        if i:
            e2e_times.append(dt)
        h2d = (case["frame_frac"].nbytes + case["frame_sigma"].nbytes
               + case["frame_epsilon"].nbytes + axes.nbytes + 9 * 8)
        d2h = res["orientation_K"].nbytes
    e2e_value = world * poses / statistics.median(e2e_times)

    extra = {}
    if rank == 0:
        # FP64 GPU kernels: the tiled FP64 oracle kernel and the plain
        # one-thread-per-pose FP64 baseline (both one field per launch)
        exact = system.field(size, axes, mode=_lib.VEXT_MODE_FP64, energy=True,
                             orientation=False)["energy"]
        fp64 = {}
        for label, mode in (("fp64_tiled", _lib.VEXT_MODE_FP64),
                            ("fp64_plain", _lib.VEXT_MODE_FP64_PLAIN)):
            times = []
            for _ in range(2):
                system.invalidate()
                torch.cuda.synchronize()
                system.field(size, axes, mode=mode, orientation=False)
                st = system.last_stats
                times.append(st["kernel_ms"] + st["list_build_ms"] + st["epilogue_ms"])
            fp64[label] = {"value": poses / (min(times) * 1e-3), "unit": "poses/s",
                           "ms_per_field": min(times)}
        extra["fp64_kernels"] = fp64
        extra["speedup_vs_fp64_plain"] = fp64["fp64_plain"]["ms_per_field"] / ms_step
        extra["speedup_vs_fp64_tiled"] = fp64["fp64_tiled"]["ms_per_field"] / ms_step
        mixed = system.field(size, axes, energy=True, orientation=False)
        stats = system.last_stats
        extra["error_vs_fp64"] = error_stats(mixed["energy"], exact)
        extra["refined_poses"] = stats["refined_poses"]
        extra["list_entries"] = stats["list_entries"]
        extra["near_entries"] = stats["near_entries"]
        del exact, mixed
        # forward + adjoint on a random pose batch of the same framework
        n_pose = 1 << 20
        rng = np.random.default_rng(9)
        cart = torch.tensor(rng.random((n_pose, 3)) @ case["cell"], device=device)
        q = torch.tensor(rng.normal(size=(n_pose, 4)), device=device)
        e = torch.empty(n_pose, dtype=torch.float64, device=device)
        gc = torch.empty((n_pose, 3), dtype=torch.float64, device=device)
        gq = torch.empty((n_pose, 4), dtype=torch.float64, device=device)
        for _ in range(2):
            system.pose_energy_grad_device(cart, q, e, gc, gq, stream=stream)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        reps = 3
        for _ in range(reps):
            system.pose_energy_grad_device(cart, q, e, gc, gq, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        adj_ms = a.elapsed_time(b) / reps
        extra["fwd_adjoint"] = {"value": n_pose / (adj_ms * 1e-3), "unit": "poses/s",
                                "poses": n_pose, "workload": "random poses, same framework",
                                "flop_per_pair": FLOP_FWD_ADJ}
        del cart, q, e, gc, gq
        if not args.no_batch:
            extra["batch"] = bench_batch(args, size, axes, device, stream)
    if world > 1:
        dist.barrier()
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu:
        cpu = cpu_reference_sample(case, size, n_axes, args.cpu_seconds, host_cores())
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    clock = clocks.summary()
    line = {"metric": METRIC, "value": value, "unit": "poses/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32x2+f64 (pairs < 6 A in FP64, beyond in packed FP32, FP64 refinement band)",
            "data": "synthetic", "config": config_of(args.workload, size),
            "e2e": {"value": e2e_value, "unit": "poses/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "path": "vext_system_create + vext_field "
                    "(host buffers) + vext_system_destroy"},
            "gpu_launches": args.steps * 7,
            "step_breakdown_ms": {"list_build": list_ms, "near_pairs_fp64": near_ms,
                                  "far_pairs_fp32x2": far_ms, "refine_epilogue": epi_ms},
            "roofline": {"bound": "fp32", "kernel": "field_far_kernel<16,8,4,4> (default variant)",
                         "achieved": achieved_far / 1e12, "peak": peak / 1e12, "unit": "TFLOP/s",
                         "frac": achieved_far / peak,
                         "peak_source": "measured on this GPU: max(FFMA, FFMA2) FMA rate x 2 "
                                        "(vext_measure_pipes); MEASURED_PEAKS.json has no FP32 figure",
                         "algorithmic": f"{far_pairs} far in-cutoff pairs x {FLOP_FWD} FLOP per field",
                         "traffic": (FAR_DRAM_BYTES_FULL_FIELD
                                     if args.workload == "full_field" else None),
                         "traffic_unit": "bytes per launch (ncu dram__bytes_read+write)",
                         "both_pair_kernels": {"achieved": achieved_pairs / 1e12,
                                               "frac": achieved_pairs / peak,
                                               "algorithmic": f"{pairs} in-cutoff pairs x {FLOP_FWD} FLOP"},
                         "pipes": pipes},
            "clocks": clock, "cpu_baseline": cpu}
    line.update(extra)
    print(json.dumps(line))


def bench_batch(args, size, axes, device, stream):
    """The batched workload: 50 seeded frameworks x 2 guests = 100 fields of
    size^3 x 64 in one persistent, graph-captured launch (autotuned)."""
    import torch
    from string_vext_b200 import synth
    from string_vext_b200.system import VextBatch, VextSystem
    t0 = time.perf_counter()
    systems = [VextSystem(c) for c in synth.batch_frameworks()]
    outs = [torch.empty((len(axes), size, size, size), dtype=torch.float32, device=device)
            for _ in systems]
    batch = VextBatch(systems, size, axes, outs)
    setup_s = time.perf_counter() - t0
    info = batch.info()
    for _ in range(max(1, args.warmup // 2)):
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
              "autotuned": {"cta_shape": ["128x4 dirs", "256x2 dirs"][info["shape"]],
                            "resident_ctas": info["grid"]},
              "workload": "50 seeded frameworks x 2 guests, one graph launch"}
    batch.close()
    for s_ in systems:
        s_.close()
    del outs
    torch.cuda.empty_cache()
    return result


def run_profile_case(kind):
    """Short, fixed cases for ncu (no timing is reported from them)."""
    import torch
    from string_vext_b200 import synth
    from string_vext_b200.orientation import normalized_directors, regular_pose_grid
    from string_vext_b200.system import VextSystem
    case = synth.full_field()
    with VextSystem(case) as system:
        if kind == "field":
            _, axes = regular_pose_grid(60, 64)
            axes = normalized_directors(axes)
            for _ in range(2):
                system.field(60, axes, orientation=False)
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
    parser.add_argument("--steps", type=int, default=5)
    parser.add_argument("--warmup", type=int, default=3)
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--workload", default="full_field",
                        choices=("full_field", "small_field", "skewed_field"))
    parser.add_argument("--cpu-seconds", type=float, default=15.0,
                        help="target length of the CPU-baseline sample")
    parser.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    parser.add_argument("--no-batch", action="store_true", help="skip the 100-field batch")
    parser.add_argument("--profile", choices=("field", "pose"),
                        help="run one short case for an ncu capture and exit: 'field' = two "
                             "mixed full_field fields, 'pose' = two 2^20-pose forward+adjoint "
                             "batches of the same framework")
    args = parser.parse_args()
    ensure_built()
    if args.profile:
        run_profile_case(args.profile)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
