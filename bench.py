#!/usr/bin/env python
"""Benchmark of the path-tracing hot path: Mpaths/s on B200.

One step renders one full frame of the workload (default: the random-spheres field,
1920x1080, 256 spp, depth 16) with the megakernel, scene resident in HBM.  Prints ONE JSON
line on rank 0.  Under torchrun each rank renders its own frame (independent seeds, weak
scaling, no data-path collective).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference estimator on the host cores: the Rust reference cannot
be built here, so its CPU restatement (oracle/, stream-RNG mode, all host threads) renders a
bounded sample of the same workload per step.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic cost per counted test (FP32 flops, bytes read): AABB 18/24, sphere 28/16,
# quad 54/64, triangle 52/36, disk 28/32; a node visit slab-tests two child boxes.  Fog
# tests (boundary roots + hash) and plane tests are charged like a disk.
COST = {
    "node_visits": (36, 48),
    "sphere_tests": (28, 16),
    "quad_tests": (54, 64),
    "triangle_tests": (52, 36),
    "disk_tests": (28, 32),
    "fog_tests": (28, 32),
    "plane_tests": (28, 32),
}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", default="random_spheres")
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--height", type=int, default=0)
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--depth", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="target CPU time of the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/forward cost block")
    ap.add_argument("--adjoint-res", type=int, default=512, help="adjoint block: image side (workload: 512)")
    ap.add_argument("--adjoint-spp", type=int, default=64, help="adjoint block: samples per pixel (workload: 64)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-workload block")
    ap.add_argument("--no-sampling", action="store_true", help="skip the adaptive / time-limit block")
    ap.add_argument("--no-rmse", action="store_true", help="skip the RMSE block (reference-estimator rows)")
    ap.add_argument("--no-configs", action="store_true", help="skip the box-room / dense-mesh / diff-quads records")
    ap.add_argument("--scenes", type=int, default=64, help="batched workload: number of scenes")
    ap.add_argument("--max-res", type=int, default=1024, help="batched workload: largest resolution")
    ap.add_argument("--batch-config", default="auto", help="batched workload: auto | default | k=v,k=v")
    return ap.parse_args()


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def workload(args, rank=0):
    from luminara_b200 import workloads as W

    world, cfg = W.CONFIGS[args.config]()
    if args.width:
        cfg.width = args.width
    if args.height:
        cfg.height = args.height
    if args.width or args.height:
        world.camera.aspect_ratio = cfg.width / cfg.height
    if args.spp:
        cfg.samples_per_pixel = args.spp
    if args.depth:
        cfg.max_depth = args.depth
    cfg.seed = cfg.seed + 7919 * rank
    return world, cfg


def strata(cfg):
    import math

    n = math.ceil(math.sqrt(cfg.samples_per_pixel))
    return n * n


def workload_name(args, cfg):
    return f"{args.config} {cfg.width}x{cfg.height} {cfg.samples_per_pixel}spp ({strata(cfg)} strata) depth {cfg.max_depth}"


# ------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples during the timed region (200 ms period)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self, wait_s=20.0):
        """Starts sampling and waits (up to wait_s) for the first sample, so nvidia-smi's own
        start-up does not overlap the timed region."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
            return
        t0 = time.time()
        while not self.lines and time.time() - t0 < wait_s and self.proc.poll() is None:
            time.sleep(0.05)
        self.lines.clear()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------------------------ peaks
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), d.get("sm_max_mhz", 1965.0), "measured"
    return 6650.0, 1965.0, "fallback"


# ------------------------------------------------------------------------------ CPU baseline
def spread_rows(h, n, offset=0.5, exclude=()):
    """n distinct image rows spread evenly over [0, h), not in `exclude`."""
    ex = set(exclude)
    rows = []
    for k in range(n):
        j = min(h - 1, int((k + offset) * h / max(n, 1)))
        while j in ex or j in rows:
            j = (j + 1) % h
        rows.append(j)
    return rows


def cpu_sample(world, cfg, target_s, threads=0, scene=None):
    """Reference estimator (oracle stream mode) on image rows spread over the frame, rendered
    with OpenMP over the row list so that every host thread is busy, sized to take about
    target_s seconds of wall time.  Returns (paths, wall seconds, rows, threads)."""
    import oracle as O

    sc = scene or O.OracleScene(world)
    nt = threads or os.cpu_count() or 1
    h = cfg.height
    rows0 = spread_rows(h, min(h, 2 * nt), 0.25)              # calibration: two rows per thread
    _, st = sc.render_row_list(cfg, rows0, mode=O.MODE_STREAM, threads=threads)
    total_paths, total_s, used = st.paths, st.seconds, st.threads
    n_rows = len(rows0)
    per_row = st.seconds / len(rows0)
    n_more = int((target_s - total_s) / max(per_row, 1e-9))
    n_more = min(h - len(rows0), (n_more // used) * used)   # whole waves of rows
    if n_more > 0:
        rows1 = spread_rows(h, n_more, 0.75, exclude=rows0)
        _, st = sc.render_row_list(cfg, rows1, mode=O.MODE_STREAM, threads=threads)
        total_paths += st.paths
        total_s += st.seconds
        n_rows += len(rows1)
    return total_paths, total_s, n_rows, used


def config_dict(args, cfg):
    """The workload description shared by both arms' JSON lines."""
    return {"workload": workload_name(args, cfg), "width": cfg.width, "height": cfg.height, "spp": strata(cfg),
            "max_depth": cfg.max_depth, "paths_per_step_per_gpu": cfg.width * cfg.height * strata(cfg),
            "l2": "GPU arm: L2 flushed before every timed step (256 MiB device write inside the timed region)",
            "parallelism": "one independent frame per GPU (seed offset by rank), no data-path collective"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    world, cfg = workload(args)
    import oracle as O

    sc = O.OracleScene(world)
    per_step = max(2.0, min(20.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_sample(world, cfg, per_step / 4, scene=sc)
    paths, secs, rows, threads = 0, 0.0, 0, 0
    for _ in range(args.steps):
        p, s, r, threads = cpu_sample(world, cfg, per_step, scene=sc)
        paths += p
        secs += s
        rows += r
    value = paths / secs / 1e6
    sample = (f"{rows} image rows spread over the frame ({cfg.width} px x {strata(cfg)} strata each) over "
              f"{args.steps} steps of about {per_step:.0f} s ({secs:.1f} s of wall time, {threads} threads, "
              f"OpenMP over the rows)")
    line = {
        "impl": "reference", "metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(args, cfg),
        "cpu_baseline": {"value": value, "unit": "Mpaths/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Mpaths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "Rust reference not buildable on this machine (no cargo/rustc); timed its C++ f64 restatement "
                "(oracle/, the reference's per-row SmallRng estimator) with OpenMP over rows, all host threads",
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------ our arm
def profile_figures(kernel="k_render", workload=None):
    """Figures recorded in profiles/<kernel>_<workload>.md by its ncu summary (lines 'key: value')."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    out = {}
    if not os.path.exists(path):
        return out
    for line in open(path):
        if ":" not in line or line.startswith((" ", "|", "#")):
            continue
        k, v = line.split(":", 1)
        if k in ("dram_bytes_per_full_launch", "issue_active", "simt_lanes_per_inst", "l1_hit_rate", "l2_hit_rate"):
            try:
                out[k] = float(v.strip())
            except ValueError:
                pass
    return out


def l1_peaks(L):
    """L1 load throughput of this device (lum_diag_l1_throughput): coalesced and 64-byte gather."""
    try:
        return {"coalesced_gbs": L.diag_l1_throughput(0), "gather_gbs": L.diag_l1_throughput(1)}
    except Exception as e:                              # reported in the line, never fatal
        return {"error": str(e)}


def roofline(counts, avg_kernel_s, l1, workload_key=None):
    """Roofline of one k_render launch from its counted tests (COST per test).  The algorithmic
    bytes are node and primitive records, which L1 and L2 serve (ncu: DRAM traffic per launch
    is ~1e-6 of them on the sphere field), so the bound reported is the L1 gather throughput of
    64-byte records measured in this run; the HBM and FP32 fractions are given beside it."""
    flops = sum(getattr(counts, k) * c[0] for k, c in COST.items())
    nbytes = sum(getattr(counts, k) * c[1] for k, c in COST.items())
    hbm_peak, sm_max_mhz, peak_kind = measured_peaks()
    import torch

    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    fp32_peak = props.multi_processor_count * 128 * 2 * sm_max_mhz * 1e6 / 1e12
    ach_gbs = nbytes / avg_kernel_s / 1e9
    ach_tflops = flops / avg_kernel_s / 1e12
    prof = profile_figures("k_render", workload_key) if workload_key else {}
    gather = l1.get("gather_gbs")
    roof = {
        "kernel": "k_render",
        "bound": "l1" if gather else "hbm",
        "achieved": ach_gbs, "unit": "GB/s",
        "peak": gather if gather else hbm_peak,
        "frac": ach_gbs / gather if gather else ach_gbs / hbm_peak,
        "traffic": int(prof["dram_bytes_per_full_launch"]) if "dram_bytes_per_full_launch" in prof else None,
        "peak_kind": ("L1 gather of 64-byte records, measured in this run (lum_diag_l1_throughput pattern 1); "
                      "the algorithmic bytes are served from L1/L2, `traffic` is the DRAM bytes of one launch"
                      if gather else "HBM " + peak_kind),
        "bytes_per_launch": nbytes, "flops_per_launch": flops,
        "l1": {**l1, "frac_gather": ach_gbs / gather if gather else None,
               "frac_coalesced": ach_gbs / l1["coalesced_gbs"] if l1.get("coalesced_gbs") else None,
               "of": "builder-measured (lum_diag_l1_throughput)"},
        "hbm": {"achieved_gbs": ach_gbs, "peak_gbs": hbm_peak, "frac": ach_gbs / hbm_peak, "of": peak_kind,
                "note": "algorithmic bytes against the HBM copy rate; they are served from L1/L2, not DRAM"},
        "fp32": {"achieved_tflops": ach_tflops, "peak_tflops": fp32_peak, "frac": ach_tflops / fp32_peak,
                 "of": "nominal (SMs x 128 lanes x 2 x max SM clock)"},
        "avg_launch_ms": avg_kernel_s * 1e3,
        "counts_per_launch": {k: int(getattr(counts, k)) for k in
                              ("node_visits", "sphere_tests", "quad_tests", "triangle_tests", "disk_tests",
                               "fog_tests", "plane_tests", "segments", "shadow_rays", "paths")},
    }
    if "issue_active" in prof:
        roof["issue"] = {"issue_active": prof["issue_active"], "simt_lanes_per_inst": prof.get("simt_lanes_per_inst"),
                         "of": f"ncu, small case of the same kernel (profiles/k_render_{workload_key}.md)"}
    return roof


def time_frames(sc, cfg, out, flush, stream, steps, warmup, barrier=lambda: None):
    """Warm-up steps are timed steps: the same flush, events and enqueue-only renders, so lazily
    loaded kernel modules (torch's fill kernel) and first-call host work stay out of the timed
    region.  A checked render before and after the timed steps supplies the segment counts and
    confirms no kernel error flags.  The timed steps are enqueued back to back (render_device
    without waiting), each bracketed by CUDA events on the launching stream for the kernel's own
    time.  Returns (timed-region seconds, per-step kernel ms, checked stats)."""
    import torch

    for _ in range(warmup):
        w0, w1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.zero_()
        w0.record(stream)
        sc.render_device(cfg, out.data_ptr(), stream.cuda_stream, wait=False)
        w1.record(stream)
    torch.cuda.synchronize()
    st0 = sc.render_device(cfg, out.data_ptr(), stream.cuda_stream)
    assert st0.error_flags == 0
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    step_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    ev0.record(stream)
    for k in range(steps):
        flush.zero_()
        step_ev[k][0].record(stream)
        sc.render_device(cfg, out.data_ptr(), stream.cuda_stream, wait=False)
        step_ev[k][1].record(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    st1 = sc.render_device(cfg, out.data_ptr(), stream.cuda_stream)      # the last frame's flags
    assert st1.error_flags == 0 and st1.segments == st0.segments
    return ev0.elapsed_time(ev1) / 1e3, [a.elapsed_time(b) for a, b in step_ev], st0


def rmse_block(world, cfg, out, rate_mpaths, target_s=25.0, ref_spp=4096):
    """Per-pixel RMSE of the device frame against the reference estimator (oracle stream mode)
    at ref_spp samples per pixel, on rows spread over the frame, beside the RMSE of an
    independent reference-estimator render at the frame's own spp (another seed) against the same
    high-spp rows: equal RMSE at equal spp is what 'at matched RMSE' asks.  Also the mean
    luminance difference in standard errors."""
    from dataclasses import replace

    import numpy as np

    import oracle as O

    sc = O.OracleScene(world)
    per_row_paths = cfg.width * ref_spp
    n_rows = int(max(4, min(32, rate_mpaths * 1e6 * target_s / per_row_paths)))
    rows = spread_rows(cfg.height, n_rows, 0.5)
    t0 = time.perf_counter()
    ref, _ = sc.render_row_list(replace(cfg, samples_per_pixel=ref_spp, seed=cfg.seed + 1000003), rows)
    cpu, _ = sc.render_row_list(replace(cfg, seed=cfg.seed + 2000003), rows)
    secs = time.perf_counter() - t0
    gpu = out[rows].float().cpu().numpy().astype(np.float64)
    rm = lambda a: float(np.sqrt(np.mean((a - ref) ** 2)))
    lum = lambda a: 0.2126 * a[..., 0] + 0.7152 * a[..., 1] + 0.0722 * a[..., 2]
    d = (lum(gpu) - lum(ref)).ravel()
    dc = (lum(cpu) - lum(ref)).ravel()
    return {"rmse": rm(gpu), "rmse_cpu_same_spp": rm(cpu), "ratio": rm(gpu) / max(rm(cpu), 1e-30),
            "mean_lum_bias_z": float(d.mean() / (d.std(ddof=1) / np.sqrt(d.size))),
            "mean_lum_bias_z_cpu": float(dc.mean() / (dc.std(ddof=1) / np.sqrt(dc.size))),
            "reference": f"oracle stream mode (the reference's estimator, f64) at {ref_spp} spp",
            "rows": rows, "pixels": len(rows) * cfg.width, "cpu_seconds": secs}


def config_record(L, name, flush, stream, l1, steps=5, warmup=3, cpu_s=4.0):
    """One of the other configurations (box room, dense mesh, differentiable quads): the same
    frame timing, roofline and CPU baseline as the headline, at the configuration's own size."""
    import torch

    from luminara_b200 import workloads as W

    world, cfg = W.CONFIGS[name]()
    t0 = time.perf_counter()
    sc = L.GpuScene(world)
    build_s = time.perf_counter() - t0
    info = sc.info()
    H, Wd = cfg.out_shape()[:2]
    out = torch.empty((H, Wd, 3), dtype=torch.float32, device="cuda")
    counts = sc.count_tests(cfg)
    region_s, kernel_ms, st0 = time_frames(sc, cfg, out, flush, stream, steps, warmup)
    paths = H * Wd * strata(cfg)
    rec = {"workload": f"{name} {cfg.width}x{cfg.height} {cfg.samples_per_pixel}spp ({strata(cfg)} strata) "
                       f"depth {cfg.max_depth}",
           "value": paths * steps / region_s / 1e6, "unit": "Mpaths/s", "ms_per_step": region_s * 1e3 / steps,
           "steps": steps, "warmup": warmup, "paths_per_step": paths,
           "mrays_per_s": (st0.segments + st0.shadow_rays) * steps / region_s / 1e6,
           "prims": info["prims"], "bvh_nodes": info["nodes"], "scene_build_s": build_s,
           "roofline": roofline(counts, statistics.mean(kernel_ms) / 1e3, l1, name)}
    import oracle as O

    t1 = time.perf_counter()
    osc = O.OracleScene(world)
    oracle_build = time.perf_counter() - t1
    p, s_, rows, threads = cpu_sample(world, cfg, cpu_s, scene=osc)
    rec["cpu_baseline"] = {"value": p / s_ / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": "port",
                           "sample": f"{rows} rows spread over the frame ({p} paths, {s_:.1f} s wall, OpenMP over "
                                     f"rows; oracle scene + BVH build {oracle_build:.1f} s not timed)"}
    sc.close()
    return rec


def run_ours(args):
    import torch

    import luminara_b200 as L

    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world_size > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    def barrier():
        if dist is not None:
            dist.barrier()

    def allmax(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    world, cfg = workload(args, rank)
    t0 = time.perf_counter()
    sc = L.GpuScene(world)
    build_s = time.perf_counter() - t0
    info = sc.info()
    H, Wd = cfg.out_shape()[:2]
    paths_per_step = H * Wd * strata(cfg)
    out = torch.empty((H, Wd, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2
    # a stream of our own (a non-zero handle): lum_render_device maps a null stream to the
    # scene's stream, and the events below must be on the stream the renders run on
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    l1 = l1_peaks(L)

    t1 = time.perf_counter()
    counts = sc.count_tests(cfg)                   # counter build, same seeds (not timed)
    t2 = time.perf_counter()
    clocks = ClockSampler(dev)
    clocks.start()
    region_s, kernel_ms, st0 = time_frames(sc, cfg, out, flush, stream, args.steps, args.warmup, barrier)
    clock_info = clocks.stop()
    log(f"scene build {build_s:.3f}s, counter build {t2 - t1:.3f}s, frames {time.perf_counter() - t2:.3f}s")
    segs, shadows = st0.segments * args.steps, st0.shadow_rays * args.steps
    region_s = allmax(region_s)
    value = world_size * paths_per_step * args.steps / region_s / 1e6
    avg_kernel_s = statistics.mean(kernel_ms) / 1e3
    default_frame = not args.width and not args.height and not args.spp and not args.depth
    roof = roofline(counts, avg_kernel_s, l1, args.config if default_frame else None)

    # end to end through the public C ABI with host buffers: scene upload + render + readback
    e2e = None
    if not args.no_e2e:
        phases = []

        def e2e_step():
            t = time.perf_counter()
            s2 = L.GpuScene(world)
            ta = time.perf_counter()
            img, st2 = s2.render(cfg)
            tb = time.perf_counter()
            s2.close()
            phases.append((ta - t, tb - ta, time.perf_counter() - tb, st2.kernel_ms / 1e3))
            return img, st2

        # warm-up: at least W steps, then until two consecutive steps agree within 10% (at most 10
        # more): the first host-side steps of a process can be several times slower
        for _ in range(max(1, args.warmup)):
            e2e_step()
        for _ in range(10):
            a, b = sum(phases[-2][:3]) if len(phases) > 1 else 0.0, sum(phases[-1][:3])
            if len(phases) > 1 and abs(a - b) <= 0.1 * min(a, b):
                break
            e2e_step()
        phases.clear()
        barrier()
        t1 = time.perf_counter()
        for _ in range(args.steps):
            img, st2 = e2e_step()
        torch.cuda.synchronize()
        e2e_s = allmax(time.perf_counter() - t1)
        barrier()
        e2e = {"value": world_size * paths_per_step * args.steps / e2e_s / 1e6, "unit": "Mpaths/s",
               "h2d_bytes_per_step": int(info["device_bytes"]), "d2h_bytes_per_step": int(H * Wd * 3 * 4),
               "path": "lum_scene_create (flatten + BVH + H2D) + lum_render (render + D2H) + lum_scene_destroy",
               "median_ms": {k: 1e3 * statistics.median(ph[i] for ph in phases) for i, k in
                             enumerate(("scene_create", "render", "scene_destroy", "render_kernel"))},
               "step_ms": [round(1e3 * sum(ph[:3]), 2) for ph in phases]}

    solo = rank == 0 and world_size == 1
    cpu = None
    if solo and not args.no_cpu_baseline:
        p, s, rows, threads = cpu_sample(world, cfg, args.cpu_seconds)
        cpu = {"value": p / s / 1e6, "unit": "Mpaths/s", "cores": threads, "kind": "port",
               "sample": f"{rows} rows spread over the same frame ({p} paths, {s:.1f} s wall), reference estimator "
                         f"restated in C++ f64 (oracle/, stream RNG), OpenMP over the rows"}
    rmse = None
    if solo and not args.no_rmse and default_frame:
        rmse = rmse_block(world, cfg, out, cpu["value"] if cpu else 1.0)
    hbm_peak = measured_peaks()[0]
    tone = tonemap_block(L, out, H, Wd, stream, hbm_peak, flush) if rank == 0 else None
    sampling = sampling_block(L, sc, cfg, out, stream) if (solo and not args.no_sampling) else None
    others = None
    if solo and not args.no_configs and default_frame:
        others = {}
        for name in ("box_room", "dense_mesh", "diff_quads"):
            if name != args.config:
                others[name] = config_record(L, name, flush, stream, l1)
    adjoint = adjoint_block(L, args.adjoint_res, args.adjoint_spp) if (solo and not args.no_adjoint) else None
    batched = None
    if solo and not args.no_batched:
        b = batched_measure(args, 2, 3, with_clocks=False)
        batched = {k: b[k] for k in ("value", "unit", "ms_per_step", "batch_mode", "sequential_megakernel",
                                     "speedup_vs_sequential", "max_rel_diff_vs_megakernel", "autotune",
                                     "scene_done_ms", "modes")}
        batched["workload"] = b["config"]["workload"]

    if rank == 0:
        line = {
            "metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": world_size, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": region_s * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
            "config": config_dict(args, cfg),
            "scene": {"prims": info["prims"], "bvh_nodes": info["nodes"], "scene_build_s": build_s},
            "mrays_per_s": world_size * (segs + shadows) / region_s / 1e6,
            "segments_per_path": segs / (paths_per_step * args.steps),
            "shadow_rays_per_path": shadows / (paths_per_step * args.steps),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "rmse": rmse, "gpu_launches": args.steps,
            "clocks": clock_info, "configs": others, "tonemap": tone, "sampling": sampling, "adjoint": adjoint,
            "batched": batched,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    sc.close()
    return 0


# ------------------------------------------------------------------------------ LDR output
def tonemap_block(L, hdr, H, Wd, stream, hbm_peak, flush):
    """The LDR colour chain (lum_tonemap_device) over the frame just rendered: ACES + sRGB,
    without and with auto-exposure (a log-luminance reduction kernel first).  Each launch is
    timed alone with CUDA events after an L2 flush.  Algorithmic bytes per call: 12 read + 4
    written per pixel, plus 12 read per pixel for the reduction."""
    import torch

    rgba = torch.empty((H, Wd, 4), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(L.abi.TONEMAP_SCRATCH_BYTES, dtype=torch.uint8, device="cuda")
    out = {}
    for name, auto in (("aces_srgb", False), ("aces_srgb_auto_exposure", True)):
        tm = L.ToneMapConfig(auto_exposure=auto)
        for _ in range(3):
            L.tonemap_device(hdr.data_ptr(), Wd, H, tm, scratch.data_ptr(), rgba.data_ptr(), stream.cuda_stream)
        times = []
        for _ in range(20):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            L.tonemap_device(hdr.data_ptr(), Wd, H, tm, scratch.data_ptr(), rgba.data_ptr(), stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        nbytes = H * Wd * (16 + (12 if auto else 0))
        out[name] = {"ms": ms, "gbs": nbytes / ms / 1e6, "frac_of_hbm_peak": nbytes / ms / 1e6 / hbm_peak,
                     "bytes_per_call": nbytes}
    # an 8K frame: its 398 MB of input exceed L2, so every call reads from HBM without a flush
    # (and without the flush's dirty lines to write back); seeded synthetic radiance
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    big_h, big_w = 4320, 7680
    big = torch.rand((big_h, big_w, 3), generator=g, device="cuda", dtype=torch.float32) * 4.0
    big_rgba = torch.empty((big_h, big_w, 4), dtype=torch.uint8, device="cuda")
    tm = L.ToneMapConfig()
    for _ in range(3):
        L.tonemap_device(big.data_ptr(), big_w, big_h, tm, scratch.data_ptr(), big_rgba.data_ptr(), stream.cuda_stream)
    times = []
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        L.tonemap_device(big.data_ptr(), big_w, big_h, tm, scratch.data_ptr(), big_rgba.data_ptr(), stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    nbytes = big_h * big_w * 16
    out["aces_srgb_8k"] = {"ms": ms, "gbs": nbytes / ms / 1e6, "frac_of_hbm_peak": nbytes / ms / 1e6 / hbm_peak,
                           "bytes_per_call": nbytes, "pixels": big_h * big_w,
                           "l2": "input (398 MB) larger than L2; no flush"}
    del big, big_rgba
    out["hbm_peak"] = {"gbs": hbm_peak, "of": measured_peaks()[2]}
    out["pixels"] = H * Wd
    out["l2"] = "flushed (256 MiB write) before each timed call (1080p frame)"
    return out


# ------------------------------------------------------------------------------ adaptive / time limit
def sampling_block(L, sc, cfg, out, stream, threshold=0.03):
    """The sample loop's in-loop branches on the headline frame (k_render_sampled): adaptive
    sampling at the reference's default threshold, and a time limit of half the plain frame
    time.  Kernel times (median of 5 after 2 warm-ups, lum_stats.kernel_ms); samples kept =
    the reference's ray count."""
    from dataclasses import replace

    def run(c, n=5):
        for _ in range(2):
            sc.render_device(c, out.data_ptr(), stream.cuda_stream)
        sts = [sc.render_device(c, out.data_ptr(), stream.cuda_stream) for _ in range(n)]
        return statistics.median(s.kernel_ms for s in sts), sts[-1]

    px = cfg.width * cfg.height
    plain_ms, plain = run(cfg)
    res = {"plain": {"ms": plain_ms, "samples": plain.paths, "segments": plain.segments}}
    a_ms, a = run(replace(cfg, adaptive=True, adaptive_threshold=threshold))
    res["adaptive"] = {"threshold": threshold, "ms": a_ms, "samples": a.paths, "avg_spp": a.paths / px,
                       "segments": a.segments, "time_vs_plain": a_ms / plain_ms,
                       "kept_mpaths_per_s": a.paths / a_ms / 1e3}
    limit_s = plain_ms * 0.5e-3
    t_ms, t = run(replace(cfg, time_limit=limit_s))
    res["time_limit"] = {"limit_ms": limit_s * 1e3, "ms": t_ms, "samples": t.paths,
                         "full_tiles_frac": (t.paths - px) / (plain.paths - px) if plain.paths > px else None}
    return res


# ------------------------------------------------------------------------------ adjoint
def adjoint_block(L, res=512, spp=64):
    """Cost of the path-replay adjoint against one forward render on the differentiable
    workload (1000 GGX quads + 4 emissive quads, 512x512, 64 spp, depth 6): device time of
    lum_forward's render kernel and of lum_backward's replay + sweep kernels, for a dense
    dL/d(image) (every pixel replayed) and for the L2 loss against a render at perturbed
    parameters (pixels with zero gradient are skipped)."""
    import numpy as np

    from luminara_b200 import workloads as W

    world, cfg = W.diff_quads(width=res, height=res, spp=spp)
    rng = np.random.default_rng(77)
    saved = [(m, m.color, m.roughness) for m in world.materials]
    for m in world.materials:
        if m.kind != 4:
            m.color = tuple(float(x) for x in np.clip(np.array(m.color) + rng.normal(0, 0.05, 3), 0, 1))
            m.roughness = float(np.clip(m.roughness + rng.normal(0, 0.05), 0.05, 1))
    target, _ = L.GpuScene(world).render(cfg)
    for m, c, r in saved:
        m.color, m.roughness = c, r
    sc = L.GpuScene(world)
    lm = world.light_material_indices()
    img, _ = sc.forward(cfg)
    grads = {"dense": np.random.default_rng(1).normal(size=img.shape).astype(np.float32),
             "l2": (2.0 * (img - target)).astype(np.float32)}
    fwd = []
    bwd = {k: [] for k in grads}
    for _ in range(4):
        _, st = sc.forward(cfg)
        fwd.append(st.kernel_ms)
        for k, g in grads.items():
            *_, st = sc.backward(cfg, g, lm)
            assert st.error_flags == 0
            bwd[k].append(st.kernel_ms)
    f = min(fwd)
    out = {"workload": f"diff_quads {res}x{res} {spp}spp depth 6 (1004 materials)", "forward_ms": f,
           "paths": int(np.prod(img.shape[:2])) * int(np.ceil(np.sqrt(spp))) ** 2}
    for k, v in bwd.items():
        out[f"backward_ms_{k}"] = min(v)
        out[f"ratio_{k}"] = min(v) / f
    sc.close()
    return out


# ------------------------------------------------------------------------------ batched
def batched_measure(args, steps, warmup, with_clocks=True):
    """The batched uneven workload: 64 seeded scenes rendered (a) one after another with the
    megakernel and (b) together by the batch (lum_batch_*, autotuned); returns the JSON line."""
    import torch

    import luminara_b200 as L
    from luminara_b200 import workloads as W

    torch.cuda.set_device(0)
    res = tuple(r for r in (128, 256, 512, 1024) if r <= args.max_res)
    items = W.batched(n_scenes=args.scenes, res_choices=res)
    scenes = [L.GpuScene(w) for w, _ in items]
    cfgs = [c for _, c in items]
    paths = sum(c.out_shape()[0] * c.out_shape()[1] * strata(c) for c in cfgs)
    outs = [torch.empty(c.out_shape(), dtype=torch.float32, device="cuda") for c in cfgs]
    stream = torch.cuda.current_stream()
    t0 = time.perf_counter()
    if args.batch_config == "auto":
        tuned, tune_ms = L.autotune(scenes, cfgs)
        batch = L.Batch(scenes, cfgs)
    else:
        kv = {} if args.batch_config == "default" else dict(x.split("=") for x in args.batch_config.split(","))
        batch = L.Batch(scenes, cfgs, config=kv or "default")
        tuned, tune_ms = batch.config(), None
    tune_s = time.perf_counter() - t0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def seq():
        for s, c, o in zip(scenes, cfgs, outs):
            s.render_device(c, o.data_ptr(), stream.cuda_stream)

    for _ in range(warmup):
        seq()
        batch.render_device([o.data_ptr() for o in outs])
    torch.cuda.synchronize()
    clocks = ClockSampler(0) if with_clocks else None
    if clocks:
        clocks.start()
    ev0.record(stream)
    for _ in range(steps):
        seq()
    ev1.record(stream)
    torch.cuda.synchronize()
    seq_s = ev0.elapsed_time(ev1) / 1e3
    seq_imgs = [o.clone() for o in outs]
    done_all, bstats = [], []
    ev0.record(stream)
    for _ in range(steps):
        done, st = batch.render_device([o.data_ptr() for o in outs])
        done_all.append(done)
        bstats.append(st)
    ev1.record(stream)
    torch.cuda.synchronize()
    bat_s = ev0.elapsed_time(ev1) / 1e3
    clock_info = clocks.stop() if clocks else None
    max_rel = max(float(((a - b).abs() / (b.abs() + 1e-3)).max()) for a, b in zip(outs, seq_imgs))
    value = paths * steps / bat_s / 1e6
    batch_mode = {0: "wavefront", 1: "megakernel", 2: "streams"}[batch.config().get("mode")]
    batch.close()
    # each batch mode on its own (default configuration otherwise), the same images
    modes = {}
    for m, mname in ((0, "wavefront"), (1, "megakernel"), (2, "streams")):
        bm = L.Batch(scenes, cfgs, config={"mode": m})
        bm.render_device([o.data_ptr() for o in outs])
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(steps):
            bm.render_device([o.data_ptr() for o in outs])
        ev1.record(stream)
        torch.cuda.synchronize()
        m_s = ev0.elapsed_time(ev1) / 1e3
        same = all(torch.equal(a, b) for a, b in zip(outs, seq_imgs))
        modes[mname] = {"value": paths * steps / m_s / 1e6, "ms_per_step": m_s * 1e3 / steps,
                        "speedup_vs_sequential": seq_s / m_s, "config": bm.config(), "images_equal": same}
        bm.close()
    done_ms = done_all[-1]
    line = {
        "metric": "Mpaths/s", "value": value, "unit": "Mpaths/s", "n_gpus": 1, "steps": steps,
        "warmup": warmup, "ms_per_step": bat_s * 1e3 / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene generator)",
        "config": {"workload": f"batched: {len(cfgs)} uneven scenes, {paths} paths per step",
                   "scenes": len(cfgs), "prims": sum(w.n_prims() for w, _ in items),
                   "l2": "working set of the batch exceeds L2 (pool, queues, 64 scenes)"},
        "batch_mode": batch_mode,
        "sequential_megakernel": {"value": paths * steps / seq_s / 1e6, "unit": "Mpaths/s",
                                  "ms_per_step": seq_s * 1e3 / steps},
        "speedup_vs_sequential": seq_s / bat_s,
        "max_rel_diff_vs_megakernel": max_rel,
        "autotune": {"config": tuned, "best_ms": tune_ms, "seconds": tune_s},
        "scene_done_ms": {"min": min(done_ms), "median": statistics.median(done_ms), "max": max(done_ms)},
        "iterations": bstats[-1].iterations, "graph_launches": bstats[-1].graph_launches,
        "modes": modes, "gpu_launches": None, "clocks": clock_info,
    }
    return line


def run_batched(args):
    line = batched_measure(args, args.steps, args.warmup)
    print(json.dumps(line), flush=True)

    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.config == "batched":
        return run_batched(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
