"""Benchmark of the splat path: one frame = project + SH + key + sort of the
4M-splat SH-degree-3 float32 workload (1920x1080, fov 50, 32-bit keys).

python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One process per GPU (torchrun for N > 1): each rank runs its own replica of
the workload (the path shards by object and view; no collective is needed),
timed on the device with CUDA events between barriers; the time is the max
over ranks and `value` counts the splats of every rank. A step is one CUDA
graph launch of the frame (rb.Batch with one view); the same frame through
rb.frame, which plans on the host every call, is timed beside it. Rank 0
prints one JSON line. --impl reference times the reference's CPU path (the float64 port of
SortKeys.compute / SortKeys.sort and of the projection) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Msplats/s (project+SH+key+sort)"
N_SPLATS = 4_000_000
SH_DEGREE = 3
BITS = 32
# Algorithmic bytes per splat (project+SH+key+sort): inputs 236, outputs 40,
# key + index 8, sort 16 per 8-bit pass + 4
FRAME_BYTES = 236 + 40 + 8 + 16 * (BITS // 8) + 4
# The projection kernel alone: inputs 236, outputs 40, the key 4
PROJECT_BYTES = 236 + 40 + 4
FALLBACK_HBM_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_SPLATS)
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-forms", action="store_true",
                   help="frame workload: skip the batched, stereo and backward forms timed after the headline frame")
    p.add_argument("--bits", type=int, default=32, choices=[16, 24, 32],
                   help="sort-key width (32 for the headline; 24 is the reference's default)")
    p.add_argument("--pose", default="scale", choices=["scale", "all-visible"],
                   help="frame: the configuration's camera at (0, 0.5, 3) (about half the splats in view), or a "
                        "camera at (0, 0.5, 30) that keeps every splat inside the culls")
    p.add_argument("--no-tune", action="store_true", help="keep the default kernel choices (no autotuning)")
    p.add_argument("--variant", type=int, default=None,
                   help="force a digit-pass variant (rdx_ctx_set_sort_variant's numbering) instead of tuning")
    p.add_argument("--spz-container", default="gzip", choices=["gzip", "ngsp"],
                   help="spz workload: version 3 in gzip (one DEFLATE stream) or SPZ 4 (NGSP, a zstd stream a column)")
    p.add_argument("--workload", default="frame",
                   choices=["frame", "batched", "stereo", "backward", "ply", "spz", "rdx", "census", "rays"],
                   help="frame: 4M SH-3 splats, one view (the headline); batched: 16 scenes x 64 views in one "
                        "CUDA graph; stereo: 16M SH-3 fp16 splats, two eyes; backward: the projection's gradient, 1M; "
                        "ply: decoding a 1M-splat PLY file; spz: decoding a 1M-splat SPZ file from host bytes; "
                        "rdx: decoding a 1M-splat RDX file from host bytes; census: every device entry point "
                        "once a step, each timed alone; rays: the 3dgut, htgs and raygs words and keys of the 4M "
                        "SH-3 frame")
    return p.parse_args()


def peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(summary="project_kernel_4m_sh3.md", scale=1.0):
    """DRAM bytes per launch of a kernel from its committed ncu summary (times
    `scale` where the summary captured a smaller launch of the same kernel), or None."""
    path = os.path.join(ROOT, "profiles", summary)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1].split()[0]) * scale
    return None


class Clocks:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(n, device):
    import numpy as np
    import torch

    from radix_b200 import synthetic as syn
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE)
    cols = ("centers", "log_scales", "quats", "opacities", "colors")
    host = {k: torch.from_numpy(np.ascontiguousarray(d[k])).pin_memory() for k in cols}
    dev = {k: v.to(device) for k, v in host.items()}
    return d, host, dev


def table_of(cols):
    import radix_b200 as rb
    return rb.Table.raw(cols["centers"], cols["log_scales"], cols["quats"], cols["opacities"], cols["colors"], SH_DEGREE)


def keys_sort_only(dist, n, reps=3):
    """The reference's own CPU path as bench-core.ts times it (SortKeys.compute
    + SortKeys.sort, one worker thread): Msplats/s, median of reps after one warm-up."""
    from oracle import oracle as orc
    ks = []
    for i in range(reps + 1):
        t0 = time.perf_counter()
        keys = orc.sort_keys(dist, BITS)
        orc.sort(keys, n, BITS)
        if i:
            ks.append(time.perf_counter() - t0)
    return n / statistics.median(ks) / 1e6


def cpu_baseline(n_sample):
    """The oracle (float64 port of the reference's CPU path) on the workload:
    projection + SH + keys on all host threads, SortKeys.sort single-threaded."""
    import radix_b200 as rb
    from oracle import oracle as orc
    from radix_b200 import synthetic as syn
    d = syn.mixture_table(n_sample, seed=0, sh_degree=SH_DEGREE)
    obj = [rb.SplatObject(rb.Table.from_dict(d))]
    cam = syn.scale_camera()
    times = []
    for i in range(4):
        t0 = time.perf_counter()
        ref = orc.project(obj, cam, None, BITS, cull_keys=True, threads=0)
        orc.sort(ref["keys"], n_sample, BITS)
        if i:
            times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    threads = os.cpu_count() or 1
    return {"value": n_sample / t / 1e6, "unit": "Msplats/s", "cores": threads, "kind": "port",
            "sample": f"{n_sample} splats of the same workload; float64 projection+SH+keys on {threads} threads "
                      f"(OpenMP), SortKeys.sort restated in C on 1 thread; median of 3 after 1 warm-up",
            "keys_sort_only_msplats_s_1thread": keys_sort_only(ref["distance"], n_sample)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import radix_b200 as rb
    from oracle import oracle as orc
    from radix_b200 import synthetic as syn
    n = args.n
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE)
    obj = [rb.SplatObject(rb.Table.from_dict(d))]
    cam = syn.scale_camera()
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ref = orc.project(obj, cam, None, BITS, cull_keys=True, threads=0)
        orc.sort(ref["keys"], n, BITS)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    value = n / t / 1e6
    threads = os.cpu_count() or 1
    line = {
        "metric": METRIC, "value": value, "unit": "Msplats/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded mulberry32)",
        "config": {"workload": f"project+SH+key+sort, {n} splats, SH degree 3 fp32, Gaussian-mixture centres, "
                               f"1920x1080 fov 50, {BITS}-bit keys, stable order",
                   "n": n, "sh_degree": SH_DEGREE, "bits": BITS},
        "cpu_baseline": {"value": value, "unit": "Msplats/s", "cores": threads, "kind": "port",
                         "sample": f"the whole workload ({n} splats) every step; float64 projection+SH+keys on "
                                   f"{threads} threads (OpenMP), SortKeys.sort restated in C on 1 thread",
                         "keys_sort_only_msplats_s_1thread": keys_sort_only(ref["distance"], n)},
        "e2e": {"value": value, "unit": "Msplats/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def max_over_ranks(value, world, device):
    """The largest of a per-rank float over the process group's ranks (the
    value itself for one rank): every rank gets it."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_throughput(units_per_rank, steps, world, ms_total):
    """Whole-job throughput in millions of units per second: `world` replicas,
    each processing units_per_rank units a step, `steps` steps in ms_total
    (the slowest rank's time)."""
    return world * units_per_rank * steps / (ms_total / 1e3) / 1e6


def timed(step, steps, warmup, world, local, after_warmup=None):
    """W untimed steps, then K steps between barriers, timed with CUDA events
    on the current stream; returns (max over ranks of the total ms, clocks)."""
    import torch
    import torch.distributed as dist
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    if after_warmup:
        after_warmup()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(steps):
        step()
    stop.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clock_info = clocks.stop()
    ms = max_over_ranks(start.elapsed_time(stop), world, torch.device("cuda", local))
    return ms, clock_info


def run_batched(args, world, rank, local, device):
    """16 scenes (log-uniform 50k-2M splats, SH 3 fp32), 64 views on a sphere
    of radius 4 (view v sees scene v mod 16): one CUDA-graph launch per step."""
    import numpy as np
    import torch

    import radix_b200 as rb
    from radix_b200 import synthetic as syn
    counts = syn.batched_counts(16, seed=2)
    tables = []
    for s, c in enumerate(counts):
        d = syn.mixture_table(c, seed=100 + s, sh_degree=SH_DEGREE, device=device)
        tables.append(rb.Table.raw(*(torch.from_numpy(np.ascontiguousarray(d[k])).to(device) for k in
                                     ("centers", "log_scales", "quats", "opacities", "colors")), SH_DEGREE))
    cams = syn.sphere_cameras(64, seed=1)
    views = [([rb.SplatObject(tables[v % 16])], cams[v]) for v in range(64)]
    n_views = sum(counts[v % 16] for v in range(64))
    names = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")
    ctx = rb.Context(local)
    batch = rb.Batch(views, None, BITS, names, device=device, ctx=ctx)
    tuning = None if args.no_tune else batch.tune(reps=5)
    graph_kernels = batch.launches()
    ms_total, clock_info = timed(batch.launch, args.steps, args.warmup, world, local)
    batch.synchronize()
    ms_step = ms_total / args.steps
    # the plain path for the same 64 views: one single-view graph each (every
    # view's own projection and sort), launched back to back
    singles = [rb.Batch([view], None, BITS, names, device=device, ctx=ctx) for view in views]

    def plain_step():
        for b in singles:
            b.launch()

    plain_total, _ = timed(plain_step, max(3, args.steps // 4), 2, world, local)
    plain_ms = plain_total / max(3, args.steps // 4)
    for b in singles:
        b.synchronize()
        b.close()
    del singles
    # the projection / sort split of the same batch, from the direct call's phase events
    out = rb._alloc_outputs(names, n_views, 1, device)
    ordering = torch.empty(n_views, dtype=torch.int32, device=device)
    visible = torch.zeros(64, dtype=torch.int32, device=device)
    for _ in range(2):
        rb.frame_batched(views, None, BITS, names, ctx=ctx, out=out, ordering=ordering, visible=visible)
    torch.cuda.synchronize()
    ctx.set_profiling(True)
    ctx.phase_times()
    for _ in range(5):
        rb.frame_batched(views, None, BITS, names, ctx=ctx, out=out, ordering=ordering, visible=visible)
    phases = ctx.phase_times()
    ctx.set_profiling(False)
    proj_ms = phases["project"][0] / max(phases["project"][1], 1)
    sort_ms = phases["sort"][0] / max(phases["sort"][1], 1)
    peak, peak_kind = peak_hbm()
    achieved = PROJECT_BYTES * n_views / (proj_ms / 1e3) / 1e9
    batch.close()
    return {
        "metric": "Msplat-views/s (batched project+SH+key+sort)",
        "value": replicas_throughput(n_views, args.steps, world, ms_total), "unit": "Msplat-views/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded mulberry32 + Box-Muller)",
        "config": {"workload": "batched: 16 scenes (log-uniform 50k-2M splats, SH 3 fp32, Gaussian mixtures), "
                               f"64 views on a sphere of radius 4, 1920x1080 fov 50, {BITS}-bit keys, "
                               "one CUDA-graph launch (projection + segmented sort) per step",
                   "scenes": counts, "splat_views": n_views, "bits": BITS, "parallelism": f"replicas{world}",
                   "l2": "inputs 2 GB > 126 MB L2 (no flush)", "frame_bytes_per_splat_view": FRAME_BYTES,
                   "hbm_frac_frame": FRAME_BYTES * n_views / (ms_step / 1e3) / 1e9 / peak,
                   "project_ms": proj_ms, "sort_ms": sort_ms,
                   "plain_ms": plain_ms, "batched_over_plain": ms_step / plain_ms,
                   "plain": "the same 64 views as 64 single-view CUDA graphs (projection + sort each)",
                   "tuning": tuning},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "k_project (raw, SH 3, 1 eye), all 64 views in one launch",
                     "bytes_per_splat": PROJECT_BYTES, "peak_kind": peak_kind},
        "e2e": None, "e2e_note": "a graph batch takes device memory only",
        "gpu_launches": graph_kernels * args.steps,
        "clocks": clock_info,
    }


def run_stereo(args, world, rank, local, device):
    """16M splats, SH 3 stored as fp16, two eyes 2064x2208 fov 100 with a
    64 mm baseline, one key per splat from the head."""
    import numpy as np
    import torch

    import radix_b200 as rb
    from radix_b200 import synthetic as syn
    n = 16_000_000 if args.n == N_SPLATS else args.n
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE, color_dtype=np.float16, device=device)
    cols = {k: torch.from_numpy(np.ascontiguousarray(d[k])).to(device)
            for k in ("centers", "log_scales", "quats", "opacities", "colors")}
    del d
    table = rb.Table.raw(cols["centers"], cols["log_scales"], cols["quats"], cols["opacities"], cols["colors"],
                         SH_DEGREE)
    cam = syn.stereo_camera()
    names = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")
    out = rb._alloc_outputs(names, n, 2, device)
    ordering = torch.empty(n, dtype=torch.int32, device=device)
    visible = torch.zeros(1, dtype=torch.int32, device=device)
    ctx = rb.Context(local)
    ctx.reserve(n)
    obj = [rb.SplatObject(table)]

    def step():
        rb.frame(obj, cam, None, BITS, names, ctx=ctx, out=out, ordering=ordering, visible=visible)

    marks = {}

    def start_counting():
        ctx.set_profiling(True)
        ctx.phase_times()
        marks["launches"] = ctx.launches()

    ms_total, clock_info = timed(step, args.steps, args.warmup, world, local, start_counting)
    launches = ctx.launches() - marks["launches"]
    phases = ctx.phase_times()
    ctx.set_profiling(False)
    runs = args.steps
    proj_ms = phases["project"][0] / max(phases["project"][1], 1)
    sort_ms = phases["sort"][0] / max(phases["sort"][1], 1)
    ms_step = ms_total / args.steps
    # the batched form of the same stereo frame (one CUDA graph, tuned), and a
    # mono frame of the same table and pose (one eye at the head, same size and fov)
    batch = rb.Batch([(obj, cam)], None, BITS, names, device=device, ctx=ctx)
    tuning = None if args.no_tune else batch.tune(reps=3)
    batched_total, _ = timed(batch.launch, args.steps, 2, world, local)
    batch.synchronize()
    batch.close()
    batched_ms = batched_total / args.steps
    mono = syn.Camera.mono((0.0, 0.5, 3.0), (0.0, 0.0, 0.0), 100.0, 2064, 2208)
    out_mono = rb._alloc_outputs(names, n, 1, device)

    def mono_step():
        rb.frame(obj, mono, None, BITS, names, ctx=ctx, out=out_mono, ordering=ordering, visible=visible)

    mono_total, _ = timed(mono_step, args.steps, 2, world, local)
    mono_ms = mono_total / args.steps
    del out_mono
    in_bytes = 12 + 12 + 16 + 4 + 96
    proj_bytes = in_bytes + 2 * 40 + 4
    frame_bytes = in_bytes + 2 * 40 + 8 + 16 * (BITS // 8) + 4
    peak, peak_kind = peak_hbm()
    achieved = proj_bytes * n / (proj_ms / 1e3) / 1e9
    return {
        "metric": "Msplats/s (stereo project+SH+key+sort)",
        "value": replicas_throughput(n, args.steps, world, ms_total), "unit": "Msplats/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f16 SH, f32+f64 maths",
        "data": "synthetic (seeded mulberry32 + Box-Muller)",
        "config": {"workload": f"stereo: {n} splats, SH 3 stored fp16, two eyes 2064x2208 fov 100, 64 mm "
                               f"baseline, one key per splat from the head, {BITS}-bit keys",
                   "n": n, "eyes": 2, "bits": BITS, "parallelism": f"replicas{world}",
                   "l2": "inputs 2.2 GB > 126 MB L2 (no flush)", "frame_bytes_per_splat": frame_bytes,
                   "hbm_frac_frame": frame_bytes * n / (ms_step / 1e3) / 1e9 / peak,
                   "project_ms": proj_ms, "sort_ms": sort_ms, "phase_runs": runs,
                   "batched_ms": batched_ms, "batched_over_plain": batched_ms / ms_step,
                   "mono_ms": mono_ms, "stereo_over_mono": ms_step / mono_ms,
                   "mono": "one eye at the head, 2064x2208 fov 100, the same table (rb.frame)",
                   "tuning": tuning},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": ncu_traffic("project_kernel_stereo_2m.md", n / 2_000_000),
                     "kernel": "k_project (raw, SH 3 fp16, 2 eyes)",
                     "bytes_per_splat": proj_bytes, "peak_kind": peak_kind},
        "e2e": None, "e2e_note": "device-resident tables; the headline workload carries the host end-to-end number",
        "gpu_launches": launches,
        "clocks": clock_info,
    }


def run_backward(args, world, rank, local, device):
    """1M splats of the SH-3 mixture: the forward projection (mean2d, conic,
    depth, opacity, rgb) and its gradient with respect to the table, upstream
    gradients N(0, 1); timed separately, the backward is the step."""
    import numpy as np
    import torch

    import radix_b200 as rb
    from radix_b200 import synthetic as syn
    n = 1_000_000 if args.n == N_SPLATS else args.n
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE, device=device)
    cols = {k: torch.from_numpy(np.ascontiguousarray(d[k])).to(device)
            for k in ("centers", "log_scales", "quats", "opacities", "colors")}
    table = rb.Table.raw(cols["centers"], cols["log_scales"], cols["quats"], cols["opacities"], cols["colors"],
                         SH_DEGREE)
    obj = [rb.SplatObject(table)]
    cam = syn.scale_camera()
    ctx = rb.Context(local)
    names = ("mean2d", "conic", "depth", "opacity", "rgb")
    out = rb._alloc_outputs(names, n, 1, device)
    g = torch.Generator(device=device).manual_seed(1)
    up = {k: torch.randn(out[k].shape, device=device, generator=g) for k in ("mean2d", "conic", "opacity", "rgb")}
    grads = [{"centers": torch.empty((n, 3), device=device), "log_scales": torch.empty((n, 3), device=device),
              "quats": torch.empty((n, 4), device=device), "opacities": torch.empty(n, device=device),
              "colors": torch.empty((n, (SH_DEGREE + 1) ** 2, 3), device=device)}]

    def forward():
        rb.project_collection(obj, cam, None, BITS, "full", True, names, ctx=ctx, out=out)

    def backward():
        rb.project_backward(obj, cam, up, out["opacity"], None, ctx=ctx, grads=grads)

    marks = {}

    def start_counting():
        marks["launches"] = ctx.launches()

    fwd_ms, _ = timed(forward, args.steps, args.warmup, world, local)
    ms_total, clock_info = timed(backward, args.steps, args.warmup, world, local, start_counting)
    launches = ctx.launches() - marks["launches"]
    ms_step = ms_total / args.steps
    fwd_step = fwd_ms / args.steps
    in_bytes = 12 + 12 + 16 + 4 + 192
    bwd_bytes = in_bytes + 36 + 4 + in_bytes  # table re-read, upstream + forward opacity, gradients
    peak, peak_kind = peak_hbm()
    achieved = bwd_bytes * n / (ms_step / 1e3) / 1e9
    return {
        "metric": "Msplats/s (projection backward)",
        "value": replicas_throughput(n, args.steps, world, ms_total), "unit": "Msplats/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 adjoint, f32 I/O",
        "data": "synthetic (seeded mulberry32 + Box-Muller; upstream N(0, 1))",
        "config": {"workload": f"backward: {n} splats, SH 3 fp32, Gaussian-mixture centres, 1920x1080 fov 50; "
                               "gradient of mean2d/conic/opacity/rgb w.r.t. centres, ln scales, quaternions, "
                               "opacities and colour rows",
                   "n": n, "parallelism": f"replicas{world}", "l2": "inputs 236 MB > 126 MB L2 (no flush)",
                   "forward_ms": fwd_step, "backward_over_forward": ms_step / fwd_step,
                   "backward_bytes_per_splat": bwd_bytes},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": ncu_traffic("backward_kernel_1m_sh3.md", n / 1_000_000),
                     "kernel": "k_project_backward (raw, SH 3, 1 eye)",
                     "bytes_per_splat": bwd_bytes, "peak_kind": peak_kind},
        "e2e": None, "e2e_note": "device-resident tensors (a training step's layout)",
        "gpu_launches": launches,
        "clocks": clock_info,
    }


def run_ply(args, world, rank, local, device):
    """A 1M-splat SH-3 standard 3DGS PLY file (59 float properties, 236 B a
    splat) in device memory decoded into a raw table each step."""
    import numpy as np
    import torch

    import radix_b200 as rb
    from radix_b200 import synthetic as syn
    n = 1_000_000 if args.n == N_SPLATS else args.n
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE, device=device)
    k = (SH_DEGREE + 1) ** 2 - 1
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2"] + [f"f_rest_{i}" for i in range(3 * k)] + \
        ["opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"]
    header = ("ply\nformat binary_little_endian 1.0\nelement vertex %d\n" % n +
              "".join(f"property float {nm}\n" for nm in names) + "end_header\n").encode()
    c0 = 0.28209479177387814
    op = np.clip(d["opacities"].astype(np.float64), 1e-6, 1 - 1e-6)
    cols = [d["centers"], (d["colors"][:, 0].astype(np.float64) - 0.5) / c0]
    cols += [d["colors"][:, 1:, ch] for ch in range(3)]
    cols += [np.log(op / (1 - op))[:, None], d["log_scales"], d["quats"][:, 3:4], d["quats"][:, :3]]
    body = np.concatenate([np.asarray(x, dtype=np.float32).reshape(n, -1) for x in cols], axis=1)
    raw = np.concatenate([np.frombuffer(header, dtype=np.uint8), body.view(np.uint8).reshape(-1)])
    data = torch.from_numpy(raw).to(device)
    del d, body
    ctx = rb.Context(local)
    table, out = rb.decode_ply(data, ctx=ctx)
    record = 4 * len(names)
    row = (k + 1) * 3 * 4

    def step():
        rb.decode_ply(data, ctx=ctx)

    marks = {}

    def start_counting():
        marks["launches"] = ctx.launches()

    ms_total, clock_info = timed(step, args.steps, args.warmup, world, local, start_counting)
    launches = ctx.launches() - marks["launches"]
    ms_step = ms_total / args.steps

    # the decode kernel's own time (CUDA events around each launch)
    def start_profiling():
        ctx.set_profiling(True)
        ctx.phase_times()

    timed(step, args.steps, 1, world, local, start_profiling)
    kernel_ms, kernel_runs = ctx.phase_times()["project"]
    ctx.set_profiling(False)
    kernel_ms /= max(kernel_runs, 1)
    peak, peak_kind = peak_hbm()
    bytes_per = record + 12 + 12 + 16 + 4 + row
    achieved = bytes_per * n / (kernel_ms / 1e3) / 1e9
    return {
        "metric": "Msplats/s (PLY decode)", "value": replicas_throughput(n, args.steps, world, ms_total),
        "unit": "Msplats/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 in, f64 maths, f32 out",
        "data": "synthetic (a PLY file written from the seeded SH-3 mixture)",
        "config": {"workload": f"PLY decode: {n} splats, standard 3DGS, SH 3 ({record} B records) in device memory "
                               "to a raw float32 table", "n": n, "parallelism": f"replicas{world}",
                   "bytes_per_splat": bytes_per, "kernel_ms": kernel_ms,
                   "note": "each step includes the header read on the host (4 KB device-to-host copies)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": ncu_traffic("ply_decode_kernel_1m_sh3.md"), "kernel": "k_decode_ply_rows<48>",
                     "bytes_per_splat": bytes_per, "peak_kind": peak_kind},
        "e2e": None, "e2e_note": "device-resident file bytes",
        "gpu_launches": launches, "clocks": clock_info,
    }


def run_spz(args, world, rank, local, device):
    """A 1M-splat SH-3 SPZ file (version 3, gzip) in host memory decoded into a
    raw table on the GPU each step: the host inflates the container, the device
    decodes the byte columns. The device decode is timed alone beside it."""
    import torch

    import radix_b200 as rb
    from radix_b200 import synthetic as syn
    from tests import spz_fixtures as sf
    n = 1_000_000 if args.n == N_SPLATS else args.n
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE)
    raw = sf.gzip_spz(d, version=3) if args.spz_container == "gzip" else sf.ngsp_spz(d)
    form = "version 3 in gzip" if args.spz_container == "gzip" else "SPZ 4 (NGSP, zstd streams)"
    del d
    ctx = rb.Context(local)
    rb.decode_spz(raw, ctx=ctx)
    k = (SH_DEGREE + 1) ** 2 - 1
    payload = n * (9 + 1 + 3 + 3 + 4 + 3 * k)

    def step():
        rb.decode_spz(raw, ctx=ctx)

    marks = {}

    def start_counting():
        marks["launches"] = ctx.launches()

    ms_total, clock_info = timed(step, args.steps, args.warmup, world, local, start_counting)
    launches = ctx.launches() - marks["launches"]
    ms_step = ms_total / args.steps
    # the device decode alone: phase events around its launch, outside the timed region
    ctx.set_profiling(True)
    ctx.phase_times()
    for _ in range(5):
        rb.decode_spz(raw, ctx=ctx)
    torch.cuda.synchronize()
    kt, kr = ctx.phase_times()["project"]
    ctx.set_profiling(False)
    kernel_ms = kt / max(kr, 1)
    peak, peak_kind = peak_hbm()
    bytes_per = payload // n + 12 + 12 + 16 + 4 + (k + 1) * 3 * 4
    achieved = bytes_per * n / (kernel_ms / 1e3) / 1e9
    value = replicas_throughput(n, args.steps, world, ms_total)
    return {
        "metric": "Msplats/s (SPZ decode, host bytes to a device table)", "value": value,
        "unit": "Msplats/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8 in, f64 maths, f32 out",
        "data": "synthetic (an SPZ file written from the seeded SH-3 mixture)",
        "config": {"workload": f"SPZ decode: {n} splats, {form} ({len(raw)} B file, {payload} B of columns), "
                               "SH 3, host bytes to a raw float32 table on the GPU", "n": n,
                   "parallelism": f"replicas{world}", "file_bytes": len(raw), "kernel_ms": kernel_ms,
                   "note": "a step: the container unpacked on the host (gzip: zlib on one thread; NGSP: libzstd, "
                           "the streams on host threads side by side), columns copied, decoded on the GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": ncu_traffic("spz_decode_kernel_1m_sh3.md", n / 1_000_000), "kernel": "k_decode_spz",
                     "bytes_per_splat": bytes_per, "peak_kind": peak_kind},
        "e2e": {"value": value, "unit": "Msplats/s", "h2d_bytes_per_step": payload, "d2h_bytes_per_step": 0},
        "gpu_launches": launches, "clocks": clock_info,
    }


def run_rdx(args, world, rank, local, device):
    """A 1M-splat RDX file in host memory decoded into device channel arrays
    each step: an extSplats bundle (extA, extB) and a degree-3 extSh bundle
    (four channels), six uint32x4 channels in 64k-row chunks, every chunk's
    channel byte-transposed and gzipped. The host inflates the payloads, the
    device un-transposes them in one launch, which is timed alone beside it.
    The words are the seeded SH-3 mixture's float32 columns, so the payloads
    compress like splat data; the decode does not interpret them."""
    import numpy as np
    import torch

    import radix_b200 as rb
    from radix_b200 import synthetic as syn
    from tests import rdx_fixtures as rf
    n = 1_000_000 if args.n == N_SPLATS else args.n
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE)

    def words(*cols):
        rows = np.concatenate([np.asarray(c, np.float32).reshape(n, -1) for c in cols], 1)
        return np.ascontiguousarray(rows).view(np.uint32)

    sh = np.asarray(d["colors"][:, 1:, :], np.float32).reshape(n, -1)[:, :16]
    chans = {"extA": words(d["centers"], d["opacities"]), "extB": words(d["log_scales"], d["quats"][:, 3])}
    sh_chans = {f"extSh{chr(65 + c)}": np.ascontiguousarray(sh[:, 4 * c:4 * c + 4]).view(np.uint32) for c in range(4)}
    bundles = {"extSplats": ({k: "uint32x4" for k in chans}, {}, chans),
               "extSh": ({k: "uint32x4" for k in sh_chans}, {"codec": "ext", "degree": SH_DEGREE}, sh_chans)}
    raw = rf.rdx_file(bundles, n, 65536, level=6)
    del d, chans, sh_chans, sh
    ctx = rb.Context(local)
    rb.decode_rdxfile(raw, ctx=ctx)
    payload = n * 6 * 16

    def step():
        rb.decode_rdxfile(raw, ctx=ctx)

    marks = {}

    def start_counting():
        marks["launches"] = ctx.launches()

    ms_total, clock_info = timed(step, args.steps, args.warmup, world, local, start_counting)
    launches = ctx.launches() - marks["launches"]
    ms_step = ms_total / args.steps
    # the un-transpose alone: phase events around its launch, outside the timed region
    ctx.set_profiling(True)
    ctx.phase_times()
    for _ in range(5):
        rb.decode_rdxfile(raw, ctx=ctx)
    torch.cuda.synchronize()
    kt, kr = ctx.phase_times()["project"]
    ctx.set_profiling(False)
    kernel_ms = kt / max(kr, 1)
    peak, peak_kind = peak_hbm()
    bytes_per = 2 * 6 * 16  # the inflated payload read, the channel arrays written
    achieved = bytes_per * n / (kernel_ms / 1e3) / 1e9
    value = replicas_throughput(n, args.steps, world, ms_total)
    return {
        "metric": "Msplats/s (RDX decode, host bytes to device channels)", "value": value,
        "unit": "Msplats/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (an RDX file of the seeded SH-3 mixture's float32 words)",
        "config": {"workload": f"RDX decode: {n} splats, extSplats + extSh degree 3 (6 uint32x4 channels, "
                               f"64k-row chunks, {len(raw)} B file), host bytes to device channel arrays", "n": n,
                   "parallelism": f"replicas{world}", "file_bytes": len(raw), "kernel_ms": kernel_ms,
                   "note": "a step: the payloads inflated on one host thread (zlib), copied, un-transposed on the GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": ncu_traffic("rdx_untranspose_kernel_1m.md", n / 1_000_000), "kernel": "k_untranspose",
                     "bytes_per_splat": bytes_per, "peak_kind": peak_kind},
        "e2e": {"value": value, "unit": "Msplats/s", "h2d_bytes_per_step": payload, "d2h_bytes_per_step": 0},
        "gpu_launches": launches, "clocks": clock_info,
    }


def run_census(args, world, rank, local, device):
    """Every device entry point once a step, each timed with CUDA events on the
    library's stream at a size above L2 (or the entry point's own limit), with
    its algorithmic bytes per unit: the census that an ncu launch list of this
    workload turns into DRAM bytes and throughput for every kernel."""
    import ctypes

    import numpy as np
    import torch

    import radix_b200 as rb
    from radix_b200 import _abi
    from radix_b200 import synthetic as syn
    ctx = rb.Context(local)
    n = 32_000_000
    rng = syn.Mulberry32(11)
    dist64 = torch.from_numpy(rng.uniform(n) * 10.0).to(device)
    dist32 = dist64.float()
    keys = torch.empty(n, dtype=torch.int32, device=device)
    out_k = torch.empty(n, dtype=torch.int32, device=device)
    out_v = torch.empty(n, dtype=torch.int32, device=device)
    count = torch.zeros(1, dtype=torch.int32, device=device)
    ctx.call("rdx_sort_keys_compute", dist64.data_ptr(), n, 32, keys.data_ptr())
    keys[::3] = -1  # a third invalid, as a frame's culled splats
    ordering = torch.empty(rb.align_capacity(n), dtype=torch.int32, device=device)
    scratch_k, scratch_v = torch.empty_like(keys), torch.empty_like(keys)
    d = syn.mixture_table(4_000_000, seed=0, sh_degree=SH_DEGREE, device=device)
    cols = {k: torch.from_numpy(np.ascontiguousarray(d[k])).to(device)
            for k in ("centers", "log_scales", "quats", "opacities", "colors")}
    del d
    table = rb.Table.raw(cols["centers"], cols["log_scales"], cols["quats"], cols["opacities"], cols["colors"],
                         SH_DEGREE)
    obj = [rb.SplatObject(table)]
    cam = syn.scale_camera()
    names = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")
    fout = rb._alloc_outputs(names, 4_000_000, 1, device)
    ford = torch.empty(4_000_000, dtype=torch.int32, device=device)
    fvis = torch.zeros(1, dtype=torch.int32, device=device)
    b1 = 1_000_000
    bobj = [rb.SplatObject(rb.Table.raw(*(cols[k][:b1] for k in ("centers", "log_scales", "quats", "opacities",
                                                                   "colors")), SH_DEGREE))]
    bout = rb._alloc_outputs(names, b1, 1, device)
    g = torch.Generator(device=device).manual_seed(1)
    up = {k: torch.randn(bout[k].shape, device=device, generator=g) for k in ("mean2d", "conic", "opacity", "rgb")}
    vis = torch.zeros(1, dtype=torch.int32, device=device)

    def sort(m, variant):
        ctx.set_sort_variant(variant)
        ctx.call("rdx_sort", keys.data_ptr(), m, 32, ordering.data_ptr(), ordering.numel(), None)

    def pairs(m):
        ctx.set_sort_variant(0)
        ctx.call("rdx_sort_pairs", scratch_k.data_ptr(), scratch_v.data_ptr(), m, 32)

    def noalloc(m):
        st = _abi.lib().rdx_sort_noalloc(ctypes.c_void_p(keys.data_ptr()), m, 32, ctypes.c_void_p(ordering.data_ptr()),
                                         ordering.numel(), ctypes.c_void_p(vis.data_ptr()),
                                         ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream))
        assert st == _abi.RDX_OK, st

    def frame():
        ctx.set_sort_variant(1)
        rb.frame(obj, cam, None, BITS, names, ctx=ctx, out=fout, ordering=ford, visible=fvis)

    # (name, call, units, algorithmic bytes a unit, before: untimed set-up of each call)
    families = [
        ("keys from float64 distances", lambda: ctx.call("rdx_sort_keys_compute", dist64.data_ptr(), n, 32,
                                                         out_k.data_ptr()), n, 12, None),
        ("keys from float32 distances", lambda: ctx.call("rdx_sort_keys_compute_f32", dist32.data_ptr(), n, 32,
                                                         out_k.data_ptr()), n, 8, None),
        ("compaction (a third invalid)", lambda: ctx.call("rdx_compact", keys.data_ptr(), n,
                                                          ctypes.c_uint32(0xFFFFFFFF), out_k.data_ptr(),
                                                          out_v.data_ptr(), count.data_ptr()), n, 4 + 8 * 2 / 3, None),
        ("SortKeys.sort 32M, onesweep passes", lambda: sort(n, 0), n, 68, None),
        ("SortKeys.sort 2M, cooperative passes", lambda: sort(2_000_000, 1), 2_000_000, 68, None),
        ("WgpuRadixSort.sort 16M in place", lambda: pairs(16_000_000), 16_000_000, 68,
         lambda: (scratch_k[:16_000_000].copy_(keys[:16_000_000]), scratch_v[:16_000_000].copy_(keys[:16_000_000]))),
        ("rdx_sort_noalloc 1M", lambda: noalloc(b1), b1, 68, None),
        ("frame 4M (projection + sort)", frame, 4_000_000, FRAME_BYTES, None),
        ("projection backward 1M", lambda: rb.project_backward(bobj, cam, up, bout["opacity"], None, ctx=ctx), b1, 512,
         lambda: rb.project_collection(bobj, cam, None, BITS, "full", True, names, ctx=ctx, out=bout)),
    ]
    for method in ("3dgut", "htgs", "raygs"):
        wout = {"words": torch.empty((4_000_000, rb.method_words(method, 1)), dtype=torch.int32, device=device),
                "keys": fout["keys"]}
        families.append((f"{method} words 4M", lambda m=method, o=wout: rb.project_words(obj, cam, m, None, BITS, True,
                                                                                      ctx=ctx, out=o),
                         4_000_000, RAY_BYTES[method], None))
    peak, peak_kind = peak_hbm()
    stream = torch.cuda.current_stream(device)
    results = []
    launches0 = ctx.launches()
    for name, call, units, per_unit, before in families:
        times = []
        for step in range(args.warmup + args.steps):
            if before:
                before()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            torch.cuda.synchronize()
            if step >= args.warmup:
                times.append(e0.elapsed_time(e1))
        ms = statistics.median(times)
        gbs = per_unit * units / (ms / 1e3) / 1e9
        results.append({"call": name, "ms": ms, "units": units, "bytes_per_unit": per_unit, "gb_s": gbs,
                        "frac": gbs / peak})
    ctx.set_sort_variant(-1)
    ctx.synchronize()
    return {
        "metric": "GB/s of algorithmic bytes per call (every device entry point)",
        "value": min(r["frac"] for r in results), "unit": "fraction of measured HBM peak (the lowest call)",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": sum(r["ms"] for r in results),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 keys, f32+f64 maths",
        "data": "synthetic (seeded mulberry32)",
        "config": {"workload": "census: each device entry point once a step, timed alone with CUDA events",
                   "results": results, "peak": peak, "peak_kind": peak_kind},
        "e2e": None, "e2e_note": "device-resident inputs; a per-call census",
        "gpu_launches": ctx.launches() - launches0,
    }


RAY_BYTES = {"3dgut": 236 + 8 * 4 + 4, "htgs": 236 + 8 * 4 + 4, "raygs": 236 + 7 * 4 + 4}


def run_rays(args, world, rank, local, device):
    """The ray projection methods (3dgut, htgs, raygs) on the frame's 4M SH-3
    table and camera: each method's words and keys (rdx_project_words), K
    steps timed between barriers with CUDA events (the slowest rank's time),
    one replica a GPU. A splat's algorithmic bytes: its 236 bytes of fields,
    read once, plus its words and key."""
    import numpy as np
    import torch

    import radix_b200 as rb
    from radix_b200 import synthetic as syn
    ctx = rb.Context(local)
    n = args.n
    d = syn.mixture_table(n, seed=0, sh_degree=SH_DEGREE, device=device)
    cols = {k: torch.from_numpy(np.ascontiguousarray(d[k])).to(device)
            for k in ("centers", "log_scales", "quats", "opacities", "colors")}
    del d
    obj = [rb.SplatObject(rb.Table.raw(cols["centers"], cols["log_scales"], cols["quats"], cols["opacities"],
                                       cols["colors"], SH_DEGREE))]
    cam = syn.scale_camera()
    peak, peak_kind = peak_hbm()
    results = {}
    launches0 = ctx.launches()
    clock_info = None
    for method in ("3dgut", "htgs", "raygs"):
        out = {"words": torch.empty((n, rb.method_words(method, 1)), dtype=torch.int32, device=device),
               "keys": torch.empty(n, dtype=torch.int32, device=device)}

        def step(m=method, o=out):
            rb.project_words(obj, cam, m, None, BITS, True, ctx=ctx, out=o)

        ms_total, clocks = timed(step, args.steps, args.warmup, world, local)
        if clock_info is None:
            clock_info = clocks
        ms = ms_total / args.steps
        gbs = RAY_BYTES[method] * n / (ms / 1e3) / 1e9
        results[method] = {"ms": ms, "msplats_s": replicas_throughput(n, args.steps, world, ms_total),
                           "bytes_per_splat": RAY_BYTES[method], "gb_s_per_gpu": gbs, "frac": gbs / peak,
                           "drawn": int((out["keys"] != -1).sum().item())}
        del out
    ctx.synchronize()
    head = results["3dgut"]
    return {
        "metric": "Msplats/s (ray projection words + keys, 3dgut)", "value": head["msplats_s"], "unit": "Msplats/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 maths, u32 words",
        "data": "synthetic (seeded mulberry32)",
        "config": {"workload": f"rays: {n} splats a GPU, SH {SH_DEGREE} fp32, 1920x1080 fov 50, {BITS}-bit keys; "
                               "each method timed alone (inputs larger than L2)", "parallelism": f"replicas x{world}",
                   "methods": results},
        "roofline": {"bound": "hbm", "achieved": head["gb_s_per_gpu"], "peak": peak, "unit": "GB/s",
                     "frac": head["frac"], "traffic": ncu_traffic("project_rays_kernel_1m_sh3.md", n / 1_000_000),
                     "kernel": "k_project_rays", "peak_kind": peak_kind},
        "clocks": clock_info, "e2e": None, "e2e_note": "device-resident inputs",
        "gpu_launches": ctx.launches() - launches0,
    }


def other_forms(args, world, rank, local, device):
    """The path's other forms, after the headline frame in the same run: the 64-view batch, the
    16M-splat stereo frame and the 1M-splat gradient, each the leg of its own workload (--workload
    batched / stereo / backward) with 10 timed steps after 3 warm-up steps; a summary of each line,
    or the error of a leg that failed (the headline line is printed either way)."""
    import copy
    import gc

    import torch
    sub = copy.copy(args)
    sub.steps, sub.warmup = 10, 3
    legs = (("batched", run_batched, ("plain_ms", "batched_over_plain", "hbm_frac_frame", "project_ms", "sort_ms",
                                      "splat_views", "tuning")),
            ("stereo", run_stereo, ("batched_ms", "batched_over_plain", "mono_ms", "stereo_over_mono", "project_ms",
                                    "sort_ms", "hbm_frac_frame", "n")),
            ("backward", run_backward, ("forward_ms", "backward_over_forward", "n")))
    forms = {}
    for name, run, keys in legs:
        try:
            r = run(sub, world, rank, local, device)
            forms[name] = {"metric": r["metric"], "value": r["value"], "unit": r["unit"], "ms_per_step": r["ms_per_step"],
                           "steps": r["steps"], "roofline_frac": r["roofline"]["frac"],
                           "roofline_kernel": r["roofline"].get("kernel"), "gpu_launches": r.get("gpu_launches"),
                           "clocks": r.get("clocks"), **{k: r["config"][k] for k in keys if k in r["config"]}}
        except Exception as e:  # noqa: BLE001 - recorded in the line, the headline stands
            forms[name] = {"error": f"{type(e).__name__}: {e}"}
        gc.collect()
        torch.cuda.empty_cache()
    return forms


def main():
    global BITS, FRAME_BYTES
    args = parse()
    BITS = args.bits
    FRAME_BYTES = 236 + 40 + 8 + 16 * (BITS // 8) + 4
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "frame":
        import torch
        import torch.distributed as dist
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        local = int(os.environ.get("LOCAL_RANK", "0"))
        torch.cuda.set_device(local)
        device = torch.device("cuda", local)
        if world > 1:
            from datetime import timedelta
            dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)
        run = {"batched": run_batched, "stereo": run_stereo, "backward": run_backward, "ply": run_ply,
               "spz": run_spz, "rdx": run_rdx, "census": run_census, "rays": run_rays}[args.workload]
        line = run(args, world, rank, local, device)
        if rank == 0:
            print(json.dumps(line))
        if world > 1:
            dist.destroy_process_group()
        return
    import torch
    import torch.distributed as dist

    import radix_b200 as rb
    from radix_b200 import synthetic as syn

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)

    n = args.n
    d, host_cols, dev_cols = make_workload(n, device)
    cam = syn.scale_camera() if args.pose == "scale" else syn.all_visible_camera()
    ctx = rb.Context(local)
    table = table_of(dev_cols)
    obj = [rb.SplatObject(table)]
    names = ("mean2d", "conic", "depth", "opacity", "rgb", "keys")
    out = rb._alloc_outputs(names, n, 1, device)
    ordering = torch.empty(n, dtype=torch.int32, device=device)
    visible = torch.zeros(1, dtype=torch.int32, device=device)
    ctx.reserve(n)
    if args.variant is not None:
        ctx.set_sort_variant(args.variant)

    def frame_step():
        rb.frame(obj, cam, None, BITS, names, ctx=ctx, out=out, ordering=ordering, visible=visible)

    # The frame captured once in a CUDA graph (rb.Batch with one view): each
    # step is one graph launch of the projection and the sort
    batch = rb.Batch([(obj, cam)], None, BITS, names, device=device, ctx=ctx)
    tuning = None if args.no_tune or args.variant is not None else batch.tune(reps=5)
    graph_kernels = batch.launches()
    ms_total, clock_info = timed(batch.launch, args.steps, args.warmup, world, local)
    batch.synchronize()
    launches = graph_kernels * args.steps
    ms_step = ms_total / args.steps
    value = replicas_throughput(n, args.steps, world, ms_total)
    # the same frame through rb.frame (host planning every call), and its phase split
    frame_ms, _ = timed(frame_step, args.steps, args.warmup, world, local)

    def start_profiling():
        ctx.set_profiling(True)
        ctx.phase_times()

    timed(frame_step, args.steps, 1, world, local, start_profiling)
    phases = ctx.phase_times()
    ctx.set_profiling(False)
    batch.close()
    drawn = int(visible.cpu().numpy()[0])

    # end to end through the public API: pinned host tables in, the order and
    # the visible count out, the host reads inside the timed region. By default
    # the kernel reads the drawn candidates' quaternion and colour rows in place
    # and the other columns are copied in; the bytes moved are the library's count.
    e2e = None
    if not args.no_e2e:
        host_table = table_of(host_cols)
        host_order = torch.empty(n, dtype=torch.int32).pin_memory()
        hobj = [rb.SplatObject(host_table)]
        table_bytes = sum(v.numel() * v.element_size() for v in host_cols.values())
        bo = n * 4 + 4
        e2e_steps = max(3, min(args.steps, 10))

        def e2e_run(in_place):
            ctx.set_host_reads(in_place)
            rb.frame(hobj, cam, None, BITS, names, ctx=ctx, out=out, ordering=host_order)
            torch.cuda.synchronize()
            ctx.host_bytes()
            if world > 1:
                dist.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(e2e_steps):
                rb.frame(hobj, cam, None, BITS, names, ctx=ctx, out=out, ordering=host_order)
            e1.record()
            torch.cuda.synchronize()
            moved = ctx.host_bytes() / e2e_steps
            return max_over_ranks(e0.elapsed_time(e1), world, device), moved

        copy_ms, copy_bytes = e2e_run(False)
        e_ms, bi = e2e_run(True)
        e2e = {"value": replicas_throughput(n, e2e_steps, world, e_ms), "unit": "Msplats/s",
               "h2d_bytes_per_step": int(bi), "d2h_bytes_per_step": bo, "ms_per_step": e_ms / e2e_steps,
               "host_reads": "in place: the colour rows of splats that pass the centre culls, staged a warp at a "
                             "time; the other columns copied",
               "table_bytes": table_bytes,
               "copy_every_column": {"value": replicas_throughput(n, e2e_steps, world, copy_ms),
                                     "ms_per_step": copy_ms / e2e_steps, "h2d_bytes_per_step": int(copy_bytes)}}

    peak, peak_kind = peak_hbm()
    proj_ms, proj_runs = phases["project"]
    sort_ms, sort_runs = phases["sort"]
    proj_avg = proj_ms / max(proj_runs, 1)
    achieved = PROJECT_BYTES * n / (proj_avg / 1e3) / 1e9
    # ncu DRAM bytes of the projection: captured on 1M splats of the same pose, scaled by the splats processed
    traffic = ncu_traffic("project_kernel_4m_sh3.md" if args.pose == "scale" else "project_kernel_allvis_1m_sh3.md",
                          n / (4_000_000 if args.pose == "scale" else 1_000_000))
    line = {
        "metric": METRIC, "value": value, "unit": "Msplats/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded mulberry32 + Box-Muller)",
        "config": {"workload": f"project+SH+key+sort, {n} splats, SH degree 3 fp32, Gaussian-mixture centres, "
                               f"1920x1080 fov 50, {BITS}-bit keys, stable order",
                   "n": n, "sh_degree": SH_DEGREE, "bits": BITS, "parallelism": f"replicas{world}",
                   "l2": "inputs 944 MB > 126 MB L2 (no flush)",
                   "frame_bytes_per_splat": FRAME_BYTES,
                   "hbm_frac_frame": FRAME_BYTES * n / (ms_step / 1e3) / 1e9 / peak,
                   "project_ms": proj_avg, "sort_ms": sort_ms / max(sort_runs, 1),
                   "step": "one CUDA-graph launch of the frame (rb.Batch, one view, autotuned)",
                   "rb_frame_ms": frame_ms / args.steps, "pose": args.pose,
                   "drawn_fraction": drawn / n, "tuning": tuning},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "k_project (raw, SH 3, 1 eye)",
                     "bytes_per_splat": PROJECT_BYTES, "peak_kind": peak_kind},
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clock_info,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(n)
    if world == 1 and not args.no_forms and args.n == N_SPLATS and args.pose == "scale" and args.variant is None:
        line["config"]["forms"] = other_forms(args, world, rank, local, device)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
