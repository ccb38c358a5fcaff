"""Benchmark of the global repetition map (SReD's block-correlation hot path).

Workload: global repetition map of a 1024x1024 float32 synthetic spot image
(80x80 jittered lattice plus 30% random spots, Poisson + Gaussian noise,
seed 0), 9x9 block (ellipse K = 49), Pearson's R, relevance constant 1.0.

A step is one complete map: moments, relevance mask, compaction, the
all-pairs contraction with its fused epilogue, finalisation and
normalisation. ``value`` is block-pairs/s with the image resident in HBM
(pairs = relevant blocks squared, the pairs the map is defined over); ``e2e``
is the same through the C ABI with host buffers (H2D of the image and D2H of
the map inside the timed region). L2 is flushed (256 MiB write) between
steps, outside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica (the map of its own
image); value = total pairs of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "global-map block-pairs/s at 1024²/9×9; split-BF16 vs FP32 speedup @≤1e-5 err"
W_IMG = H_IMG = 1024
BW = BH = 9
SIM = "Pearson's R"
RELC = 1.0
WORKLOAD = ("global repetition map, 1024x1024 float32 spot image (80x80 lattice + 30% random spots), "
            "9x9 block (ellipse K=49), Pearson's R, relevance constant 1.0")


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"],
                "bf16_tflops_sustained": d["bf16_tflops_sustained"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0, "source": "fallback"}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                self.out, _ = self.p.communicate()

    def summary(self) -> dict:
        rows = [r.split(", ") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, local, world


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def image(seed: int) -> np.ndarray:
    from sred_b200 import synth
    if W_IMG == 1024 and H_IMG == 1024:
        return synth.normalize_input(synth.image_1024_spots_random(seed=seed))
    if W_IMG == 2048 and H_IMG == 2048:
        return synth.normalize_input(synth.image_2048_elongated(seed=seed))
    if W_IMG == 256 and H_IMG == 256:
        return synth.normalize_input(synth.image_256_spots(seed=seed))
    # Same spot density and layout at another side (used for profiling captures).
    return synth.normalize_input(synth.spot_image(W_IMG, H_IMG, max(2, W_IMG * 80 // 1024), seed=seed,
                                                  random_fraction=0.3))


def time_engine(ctx, engine, d_img, d_out, flush, steps, warmup, stream):
    """Device-resident steps; returns (per-step ms list, last run info, launches)."""
    import torch
    from sred_b200 import clutils
    ctx.set_engine(engine)
    for _ in range(warmup):
        clutils.global_map_device(SIM, d_img.data_ptr(), W_IMG, H_IMG, BW, BH, RELC, True, d_out.data_ptr(),
                                  stream.cuda_stream, ctx=ctx)
    ms, gram_ms, launches, info = [], [], 0, None
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        info = clutils.global_map_device(SIM, d_img.data_ptr(), W_IMG, H_IMG, BW, BH, RELC, True,
                                         d_out.data_ptr(), stream.cuda_stream, ctx=ctx)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        gram_ms.append(info["ms_gram"])
        launches += info["launches"]
    return ms, gram_ms, info, launches


def cpu_baseline(img: np.ndarray, gpu_map: np.ndarray | None, budget_s: float = 12.0) -> dict:
    """The reference's own kernel (oracle/_ref, compiled for the CPU) on a
    bounded sample of reference pixels against all test blocks, on all host
    cores; falls back to the oracle's FP32 port if _ref was not built."""
    import oracle
    kind = "reference" if oracle.refshim() is not None else "port"
    means, stds = oracle.local_stats(img, BW, BH)
    mask, thr, nv = oracle.relevance_mask(img, BW, BH, stds, RELC)
    H, W = img.shape
    rel = np.flatnonzero((stds.ravel() * stds.ravel() >= thr) & (np.arange(W * H) % W >= BW // 2) &
                         (np.arange(W * H) % W < W - BW // 2) & (np.arange(W * H) // W >= BH // 2) &
                         (np.arange(W * H) // W < H - BH // 2))
    n_rel = rel.size
    rng = np.random.default_rng(123)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    rows = rng.choice(rel, size=min(n_rel, 2 * cores), replace=False).astype(np.int32)
    t0 = time.perf_counter()
    oracle.global_sums_f32(SIM, img, BW, BH, means, stds, nv, thr, rows, use_refshim=(kind == "reference"))
    t_probe = time.perf_counter() - t0
    n_rows = int(max(cores, min(n_rel, budget_s / max(t_probe, 1e-6) * rows.size)))
    rows = rng.choice(rel, size=n_rows, replace=False).astype(np.int32)
    t0 = time.perf_counter()
    num, den = oracle.global_sums_f32(SIM, img, BW, BH, means, stds, nv, thr, rows,
                                      use_refshim=(kind == "reference"))
    dt = time.perf_counter() - t0
    pairs = float(rows.size) * n_rel
    res = {"value": pairs / dt, "unit": "block-pairs/s", "cores": cores, "kind": kind,
           "sample": f"{rows.size} relevant reference pixels x all {n_rel} relevant test blocks "
                     f"({pairs:.3g} pairs, {dt:.1f} s); rate extrapolates per pair"}
    if gpu_map is not None:
        npx = float(oracle.n_pixels(mask, BW // 2, BH // 2))
        raw = num / (den * np.float32(npx) + np.float32(1e-7))
        res["gpu_raw_rel_err_vs_reference_sample"] = None if gpu_map is None else float(
            np.max(np.abs(gpu_map.ravel()[rows] - raw) / np.maximum(np.abs(raw), 1e-30)))
    return res


def run_ours(args, rank, local, world):
    import torch
    from sred_b200 import _lib, clutils
    torch.cuda.set_device(local)
    ctx = _lib.Context(local, "tc")
    stream = torch.cuda.Stream()
    img = image(seed=rank)
    d_img = torch.from_numpy(img).cuda()
    d_out = torch.empty_like(d_img)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    engines = [args.engine] + (["fp32"] if args.engine == "tc" and not args.no_compare else [])
    results = {}
    for eng in engines:
        steps = args.steps if eng == args.engine else max(2, min(args.steps, 3))
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        with Clocks(local) as clk:
            ms, gram_ms, info, launches = time_engine(ctx, eng, d_img, d_out, flush, steps, args.warmup, stream)
        torch.cuda.synchronize()
        total_ms = max_over_ranks(sum(ms), world)
        pairs = sum_over_ranks(info["pairs"] * steps, world)
        results[eng] = {"ms": ms, "gram_ms": gram_ms, "info": info, "launches": launches, "total_ms": total_ms,
                        "pairs": pairs, "clocks": clk.summary(), "steps": steps}

    # End to end through the C ABI with host buffers (pinned).
    ctx.set_engine(args.engine)
    h_img = torch.from_numpy(img).pin_memory()
    h_out = torch.empty_like(h_img).pin_memory()
    for _ in range(args.warmup):
        clutils.global_map_host(SIM, h_img.numpy(), BW, BH, RELC, True, out=h_out.numpy(), ctx=ctx)
    e2e_s = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, info_e = clutils.global_map_host(SIM, h_img.numpy(), BW, BH, RELC, True, out=h_out.numpy(), ctx=ctx)
        e2e_s.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(sum(e2e_s), world)
    e2e_pairs = sum_over_ranks(info_e["pairs"] * args.steps, world)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()

    if rank != 0:
        return
    r = results[args.engine]
    pk = peaks()
    K = r["info"]["k"]
    gram_s = statistics.mean(r["gram_ms"]) / 1e3
    per_launch_pairs = r["info"]["pairs"]
    line = {
        "metric": METRIC,
        "value": r["pairs"] / (r["total_ms"] / 1e3),
        "unit": "block-pairs/s",
        "n_gpus": world,
        "steps": r["steps"],
        "warmup": args.warmup,
        "ms_per_step": r["total_ms"] / r["steps"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "bf16x3 split (hi/lo) tensor-core Gram, f32 accumulate, f64 moments" if r["info"]["engine"] == 0
                 else "f32 CUDA-core Gram, f64 moments",
        "data": "synthetic (seeded spot image, numpy default_rng; no dataset)",
        "config": {"workload": WORKLOAD, "image": f"{W_IMG}x{H_IMG}", "block": f"{BW}x{BH}", "K": K,
                   "metric": SIM, "relevance_constant": RELC, "engine": args.engine,
                   "relevant_blocks": r["info"]["n_relevant"], "pairs_per_step": per_launch_pairs,
                   "l2": "flushed between steps (256 MiB write, outside the timed region)",
                   "parallelism": f"{world} independent replica(s)"},
        "gpu_launches": r["launches"],
        "clocks": r["clocks"],
    }
    if r["info"]["engine"] == 0:  # tensor-core engine
        eff_peak = pk["bf16_tflops_sustained"] / 3.0
        n_g = r["info"]["n_relevant"] - r["info"]["n_flat"]
        evaluated = n_g * (n_g + 1) / 2  # each unordered pair of non-flat blocks once
        achieved = evaluated * 2 * K / gram_s / 1e12
        line["roofline"] = {
            "bound": "tensor", "achieved": achieved, "peak": eff_peak, "unit": "TFLOP/s",
            "frac": achieved / eff_peak, "traffic": traffic_from_profile(),
            "evaluated_pairs_per_launch": evaluated,
            "note": f"all-pairs Gram kernel; algorithmic FLOPs = contracted pairs x 2K (K={K}), contracted pairs = "
                    f"n(n+1)/2 of the n non-flat relevant blocks (symmetric schedule: each unordered pair once; "
                    f"value counts all relevant^2 ordered pairs the map is defined over); peak = {pk['source']} "
                    f"sustained BF16 / 3 (three hi/lo products per FP32-accurate product)"}
    if "fp32" in results and args.engine != "fp32":
        f = results["fp32"]
        fv = f["pairs"] / (f["total_ms"] / 1e3)
        line["fp32_engine"] = {"value": fv, "ms_per_step": f["total_ms"] / f["steps"], "steps": f["steps"],
                               "gram_ms": statistics.mean(f["gram_ms"])}
        line["speedup_tc_vs_fp32"] = line["value"] / fv
        line["gram_speedup_tc_vs_fp32"] = statistics.mean(f["gram_ms"]) / (gram_s * 1e3)
    line["e2e"] = {"value": e2e_pairs / e2e_total, "unit": "block-pairs/s",
                   "h2d_bytes_per_step": 4 * W_IMG * H_IMG, "d2h_bytes_per_step": 4 * W_IMG * H_IMG,
                   "ms_per_step": 1e3 * e2e_total / args.steps}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(img, None)
    print(json.dumps(line), flush=True)


def traffic_from_profile():
    """ncu DRAM bytes per Gram launch, recorded for the default workload only."""
    if (W_IMG, H_IMG, BW, BH, RELC, SIM) != (1024, 1024, 9, 9, 1.0, "Pearson's R"):
        return None
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("gram_tc_bytes_per_launch")
        except Exception:
            return None
    return None


BLOCK_METRICS = ["Pearson's R", "SSIM", "NRMSE (inverted)", "Abs. Diff. of StdDevs.", "Cosine", "Hu moments",
                 "Phase correlation", "Hu distance"]
# FP64 shape metrics run on the first frames of the stack only (they are compute-bound: ~1 ms and ~21 ms per
# 1024x1024 frame at 15x15), so the block workload still ends within a few minutes.
SHAPE_FRAMES = 8


def run_block(args, rank, local, world):
    """Block (local) repetition map: a stack of 1024x1024 frames (6,400-spot
    lattice images, one seed per frame) against one 15x15 reference block cut
    at a seeded position from frame 0, relevance 0, normalised per frame; the
    stack (frames x 4 MB) is larger than L2. Reports frames x pixels / s and
    GB/s of the 8 algorithmic bytes per pixel (4 B read, 4 B written)."""
    import torch
    from sred_b200 import _lib, clutils, synth, utils
    torch.cuda.set_device(local)
    ctx = _lib.Context(local, "tc")
    frames = args.frames
    base = [synth.normalize_input(synth.image_1024_spots(seed=100 * rank + f)) for f in range(4)]
    stack = np.stack([base[f % 4] for f in range(frames)])
    rng = np.random.default_rng(7)
    y0, x0 = rng.integers(0, 1024 - 15, 2)
    ref = utils.get_reference_block_2d(base[0][y0:y0 + 15, x0:x0 + 15])
    d_in = torch.from_numpy(stack).cuda()
    d_out = torch.empty_like(d_in)
    stream = torch.cuda.Stream()
    res = {}
    clocks = Clocks(local)
    clocks.__enter__()
    for metric in BLOCK_METRICS:
        nf = min(frames, SHAPE_FRAMES) if metric in ("Hu moments", "Phase correlation", "Hu distance") else frames
        for _ in range(args.warmup):
            clutils.block_map_device(metric, d_in.data_ptr(), 1024, 1024, nf, ref, 0.0, True, d_out.data_ptr(),
                                     stream.cuda_stream, ctx=ctx)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            clutils.block_map_device(metric, d_in.data_ptr(), 1024, 1024, nf, ref, 0.0, True, d_out.data_ptr(),
                                     stream.cuda_stream, ctx=ctx)
        e1.record(stream)
        e1.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
        px = 1024 * 1024 * nf * world
        res[metric] = {"frames": nf, "ms_per_step": ms, "ms_per_frame": ms / nf, "pixels_per_s": px / (ms / 1e3),
                       "gbs_8B_per_pixel": 8 * px / (ms / 1e3) / 1e9}
    clocks.__exit__(None, None, None)
    # end to end: host stack in, host maps out, through the public call (page-locked host buffers, as a
    # caller streaming time-lapses would hold); pipelined in chunks, and as one chunk (copies not overlapped)
    h_in = torch.from_numpy(stack).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    e2e = {}
    for name, chunk in (("pipelined", 0), ("one_chunk", frames)):
        for _ in range(args.warmup):
            clutils.block_map_stack("Pearson's R", h_in.numpy(), ref, 0.0, True, chunk_frames=chunk,
                                    out=h_out.numpy(), ctx=ctx)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            clutils.block_map_stack("Pearson's R", h_in.numpy(), ref, 0.0, True, chunk_frames=chunk,
                                    out=h_out.numpy(), ctx=ctx)
        e2e[name] = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps, world)
    if rank != 0:
        return
    pk = peaks()
    p = res["Pearson's R"]
    line = {"metric": "block-map pixels/s at 1024²/15×15 (HBM-streaming local map)", "value": p["pixels_per_s"],
            "unit": "pixels/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": p["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (reference evaluation order, bit-exact)", "data": "synthetic",
            "config": {"workload": f"block repetition map, {frames} frames of 1024x1024 float32 spot images, "
                                   f"15x15 reference block (K=149), relevance 0, normalised per frame",
                       "frames": frames, "l2": f"stack of {4 * frames} MB > L2"},
            "per_metric": res,
            "e2e": {"value": 1024 * 1024 * frames * world / (e2e["pipelined"] / 1e3), "unit": "pixels/s",
                    "h2d_bytes_per_step": int(stack.nbytes), "d2h_bytes_per_step": int(stack.nbytes),
                    "ms_per_step": e2e["pipelined"], "ms_per_step_one_chunk": e2e["one_chunk"],
                    "call": "clutils.block_map_stack (sred_block_map_2d_stack), Pearson's R, page-locked buffers"},
            "clocks": clocks.summary(),
            # per Pearson call: map, min-max initialisation, min-max, remap
            "gpu_launches": 4 * args.steps,
            "roofline": {"bound": "hbm", "achieved": p["gbs_8B_per_pixel"], "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": p["gbs_8B_per_pixel"] / pk["hbm_gbs"], "traffic": None,
                         "note": "8 algorithmic bytes per pixel over the whole call (map kernel plus per-frame "
                                 "normalisation passes); the map kernel evaluates 149-element sums in the "
                                 "reference's sequential FP32 order, so it is issue-bound, not HBM-bound"}}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = block_cpu_baseline(stack, ref)
    print(json.dumps(line), flush=True)


def block_cpu_baseline(frames: np.ndarray, ref, budget_s: float = 10.0) -> dict:
    """The reference's 2D block kernel (oracle/_ref, compiled for the CPU; the
    oracle's FP32 port if not built) with the Java host steps, Pearson's R,
    15x15, on whole 1024x1024 frames until about budget_s, on all host cores."""
    import oracle
    kind = "reference" if oracle.refshim() is not None else "port"
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    n, t0 = 0, time.perf_counter()
    while n < frames.shape[0] and (n == 0 or time.perf_counter() - t0 < budget_s):
        oracle.block_map("Pearson's R", frames[n], ref.pixels, ref.width, ref.height, ref.mean, ref.std, 0.0, True,
                         use_refshim=(kind == "reference"))
        n += 1
    dt = time.perf_counter() - t0
    px = n * frames.shape[1] * frames.shape[2]
    return {"value": px / dt, "unit": "pixels/s", "cores": cores, "kind": kind,
            "sample": f"Pearson's R on {n} whole 1024x1024 frame(s) ({dt:.1f} s): kernel and host steps"}


def volume_cpu_baseline(vol: np.ndarray, ref, bw: int, budget_s: float = 12.0) -> dict:
    """The reference's 3D kernels (oracle/_ref, compiled for the CPU; the
    oracle's FP32 port if not built) with the Java host steps, Pearson, on a
    slab of the volume sized to about budget_s, on all host cores."""
    import oracle
    kind = "reference" if oracle.refshim() is not None else "port"
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    r = bw // 2

    def run(depth):
        slab = np.ascontiguousarray(vol[:depth])
        t0 = time.perf_counter()
        oracle.block_map3d("Pearson's R", slab, ref.pixels, bw, bw, bw, ref.mean, ref.std, 0.0, True,
                           use_refshim=(kind == "reference"))
        return slab.size, time.perf_counter() - t0

    n, dt = run(2 * r + 2)
    depth = int(min(vol.shape[0], max(2 * r + 2, (2 * r + 2) * budget_s / max(dt, 1e-6))))
    n, dt = run(depth)
    return {"value": n / dt, "unit": "voxels/s", "cores": cores, "kind": kind,
            "sample": f"Pearson's R over the first {depth} slices ({n} voxels, {dt:.1f} s): kernels and host steps"}


def run_volume(args, rank, local, world):
    """3D block repetition map: a 512x512x128 spot volume (134 MB, larger than
    L2) against one 5x5x5 reference block (ellipsoid K=33) cut at a seeded
    position, relevance 0, normalised; the four metrics of the reference's 3D
    command. Reports voxels/s (Pearson's R, the first metric) over the whole
    call (local statistics, map kernel, metric transform, normalisation)."""
    import torch
    from sred_b200 import _lib, clutils, synth, utils
    torch.cuda.set_device(local)
    ctx = _lib.Context(local, "tc")
    vol = synth.normalize_input(synth.volume_512_spots(seed=rank))
    D, H, W = vol.shape
    bw = 5
    rng = np.random.default_rng(11)
    z0, y0, x0 = (int(v) for v in rng.integers(0, [D - bw, H - bw, W - bw]))
    ref = utils.get_reference_block_3d(vol[z0:z0 + bw, y0:y0 + bw, x0:x0 + bw])
    d_in = torch.from_numpy(vol).cuda()
    d_out = torch.empty_like(d_in)
    stream = torch.cuda.Stream()
    res = {}
    clocks = Clocks(local)
    with clocks:
        for metric in clutils.BLOCK_METRICS_3D:
            for _ in range(args.warmup):
                clutils.block_map_3d_device(metric, d_in.data_ptr(), W, H, D, ref, 0.0, True, d_out.data_ptr(),
                                            stream.cuda_stream, ctx=ctx)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                clutils.block_map_3d_device(metric, d_in.data_ptr(), W, H, D, ref, 0.0, True, d_out.data_ptr(),
                                            stream.cuda_stream, ctx=ctx)
            e1.record(stream)
            e1.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
            nvox = vol.size * world
            res[metric] = {"ms_per_step": ms, "voxels_per_s": nvox / (ms / 1e3),
                           "gbs_8B_per_voxel": 8 * nvox / (ms / 1e3) / 1e9}
        # end to end: host volume in, host map out, through the public call
        # (pinned host buffers, as a caller that streams volumes would hold)
        h_in = torch.from_numpy(vol.ravel()).pin_memory()
        h_out = torch.empty_like(h_in).pin_memory()
        inp = utils.InputImage3D(h_in.numpy(), W, H, D)
        for _ in range(args.warmup):
            clutils.calculate_block_repetition_map_3d("Pearson's R", inp, ref, 0.0, True, ctx=ctx,
                                                      out=h_out.numpy())
        n_e2e = max(5, 2 * args.steps)  # ~6 ms each: enough calls to average out host-side jitter
        t0 = time.perf_counter()
        for _ in range(n_e2e):
            clutils.calculate_block_repetition_map_3d("Pearson's R", inp, ref, 0.0, True, ctx=ctx, out=h_out.numpy())
        e2e_ms = (time.perf_counter() - t0) * 1e3 / n_e2e
        e2e_ms = max_over_ranks(e2e_ms, world)
    if rank != 0:
        return
    pk = peaks()
    p = res["Pearson's R"]
    line = {"metric": "3D block-map voxels/s at 512x512x128/5x5x5", "value": p["voxels_per_s"],
            "unit": "voxels/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": p["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (reference evaluation order, bit-exact)", "data": "synthetic",
            "config": {"workload": "3D block repetition map, 512x512x128 float32 spot volume (40x40x16 lattice), "
                                   f"5x5x5 reference block (ellipsoid K={ref.size}), relevance 0, normalised",
                       "l2": "volume of 134 MB > L2"},
            "per_metric": res,
            "e2e": {"value": vol.size * world / (e2e_ms / 1e3), "unit": "voxels/s",
                    "h2d_bytes_per_step": vol.nbytes, "d2h_bytes_per_step": vol.nbytes},
            "clocks": clocks.summary(),
            # per Pearson call: local statistics, map, min-max initialisation, min-max, remap
            "gpu_launches": 5 * args.steps,
            "roofline": {"bound": "hbm", "achieved": p["gbs_8B_per_voxel"], "peak": pk["hbm_gbs"], "unit": "GB/s",
                         "frac": p["gbs_8B_per_voxel"] / pk["hbm_gbs"], "traffic": None,
                         "note": "8 algorithmic bytes per voxel over the whole call; the kernels evaluate "
                                 "K-element sums in the reference's sequential FP32 order"}}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = volume_cpu_baseline(vol, ref, bw)
    print(json.dumps(line), flush=True)


def run_volume_global(args, rank, local, world):
    """3D global repetition map: a 192x192x64 spot volume (9.4 MB), 5x5x5
    block (ellipsoid K=33), relevance constant 1.0, Pearson's R, normalised;
    L2 flushed between steps. Reports block-pairs/s (reference voxels x test
    voxels per second) over the whole call; the tensor-core Gram kernel is
    the dominant kernel."""
    import torch
    from sred_b200 import _lib, clutils, synth, utils
    torch.cuda.set_device(local)
    ctx = _lib.Context(local, args.engine)
    vol = synth.normalize_input(synth.spot_volume(192, 192, 64, 24, 8, seed=rank))
    D, H, W = vol.shape
    b, relc, metric = 5, 1.0, "Pearson's R"
    d_in = torch.from_numpy(vol).cuda()
    d_out = torch.empty_like(d_in)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    for _ in range(args.warmup):
        clutils.global_map_3d_device(metric, d_in.data_ptr(), W, H, D, b, b, b, relc, True, d_out.data_ptr(),
                                     stream.cuda_stream, ctx=ctx)
    torch.cuda.synchronize()
    ms, gram_ms, launches, info = [], [], 0, None
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            info = clutils.global_map_3d_device(metric, d_in.data_ptr(), W, H, D, b, b, b, relc, True,
                                                d_out.data_ptr(), stream.cuda_stream, ctx=ctx)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
            gram_ms.append(info["ms_gram"])
            launches += info["launches"]
    total_ms = max_over_ranks(sum(ms), world)
    pairs = sum_over_ranks(info["pairs"] * args.steps, world)
    # end to end: host volume in, host map out (pinned host buffers)
    h_in = torch.from_numpy(vol.ravel()).pin_memory()
    h_out = torch.empty_like(h_in).pin_memory()
    inp = utils.InputImage3D(h_in.numpy(), W, H, D)
    e2e = []
    for _ in range(max(2, args.steps // 2)):
        t0 = time.perf_counter()
        clutils.calculate_global_repetition_map_3d(metric, inp, b, b, b, relc, True, ctx=ctx, out=h_out.numpy())
        e2e.append(time.perf_counter() - t0)
    e2e_total = max_over_ranks(sum(e2e), world)
    e2e_pairs = sum_over_ranks(info["pairs"] * len(e2e), world)
    if rank != 0:
        return
    pk = peaks()
    K = info["k"]
    gram_s = statistics.mean(gram_ms) / 1e3
    line = {"metric": "3D global-map block-pairs/s at 192x192x64/5x5x5", "value": pairs / (total_ms / 1e3),
            "unit": "block-pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3 split tensor-core Gram, f32 accumulate, f64 sums" if args.engine == "tc"
                     else "f32 CUDA-core Gram, f64 sums",
            "data": "synthetic (seeded spot volume, numpy default_rng; no dataset)",
            "config": {"workload": "3D global repetition map, 192x192x64 float32 spot volume (24x24x8 lattice), "
                                   f"5x5x5 block (ellipsoid K={K}), Pearson's R, relevance constant 1.0",
                       "engine": args.engine, "relevant_blocks": info["n_relevant"],
                       "pairs_per_step": info["pairs"],
                       "l2": "flushed between steps (256 MiB write, outside the timed region)"},
            "gpu_launches": launches, "clocks": clk.summary(),
            "e2e": {"value": e2e_pairs / e2e_total, "unit": "block-pairs/s", "h2d_bytes_per_step": vol.nbytes,
                    "d2h_bytes_per_step": vol.nbytes, "ms_per_step": 1e3 * e2e_total / len(e2e)}}
    if args.engine == "tc":
        eff_peak = pk["bf16_tflops_sustained"] / 3.0
        n_g = info["n_relevant"] - info["n_flat"]
        evaluated = n_g * (n_g + 1) / 2
        achieved = evaluated * 2 * K / gram_s / 1e12
        line["roofline"] = {"bound": "tensor", "achieved": achieved, "peak": eff_peak, "unit": "TFLOP/s",
                            "frac": achieved / eff_peak, "traffic": None, "evaluated_pairs_per_launch": evaluated,
                            "note": f"all-pairs Gram kernel; algorithmic FLOPs = contracted pairs x 2K (K={K}), "
                                    f"contracted pairs = n(n+1)/2 of the n non-flat relevant blocks (each unordered "
                                    f"pair once); peak = {pk['source']} sustained BF16 / 3"}
    if not args.no_cpu_baseline:
        import oracle
        kind = "reference" if oracle.refshim() is not None else "port"
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        means, stds = oracle.local_stats3d(vol, b, b, b)
        mask, nv = oracle.relevance_mask3d(stds, b, b, b, relc)
        thr = np.float32(nv * np.float32(relc))
        rel = np.flatnonzero(mask.ravel() > 0).astype(np.int32)
        rng = np.random.default_rng(5)
        rows = rng.choice(rel, size=min(rel.size, 2 * cores), replace=False).astype(np.int32)
        t0 = time.perf_counter()
        oracle.global3d_sums_f32(metric, vol, b, b, b, means, stds, nv, thr, rows, use_refshim=(kind == "reference"))
        dt = time.perf_counter() - t0
        n_rows = int(max(cores, min(rel.size, 12.0 / max(dt, 1e-6) * rows.size)))
        rows = rng.choice(rel, size=n_rows, replace=False).astype(np.int32)
        t0 = time.perf_counter()
        oracle.global3d_sums_f32(metric, vol, b, b, b, means, stds, nv, thr, rows, use_refshim=(kind == "reference"))
        dt = time.perf_counter() - t0
        test_blocks = int(np.count_nonzero(stds.ravel() ** 2 >= thr) )
        line["cpu_baseline"] = {"value": rows.size * test_blocks / dt, "unit": "block-pairs/s", "cores": cores,
                                "kind": kind, "sample": f"{rows.size} reference voxels x all {test_blocks} test "
                                                        f"voxels ({dt:.1f} s); rate extrapolates per pair"}
    print(json.dumps(line), flush=True)


def run_aux(args, rank, local, world):
    """The widened rows on one 1024x1024 image: variance stabilisation (GAT
    fit and transform), the relevance-mask sweep (11 constants), the
    constant-range search, and the redundancy classification (k = 3) of the
    image's 9x9 global map. Host image in, host result out, timed per call
    (wall clock around the synchronous C ABI call). Each line item also has
    the oracle's single-thread CPU restatement timed on the same input (one
    run), the reference-order baseline for these host-side Java steps."""
    import torch
    import oracle
    from sred_b200 import _lib, clutils, plugins, synth, utils
    torch.cuda.set_device(local)
    ctx = _lib.Context(local, "tc")
    rng = np.random.default_rng(rank)
    lam = synth.image_1024_spots(seed=rank).clip(0, None) / 4.0
    raw = (2.0 * rng.poisson(lam) + 100.0 + rng.normal(0, 5.0, lam.shape)).astype(np.float32)
    inp = synth.normalize_input(raw)
    gmap, _ = clutils.global_map_host("Pearson's R", inp, 9, 9, 1.0, True, ctx=ctx)

    def timed(fn, reps):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            r = fn()
        return (time.perf_counter() - t0) / reps, r

    res = {}
    t, (g, sg, o, _) = timed(lambda: utils.fit_gat_2d(raw, 5000, ctx=ctx), 1)
    res["gat_fit_2d"] = {"ms": 1e3 * t, "params": [g, sg, o]}
    t_cpu, _ = timed(lambda: oracle.gat_objective(raw, g, sg, o), 1)
    res["gat_fit_2d"]["cpu_ms_per_objective"] = 1e3 * t_cpu
    t, _ = timed(lambda: utils.get_gat_2d(raw, g, sg, o, ctx=ctx), max(3, args.steps))
    res["gat_transform_2d"] = {"ms": 1e3 * t}
    t_cpu, _ = timed(lambda: oracle.gat(raw, g, sg, o), 1)
    res["gat_transform_2d"]["cpu_ms"] = 1e3 * t_cpu
    t, _ = timed(lambda: clutils.relevance_mask_sweep_2d(inp, 3, 3, 0.0, 0.1, 11, ctx=ctx), max(3, args.steps))
    var = oracle.local_var2d(inp, 3, 3, 0)
    nv = oracle.tool_noise_var(inp, 0)
    t_cpu, _ = timed(lambda: [oracle.tool_mask(var, 3, 3, nv, np.float32(0.1 * i)) for i in range(11)], 1)
    res["relevance_sweep_11"] = {"ms": 1e3 * t, "cpu_ms_masks_only": 1e3 * t_cpu}
    t, rr = timed(lambda: clutils.relevance_constant_range_2d(inp, 3, 3, 0.05, ctx=ctx), max(3, args.steps))
    res["relevance_range"] = {"ms": 1e3 * t, "range": [float(rr[0]), float(rr[1])]}
    t, (cm, kc, w) = timed(lambda: plugins.classify_redundancy(gmap, 1, 3, seed=1, ctx=ctx), 1)
    t_cpu, _ = timed(lambda: oracle.classify_redundancy(gmap, 1, 3, seed=1), 1)
    res["classify_k3"] = {"ms": 1e3 * t, "cpu_ms": 1e3 * t_cpu}
    if rank != 0:
        return
    line = {"metric": "auxiliary steps on 1024x1024 (GAT fit, relevance tools, classification), ms per call",
            "value": res["gat_fit_2d"]["ms"], "unit": "ms (GAT fit)", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["gat_fit_2d"]["ms"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64 objective, f32 masks, f64 k-means",
            "data": "synthetic (Poisson-Gaussian spot image: gain 2, offset 100, read noise 5)",
            "config": {"workload": "1024x1024 spot image; GAT fit from (1, 10, 100), relevance sweep 0..1 step "
                                   "0.1, range search step 0.05, k-means k = 3 on its 9x9 global map"},
            "per_step": res, "cpu_baseline": {"kind": "port", "cores": 1,
                                              "sample": "oracle restatements, single thread, one run each"}}
    print(json.dumps(line), flush=True)


def run_shard(args, rank, local, world):
    """One global map of the default workload split by rows across the ranks
    (strong scaling): every rank prepares the same image, computes the sums
    of its row blocks, the ranks sum them with one NCCL all-reduce, and every
    rank finishes the map. Timed on the device, max over ranks."""
    import torch
    from sred_b200 import _lib, clutils
    torch.cuda.set_device(local)
    ctx = _lib.Context(local, "tc")
    img = image(0)
    d_img = torch.from_numpy(img).cuda()
    d_out = torch.empty_like(d_img)
    stream = torch.cuda.current_stream()
    if world > 1:
        import torch.distributed as dist
        allreduce = dist.all_reduce
    else:
        def allreduce(t):
            return None
    info = {}

    def step():
        nonlocal info
        info = clutils.global_map_device_sharded(SIM, d_img.data_ptr(), W_IMG, H_IMG, BW, BH, RELC, True,
                                                 d_out.data_ptr(), rank, world, allreduce, stream.cuda_stream,
                                                 ctx=ctx)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    if rank != 0:
        return
    pairs = float(info["pairs"])
    line = {"metric": METRIC.replace("split-BF16 vs FP32 speedup @≤1e-5 err", "one map sharded across GPUs by work items"),
            "value": pairs / (ms / 1e3), "unit": "block-pairs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "bf16x3 split (hi/lo) tensor-core Gram, f32 accumulate, f64 moments",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "image": f"{W_IMG}x{H_IMG}", "block": f"{BW}x{BH}",
                       "pairs_per_step": pairs,
                       "parallelism": f"work items of the pair triangle sharded over {world} GPU(s), one all-reduce "
                                      "of the per-block sums"}}
    print(json.dumps(line), flush=True)


BATCH_SIDES = [256, 384, 512, 768, 1024]
BATCH_BLOCKS = [3, 5, 9, 13, 15]


def run_batch(args, rank, local, world):
    """Batched global maps (the multi-scale set): `--images` seeded spot
    images with sides from {256, 384, 512, 768, 1024} (width and height drawn
    independently, so most are not square), each mapped with 3x3, 5x5, 9x9,
    13x13 and 15x15 blocks (K = 5, 13, 49, 113, 149) and with Pearson's R and
    SSIM at relevance 1.0: 10 maps per image through sred_global_map_2d_batch
    with host buffers. Reports the sum over maps of relevant^2 block pairs per
    second of wall time (transfers included) and maps per second.

    Before the warm-up, unless --no-tune, a tuning pass (one worker, untimed)
    maps one image per (block, metric, block-count class) with
    sred_set_gram_tuning on, so the tensor-core engine times its launch shapes
    for each key the process table lacks; the table is saved next to the
    library and its entries go into the line. Tuning is off in the timed
    run."""
    import torch
    from sred_b200 import _lib, clutils, synth
    torch.cuda.set_device(local)
    ctx = _lib.Context(local, "tc")
    rng = np.random.default_rng(11 + rank)
    jobs = []
    for i in range(args.images):
        w, h = (int(v) for v in rng.choice(BATCH_SIDES, 2))
        img = synth.normalize_input(synth.spot_image(w, h, max(4, min(w, h) // 13), seed=1000 * rank + i))
        for b in BATCH_BLOCKS:
            for metric in ("Pearson's R", "SSIM"):
                jobs.append({"metric": metric, "img": img, "block_width": b, "block_height": b,
                             "relevance_constant": 1.0})
    tuning = []
    if args.tune:
        groups = {}
        for j in jobs:
            hh, ww = j["img"].shape
            nb = (ww - j["block_width"] + 1) * (hh - j["block_height"] + 1)
            key = (j["block_width"], j["metric"], 0 if nb < 1 << 16 else 1 if nb < 1 << 18 else 2)
            groups.setdefault(key, []).append(j)
        pick = [sorted(g, key=lambda j: j["img"].size)[len(g) // 2] for g in groups.values()]
        ctx.set_gram_tuning(True)
        clutils.global_map_batch(pick, n_workers=1, ctx=ctx)
        ctx.set_gram_tuning(False)
        torch.cuda.synchronize()
        if rank == 0:
            _lib.gram_tuning_save(device=torch.cuda.get_device_name(local))
        tuning = [f"K'={t['kq']} {t['metric_name']} class {t['size_class']}: {t['bn']} cols, "
                  f"{'A resident' if t['a_resident'] else 'A chunk ring'}, L<={t['max_l']} ({t['ms']:.3f} ms)"
                  for t in _lib.gram_tuning_entries()]
    # warm-up: the largest image's ten maps, W times (this also sizes every
    # worker's workspaces)
    big = max(range(args.images), key=lambda i: jobs[10 * i]["img"].size)
    for _ in range(args.warmup):
        clutils.global_map_batch(jobs[10 * big:10 * big + 10], n_workers=args.workers, ctx=ctx)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    res = clutils.global_map_batch(jobs, n_workers=args.workers, ctx=ctx)
    torch.cuda.synchronize()
    dt = max_over_ranks(time.perf_counter() - t0, world)
    pairs = sum_over_ranks(float(sum(info["pairs"] for _, info in res)), world)
    if rank != 0:
        return
    line = {"metric": "batched global maps: block-pairs/s summed over maps (wall time, host buffers)",
            "value": pairs / dt, "unit": "block-pairs/s", "n_gpus": world, "steps": 1, "warmup": args.warmup,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3 split (hi/lo) tensor-core Gram, f32 accumulate, f64 moments", "data": "synthetic",
            "config": {"workload": f"{args.images} images x 5 block sizes x 2 metrics = {len(jobs)} global maps, "
                                   "sides 256-1024, relevance 1.0; warm-up: the largest image's 10 maps",
                       "images": args.images, "maps": len(jobs),
                       "workers": args.workers, "pairs": pairs,
                       "launch_shapes": tuning if args.tune else "default (tuning off)"},
            "maps_per_s": len(jobs) * world / dt,
            # per-map CUDA-event times on the workers' streams, summed (with
            # several workers a map's events also span other maps' kernels)
            "sum_ms_gram": sum(info["ms_gram"] for _, info in res),
            "sum_ms_total": sum(info["ms_total"] for _, info in res)}
    print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    if rank != 0:
        return
    img = image(seed=0)
    vals, secs = [], []
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline(img, None, budget_s=4.0 if i < args.warmup else 8.0)
        if i >= args.warmup:
            vals.append(b["value"])
            base = b
    v = statistics.mean(vals)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "block-pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (reference kernels on host cores)",
            "data": "synthetic (seeded spot image, numpy default_rng; no dataset)",
            "config": {"workload": WORKLOAD, "image": f"{W_IMG}x{H_IMG}", "block": f"{BW}x{BH}",
                       "metric": SIM, "relevance_constant": RELC, "engine": "reference CPU kernels"},
            "cpu_baseline": {"value": v, "unit": "block-pairs/s", "cores": base["cores"], "kind": base["kind"],
                             "sample": base["sample"]},
            "e2e": {"value": v, "unit": "block-pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--engine", choices=["tc", "fp32"], default="tc")
    ap.add_argument("--no-compare", action="store_true", help="skip the FP32-engine comparison")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["global", "block", "batch", "volume", "volume-global", "aux"],
                    default="global",
                    help="global repetition map (default, the headline), the block (local) map, batched "
                         "global maps of many images, the 3D block map of a volume, or the 3D global map")
    ap.add_argument("--metric", default="Pearson's R",
                    help="metric of the global workload (the reference's names; default Pearson's R)")
    ap.add_argument("--mode", choices=["replicas", "shard"], default="replicas",
                    help="global workload on N GPUs: independent replicas (default, weak scaling) or one map "
                         "sharded across the GPUs by work items (strong scaling)")
    ap.add_argument("--images", type=int, default=8, help="images of the batch workload (10 maps each)")
    ap.add_argument("--workers", type=int, default=4, help="host workers of the batch workload")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="batch workload: skip the launch-shape tuning pass (default shapes)")
    ap.add_argument("--frames", type=int, default=64, help="frames of the block-map workload")
    ap.add_argument("--size", type=int, default=1024,
                    help="image side (default 1024, the benchmark workload; smaller sides for profiling)")
    ap.add_argument("--block", type=int, default=9, help="block side of the global workload (default 9)")
    ap.add_argument("--relevance", type=float, default=1.0, help="relevance constant of the global workload")
    args = ap.parse_args()
    global W_IMG, H_IMG, WORKLOAD, BW, BH, METRIC, RELC, SIM
    if args.metric != SIM:
        SIM = args.metric
        WORKLOAD = WORKLOAD.replace("Pearson's R", SIM)
        METRIC = METRIC.replace("global-map", f"global-map ({SIM})")
    if args.size == 256:
        W_IMG = H_IMG = 256
        WORKLOAD = ("global repetition map, 256x256 float32 spot image (20x20 lattice, 400 spots), "
                    "9x9 block (ellipse K=49), Pearson's R, relevance constant 1.0")
    elif args.size == 2048:
        W_IMG = H_IMG = 2048
        WORKLOAD = ("global repetition map, 2048x2048 float32 spot image (160x160 lattice, 10% elongated "
                    "spots), 9x9 block (ellipse K=49), Pearson's R, relevance constant 1.0")
    elif args.size != 1024:
        W_IMG = H_IMG = args.size
        WORKLOAD = WORKLOAD.replace("1024x1024", f"{args.size}x{args.size}").replace(
            "80x80 lattice", f"{max(2, args.size * 80 // 1024)}x{max(2, args.size * 80 // 1024)} lattice")
    if args.block != 9:
        from sred_b200 import utils
        BW = BH = args.block
        WORKLOAD = WORKLOAD.replace("9x9 block (ellipse K=49)",
                                    f"{BW}x{BH} block (ellipse K={utils.block_size(BW, BH)})")
    if args.relevance != 1.0:
        RELC = args.relevance
        WORKLOAD = WORKLOAD.replace("relevance constant 1.0", f"relevance constant {RELC:g}")
    if args.size != 1024 or args.block != 9:
        METRIC = METRIC.replace("1024²/9×9", f"{W_IMG}²/{BW}×{BH}")
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank, int(os.environ.get("WORLD_SIZE", "1")))
        return
    rank, local, world = dist_init()
    try:
        if args.workload == "block":
            run_block(args, rank, local, world)
        elif args.workload == "volume":
            run_volume(args, rank, local, world)
        elif args.workload == "volume-global":
            run_volume_global(args, rank, local, world)
        elif args.workload == "aux":
            run_aux(args, rank, local, world)
        elif args.workload == "batch":
            run_batch(args, rank, local, world)
        elif args.mode == "shard":
            run_shard(args, rank, local, world)
        else:
            run_ours(args, rank, local, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
