"""Host-side mirror of the reference's ``CLUtils`` (java/CLUtils.java).

The OpenCL orchestration of the reference is replaced by libsred (CUDA,
sm_100a); the method names, arguments and results stay. ``OpenCLResources``
becomes a libsred ``Context``; ``CLLocalStatistics`` holds the FP32 local
means and stds.

Errors follow the reference: an unknown metric returns None
(java/CLUtils.java:2193-2195, :1007-1009); bad arguments raise.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .utils import InputImage2D, InputImage3D, ReferenceBlock2D, ReferenceBlock3D, RelevanceMask

GLOBAL_METRICS = ["Pearson's R", "SSIM", "NRMSE", "Abs. diff. of StdDevs"]  # java/GlobalRepetition2D_.java:20-25
BLOCK_METRICS = ["Pearson's R", "SSIM", "NRMSE (inverted)", "Abs. Diff. of StdDevs."]  # java/BlockRepetition2D_.java:18-23
COSINE = "Cosine"  # raw-vector cosine similarity; no reference counterpart
# Block-map forms of the reference's shape-metric kernels (no dialog entry in the reference).
HU = "Hu moments"  # cl/kernelGetPatchHu2D.cl
PHASE = "Phase correlation"  # cl/kernelGetPhaseCorrelationMap.cl (repaired)
HU7 = "Hu distance"  # L2 distance of the seven Hu invariants; no reference counterpart (it outputs Hu1 only)
EXTRA_BLOCK_METRICS = [COSINE, HU, PHASE, HU7]
BLOCK_METRICS_3D = ["Pearson's R", "SSIM", "NRMSE (inverted)", "Abs. Diff. of StdDevs."]  # java/BlockRepetition3D_.java:19-24


@dataclass
class CLLocalStatistics:
    """java/CLUtils.java:84-158 (the device buffers live in libsred)."""
    local_means: np.ndarray
    local_stds: np.ndarray


def get_open_cl_resources(use_device: bool = False, device: int = 0, engine: str = "tc") -> _lib.Context:
    """java/CLUtils.java:169-238 counterpart: a libsred context on a CUDA device."""
    return _lib.Context(device, engine)


def _ctx(ctx):
    return ctx if ctx is not None else _lib.default_context()


def get_local_statistics_2d(input_image: InputImage2D, block_width: int, block_height: int,
                            ctx=None) -> CLLocalStatistics:
    """java/CLUtils.java:376-467."""
    c = _ctx(ctx)
    n = input_image.size
    m = np.zeros(n, np.float32)
    s = np.zeros(n, np.float32)
    c.check(c._L.sred_local_statistics_2d(c.h, np.ascontiguousarray(input_image.image_array, np.float32).ravel(),
                                          input_image.width, input_image.height, block_width, block_height, m, s),
            "sred_local_statistics_2d")
    return CLLocalStatistics(m, s)


def calculate_global_repetition_map_2d(metric: str, input_image: InputImage2D, block_width: int,
                                       block_height: int, block_size: int, local_statistics: CLLocalStatistics,
                                       relevance_mask: RelevanceMask, n_pixels: float, normalize_output: bool,
                                       ctx=None, run_info: dict | None = None):
    """java/CLUtils.java:2174-2196: dispatch on the metric string to the global map."""
    if metric not in GLOBAL_METRICS:
        return None
    c = _ctx(ctx)
    n = input_image.size
    out = np.zeros(n, np.float32)
    info = _lib.RunInfo()
    c.check(c._L.sred_calculate_global_repetition_map_2d(
        c.h, metric.encode(), np.ascontiguousarray(input_image.image_array, np.float32).ravel(),
        input_image.width, input_image.height, block_width, block_height, block_size,
        np.ascontiguousarray(local_statistics.local_means, np.float32).ravel(),
        np.ascontiguousarray(local_statistics.local_stds, np.float32).ravel(),
        np.ascontiguousarray(relevance_mask.relevance_mask, np.float32).ravel(),
        float(relevance_mask.relevance_constant), float(relevance_mask.relevance_threshold),
        float(relevance_mask.noise_mean_variance), float(n_pixels), int(bool(normalize_output)), out,
        C.byref(info)), "sred_calculate_global_repetition_map_2d")
    if run_info is not None:
        run_info.update(info.as_dict())
    return out


def _global_getter(metric):
    def f(input_image, local_statistics, block_width, block_height, block_size, relevance_mask, n_pixels,
          normalize_output, ctx=None):
        return calculate_global_repetition_map_2d(metric, input_image, block_width, block_height, block_size,
                                                  local_statistics, relevance_mask, n_pixels, normalize_output, ctx)
    f.__doc__ = f"getGlobal*2D for {metric!r} (java/CLUtils.java:1680-2156)."
    return f


get_global_pearson_2d = _global_getter("Pearson's R")
get_global_ssim_2d = _global_getter("SSIM")
get_global_nrmse_2d = _global_getter("NRMSE")


def get_global_abs_diff_stds_2d(input_image, local_statistics, block_width, block_height, relevance_mask, n_pixels,
                                normalize_output, ctx=None):
    """java/CLUtils.java:2049-2156 (no block size argument, as the reference)."""
    from .utils import block_size
    return calculate_global_repetition_map_2d("Abs. diff. of StdDevs", input_image, block_width, block_height,
                                              block_size(block_width, block_height), local_statistics,
                                              relevance_mask, n_pixels, normalize_output, ctx)


def calculate_block_repetition_map_2d(metric: str, input_image: InputImage2D, reference_block: ReferenceBlock2D,
                                      relevance_constant: float, normalize_output: bool, use_device: bool = False,
                                      ctx=None):
    """java/CLUtils.java:995-1010."""
    if metric not in BLOCK_METRICS and metric not in EXTRA_BLOCK_METRICS:
        return None
    c = _ctx(ctx)
    out = np.zeros(input_image.size, np.float32)
    c.check(c._L.sred_calculate_block_repetition_map_2d(
        c.h, metric.encode(), np.ascontiguousarray(input_image.image_array, np.float32).ravel(),
        input_image.width, input_image.height, np.ascontiguousarray(reference_block.pixels, np.float32).ravel(),
        int(reference_block.size), reference_block.width, reference_block.height, float(reference_block.mean),
        float(reference_block.std), float(relevance_constant), int(bool(normalize_output)), out),
        "sred_calculate_block_repetition_map_2d")
    return out


def _block_getter(metric):
    def f(input_image, reference_block, relevance_constant, normalize_output, use_device=False, ctx=None):
        return calculate_block_repetition_map_2d(metric, input_image, reference_block, relevance_constant,
                                                 normalize_output, use_device, ctx)
    f.__doc__ = f"getBlock*2D for {metric!r} (java/CLUtils.java:486-981)."
    return f


get_block_pearson_2d = _block_getter("Pearson's R")
get_block_ssim_2d = _block_getter("SSIM")
get_block_nrmse_2d = _block_getter("NRMSE (inverted)")
get_block_abs_diff_stds_2d = _block_getter("Abs. Diff. of StdDevs.")


# ---------------------------------------------------------------------------
# The reference's shape-metric kernels (src/main/resources/, never loaded by
# its Java code): Hu moments and phase correlation.
# ---------------------------------------------------------------------------

def get_patch_hu_map_2d(input_image: InputImage2D, patch: np.ndarray, block_width: int, block_height: int,
                        patch_size: int | None = None, ctx=None) -> np.ndarray:
    """cl/kernelGetPatchHu2D.cl: sqrt(hu1(patch) * hu1(block)) per interior pixel.
    ``patch`` is the bw x bh grid the kernel reads at the ellipse positions;
    ``patch_size`` defaults to the ellipse count K."""
    from .utils import block_size
    c = _ctx(ctx)
    out = np.zeros(input_image.size, np.float32)
    ps = block_size(block_width, block_height) if patch_size is None else int(patch_size)
    c.check(c._L.sred_patch_hu_map_2d(c.h, np.ascontiguousarray(patch, np.float32).ravel(),
                                      np.ascontiguousarray(input_image.image_array, np.float32).ravel(),
                                      input_image.width, input_image.height, block_width, block_height, ps, out),
            "sred_patch_hu_map_2d")
    return out


def _stats_args(input_image, local_statistics):
    return (np.ascontiguousarray(input_image.image_array, np.float32).ravel(),
            np.ascontiguousarray(local_statistics.local_means, np.float32).ravel(),
            np.ascontiguousarray(local_statistics.local_stds, np.float32).ravel())


def get_hu_map_2d(input_image: InputImage2D, local_statistics: CLLocalStatistics, block_width: int,
                  block_height: int, ctx=None) -> np.ndarray:
    """cl/kernelGetHuMap.cl over all interior pairs (raw sums)."""
    c = _ctx(ctx)
    out = np.zeros(input_image.size, np.float32)
    c.check(c._L.sred_hu_map_2d(c.h, *_stats_args(input_image, local_statistics), input_image.width,
                                input_image.height, block_width, block_height, out), "sred_hu_map_2d")
    return out


def get_phase_correlation_map_2d(input_image: InputImage2D, local_statistics: CLLocalStatistics, block_width: int,
                                 block_height: int, ctx=None) -> np.ndarray:
    """cl/kernelGetPhaseCorrelationMap.cl (defects repaired) over all interior pairs (raw sums)."""
    c = _ctx(ctx)
    out = np.zeros(input_image.size, np.float32)
    c.check(c._L.sred_phase_correlation_map_2d(c.h, *_stats_args(input_image, local_statistics),
                                               input_image.width, input_image.height, block_width, block_height,
                                               out), "sred_phase_correlation_map_2d")
    return out


get_block_hu_2d = _block_getter(HU)
get_block_phase_correlation_2d = _block_getter(PHASE)


def global_map_device(metric: str, d_img_ptr: int, width: int, height: int, block_width: int, block_height: int,
                      relevance_constant: float, normalize_output: bool, d_out_ptr: int, stream_ptr: int = 0,
                      ctx=None) -> dict:
    """Global map on device-resident buffers (raw CUDA pointers); returns run info."""
    c = _ctx(ctx)
    info = _lib.RunInfo()
    c.check(c._L.sred_global_map_2d_device(c.h, metric.encode(), C.c_void_p(d_img_ptr), width, height, block_width,
                                           block_height, float(relevance_constant), int(bool(normalize_output)),
                                           C.c_void_p(d_out_ptr), C.c_void_p(stream_ptr or None), C.byref(info)),
            "sred_global_map_2d_device")
    return info.as_dict()


def _out_buffer(out, n: int, what: str) -> np.ndarray:
    """A caller's output buffer, flat, if the library can write it in place."""
    if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != n:
        raise ValueError(f"out must be a C-contiguous float32 array of {what}")
    return out.reshape(-1)


def global_map_host(metric: str, img: np.ndarray, block_width: int, block_height: int, relevance_constant: float,
                    normalize_output: bool = True, out: np.ndarray | None = None, ctx=None) -> tuple:
    """The whole global-map command on host buffers (sred_global_map_2d):
    returns (map, run info). ``img`` may be pinned memory."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(img, np.float32)
    h, w = a.shape
    if out is None:
        out = np.empty((h, w), np.float32)
    else:
        _out_buffer(out, h * w, "h * w elements")
    info = _lib.RunInfo()
    c.check(c._L.sred_global_map_2d(c.h, metric.encode(), C.c_void_p(a.ctypes.data), w, h, block_width,
                                    block_height, float(relevance_constant), int(bool(normalize_output)),
                                    C.c_void_p(out.ctypes.data), C.byref(info)), "sred_global_map_2d")
    return out, info.as_dict()


def global_map_batch(jobs: list[dict], n_workers: int = 4, ctx=None) -> list[tuple]:
    """Many global maps in one call (sred_global_map_2d_batch). Each job is a
    dict with metric, img (float32 [h, w]), block_width, block_height,
    relevance_constant and optionally normalize_output; returns one
    (map, run info) per job, in order."""
    c = _ctx(ctx)
    arr = (_lib.SredJob * len(jobs))()
    keep = []
    for i, j in enumerate(jobs):
        img = np.ascontiguousarray(j["img"], np.float32)
        h, w = img.shape
        out = np.empty((h, w), np.float32)
        info = _lib.RunInfo()
        m = j["metric"].encode()
        keep.append((img, out, info, m))
        arr[i] = _lib.SredJob(m, img.ctypes.data, w, h, int(j["block_width"]), int(j["block_height"]),
                              float(j["relevance_constant"]), int(bool(j.get("normalize_output", True))),
                              out.ctypes.data, C.pointer(info), -1)
    c.check(c._L.sred_global_map_2d_batch(c.h, arr, len(jobs), int(n_workers)), "sred_global_map_2d_batch")
    return [(out, info.as_dict()) for _, out, info, _ in keep]


# ---------------------------------------------------------------------------
# Sharded global map (one map across several processes / GPUs, split by work items)
# ---------------------------------------------------------------------------

def _items_before_run(j: int, n_ct: int, h: int) -> int:
    """Work items of runs [0, j): run j' has the column tiles j' h .. n_ct - 1."""
    return j * n_ct - h * j * (j - 1) // 2


def _panel_items_before_run(j: int, c0: int, c1: int, h: int) -> int:
    """Items of runs [0, j) in the panel of column tiles [c0, c1): each run j'
    takes the tiles max(c0, j' h) .. c1 - 1 (global_tc.cu: panel_items_before_run)."""
    a = min(j, c0 // h + 1)
    s = a * (c1 - c0)
    if j > a:
        s += (j - a) * c1 - h * (j * (j - 1) // 2 - a * (a - 1) // 2)
    return s


def gram_panel(bn: int, kq: int) -> int:
    """Column tiles per panel: as many bn-column B tiles of K' = kq bf16 as fit
    in 48 MB (the rule libsred applies, global_tc.cu: launch_gram_tc)."""
    return max(1, (48 << 20) // (bn * kq * 2))


def gram_items(n_gram: int, bn: int = 256, num_sms: int = 148) -> tuple[int, int]:
    """(items, L) of the tensor-core engine's symmetric schedule for n_gram
    blocks and bn-column tiles: the upper triangle of 128-row x bn-column
    tiles, cut into items (a run of L row blocks against one column tile that
    reaches it), L the largest of 32, 16, 8, 4, 2 that leaves at least 4 items
    per SM (the rule libsred applies, global_tc.cu: gram_tc_items)."""
    m = bn // 128
    n_rb, n_ct = (n_gram + 127) // 128, (n_gram + bn - 1) // bn

    def items(L):
        return _items_before_run((n_rb + L - 1) // L, n_ct, L // m)

    L = 32
    while L > 2 and items(L) < 4 * num_sms:
        L //= 2
    L = max(L, m)
    return items(L), L


def decode_items(n_gram: int, i0: int, i1: int, bn: int = 256, num_sms: int = 148, panel: int | None = None):
    """Items [i0, i1) of the schedule in libsred's order (panels of `panel`
    column tiles, within a panel run by run, within a run by column tile; None:
    one panel), each as (column tile, first row block, end row block), empty
    items left out (global_tc.cu: decode_item)."""
    _, L = gram_items(n_gram, bn, num_sms)
    m, h = bn // 128, L // (bn // 128)
    n_rb, n_ct = (n_gram + 127) // 128, (n_gram + bn - 1) // bn
    n_runs = (n_rb + L - 1) // L
    if n_ct == 0 or i1 <= i0:
        return []
    P = n_ct if not panel else panel
    spans = []  # (first item, c0, c1, runs)
    base = 0
    for c0 in range(0, n_ct, P):
        c1 = min(c0 + P, n_ct)
        J = min((c1 - 1) // h + 1, n_runs)
        spans.append((base, c0, c1, J))
        base += _panel_items_before_run(J, c0, c1, h)
    out = []
    k = 0
    for it in range(i0, i1):
        while k + 1 < len(spans) and spans[k + 1][0] <= it:
            k += 1
        b0, c0, c1, J = spans[k]
        r = it - b0
        lo, hi = 0, J - 1
        while lo < hi:
            mid = (lo + hi + 1) // 2
            if _panel_items_before_run(mid, c0, c1, h) <= r:
                lo = mid
            else:
                hi = mid - 1
        ct = max(c0, lo * h) + (r - _panel_items_before_run(lo, c0, c1, h))
        rb0 = lo * L
        rb1 = min(rb0 + L, (ct + 1) * m, n_rb)
        if rb0 < rb1:
            out.append((ct, rb0, rb1))
    return out


def shard_items(n_gram: int, shard: int, n_shards: int, bn: int = 256, num_sms: int = 148,
                panel: int | None = None):
    """Tiles of shard `shard` of `n_shards`: the work items [I s / S, I (s + 1) / S)
    of the symmetric schedule, each as (column tile, first row block, end row
    block). Every pair (p <= q) of the n_gram blocks lies in exactly one tile
    of exactly one shard."""
    items, _ = gram_items(n_gram, bn, num_sms)
    return decode_items(n_gram, items * shard // n_shards, items * (shard + 1) // n_shards, bn, num_sms, panel)


def sharded_exchange(compute_sums, finish, allreduce):
    """The sharded global map's one exchange step: this rank's per-block
    sums over its tiles of block pairs -> summed over all ranks in place (the
    only collective) -> the map finished from the summed sums."""
    sums, n_gram = compute_sums()
    allreduce(sums[:2 * n_gram])
    return finish(sums)


def global_map_device_sharded(metric: str, d_img_ptr: int, width: int, height: int, block_width: int,
                              block_height: int, relevance_constant: float, normalize_output: bool, d_out_ptr: int,
                              rank: int, world: int, allreduce=None, stream_ptr: int = 0, ctx=None) -> dict:
    """One global map computed by `world` ranks (each its own GPU and
    context), every rank finishing the full map into d_out. `allreduce`
    (default torch.distributed.all_reduce) sums a float64 CUDA tensor across
    the ranks in place."""
    import torch
    c = _ctx(ctx)
    cap = 2 * max(1, width * height)
    dev = torch.device("cuda", torch.cuda.current_device())
    sums = torch.zeros(cap, dtype=torch.float64, device=dev)
    info1, info2 = _lib.RunInfo(), _lib.RunInfo()
    if allreduce is None:
        import torch.distributed as dist
        allreduce = dist.all_reduce

    def compute():
        c.check(c._L.sred_global_map_2d_shard_sums(
            c.h, metric.encode(), C.c_void_p(d_img_ptr), width, height, block_width, block_height,
            float(relevance_constant), int(rank), int(world), C.c_void_p(sums.data_ptr()), cap,
            C.c_void_p(stream_ptr or None), C.byref(info1)), "sred_global_map_2d_shard_sums")
        return sums, int(info1.n_relevant - info1.n_flat)

    def fin(summed):
        c.check(c._L.sred_global_map_2d_shard_finish(c.h, C.c_void_p(summed.data_ptr()), int(bool(normalize_output)),
                                                     C.c_void_p(d_out_ptr), C.c_void_p(stream_ptr or None),
                                                     C.byref(info2)), "sred_global_map_2d_shard_finish")
        return info2.as_dict()

    return sharded_exchange(compute, fin, allreduce)


def block_map_device(metric: str, d_img_ptr: int, width: int, height: int, frames: int,
                     reference_block: ReferenceBlock2D, relevance_constant: float, normalize_output: bool,
                     d_out_ptr: int, stream_ptr: int = 0, ctx=None) -> None:
    """Block map over a device-resident stack of frames (raw CUDA pointers)."""
    c = _ctx(ctx)
    c.check(c._L.sred_block_map_2d_device(
        c.h, metric.encode(), C.c_void_p(d_img_ptr), width, height, frames,
        np.ascontiguousarray(reference_block.pixels, np.float32).ravel(), int(reference_block.size),
        reference_block.width, reference_block.height, float(reference_block.mean), float(reference_block.std),
        float(relevance_constant), int(bool(normalize_output)), C.c_void_p(d_out_ptr),
        C.c_void_p(stream_ptr or None)), "sred_block_map_2d_device")


def block_map_stack(metric: str, stack: np.ndarray, reference_block: ReferenceBlock2D, relevance_constant: float,
                    normalize_output: bool, chunk_frames: int = 0, out: np.ndarray | None = None,
                    ctx=None) -> np.ndarray:
    """Block maps of a host stack of frames [frames, h, w] (the time-lapse loop
    of java/BlockRepetition2D_.java:95-130), each frame mapped and normalised
    on its own. The stack streams through the GPU in chunks whose uploads,
    maps and downloads overlap; pass page-locked arrays (e.g. a pinned torch
    tensor's .numpy()) for stack and out to let the copies run concurrently."""
    if metric not in BLOCK_METRICS and metric not in EXTRA_BLOCK_METRICS:
        return None
    c = _ctx(ctx)
    a = np.ascontiguousarray(stack, np.float32)
    if a.ndim == 2:
        a = a[None]
    frames, h, w = a.shape
    if out is None:
        out = np.empty_like(a)
    res = _out_buffer(out, a.size, "frames * h * w elements").reshape(frames, h, w)
    st = c._L.sred_block_map_2d_stack(
        c.h, metric.encode(), a.reshape(-1), w, h, frames,
        np.ascontiguousarray(reference_block.pixels, np.float32).ravel(), int(reference_block.size),
        reference_block.width, reference_block.height, float(reference_block.mean), float(reference_block.std),
        float(relevance_constant), int(bool(normalize_output)), int(chunk_frames), res.reshape(-1))
    c.check(st, "sred_block_map_2d_stack")
    return res


def shard_frames(frames: int, rank: int, world: int) -> tuple[int, int]:
    """Frames [f0, f1) of a time-lapse that rank `rank` of `world` maps:
    contiguous, sizes differing by at most one."""
    return frames * rank // world, frames * (rank + 1) // world


def block_map_stack_sharded(metric: str, stack: np.ndarray, reference_block: ReferenceBlock2D,
                            relevance_constant: float, normalize_output: bool, rank: int, world: int,
                            gather: bool = True, all_gather=None, compute=None, ctx=None):
    """A time-lapse block map across `world` ranks (one GPU each): frames are
    independent, so rank r maps frames shard_frames(F, r, world) with
    block_map_stack and no data moves between ranks while mapping. With
    gather, one all-gather (default torch.distributed.all_gather, padded to
    the largest shard) gives every rank the whole [F, h, w] result; without
    it, the rank's own (f0, f1, maps) is returned. `compute(sub_stack)`
    replaces the per-rank mapping (tests)."""
    a = np.ascontiguousarray(stack, np.float32)
    frames, h, w = a.shape
    f0, f1 = shard_frames(frames, rank, world)
    if compute is None:
        def compute(sub):
            if sub.shape[0] == 0:
                return np.zeros_like(sub)
            return block_map_stack(metric, sub, reference_block, relevance_constant, normalize_output, ctx=ctx)
    mine = compute(a[f0:f1])
    if mine is None:
        return None
    if not gather:
        return f0, f1, mine
    import torch
    import torch.distributed as dist
    if all_gather is None:
        all_gather = dist.all_gather
    span = max(shard_frames(frames, r, world)[1] - shard_frames(frames, r, world)[0] for r in range(world))
    on_gpu = dist.is_initialized() and dist.get_backend() == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    buf = torch.zeros((span, h, w), dtype=torch.float32, device=dev)
    buf[:f1 - f0] = torch.from_numpy(np.ascontiguousarray(mine, np.float32)).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    all_gather(parts, buf)
    out = np.empty((frames, h, w), np.float32)
    for r in range(world):
        g0, g1 = shard_frames(frames, r, world)
        out[g0:g1] = parts[r][:g1 - g0].cpu().numpy()
    return out


# ---------------------------------------------------------------------------
# Volumes (java/CLUtils.java:1030-1653)
# ---------------------------------------------------------------------------

def get_local_statistics_3d(input_image: InputImage3D, block_width: int, block_height: int, block_depth: int,
                            ctx=None) -> CLLocalStatistics:
    """java/CLUtils.java:1030-1131."""
    c = _ctx(ctx)
    n = input_image.size
    m = np.zeros(n, np.float32)
    s = np.zeros(n, np.float32)
    c.check(c._L.sred_local_statistics_3d(c.h, np.ascontiguousarray(input_image.image_array, np.float32).ravel(),
                                          input_image.width, input_image.height, input_image.depth, block_width,
                                          block_height, block_depth, m, s), "sred_local_statistics_3d")
    return CLLocalStatistics(m, s)


def calculate_block_repetition_map_3d(metric: str, input_image: InputImage3D, reference_block: ReferenceBlock3D,
                                      relevance_constant: float, normalize_output: bool, use_device: bool = False,
                                      ctx=None, out: np.ndarray | None = None):
    """java/CLUtils.java:1639-1653 (None for an unknown metric). ``out``: an
    optional float32 buffer of the volume's size to write into (pinned host
    memory makes the copies faster)."""
    if metric not in BLOCK_METRICS_3D:
        return None
    c = _ctx(ctx)
    out = np.zeros(input_image.size, np.float32) if out is None else _out_buffer(out, input_image.size,
                                                                                  "the volume's size")
    rb = reference_block
    c.check(c._L.sred_calculate_block_repetition_map_3d(
        c.h, metric.encode(), np.ascontiguousarray(input_image.image_array, np.float32).ravel(), input_image.width,
        input_image.height, input_image.depth, np.ascontiguousarray(rb.pixels, np.float32).ravel(), int(rb.size),
        rb.width, rb.height, rb.depth, float(rb.mean), float(rb.std), float(relevance_constant),
        int(bool(normalize_output)), out), "sred_calculate_block_repetition_map_3d")
    return out


def _block3d_getter(metric):
    def f(input_image, reference_block, relevance_constant, normalize_output, use_device=False, ctx=None):
        return calculate_block_repetition_map_3d(metric, input_image, reference_block, relevance_constant,
                                                 normalize_output, use_device, ctx)
    f.__doc__ = f"getBlock*3D for {metric!r} (java/CLUtils.java:1133-1637)."
    return f


get_block_pearson_3d = _block3d_getter("Pearson's R")
get_block_ssim_3d = _block3d_getter("SSIM")
get_block_nrmse_3d = _block3d_getter("NRMSE (inverted)")
get_block_abs_diff_stds_3d = _block3d_getter("Abs. Diff. of StdDevs.")


def block_map_3d_device(metric: str, d_vol_ptr: int, width: int, height: int, depth: int,
                        reference_block: ReferenceBlock3D, relevance_constant: float, normalize_output: bool,
                        d_out_ptr: int, stream_ptr: int = 0, ctx=None) -> None:
    """3D block map over a device-resident volume (raw CUDA pointers)."""
    c = _ctx(ctx)
    rb = reference_block
    c.check(c._L.sred_block_map_3d_device(
        c.h, metric.encode(), C.c_void_p(d_vol_ptr), width, height, depth,
        np.ascontiguousarray(rb.pixels, np.float32).ravel(), int(rb.size), rb.width, rb.height, rb.depth,
        float(rb.mean), float(rb.std), float(relevance_constant), int(bool(normalize_output)),
        C.c_void_p(d_out_ptr), C.c_void_p(stream_ptr or None)), "sred_block_map_3d_device")


def calculate_global_repetition_map_3d(metric: str, input_image: InputImage3D, block_width: int, block_height: int,
                                       block_depth: int, relevance_constant: float, normalize_output: bool = True,
                                       ctx=None, return_info: bool = False, out: np.ndarray | None = None):
    """java/CLUtils.java:2793-2816 with the preprocessing of
    java/GlobalRepetition3D_.java:97-143 (local statistics, the 3D relevance
    mask, nPixels) done inside libsred. None for an unknown metric; with
    ``return_info`` a (map, run info) pair."""
    if metric not in GLOBAL_METRICS:
        return None
    c = _ctx(ctx)
    out = np.zeros(input_image.size, np.float32) if out is None else _out_buffer(out, input_image.size,
                                                                                  "the volume's size")
    info = _lib.RunInfo()
    c.check(c._L.sred_calculate_global_repetition_map_3d(
        c.h, metric.encode(), np.ascontiguousarray(input_image.image_array, np.float32).ravel(), input_image.width,
        input_image.height, input_image.depth, block_width, block_height, block_depth, float(relevance_constant),
        int(bool(normalize_output)), out, C.byref(info)), "sred_calculate_global_repetition_map_3d")
    return (out, info.as_dict()) if return_info else out


def global_map_3d_device(metric: str, d_vol_ptr: int, width: int, height: int, depth: int, block_width: int,
                         block_height: int, block_depth: int, relevance_constant: float, normalize_output: bool,
                         d_out_ptr: int, stream_ptr: int = 0, ctx=None) -> dict:
    """3D global map on device-resident buffers (raw CUDA pointers); returns run info."""
    c = _ctx(ctx)
    info = _lib.RunInfo()
    c.check(c._L.sred_global_map_3d_device(c.h, metric.encode(), C.c_void_p(d_vol_ptr), width, height, depth,
                                           block_width, block_height, block_depth, float(relevance_constant),
                                           int(bool(normalize_output)), C.c_void_p(d_out_ptr),
                                           C.c_void_p(stream_ptr or None), C.byref(info)), "sred_global_map_3d_device")
    return info.as_dict()


# ---------------------------------------------------------------------------
# Relevance-mask tools on a preprocessed image (variance-stabilised and
# min-max normalised); the commands themselves are in plugins.py.
# ---------------------------------------------------------------------------

def relevance_mask_tool_2d(image: np.ndarray, block_width: int, block_height: int, filter_constant: float,
                           ctx=None) -> RelevanceMask:
    """The mask of java/RelevanceMask2D_.java (local std, FP64 noise tiles)."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(image, np.float32)
    h, w = a.shape
    mask = np.zeros(w * h, np.float32)
    thr, nv = C.c_float(), C.c_float()
    c.check(c._L.sred_relevance_mask_tool_2d(c.h, a.ravel(), w, h, block_width, block_height, float(filter_constant),
                                             mask, C.byref(thr), C.byref(nv)), "sred_relevance_mask_tool_2d")
    return RelevanceMask(mask.reshape(h, w), np.float32(filter_constant), np.float32(thr.value), np.float32(nv.value))


def relevance_mask_sweep_2d(image: np.ndarray, block_width: int, block_height: int, lower: float, step: float,
                            n: int, ctx=None) -> tuple:
    """The n masks of java/RelevanceMaskStack2D_.java: (masks [n, h, w],
    constants [n], noise variance)."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(image, np.float32)
    h, w = a.shape
    masks = np.zeros(n * w * h, np.float32)
    consts = np.zeros(n, np.float32)
    nv = C.c_float()
    c.check(c._L.sred_relevance_mask_sweep_2d(c.h, a.ravel(), w, h, block_width, block_height, float(lower),
                                              float(step), int(n), masks, consts, C.byref(nv)),
            "sred_relevance_mask_sweep_2d")
    return masks.reshape(n, h, w), consts, np.float32(nv.value)


def relevance_constant_range_2d(image: np.ndarray, block_width: int, block_height: int, step: float,
                                ctx=None) -> tuple:
    """java/OptimiseRelevanceMask_.java's result: (last constant with an
    all-1 interior, first constant with an all-0 mask, noise variance)."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(image, np.float32)
    h, w = a.shape
    ones, zeros, nv = C.c_float(), C.c_float(), C.c_float()
    c.check(c._L.sred_relevance_constant_range_2d(c.h, a.ravel(), w, h, block_width, block_height, float(step),
                                                  C.byref(ones), C.byref(zeros), C.byref(nv)),
            "sred_relevance_constant_range_2d")
    return np.float32(ones.value), np.float32(zeros.value), np.float32(nv.value)


def global_map_3d_device_sharded(metric: str, d_vol_ptr: int, width: int, height: int, depth: int, block_width: int,
                                 block_height: int, block_depth: int, relevance_constant: float,
                                 normalize_output: bool, d_out_ptr: int, rank: int, world: int, allreduce=None,
                                 stream_ptr: int = 0, ctx=None) -> dict:
    """One 3D global map computed by `world` ranks, as global_map_device_sharded."""
    import torch
    c = _ctx(ctx)
    cap = 2 * max(1, width * height * depth)
    dev = torch.device("cuda", torch.cuda.current_device())
    sums = torch.zeros(cap, dtype=torch.float64, device=dev)
    info1, info2 = _lib.RunInfo(), _lib.RunInfo()
    if allreduce is None:
        import torch.distributed as dist
        allreduce = dist.all_reduce

    def compute():
        c.check(c._L.sred_global_map_3d_shard_sums(
            c.h, metric.encode(), C.c_void_p(d_vol_ptr), width, height, depth, block_width, block_height, block_depth,
            float(relevance_constant), int(rank), int(world), C.c_void_p(sums.data_ptr()), cap,
            C.c_void_p(stream_ptr or None), C.byref(info1)), "sred_global_map_3d_shard_sums")
        return sums, int(info1.n_relevant - info1.n_flat)

    def fin(summed):
        c.check(c._L.sred_global_map_3d_shard_finish(c.h, C.c_void_p(summed.data_ptr()), int(bool(normalize_output)),
                                                     C.c_void_p(d_out_ptr), C.c_void_p(stream_ptr or None),
                                                     C.byref(info2)), "sred_global_map_3d_shard_finish")
        return info2.as_dict()

    return sharded_exchange(compute, fin, allreduce)
