"""Row sharding of one global map across ranks (host logic, CPU only).

The exchange is checked with two gloo ranks on the CPU: each rank computes
the FP64 oracle's per-row sums of its own row blocks (zero elsewhere), the
ranks sum them with one all-reduce, and every rank finishes the map; the
result must equal the unsharded map. The partition rule is the one libsred
applies (clutils.shard_row_blocks).
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from sred_b200 import clutils


@pytest.mark.parametrize("n_gram", [0, 1, 127, 128, 129, 1000, 754587])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_row_blocks_partition(n_gram, world):
    n_rb = (n_gram + 127) // 128
    spans = [clutils.shard_row_blocks(n_gram, s, world) for s in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == n_rb
    for (a0, a1), (b0, b1) in zip(spans, spans[1:]):
        assert a1 == b0 and a0 <= a1
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, metric, out_q):
    import torch
    import torch.distributed as dist

    import oracle
    from sred_b200 import synth
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        img = synth.normalize_input(synth.spot_image(48, 40, 4, seed=31))
        H, W = img.shape
        bw = bh = 3
        c = 1.0
        means, stds = oracle.local_stats(img, bw, bh)
        mask, thr, nv = oracle.relevance_mask(img, bw, bh, stds, c)
        ys, xs = np.mgrid[1:H - 1, 1:W - 1]
        pix = (ys * W + xs).ravel()
        s = stds.ravel()[pix]
        listed = pix[s * s >= thr].astype(np.int32)  # the compacted list, raster order
        n = listed.size
        rb0, rb1 = clutils.shard_row_blocks(n, rank, world)

        def compute():
            rows = listed[rb0 * 128:rb1 * 128]
            sums = torch.zeros(2 * n, dtype=torch.float64)
            if rows.size:
                num, den = oracle.global_sums_f64(metric, img, bw, bh, stds, nv, thr, rows)
                sums[rb0 * 128:rb0 * 128 + rows.size] = torch.from_numpy(num)
                sums[n + rb0 * 128:n + rb0 * 128 + rows.size] = torch.from_numpy(den)
            return sums, n

        def finish(summed):
            nf = np.zeros(W * H)
            df = np.zeros(W * H)
            nf[listed] = summed[:n].numpy()
            df[listed] = summed[n:2 * n].numpy()
            out = np.zeros(W * H)
            npx = float(oracle.n_pixels(mask, 1, 1))
            oracle.lib().orc_global_finalize_f64(oracle.GLOBAL_METRICS[metric], nf, df, W, H, 1, 1,
                                                 mask.ravel().copy(), np.float32(c), npx, 1, out)
            return out.reshape(H, W)

        got = clutils.sharded_exchange(compute, finish, dist.all_reduce)
        exp = oracle.global_map(metric, img, bw, bh, c, precision="f64")["map"]
        out_q.put((rank, float(np.max(np.abs(got - exp)))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("metric", ["Pearson's R", "NRMSE"])
def test_sharded_exchange_gloo_two_ranks(metric):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, metric, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r for r, _ in res] == [0, 1]
    assert all(err < 1e-12 for _, err in res), res


@pytest.mark.parametrize("frames,world", [(0, 2), (1, 2), (7, 2), (8, 3), (5, 8)])
def test_shard_frames_partition(frames, world):
    spans = [clutils.shard_frames(frames, r, world) for r in range(world)]
    assert spans[0][0] == 0 and spans[-1][1] == frames
    assert all(a1 == b0 for (_, a1), (b0, _) in zip(spans, spans[1:]))
    sizes = [b - a for a, b in spans]
    assert max(sizes) - min(sizes) <= 1


def _stack_rank(rank, world, port, out_q):
    import torch.distributed as dist

    import oracle
    from sred_b200 import synth, utils
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        stack = np.stack([synth.normalize_input(synth.spot_image(36, 30, 4, seed=s)) for s in range(5)])
        rb = utils.ReferenceBlock2D(stack[0, 10:13, 10:13].ravel()[[1, 3, 4, 5, 7]].copy(), 3, 3, 1, 1, 5,
                                    np.float32(0.5), np.float32(0.2))
        seen = []

        def compute(sub):  # the oracle maps this rank's frames (no GPU here)
            seen.append(sub.shape[0])
            return np.stack([oracle.block_map("Pearson's R", f, rb.pixels, 3, 3, rb.mean, rb.std)["map"]
                             for f in sub]) if sub.shape[0] else np.zeros_like(sub)

        got = clutils.block_map_stack_sharded("Pearson's R", stack, rb, 0.0, True, rank, world, compute=compute)
        exp = np.stack([oracle.block_map("Pearson's R", f, rb.pixels, 3, 3, rb.mean, rb.std)["map"] for f in stack])
        f0, f1 = clutils.shard_frames(5, rank, world)
        out_q.put((rank, seen == [f1 - f0], bool(np.array_equal(got.reshape(exp.shape), exp))))
    finally:
        dist.destroy_process_group()


def test_sharded_time_lapse_gloo_two_ranks():
    """Frames split across two gloo ranks, each mapping its own (the oracle
    standing in for the GPU), one all-gather: every rank holds the whole
    stack's maps, equal to mapping all frames in one place."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_stack_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res == [(0, True, True), (1, True, True)], res
