"""Sharding of one global map across ranks (host logic, CPU only).

libsred evaluates each unordered block pair once: the work is the upper
triangle of 128-row x 256-column tiles, cut into work items, and shard s of
S takes the items [I s / S, I (s + 1) / S) (clutils.shard_items mirrors the
rule). The partition test checks that every pair lies in exactly one tile of
one shard. The exchange is checked with two gloo ranks on the CPU: each rank
adds the FP64 pair terms of its tiles to both blocks of each pair (the self
pair once), the ranks sum their per-block sums with one all-reduce, and every
rank finishes the map; the result must equal the oracle's unsharded FP64 map.
"""
import datetime
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from sred_b200 import clutils


@pytest.mark.parametrize("n_gram", [0, 1, 127, 128, 129, 255, 256, 257, 1000, 4097, 30001])
@pytest.mark.parametrize("world", [1, 2, 3, 8])
@pytest.mark.parametrize("bn,sms,panel", [(256, 148, None), (128, 148, None), (256, 4, None), (256, 4, 3),
                                          (128, 2, 5), (256, 148, 7)])
def test_shard_items_cover_each_pair_once(n_gram, world, bn, sms, panel):
    n_rb = (n_gram + 127) // 128
    n_ct = (n_gram + bn - 1) // bn
    seen = {}
    for s in range(world):
        for ct, rb0, rb1 in clutils.shard_items(n_gram, s, world, bn, sms, panel):
            for rb in range(rb0, rb1):
                assert (rb, ct) not in seen, (rb, ct)
                seen[(rb, ct)] = s
    # exactly the tiles holding a pair p <= q with both below n_gram
    want = {(rb, ct) for ct in range(n_ct) for rb in range(n_rb) if rb * 128 <= ct * bn + bn - 1}
    assert set(seen) == want


@pytest.mark.parametrize("n_gram,bn,panel", [(5000, 256, 4), (30001, 128, 13), (9000, 256, None)])
def test_item_order_is_panel_major(n_gram, bn, panel):
    """Items go panel by panel (column tiles [kP, (k+1)P)), within a panel run by
    run, within a run by column tile: the decoded list equals that enumeration."""
    _, L = clutils.gram_items(n_gram, bn)
    m, h = bn // 128, L // (bn // 128)
    n_rb, n_ct = (n_gram + 127) // 128, (n_gram + bn - 1) // bn
    P = panel or n_ct
    want = []
    for c0 in range(0, n_ct, P):
        for j in range((n_rb + L - 1) // L):
            for ct in range(max(c0, j * h), min(c0 + P, n_ct)):
                rb0, rb1 = j * L, min(j * L + L, (ct + 1) * m, n_rb)
                if rb0 < rb1:
                    want.append((ct, rb0, rb1))
    items, _ = clutils.gram_items(n_gram, bn)
    assert clutils.decode_items(n_gram, 0, items, bn, panel=panel) == want


def test_gram_panel_fits_48_mb():
    assert clutils.gram_panel(256, 160) == (48 << 20) // (256 * 160 * 2)
    assert clutils.gram_panel(256, 160) * 256 * 160 * 2 <= 48 << 20
    assert clutils.gram_panel(128, 1 << 20) == 1


@pytest.mark.parametrize("world", [1, 2, 8])
def test_shard_items_balanced(world):
    n = 754587  # relevant blocks of the 1024^2 / 9x9 benchmark map
    items, _ = clutils.gram_items(n)
    sizes = [items * (s + 1) // world - items * s // world for s in range(world)]
    assert sum(sizes) == items and max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _pair_terms_f64(metric, img, bw, bh, listed, nv):
    """FP64 numerator and denominator terms of every pair of the listed
    blocks, as the oracle's FP64 judge evaluates them (orc_global_f64): FP64
    block moments, weight exp(-(s_p - s_q)^2 / (nv + eps)), Pearson
    max(0, cov / (s_p s_q + eps)) (flat pairs: 1 if both flat, else 0), NRMSE
    sqrt(mse / K) unweighted."""
    import oracle
    H, W = img.shape
    rw, rh = bw // 2, bh // 2
    off = [(dy, dx) for dy in range(-rh, rh + 1) for dx in range(-rw, rw + 1)
           if (dx * dx) / float(rw * rw) + (dy * dy) / float(rh * rh) <= 1.0]
    K = oracle.block_size(bw, bh)
    assert len(off) == K
    x = img.astype(np.float64)
    ys, xs = np.divmod(listed, W)
    V = np.stack([x[ys + dy, xs + dx] for dy, dx in off], axis=1)
    mu = V.mean(axis=1, keepdims=True)
    C = V - mu
    sig = np.sqrt((C * C).sum(axis=1) / (K - 1))
    h = float(np.float32(nv)) + float(np.float32(oracle.EPSILON))
    w = np.exp(-((sig[:, None] - sig[None, :]) ** 2) / h)
    if metric == "NRMSE":
        d2 = (C * C).sum(1)[:, None] + (C * C).sum(1)[None, :] - 2.0 * (C @ C.T)
        tn = np.sqrt(np.maximum(d2, 0.0) / K)
        np.fill_diagonal(tn, 0.0)
        return tn, w
    cov = (C @ C.T) / (K - 1)
    r = cov / (sig[:, None] * sig[None, :] + float(np.float32(oracle.EPSILON)))
    flat = sig == 0.0
    tn = np.maximum(r, 0.0) * w
    tn = np.where(flat[:, None] & flat[None, :], w, np.where(flat[:, None] | flat[None, :], 0.0, tn))
    return tn, w


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
        terms_n, terms_d = _pair_terms_f64(metric, img, bw, bh, listed, nv)

        def compute():
            sums = torch.zeros(2 * n, dtype=torch.float64)
            num = np.zeros(n)
            den = np.zeros(n)
            for ct, rb0, rb1 in clutils.shard_items(n, rank, world):
                q0, q1 = ct * 256, min(ct * 256 + 256, n)
                for rb in range(rb0, rb1):
                    p0, p1 = rb * 128, min(rb * 128 + 128, n)
                    P, Q = np.meshgrid(np.arange(p0, p1), np.arange(q0, q1), indexing="ij")
                    keep = Q >= P
                    tn = np.where(keep, terms_n[p0:p1, q0:q1], 0.0)
                    td = np.where(keep, terms_d[p0:p1, q0:q1], 0.0)
                    num[p0:p1] += tn.sum(axis=1)
                    den[p0:p1] += td.sum(axis=1)
                    off = Q > P  # the pair's second block (the self pair once)
                    num[q0:q1] += np.where(off, tn, 0.0).sum(axis=0)
                    den[q0:q1] += np.where(off, td, 0.0).sum(axis=0)
            sums[:n] = torch.from_numpy(num)
            sums[n:] = torch.from_numpy(den)
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


def _failing_rank(rank, world, port, out_q):
    """Rank 1's shard fails before the exchange (as a failed
    sred_global_map_2d_shard_sums raises SredError) and leaves; rank 0 is
    already in the all-reduce and must get an error, not wait for good."""
    import time

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    n = 64

    def compute():
        if rank == 1:
            raise RuntimeError("injected shard failure")
        return torch.ones(2 * n, dtype=torch.float64), n

    t0 = time.monotonic()
    try:
        clutils.sharded_exchange(compute, lambda s: s, dist.all_reduce)
        out_q.put((rank, "completed", time.monotonic() - t0))
    except Exception as e:  # noqa: BLE001 - the test reports any failure kind
        out_q.put((rank, type(e).__name__ + ": " + str(e)[:80], time.monotonic() - t0))
    finally:
        dist.destroy_process_group()


def test_sharded_exchange_rank_failure_ends_the_collective():
    """A rank that fails between steps leaves without joining the all-reduce;
    the other rank's collective ends with an error within the process
    group's timeout instead of hanging."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode is not None for p in procs), "a rank did not end"
    res = dict((r, (msg, t)) for r, msg, t in (q.get(timeout=5) for _ in range(2)))
    assert res[1][0].startswith("RuntimeError: injected shard failure"), res
    assert res[0][0] != "completed" and res[0][1] < 60.0, res


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
