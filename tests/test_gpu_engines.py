"""The two contraction engines on caller-given vectors, through the C ABI.

num[p] = sum_q <u_p, u_q> w1[p] w1[q] and den[p] = sum_q (w2[p] + w2[q])
(symmetric pair terms, as the engines evaluate the upper triangle) are checked
against an FP64 evaluation for every K' chunk count the tensor-core engine
uses (K' = round_up(3K, 16) from 16 to 448) and for ragged N (partial row
blocks and column tiles). Bound: |err| <= tol * sum_q |G_pq w1_p w1_q| with
tol = 2e-6 for the FP32 engine and 4e-5 for split-BF16 (the omitted lo*lo
term and bf16 rounding of lo are below 2^-15 of |u_p||u_q|).
"""
import ctypes as C

import numpy as np
import pytest

from sred_b200 import _lib

pytestmark = pytest.mark.gpu
TOL = {"fp32": 2e-6, "tc": 4e-5}


@pytest.fixture(scope="module")
def ctx():
    return _lib.Context(0, "fp32")


def rowdot(ctx, engine, u, w1, w2):
    n, k = u.shape
    num = np.zeros(n, np.float64)
    den = np.zeros(n, np.float64)
    e = {"tc": _lib.ENGINE_TC, "fp32": _lib.ENGINE_FP32}[engine]
    ctx.check(ctx._L.sred_debug_gram_rowdot(ctx.h, e, np.ascontiguousarray(u, np.float32),
                                            np.ascontiguousarray(w1, np.float32),
                                            np.ascontiguousarray(w2, np.float32), n, k, num, den),
              "sred_debug_gram_rowdot")
    return num, den


@pytest.mark.parametrize("engine", ["fp32", "tc"])
@pytest.mark.parametrize("n,k", [(1, 5), (100, 5), (300, 13), (1000, 49), (777, 81), (513, 113), (260, 149)])
def test_rowdot_matches_fp64(ctx, engine, n, k):
    rng = np.random.default_rng(n * 1000 + k)
    u = rng.normal(size=(n, k)).astype(np.float32)
    u /= np.linalg.norm(u, axis=1, keepdims=True).astype(np.float32)
    w1 = rng.uniform(-1, 1, n).astype(np.float32)
    w2 = rng.uniform(0, 1, n).astype(np.float32)
    num, den = rowdot(ctx, engine, u, w1, w2)
    U = u.astype(np.float64)
    G = U @ U.T
    w = w1.astype(np.float64)
    exp = w * (G @ w)
    scale = np.abs(w) * (np.abs(G) @ np.abs(w))
    err = np.abs(num - exp) / np.maximum(scale, 1e-30)
    assert float(err.max()) <= TOL[engine], float(err.max())
    w2d = w2.astype(np.float64)
    np.testing.assert_allclose(den, n * w2d + w2d.sum(), rtol=1e-6)


def test_tc_matches_fp32_unnormalised(ctx):
    """Vectors of mixed magnitude (the engine must not assume unit norm)."""
    rng = np.random.default_rng(5)
    n, k = 700, 49
    u = (rng.normal(size=(n, k)) * rng.uniform(0.01, 10, (n, 1))).astype(np.float32)
    w1 = rng.uniform(0, 1, n).astype(np.float32)
    a, _ = rowdot(ctx, "fp32", u, w1, w1)
    b, _ = rowdot(ctx, "tc", u, w1, w1)
    U = u.astype(np.float64)
    w = w1.astype(np.float64)
    scale = w * (np.abs(U @ U.T) @ w)
    assert float(np.max(np.abs(a - b) / scale)) <= TOL["tc"]


def test_global_map_batch_equals_single_maps(ctx):
    """A batch of maps of mixed sizes, blocks and metrics on several workers
    returns each map exactly as a single call does."""
    from sred_b200 import clutils, synth
    jobs = []
    for i, (w, h, b, metric) in enumerate([(96, 80, 3, "Pearson's R"), (64, 64, 5, "SSIM"), (120, 72, 9, "NRMSE"),
                                          (80, 96, 5, "Pearson's R"), (72, 72, 11, "SSIM"),
                                          (64, 96, 3, "Abs. diff. of StdDevs")]):
        img = synth.normalize_input(synth.spot_image(w, h, 4, seed=40 + i))
        jobs.append({"metric": metric, "img": img, "block_width": b, "block_height": b, "relevance_constant": 1.0})
    for engine in ("tc", "fp32"):
        ctx.set_engine(engine)
        res = clutils.global_map_batch(jobs, n_workers=3, ctx=ctx)
        for j, (out, info) in zip(jobs, res):
            single, _ = clutils.global_map_host(j["metric"], j["img"], j["block_width"], j["block_height"], 1.0,
                                                ctx=ctx)
            np.testing.assert_array_equal(out, single)
            assert info["n_relevant"] > 0
    ctx.set_engine("fp32")


def test_sharded_map_equals_full_map(ctx):
    """The sharded entry points, every shard run in turn on one GPU and
    their sums added (what the all-reduce does across GPUs), give the map of
    sred_global_map_2d_device."""
    import ctypes as C

    import torch
    from sred_b200 import clutils, synth
    img = synth.normalize_input(synth.spot_image(176, 144, 8, seed=7))
    H, W = img.shape
    d_in = torch.from_numpy(img).cuda()
    for engine in ("tc", "fp32"):
        ctx.set_engine(engine)
        for metric in ("Pearson's R", "SSIM", "NRMSE"):
            full = torch.empty_like(d_in)
            clutils.global_map_device(metric, d_in.data_ptr(), W, H, 5, 5, 1.0, True, full.data_ptr(), ctx=ctx)
            torch.cuda.synchronize()
            for world in (2, 3):
                cap = 2 * W * H
                acc = torch.zeros(cap, dtype=torch.float64, device="cuda")
                for s in range(world):
                    part = torch.zeros(cap, dtype=torch.float64, device="cuda")
                    info = _lib.RunInfo()
                    ctx.check(ctx._L.sred_global_map_2d_shard_sums(
                        ctx.h, metric.encode(), C.c_void_p(d_in.data_ptr()), W, H, 5, 5, 1.0, s, world,
                        C.c_void_p(part.data_ptr()), cap, None, C.byref(info)), "shard_sums")
                    acc += part
                out = torch.empty_like(d_in)
                ctx.check(ctx._L.sred_global_map_2d_shard_finish(ctx.h, C.c_void_p(acc.data_ptr()), 1,
                                                                 C.c_void_p(out.data_ptr()), None, None),
                          "shard_finish")
                torch.cuda.synchronize()
                np.testing.assert_allclose(out.cpu().numpy(), full.cpu().numpy(), rtol=0, atol=1e-6)
    # phase 2 without phase 1 is refused
    st = ctx._L.sred_global_map_2d_shard_finish(ctx.h, C.c_void_p(d_in.data_ptr()), 1, C.c_void_p(d_in.data_ptr()),
                                                None, None)
    assert st == _lib.ERR_ARG
    ctx.set_engine("fp32")


def test_log_callback(ctx):
    """Messages reach the callback: one line per global map, and errors."""
    from sred_b200 import clutils, synth
    got = []
    ctx.set_log_callback(got.append)
    img = synth.normalize_input(synth.spot_image(64, 48, 4, seed=3))
    clutils.global_map_host("Pearson's R", img, 5, 5, 1.0, ctx=ctx)
    assert any(m.startswith("global map 64x48 K=13") for m in got), got
    with pytest.raises(_lib.SredError):
        clutils.global_map_host("no such metric", img, 5, 5, 1.0, ctx=ctx)
    assert any(m.startswith("error: unknown global metric") for m in got), got
    ctx.set_log_callback(None)
    n = len(got)
    clutils.global_map_host("Pearson's R", img, 5, 5, 1.0, ctx=ctx)
    assert len(got) == n


@pytest.fixture
def clean_tuning():
    _lib.gram_tuning_clear()
    yield
    _lib.gram_tuning_clear()


# (NRMSE takes three split levels, so 15x15 (K' = 6 x 149 > 576) runs on the FP32 engine and is not tuned.)
@pytest.mark.parametrize("metric,b", [("Pearson's R", 9), ("SSIM", 5), ("NRMSE", 9), ("SSIM", 15)])
def test_gram_tuning_shapes_give_the_same_map(ctx, clean_tuning, metric, b):
    """The tuner times every launch shape and stores the fastest; the map it
    returns, and the map of every other shape stored by hand, equal the
    default shape's map (the pair terms are the same; only the FP64 sum order
    differs)."""
    from sred_b200 import clutils, synth
    img = synth.normalize_input(synth.spot_image(300, 260, 6, seed=17))
    ctx.set_engine("tc")
    base, _ = clutils.global_map_host(metric, img, b, b, 1.0, ctx=ctx)
    ctx.set_gram_tuning(True)
    tuned, info = clutils.global_map_host(metric, img, b, b, 1.0, ctx=ctx)
    ctx.set_gram_tuning(False)
    ent = _lib.gram_tuning_entries()
    n_g = info["n_relevant"] - info["n_flat"]
    ncls = 0 if n_g < 1 << 16 else 1 if n_g < 1 << 18 else 2
    assert len(ent) == 1 and ent[0]["size_class"] == ncls and ent[0]["ms"] > 0, (ent, n_g)
    np.testing.assert_allclose(tuned, base, rtol=0, atol=2e-6)
    key = {k: ent[0][k] for k in ("kq", "metric", "size_class")}
    tried = 0
    for bn in (256, 128):
        for tr in (True, False):
            for ml in (32, 16, 8, 4):
                if _lib.gram_tuning_set([dict(key, bn=bn, a_resident=tr, max_l=ml)]) != 1:
                    continue
                tried += 1
                out, _ = clutils.global_map_host(metric, img, b, b, 1.0, ctx=ctx)
                np.testing.assert_allclose(out, base, rtol=0, atol=2e-6, err_msg=f"{bn} {tr} {ml}")
    # every K' admits at least one tile width with 32 / 16 / 8 / 4 row blocks per run
    # (NRMSE 9x9, K' = 320, fits only 128-column tiles with the chunk ring)
    assert tried >= 3
    # a shape the K' does not admit is refused
    assert _lib.gram_tuning_set([dict(key, bn=192, a_resident=False, max_l=16)]) == 0
    ctx.set_engine("fp32")


def test_gram_tuning_table_round_trip(tmp_path, clean_tuning):
    """gram_tuning_save / gram_tuning_load restore the table."""
    n = _lib.gram_tuning_set([{"kq": 160, "metric": 0, "size_class": 2, "bn": 128, "a_resident": False,
                               "max_l": 8, "ms": 1.5}])
    assert n == 1
    p = _lib.gram_tuning_save(tmp_path / "t.json", device="test")
    _lib.gram_tuning_clear()
    assert _lib.gram_tuning_entries() == []
    assert _lib.gram_tuning_load(p) == 1
    e = _lib.gram_tuning_entries()
    assert e[0]["bn"] == 128 and not e[0]["a_resident"] and e[0]["max_l"] == 8
