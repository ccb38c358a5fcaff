"""The ImageJ commands as functions over arrays, with the dialog fields as
keyword arguments (same defaults) and the windowing left out.

``global_repetition_2d`` follows GlobalRepetition2D_.run
(java/GlobalRepetition2D_.java:35-156), ``block_repetition_2d``
BlockRepetition2D_.run (java/BlockRepetition2D_.java:32-158), the 3D pair
GlobalRepetition3D_ / BlockRepetition3D_, and the relevance-mask tools
RelevanceMask2D_, RelevanceMaskStack2D_ and OptimiseRelevanceMask_,
ClassifyRedundancy_, CalculateLocalMeans_, and the variance-stabilisation
commands VarianceStabilisingTransform2D_ / 3D_ (Simplex) and QuadTree_ /
OcTree_. Variance stabilisation inside the map commands uses either GAT method
("Simplex" or "Quad/Octree").
"""
from __future__ import annotations

import numpy as np

from . import clutils, utils


def global_repetition_2d(image: np.ndarray, block_width: int = 5, block_height: int = 5,
                         relevance_constant: float = 0.0, metric: str = "Pearson's R",
                         stabilise_noise_variance: bool = False, normalize_output: bool = True, ctx=None,
                         run_info: dict | None = None):
    if block_width % 2 == 0 or block_height % 2 == 0:
        raise ValueError("Patch dimensions must be odd. Please try again.")
    bs = utils.block_size(block_width, block_height)
    inp = utils.get_input_image_2d(image, True, stabilise_noise_variance, ctx=ctx)
    stats = clutils.get_local_statistics_2d(inp, block_width, block_height, ctx)
    mask = utils.get_relevance_mask(inp.image_array, inp.width, inp.height, block_width // 2, block_height // 2,
                                    stats.local_stds, relevance_constant, ctx)
    m2 = mask.relevance_mask.reshape(inp.height, inp.width)
    rw, rh = block_width // 2, block_height // 2
    count = int(np.count_nonzero(m2[rh:inp.height - rh, rw:inp.width - rw] > 0))
    n_pixels = np.float32(min(count, 1 << 24))  # FP32 accumulation of 1.0f saturates at 2^24
    out = clutils.calculate_global_repetition_map_2d(metric, inp, block_width, block_height, bs, stats, mask,
                                                     n_pixels, normalize_output, ctx, run_info)
    return None if out is None else out.reshape(inp.height, inp.width)


def block_repetition_2d(block: np.ndarray, image: np.ndarray, relevance_constant: float = 0.0,
                        metric: str = "Pearson's R", stabilise_noise_variance: bool = False,
                        normalize_output: bool = True, ctx=None):
    ref = utils.get_reference_block_2d(block)
    if ref is None:
        raise ValueError("Block dimensions must be odd (e.g., 3x3 or 5x5). Please try again.")
    if image.ndim == 2:
        inp = utils.get_input_image_2d(image, True, stabilise_noise_variance, ctx=ctx)
        out = clutils.calculate_block_repetition_map_2d(metric, inp, ref, relevance_constant, normalize_output,
                                                        ctx=ctx)
        return None if out is None else out.reshape(inp.height, inp.width)
    # time-lapse: each frame prepared on its own (java/BlockRepetition2D_.java:104-130), then the whole
    # stack streams through the GPU with its copies overlapping the maps
    h, w = image.shape[1:]
    stack = np.stack([utils.get_input_image_2d(f, True, stabilise_noise_variance, ctx=ctx).image_array.reshape(h, w)
                      for f in image])
    return clutils.block_map_stack(metric, stack, ref, relevance_constant, normalize_output, ctx=ctx)


def global_repetition_3d(volume: np.ndarray, block_width: int = 3, block_height: int = 3, block_depth: int = 3,
                         relevance_constant: float = 0.0, metric: str = "Pearson's R",
                         normalize_output: bool = True, ctx=None, run_info: dict | None = None):
    """GlobalRepetition3D_.run (java/GlobalRepetition3D_.java:40-158) on a
    [depth, height, width] volume; see sred_calculate_global_repetition_map_3d
    for the repairs that make the reference's path run."""
    if block_width % 2 == 0 or block_height % 2 == 0 or block_depth % 2 == 0:
        raise ValueError("Block dimensions must be odd. Please try again.")
    if block_depth < 3:
        raise ValueError("Block depth must be at least 3. Please try again.")
    inp = utils.get_input_image_3d(volume)
    res = clutils.calculate_global_repetition_map_3d(metric, inp, block_width, block_height, block_depth,
                                                     relevance_constant, normalize_output, ctx=ctx, return_info=True)
    if res is None:
        return None
    out, info = res
    if run_info is not None:
        run_info.update(info)
    return out.reshape(inp.depth, inp.height, inp.width)


def block_repetition_3d(block: np.ndarray, volume: np.ndarray, relevance_constant: float = 0.0,
                        metric: str = "Pearson's R", normalize_output: bool = True, ctx=None):
    """BlockRepetition3D_.run (java/BlockRepetition3D_.java:40-115)."""
    ref = utils.get_reference_block_3d(block)
    inp = utils.get_input_image_3d(volume)
    out = clutils.calculate_block_repetition_map_3d(metric, inp, ref, relevance_constant, normalize_output, ctx=ctx)
    return None if out is None else out.reshape(inp.depth, inp.height, inp.width)


def relevance_tools_input(image: np.ndarray, max_iter: int = 5000, ctx=None) -> np.ndarray:
    """The preprocessing the relevance-mask tools share (e.g.
    java/RelevanceMask2D_.java, GAT section and normalisation): the GAT
    parameters fitted from gain 0, sigma 100, offset 0, the transform, then
    min-max to [0, 1] in FP64 with epsilon, stored as float."""
    a = np.ascontiguousarray(image, np.float32)
    g, s, o, _ = utils.fit_gat_2d(a, max_iter, gain=0.0, sigma=100.0, offset=0.0, ctx=ctx)
    t = utils.get_gat_2d(a, g, s, o, ctx=ctx).astype(np.float64)
    mn, mx = t.min(), t.max()
    return ((t - mn) / (mx - mn + float(utils.EPSILON))).astype(np.float32)


def relevance_mask_2d(image: np.ndarray, block_width: int = 3, block_height: int = 3, filter_constant: float = 0.0,
                      ctx=None) -> utils.RelevanceMask:
    """RelevanceMask2D_.run: the relevance mask of one filter constant."""
    return clutils.relevance_mask_tool_2d(relevance_tools_input(image, ctx=ctx), block_width, block_height,
                                          filter_constant, ctx=ctx)


def relevance_mask_stack_2d(image: np.ndarray, block_width: int = 3, block_height: int = 3,
                            lower_limit: float = 0.0, upper_limit: float = 1.0, step: float = 0.1, ctx=None):
    """RelevanceMaskStack2D_.run: masks at lower, lower + step, ... with
    ceil((upper - lower) / step) + 1 slices (FP32, as the command computes
    it); returns (masks [n, h, w], constants, the preprocessed input)."""
    f = np.float32
    n = int(np.ceil(np.float64((f(upper_limit) - f(lower_limit)) / f(step)))) + 1
    inp = relevance_tools_input(image, ctx=ctx)
    masks, consts, _ = clutils.relevance_mask_sweep_2d(inp, block_width, block_height, lower_limit, step, n, ctx=ctx)
    return masks, consts, inp


def optimise_relevance_mask(image: np.ndarray, block_width: int = 3, block_height: int = 3, step: float = 1.0,
                            ctx=None) -> tuple:
    """OptimiseRelevanceMask_.run: the filter-constant range (all-relevant,
    all-irrelevant) the command logs."""
    ones, zeros, _ = clutils.relevance_constant_range_2d(relevance_tools_input(image, ctx=ctx), block_width,
                                                         block_height, step, ctx=ctx)
    return ones, zeros


def classify_redundancy(redundancy_map: np.ndarray, border: int = 1, k: int = 3, optimal_k: bool = False,
                        max_k: int = 10, seed: int = 0, ctx=None) -> tuple:
    """ClassifyRedundancy_.run (java/ClassifyRedundancy_.java): (class map,
    classes used, WCSS); see sred_classify_redundancy_2d."""
    import ctypes as C
    from . import _lib
    c = ctx if ctx is not None else _lib.default_context()
    m = np.ascontiguousarray(redundancy_map, np.float32)
    h, w = m.shape
    out = np.zeros(w * h, np.float32)
    kc, wcss = C.c_int(), C.c_double()
    c.check(c._L.sred_classify_redundancy_2d(c.h, m.ravel(), w, h, border, k, int(bool(optimal_k)), max_k, seed, out,
                                             C.byref(kc), C.byref(wcss)), "sred_classify_redundancy_2d")
    return out.reshape(h, w), kc.value, wcss.value


def calculate_local_means(image: np.ndarray, block_width: int = 3, block_height: int = 3, ctx=None) -> np.ndarray:
    """CalculateLocalMeans_.run (java/CalculateLocalMeans_.java): the relevance
    tools' preprocessing, then the local means and standard deviations as a
    2-slice stack [2, h, w]. As shipped the command asks its program for a
    kernel, kernelGetPatchMeans2D, that the program (kernelGetLocalStatistics2D.cl)
    does not define, and stops there; this returns what it evidently meant to
    show."""
    inp = relevance_tools_input(image, ctx=ctx)
    h, w = inp.shape
    st = clutils.get_local_statistics_2d(utils.InputImage2D(inp.ravel(), w, h), block_width, block_height, ctx)
    return np.stack([st.local_means.reshape(h, w), st.local_stds.reshape(h, w)])


def quadtree_gat_2d(image: np.ndarray, min_size: int = 4, alpha: float = 0.01, max_iterations: int = 50,
                    lts_fraction: float = 0.75, ctx=None) -> tuple:
    """QuadTree_.run (java/QuadTree_.java): (variance-stabilised image, g0, eDC, leaves)."""
    return utils.gat_quadtree_2d(image, min_size, alpha, max_iterations, lts_fraction, ctx=ctx)


def octree_gat_3d(volume: np.ndarray, min_size: int = 4, alpha: float = 0.01, max_iterations: int = 50,
                  lts_fraction: float = 0.75, ctx=None) -> tuple:
    """OcTree_.run (java/OcTree_.java): (variance-stabilised volume, g0, eDC, leaves)."""
    return utils.gat_octree_3d(volume, min_size, alpha, max_iterations, lts_fraction, ctx=ctx)


def roi_offset_and_sigma(image: np.ndarray, roi: tuple) -> tuple:
    """The ROI estimate of VarianceStabilisingTransform2D_ (meanAndStdDev,
    java/VarianceStabilisingTransform2D_.java:116-133): over the rectangle
    roi = (x, y, width, height), row by row, the one-pass FP64 mean and
    sqrt(sum(v^2)/n - mean^2), summed in raster order (NaN if rounding makes
    the variance negative, as Math.sqrt does)."""
    x, y, w, h = (int(v) for v in roi)
    v = np.asarray(image, np.float64)[y:y + h, x:x + w].ravel()
    if v.size == 0:
        return 0.0, 0.0
    s = float(np.cumsum(v)[-1])           # sequential, as the Java loop
    sq = float(np.cumsum(v * v)[-1])
    mean = s / v.size
    with np.errstate(invalid="ignore"):
        return mean, float(np.sqrt(np.float64(sq / v.size - mean * mean)))


def variance_stabilising_transform_2d(image: np.ndarray, gain: float = 1.0, offset: float = 10.0,
                                      sigma: float = 100.0, roi: tuple | None = None, max_iterations: int = 5000,
                                      ctx=None) -> tuple:
    """VarianceStabilisingTransform2D_.run (java/VarianceStabilisingTransform2D_.java:17-113): the
    GATMinimizer2D Simplex fit from the dialog's starting guesses (or with the offset and noise std
    estimated from a rectangular ROI), then getGAT with the fitted parameters. Returns
    (variance-stabilised image, gain, sigma, offset)."""
    a = np.ascontiguousarray(image, np.float32)
    if a.ndim != 2:
        raise ValueError("expected a 2D image")
    if roi is not None:
        offset, sigma = roi_offset_and_sigma(a, roi)
    g, s, o, _ = utils.fit_gat_2d(a, max_iterations, gain, sigma, offset, ctx=ctx)
    return utils.get_gat_2d(a, g, s, o, ctx=ctx), g, s, o


def variance_stabilising_transform_3d(volume: np.ndarray, gain: float = 1.0, offset: float = 10.0,
                                      sigma: float = 100.0, max_iterations: int = 5000, ctx=None) -> tuple:
    """VarianceStabilisingTransform3D_.run (java/VarianceStabilisingTransform3D_.java): the
    GATMinimizer3D Simplex fit from the dialog's starting guesses, then getGAT over every voxel.
    Returns (variance-stabilised volume, gain, sigma, offset)."""
    a = np.ascontiguousarray(volume, np.float32)
    if a.ndim != 3 or a.shape[0] < 2:
        raise ValueError("Image is not 3D. Please open a 3D image and try again.")
    g, s, o, _ = utils.fit_gat_3d(a, max_iterations, gain, sigma, offset, ctx=ctx)
    return utils.get_gat_3d(a, g, s, o, ctx=ctx), g, s, o
