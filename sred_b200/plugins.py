"""The ImageJ commands of the hot path as functions over arrays.

``global_repetition_2d`` follows GlobalRepetition2D_.run
(java/GlobalRepetition2D_.java:35-156) and ``block_repetition_2d`` follows
BlockRepetition2D_.run (java/BlockRepetition2D_.java:32-158), with the dialog
fields as keyword arguments (same defaults) and the windowing left out.
Noise-variance stabilisation (GAT) is not part of this path: pass an image
that is already stabilised, or leave ``stabilise_noise_variance`` False.
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
    if stabilise_noise_variance:
        raise NotImplementedError("variance stabilisation is outside the accelerated path")
    bs = utils.block_size(block_width, block_height)
    inp = utils.get_input_image_2d(image, True)
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
    if stabilise_noise_variance:
        raise NotImplementedError("variance stabilisation is outside the accelerated path")
    ref = utils.get_reference_block_2d(block)
    if ref is None:
        raise ValueError("Block dimensions must be odd (e.g., 3x3 or 5x5). Please try again.")
    frames = image if image.ndim == 3 else image[None]
    outs = []
    for f in frames:  # time-lapse: each frame normalised on its own (java/BlockRepetition2D_.java:104-130)
        inp = utils.get_input_image_2d(f, True)
        out = clutils.calculate_block_repetition_map_2d(metric, inp, ref, relevance_constant, normalize_output,
                                                        ctx=ctx)
        if out is None:
            return None
        outs.append(out.reshape(inp.height, inp.width))
    return np.stack(outs) if image.ndim == 3 else outs[0]
