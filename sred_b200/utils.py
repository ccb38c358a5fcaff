"""Host-side mirror of the reference's ``Utils`` (java/Utils.java).

Same names (snake_case), argument meaning and error behaviour: the data types
``InputImage2D``, ``ReferenceBlock2D``, ``RelevanceMask`` and their 3D
counterparts, and the host
numerics that run between the plugin commands and the maps. The numerics run
in libsred (``include/sred.h``); this module only marshals arrays.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

EPSILON = np.float32(1e-7)  # java/Utils.java:20


@dataclass
class InputImage2D:
    """java/Utils.java InputImage2D: a float32 image and its dimensions."""
    image_array: np.ndarray  # float32 [height * width] or [height, width]
    width: int
    height: int

    @property
    def size(self) -> int:
        return self.width * self.height

    def array2d(self) -> np.ndarray:
        return np.ascontiguousarray(self.image_array, np.float32).reshape(self.height, self.width)


@dataclass
class ReferenceBlock2D:
    """java/Utils.java:108-216 ReferenceBlock2D: ellipse pixels and their stats."""
    pixels: np.ndarray
    width: int
    height: int
    radius_width: int
    radius_height: int
    size: int
    mean: float
    std: float


@dataclass
class RelevanceMask:
    """java/Utils.java:35-96 RelevanceMask."""
    relevance_mask: np.ndarray
    relevance_constant: float
    relevance_threshold: float
    noise_mean_variance: float


def _ctx(ctx):
    return ctx if ctx is not None else _lib.default_context()


def get_gat_2d(image: np.ndarray, gain: float, sigma: float, offset: float, ctx=None) -> np.ndarray:
    """VarianceStabilisingTransform2D_.getGAT
    (java/VarianceStabilisingTransform2D_.java:136-151) on the GPU."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(image, dtype=np.float32).copy()
    h, w = a.shape
    c.check(c._L.sred_gat_2d(c.h, a, w, h, float(gain), float(sigma), float(offset)), "sred_gat_2d")
    return a


def gat_objective_2d(image: np.ndarray, gain: float, sigma: float, offset: float, ctx=None) -> float:
    """GATMinimizer2D.userFunction (java/GATMinimizer2D.java) on the GPU."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(image, dtype=np.float32)
    h, w = a.shape
    e = C.c_double()
    c.check(c._L.sred_gat_objective_2d(c.h, a, w, h, float(gain), float(sigma), float(offset), C.byref(e)),
            "sred_gat_objective_2d")
    return e.value


def fit_gat_2d(image: np.ndarray, max_iter: int = 5000, gain: float = 1.0, sigma: float = 10.0,
               offset: float = 100.0, ctx=None) -> tuple:
    """GATMinimizer2D.run: (gain, sigma, offset, objective) minimising the
    objective from the reference's starting point (java/Utils.java:676)."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(image, dtype=np.float32)
    h, w = a.shape
    g, s, o, e = C.c_double(gain), C.c_double(sigma), C.c_double(offset), C.c_double()
    c.check(c._L.sred_gat_fit_2d(c.h, a, w, h, int(max_iter), C.byref(g), C.byref(s), C.byref(o), C.byref(e)),
            "sred_gat_fit_2d")
    return g.value, s.value, o.value, e.value


def gat_quadtree_2d(image: np.ndarray, min_size: int = 4, alpha: float = 0.01, max_iter: int = 50,
                    lts_fraction: float = 0.75, ctx=None) -> tuple:
    """Quadtree variance stabilisation (java/QuadTree_.java) on the GPU:
    (transformed image, g0, eDC, leaves)."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(image, dtype=np.float32).copy()
    h, w = a.shape
    g0, edc, nl = C.c_double(), C.c_double(), C.c_int()
    c.check(c._L.sred_gat_quadtree_2d(c.h, a, w, h, int(min_size), float(alpha), int(max_iter), float(lts_fraction),
                                      C.byref(g0), C.byref(edc), C.byref(nl)), "sred_gat_quadtree_2d")
    return a, g0.value, edc.value, nl.value


def gat_octree_3d(volume: np.ndarray, min_size: int = 4, alpha: float = 0.01, max_iter: int = 50,
                  lts_fraction: float = 0.75, ctx=None) -> tuple:
    """Octree variance stabilisation (java/OcTree_.java) on the GPU:
    (transformed volume, g0, eDC, leaves)."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(volume, dtype=np.float32).copy()
    d, h, w = a.shape
    g0, edc, nl = C.c_double(), C.c_double(), C.c_int()
    c.check(c._L.sred_gat_octree_3d(c.h, a, w, h, d, int(min_size), float(alpha), int(max_iter), float(lts_fraction),
                                    C.byref(g0), C.byref(edc), C.byref(nl)), "sred_gat_octree_3d")
    return a, g0.value, edc.value, nl.value


def get_input_image_2d(image: np.ndarray, normalize_output: bool = True, stabilise_noise_variance: bool = False,
                       gat_method: str = "Simplex", max_iter: int = 5000, ctx=None) -> InputImage2D:
    """java/Utils.java:653-725 for an image given as an array: float
    conversion, optional variance stabilisation ("Simplex": the GAT
    parameters fitted on the GPU, then the transform; "Quad/Octree": the
    quadtree method with the reference's fixed parameters, java/Utils.java:686-705),
    and min-max to [0, 1] with epsilon, in FP32."""
    a = np.ascontiguousarray(image, dtype=np.float32)
    h, w = a.shape
    if stabilise_noise_variance:
        if gat_method == "Simplex":
            gain, sigma, offset, _ = fit_gat_2d(a, max_iter, ctx=ctx)
            a = get_gat_2d(a, np.float32(gain), np.float32(sigma), np.float32(offset), ctx=ctx)
        elif gat_method == "Quad/Octree":
            a = gat_quadtree_2d(a, 4, 0.01, 50, 0.75, ctx=ctx)[0]
        else:
            raise ValueError(f"unknown GAT method {gat_method!r}")
    if normalize_output:
        mn, mx = np.float32(a.min()), np.float32(a.max())
        a = ((a - mn) / (mx - mn + EPSILON)).astype(np.float32)
    return InputImage2D(a.ravel(), w, h)


def get_reference_block_2d(block: np.ndarray) -> ReferenceBlock2D:
    """java/Utils.java:557-639: ellipse-flatten, min-max, mean-subtract and std
    of a block image (odd dimensions; otherwise None, as the reference)."""
    b = np.ascontiguousarray(block, dtype=np.float32)
    bh, bw = b.shape
    if bw % 2 == 0 or bh % 2 == 0:
        return None
    L = _lib.load()
    px = np.zeros(bw * bh, np.float32)
    k, m, s = C.c_int(), C.c_float(), C.c_float()
    st = L.sred_reference_block_2d(b, bw, bh, px, C.byref(k), C.byref(m), C.byref(s))
    if st != _lib.OK:
        raise ValueError(_lib.status_string(st))
    return ReferenceBlock2D(px[:k.value].copy(), bw, bh, bw // 2, bh // 2, k.value, np.float32(m.value),
                            np.float32(s.value))


def get_mean_noise_var_2d(ref_pixels: np.ndarray, w: int, h: int, ctx=None) -> np.float32:
    """java/Utils.java:790-837."""
    c = _ctx(ctx)
    out = C.c_float()
    c.check(c._L.sred_mean_noise_var_2d(c.h, np.ascontiguousarray(ref_pixels, np.float32).ravel(), w, h,
                                        C.byref(out)), "sred_mean_noise_var_2d")
    return np.float32(out.value)


def get_relevance_mask(image_array: np.ndarray, image_width: int, image_height: int, block_radius_width: int,
                       block_radius_height: int, local_stds: np.ndarray, relevance_constant: float,
                       ctx=None) -> RelevanceMask:
    """java/Utils.java:944-968."""
    c = _ctx(ctx)
    n = image_width * image_height
    mask = np.zeros(n, np.float32)
    thr, nv = C.c_float(), C.c_float()
    c.check(c._L.sred_relevance_mask_2d(
        c.h, np.ascontiguousarray(image_array, np.float32).ravel(), image_width, image_height,
        2 * block_radius_width + 1, 2 * block_radius_height + 1,
        np.ascontiguousarray(local_stds, np.float32).ravel(), relevance_constant, mask, C.byref(thr),
        C.byref(nv)), "sred_relevance_mask_2d")
    return RelevanceMask(mask, np.float32(relevance_constant), np.float32(thr.value), np.float32(nv.value))


def apply_mask_2d(image_array: np.ndarray, image_width: int, image_height: int, mask: np.ndarray) -> np.ndarray:
    """java/Utils.java:919-930 (in place; returns the array)."""
    image_array *= np.asarray(mask, np.float32).reshape(image_array.shape)
    return image_array


def normalize_image_2d(image_array: np.ndarray, image_width: int, image_height: int, border_width: int,
                       border_height: int, mask: np.ndarray | None) -> np.ndarray:
    """java/Utils.java:985-1031. Raises ValueError for a non-binary mask, as the
    reference throws IllegalArgumentException."""
    a = np.ascontiguousarray(image_array, np.float32).ravel().copy()
    mp = None
    if mask is not None:
        mp = np.ascontiguousarray(mask, np.float32).ravel()
    st = _lib.load().sred_normalize_image_2d(a, image_width, image_height, border_width, border_height,
                                             None if mp is None else mp.ctypes.data)
    if st != _lib.OK:
        raise ValueError("Relevance mask must be binary (0.0f or 1.0f)")
    return a.reshape(np.shape(image_array))


def block_size(block_width: int, block_height: int) -> int:
    """Ellipse block size (java/GlobalRepetition2D_.java:102-111)."""
    return _lib.load().sred_block_size(block_width, block_height)


# ---------------------------------------------------------------------------
# Volumes (java/Utils.java:291-470, 1047-1660). A volume is float32 [depth,
# height, width], flattened as the reference's w*h*z + y*w + x.
# ---------------------------------------------------------------------------

@dataclass
class InputImage3D:
    """java/Utils.java:427-470 InputImage3D."""
    image_array: np.ndarray
    width: int
    height: int
    depth: int

    @property
    def size(self) -> int:
        return self.width * self.height * self.depth


@dataclass
class ReferenceBlock3D:
    """java/Utils.java:291-425 ReferenceBlock3D: ellipsoid voxels and their stats."""
    pixels: np.ndarray
    width: int
    height: int
    depth: int
    radius_width: int
    radius_height: int
    radius_depth: int
    size: int
    mean: float
    std: float


def get_gat_3d(volume: np.ndarray, gain: float, sigma: float, offset: float, ctx=None) -> np.ndarray:
    """getGAT over every voxel of a [depth, height, width] volume, on the GPU."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(volume, dtype=np.float32).copy()
    d, h, w = a.shape
    c.check(c._L.sred_gat_3d(c.h, a, w, h, d, float(gain), float(sigma), float(offset)), "sred_gat_3d")
    return a


def gat_objective_3d(volume: np.ndarray, gain: float, sigma: float, offset: float, ctx=None) -> float:
    """GATMinimizer3D.userFunction (java/GATMinimizer3D.java) on the GPU."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(volume, dtype=np.float32)
    d, h, w = a.shape
    e = C.c_double()
    c.check(c._L.sred_gat_objective_3d(c.h, a, w, h, d, float(gain), float(sigma), float(offset), C.byref(e)),
            "sred_gat_objective_3d")
    return e.value


def fit_gat_3d(volume: np.ndarray, max_iter: int = 5000, gain: float = 0.0, sigma: float = 100.0,
               offset: float = 0.0, ctx=None) -> tuple:
    """GATMinimizer3D.run from the 3D command's starting point (gain 0, sigma
    100, offset 0; java/Utils.java:1222): (gain, sigma, offset, objective)."""
    c = _ctx(ctx)
    a = np.ascontiguousarray(volume, dtype=np.float32)
    d, h, w = a.shape
    g, s, o, e = C.c_double(gain), C.c_double(sigma), C.c_double(offset), C.c_double()
    c.check(c._L.sred_gat_fit_3d(c.h, a, w, h, d, int(max_iter), C.byref(g), C.byref(s), C.byref(o), C.byref(e)),
            "sred_gat_fit_3d")
    return g.value, s.value, o.value, e.value


def get_input_image_3d(volume: np.ndarray, stabilise_noise_variance: bool = False,
                       normalize_output: bool = True, gat_method: str = "Simplex", max_iter: int = 5000,
                       ctx=None) -> InputImage3D:
    """java/Utils.java:1167-1277 for a volume given as an array: float
    conversion, optional variance stabilisation (Simplex: the GAT parameters
    fitted on the GPU, then the transform) and normalizeArray (min-max over the
    whole volume with epsilon, FP32). Neither of the reference's two versions
    returns the transformed volume: the image-ID version transforms copies it
    then drops (java/Utils.java:1216-1232), the array version normalises an
    array it never filled (java/Utils.java:1311-1327, a volume of zeros); here
    the volume is transformed, then normalised. "Quad/Octree": the octree
    method with the reference's fixed parameters (java/Utils.java:1235-1250),
    every voxel transformed."""
    a = np.ascontiguousarray(volume, dtype=np.float32)
    d, h, w = a.shape
    if stabilise_noise_variance:
        if gat_method == "Simplex":
            gain, sigma, offset, _ = fit_gat_3d(a, max_iter, ctx=ctx)
            a = get_gat_3d(a, gain, sigma, offset, ctx=ctx)
        elif gat_method == "Quad/Octree":
            a = gat_octree_3d(a, 4, 0.01, 50, 0.75, ctx=ctx)[0]
        else:
            raise ValueError(f"unknown GAT method {gat_method!r}")
    if normalize_output:
        mn, mx = np.float32(a.min()), np.float32(a.max())
        a = ((a - mn) / (mx - mn + EPSILON)).astype(np.float32)
    return InputImage3D(a.ravel(), w, h, d)


def block_size_3d(block_width: int, block_height: int, block_depth: int) -> int:
    """Ellipsoid block size (java/Utils.java:1075-1085)."""
    return _lib.load().sred_block_size_3d(block_width, block_height, block_depth)


def get_reference_block_3d(block: np.ndarray) -> ReferenceBlock3D:
    """java/Utils.java:1047-1160 for a block given as an array [bd, bh, bw].
    Raises ValueError for even dimensions or fewer than 3 slices, as the
    reference throws IllegalArgumentException."""
    b = np.ascontiguousarray(block, dtype=np.float32)
    bd, bh, bw = b.shape
    if bw % 2 == 0 or bh % 2 == 0 or bd % 2 == 0:
        raise ValueError("Block dimensions must be odd.")
    if bd < 3:
        raise ValueError("Reference block must have at least 3 slices.")
    px = np.zeros(b.size, np.float32)
    k, m, s = C.c_int(), C.c_float(), C.c_float()
    st = _lib.load().sred_reference_block_3d(b.ravel(), bw, bh, bd, px, C.byref(k), C.byref(m), C.byref(s))
    if st != _lib.OK:
        raise ValueError(_lib.status_string(st))
    return ReferenceBlock3D(px[:k.value].copy(), bw, bh, bd, bw // 2, bh // 2, bd // 2, k.value,
                            np.float32(m.value), np.float32(s.value))


def get_relevance_mask_3d(image_width: int, image_height: int, image_depth: int, block_radius_width: int,
                          block_radius_height: int, block_radius_depth: int, local_stds: np.ndarray,
                          relevance_constant: float, ctx=None) -> RelevanceMask:
    """java/Utils.java:1501-1525 (the reference returns the mask alone; here
    with its threshold and noise variance, as RelevanceMask)."""
    c = _ctx(ctx)
    mask = np.zeros(image_width * image_height * image_depth, np.float32)
    nv = C.c_float()
    c.check(c._L.sred_relevance_mask_3d(
        c.h, image_width, image_height, image_depth, 2 * block_radius_width + 1, 2 * block_radius_height + 1,
        2 * block_radius_depth + 1, np.ascontiguousarray(local_stds, np.float32).ravel(),
        float(relevance_constant), mask, C.byref(nv)), "sred_relevance_mask_3d")
    nvf = np.float32(nv.value)
    return RelevanceMask(mask, np.float32(relevance_constant), np.float32(nvf * np.float32(relevance_constant)), nvf)
