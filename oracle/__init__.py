"""CPU oracle for the SReD block-correlation path (numpy/ctypes front end).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker. The product
(``sred_b200``) never imports it.

Layers:
  * ``liboracle.so``  (``oracle/sred_oracle.c``): FP32 restatement of the
    reference kernels and Java host code (bit-exact target) and the FP64 judge.
  * ``_ref/librefshim.so``: the reference's own OpenCL kernels compiled as C++
    by ``oracle/refshim/build.py`` (present only where a reference checkout
    was available at build time; it travels with the built tree).
  * Pure-Python helpers below: the Java-side orchestration of
    ``java/GlobalRepetition2D_.java:97-145`` and
    ``java/CLUtils.java:486-981`` expressed over those primitives.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
EPSILON = np.float32(1e-7)

# Metric names exactly as the reference's dialogs spell them
# (java/GlobalRepetition2D_.java:20-25, java/BlockRepetition2D_.java:18-23).
GLOBAL_METRICS = {"Pearson's R": 0, "SSIM": 1, "NRMSE": 2, "Abs. diff. of StdDevs": 3}
BLOCK_METRICS = {"Pearson's R": 0, "SSIM": 1, "NRMSE (inverted)": 2, "Abs. Diff. of StdDevs.": 3}
COSINE = 4

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)

_lib = None
_ref = None


def _build() -> None:
    import importlib.util
    spec = importlib.util.spec_from_file_location("_oracle_build", HERE / "refshim" / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build_oracle()
    mod.build_refshim(mod.reference_root())


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        so = HERE / "liboracle.so"
        if not so.exists():
            _build()
        L = C.CDLL(str(so))
        L.orc_block_size.restype = C.c_int
        L.orc_local_stats_f32.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p]
        L.orc_mean_noise_var.argtypes = [_f32p, C.c_int, C.c_int, _fp]
        L.orc_relevance_mask.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, C.c_float,
                                         _f32p, _fp, _fp]
        L.orc_normalize_image.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]
        L.orc_n_pixels.restype = C.c_float
        L.orc_n_pixels.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_global_f32.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, _f32p,
                                     C.c_float, C.c_float, _i32p, C.c_int, _f32p, _f32p]
        L.orc_global_f64.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p,
                                     C.c_float, C.c_float, _i32p, C.c_int, _f64p, _f64p]
        L.orc_global_finalize_f32.argtypes = [C.c_int, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                              _f32p, C.c_float, C.c_float, C.c_int, _f32p]
        L.orc_global_finalize_f64.argtypes = [C.c_int, _f64p, _f64p, C.c_int, C.c_int, C.c_int, C.c_int,
                                              _f32p, C.c_float, C.c_double, C.c_int, _f64p]
        L.orc_reference_block.argtypes = [_f32p, C.c_int, C.c_int, _f32p, _fp, _fp]
        L.orc_block_kernel_f32.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p,
                                           _f32p, _f32p, C.c_int, C.c_float, C.c_float, _f32p]
        L.orc_block_postprocess_f32.argtypes = [C.c_int, _f32p, _f32p, C.c_int, C.c_int, C.c_int,
                                                C.c_int, _f32p, C.c_float, C.c_int]
        L.orc_block_kernel_f64.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p,
                                           _f32p, C.c_int, C.c_float, C.c_float, _f64p]
        L.orc_java_random_floats.argtypes = [C.c_int64, C.c_int, _f32p]
        L.orc_gat.argtypes = [_f32p, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_block_size3d.restype = C.c_int
        L.orc_block_size3d.argtypes = [C.c_int, C.c_int, C.c_int]
        L.orc_local_stats3d_f32.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p,
                                            _f32p]
        L.orc_reference_block3d.restype = C.c_int
        L.orc_reference_block3d.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _f32p, _fp, _fp]
        L.orc_block3d_kernel_f32.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             _f32p, _f32p, _f32p, C.c_int, C.c_float, C.c_float, _f32p]
        L.orc_noise_var3d.restype = C.c_float
        L.orc_noise_var3d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_relevance_mask3d.restype = C.c_float
        L.orc_relevance_mask3d.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p, C.c_float,
                                           _f32p]
        L.orc_block3d_postprocess_f32.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                                  C.c_int, _f32p, C.c_float, C.c_int]
        i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        L.orc_global3d_f32.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       _f32p, _f32p, C.c_float, C.c_float, i32, C.c_int, _f32p, _f32p]
        L.orc_global3d_f64.argtypes = [C.c_int, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       _f32p, C.c_float, C.c_float, i32, C.c_int, _f64p, _f64p]
        L.orc_n_pixels3d.restype = C.c_float
        L.orc_n_pixels3d.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_global3d_finalize_f32.argtypes = [C.c_int, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.c_int, C.c_int, _f32p, C.c_float, C.c_float, C.c_int, _f32p]
        L.orc_global3d_finalize_f64.argtypes = [C.c_int, _f64p, _f64p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.c_int, C.c_int, _f32p, C.c_float, C.c_double, C.c_int, _f64p]
        L.orc_local_var2d.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_tool_noise_var.restype = C.c_int
        L.orc_tool_noise_var.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, _fp]
        L.orc_tool_mask.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _f32p]
        L.orc_tool_range.restype = C.c_int
        L.orc_tool_range.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int,
                                     _fp, _fp]
        L.orc_gat_objective3d.restype = C.c_double
        L.orc_gat_objective3d.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_classify_redundancy.restype = C.c_int
        L.orc_classify_redundancy.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                              C.c_int64, _f32p, C.POINTER(C.c_double)]
        L.orc_java_random_next.argtypes = [C.c_int64, C.c_int, C.c_int, np.ctypeslib.ndpointer(np.int32)]
        L.orc_java_random_doubles.argtypes = [C.c_int64, C.c_int, _f64p]
        L.orc_f_quantile.restype = C.c_double
        L.orc_f_quantile.argtypes = [C.c_double, C.c_double]
        L.orc_gat_tree.restype = C.c_int
        L.orc_gat_tree.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int,
                                   C.c_float, _dp, _dp, np.ctypeslib.ndpointer(np.int32), _f32p, _f32p, C.c_int]
        L.orc_gat_objective.restype = C.c_double
        L.orc_gat_objective.argtypes = [_f32p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double]
        L.orc_patch_hu1_ref.restype = C.c_double
        L.orc_patch_hu1_ref.argtypes = [_f32p, C.c_int, C.c_int]
        L.orc_patch_hu.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f32p]
        L.orc_hu_prepare_patch.argtypes = [_f32p, C.c_int, C.c_int, _f32p]
        L.orc_hu_feature.restype = C.c_float
        L.orc_hu_feature.argtypes = [_f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_hu_map.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f64p]
        L.orc_phase_map.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _f64p]
        L.orc_block_hu7.argtypes = [_f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p,
                                    np.ctypeslib.ndpointer(np.float64, flags="C"),
                                    np.ctypeslib.ndpointer(np.float64, flags="C")]
        L.orc_block_phase.argtypes = [_f32p, _f32p, _f32p, C.c_int, C.c_int, C.c_int, C.c_int, _f32p,
                                      C.c_float, _f64p]
        _lib = L
    return _lib


def refshim() -> C.CDLL | None:
    """The reference's own kernels compiled for the CPU, or None if not built here."""
    global _ref
    if _ref is None:
        so = HERE / "_ref" / "librefshim.so"
        if not so.exists():
            return None
        _ref = C.CDLL(str(so))
    return _ref


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


# --------------------------------------------------------------------------
# Host numerics (java/Utils.java)
# --------------------------------------------------------------------------

def block_size(bw: int, bh: int) -> int:
    """Ellipse block size K (java/GlobalRepetition2D_.java:102-111)."""
    return lib().orc_block_size(bw, bh)


def normalize_input(img: np.ndarray) -> np.ndarray:
    """Min-max to [0,1] with epsilon (java/Utils.java:707-722)."""
    a = _f32(img).copy()
    lib().orc_normalize_input(a.ctypes.data_as(_fp), C.c_int(a.size))
    return a


def local_stats(img: np.ndarray, bw: int, bh: int):
    """(means, stds) per pixel, FP32 reference order (cl/kernelGetLocalStatistics2D.cl)."""
    img = _f32(img)
    H, W = img.shape
    m = np.zeros_like(img)
    s = np.zeros_like(img)
    lib().orc_local_stats_f32(img, W, H, bw, bh, m, s)
    return m, s


def mean_noise_var(img: np.ndarray) -> float:
    img = _f32(img)
    H, W = img.shape
    out = C.c_float()
    if lib().orc_mean_noise_var(img, W, H, C.byref(out)) != 0:
        raise IndexError("image smaller than one noise tile")
    return np.float32(out.value)


def relevance_mask(img: np.ndarray, bw: int, bh: int, stds: np.ndarray, c: float):
    """(mask, threshold, noise_var) as java/Utils.java:944-968."""
    img = _f32(img)
    H, W = img.shape
    mask = np.zeros_like(img)
    thr, nv = C.c_float(), C.c_float()
    if lib().orc_relevance_mask(img, W, H, bw // 2, bh // 2, _f32(stds), C.c_float(c), mask,
                                C.byref(thr), C.byref(nv)) != 0:
        raise IndexError("image smaller than one noise tile")
    return mask, np.float32(thr.value), np.float32(nv.value)


def normalize_image(a: np.ndarray, rw: int, rh: int, mask: np.ndarray | None) -> np.ndarray:
    a = _f32(a).copy()
    H, W = a.shape
    mp = None if mask is None else _f32(mask)
    rc = lib().orc_normalize_image(a, W, H, rw, rh, None if mp is None else mp.ctypes.data)
    if rc != 0:
        raise ValueError("Relevance mask must be binary (0.0f or 1.0f)")
    return a


def n_pixels(mask: np.ndarray, rw: int, rh: int) -> np.float32:
    H, W = mask.shape
    return np.float32(lib().orc_n_pixels(_f32(mask), W, H, rw, rh))


def reference_block(block_img: np.ndarray):
    """(pixels[K], mean, std) as java/Utils.java:557-639."""
    b = _f32(block_img)
    bh, bw = b.shape
    px = np.zeros(bw * bh, np.float32)
    m, s = C.c_float(), C.c_float()
    K = lib().orc_reference_block(b, bw, bh, px, C.byref(m), C.byref(s))
    return px[:K].copy(), np.float32(m.value), np.float32(s.value)


def java_random_floats(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    lib().orc_java_random_floats(seed, n, out)
    return out


# --------------------------------------------------------------------------
# Global repetition map
# --------------------------------------------------------------------------

def _pix(W, H, rw, rh, pix):
    if pix is None:
        ys, xs = np.mgrid[rh:H - rh, rw:W - rw]
        pix = (ys * W + xs).ravel()
    return np.ascontiguousarray(pix, dtype=np.int32)


def global_sums_f32(metric: str, img, bw, bh, means, stds, filter_param, threshold, pix=None,
                    use_refshim: bool = False):
    """(num, den) per listed reference pixel, FP32 reference semantics.

    With ``use_refshim`` the reference's own kernel (compiled for the CPU) runs
    instead of the restatement."""
    img = _f32(img)
    H, W = img.shape
    pix = _pix(W, H, bw // 2, bh // 2, pix)
    m = GLOBAL_METRICS[metric]
    if use_refshim:
        R = refshim()
        if R is None:
            raise RuntimeError("refshim not built (no reference checkout at build time)")
        K = block_size(bw, bh)
        num = np.zeros(W * H, np.float32)
        den = np.zeros(W * H, np.float32)
        name = ["kernelGetGlobalPearson2D", "kernelGetGlobalSsim2D", "kernelGetGlobalNrmse2D",
                "kernelGetGlobalAbsDiffStds2D"][m]
        fn = getattr(R, f"rs_{name}")
        args = [C.c_int(K), C.c_int(W), C.c_int(H), C.c_int(bw), C.c_int(bh), C.c_float(filter_param),
                C.c_float(threshold), C.c_float(EPSILON), C.c_float(0), C.c_float(0),
                pix.ctypes.data_as(C.c_void_p), C.c_int(pix.size), img.ctypes.data_as(C.c_void_p)]
        if m != 3:
            args.append(_f32(means).ctypes.data_as(C.c_void_p))
        args += [_f32(stds).ctypes.data_as(C.c_void_p), den.ctypes.data_as(C.c_void_p),
                 num.ctypes.data_as(C.c_void_p)]
        if fn(*args) != 0:
            raise ValueError(f"refshim has no instantiation for K={K}")
        return num[pix], den[pix]
    num = np.zeros(pix.size, np.float32)
    den = np.zeros(pix.size, np.float32)
    lib().orc_global_f32(m, img, W, H, bw, bh, _f32(means), _f32(stds), C.c_float(filter_param),
                         C.c_float(threshold), pix, pix.size, num, den)
    return num, den


def global_sums_f64(metric: str, img, bw, bh, stds, filter_param, threshold, pix=None):
    """(num, den) per listed reference pixel, FP64 judge."""
    img = _f32(img)
    H, W = img.shape
    pix = _pix(W, H, bw // 2, bh // 2, pix)
    num = np.zeros(pix.size, np.float64)
    den = np.zeros(pix.size, np.float64)
    lib().orc_global_f64(GLOBAL_METRICS[metric], img, W, H, bw, bh, _f32(stds),
                         C.c_float(filter_param), C.c_float(threshold), pix, pix.size, num, den)
    return num, den


def global_map(metric: str, img, bw: int, bh: int, relevance_constant: float, normalize=True,
               precision: str = "f32", use_refshim: bool = False):
    """Full global repetition map as GlobalRepetition2D_ computes it after
    preprocessing (java/GlobalRepetition2D_.java:97-145, java/CLUtils.java:2174).

    Returns a dict with the map and every intermediate."""
    img = _f32(img)
    H, W = img.shape
    rw, rh = bw // 2, bh // 2
    means, stds = local_stats(img, bw, bh)
    mask, thr, nv = relevance_mask(img, bw, bh, stds, relevance_constant)
    npx = n_pixels(mask, rw, rh)
    pix = _pix(W, H, rw, rh, None)
    m = GLOBAL_METRICS[metric]
    if precision == "f32":
        num, den = global_sums_f32(metric, img, bw, bh, means, stds, nv, thr, pix, use_refshim)
        nf = np.zeros(W * H, np.float32); df = np.zeros(W * H, np.float32)
        nf[pix] = num; df[pix] = den
        out = np.zeros(W * H, np.float32)
        rc = lib().orc_global_finalize_f32(m, nf, df, W, H, rw, rh, mask.ravel().copy(),
                                           C.c_float(relevance_constant), C.c_float(npx),
                                           int(normalize), out)
        if rc != 0:
            raise ValueError("non-binary mask")
    else:
        num, den = global_sums_f64(metric, img, bw, bh, stds, nv, thr, pix)
        nf = np.zeros(W * H, np.float64); df = np.zeros(W * H, np.float64)
        nf[pix] = num; df[pix] = den
        out = np.zeros(W * H, np.float64)
        lib().orc_global_finalize_f64(m, nf, df, W, H, rw, rh, mask.ravel().copy(),
                                      C.c_float(relevance_constant), C.c_double(float(npx)),
                                      int(normalize), out)
    return {"map": out.reshape(H, W), "num": nf.reshape(H, W), "den": df.reshape(H, W),
            "means": means, "stds": stds, "mask": mask, "threshold": thr, "noise_var": nv,
            "n_pixels": npx}


# --------------------------------------------------------------------------
# Block (local) repetition map
# --------------------------------------------------------------------------

def block_map(metric: str, img, ref_pixels, bw: int, bh: int, ref_mean: float, ref_std: float,
              relevance_constant: float = 0.0, normalize: bool = True, use_refshim: bool = False):
    """Block repetition map as java/CLUtils.java:995-1010 computes it, FP32."""
    img = _f32(img)
    H, W = img.shape
    means, stds = local_stats(img, bw, bh)
    ref = _f32(ref_pixels)
    K = ref.size
    m = BLOCK_METRICS[metric]
    out = np.zeros(W * H, np.float32)
    if use_refshim:
        R = refshim()
        if R is None:
            raise RuntimeError("refshim not built")
        name = ["kernelGetBlockPearson2D", "kernelGetBlockSsim2D", "kernelGetBlockNrmse2D",
                "kernelGetBlockAbsDiffStds2D"][m]
        pix = np.arange(W * H, dtype=np.int32)
        bufs = {"ref": ref, "img": img, "means": means, "stds": stds, "map": out}
        args = [C.c_int(K), C.c_int(W), C.c_int(H), C.c_int(bw), C.c_int(bh), C.c_float(0),
                C.c_float(0), C.c_float(EPSILON), C.c_float(ref_std), C.c_float(ref_mean),
                pix.ctypes.data_as(C.c_void_p), C.c_int(pix.size)]
        kind_args = {0: ["ref", "img", "means", "stds", "map"], 1: ["ref", "img", "means", "stds", "map"],
                     2: ["ref", "img", "means", "map"], 3: ["stds", "map"]}[m]
        args += [bufs[a].ctypes.data_as(C.c_void_p) for a in kind_args]
        if getattr(R, f"rs_{name}")(*args) != 0:
            raise ValueError(f"refshim has no instantiation for K={K}")
    else:
        lib().orc_block_kernel_f32(m, img, W, H, bw, bh, means, stds, ref, K, C.c_float(ref_mean),
                                   C.c_float(ref_std), out)
    raw = out.copy()
    rc = lib().orc_block_postprocess_f32(m, out, img, W, H, bw // 2, bh // 2, stds,
                                         C.c_float(relevance_constant), int(normalize))
    if rc != 0:
        raise IndexError("image smaller than one noise tile")
    return {"map": out.reshape(H, W), "raw": raw.reshape(H, W), "means": means, "stds": stds}


def block_raw_f64(metric: int, img, ref_pixels, bw, bh, ref_mean, ref_std, stds32):
    """FP64 judge of the block-map kernel output (before host post-processing).
    ``metric`` is 0..3 as BLOCK_METRICS, or COSINE."""
    img = _f32(img)
    H, W = img.shape
    out = np.zeros(W * H, np.float64)
    ref = _f32(ref_pixels)
    lib().orc_block_kernel_f64(metric, img, W, H, bw, bh, _f32(stds32), ref, ref.size,
                               C.c_float(ref_mean), C.c_float(ref_std), out)
    return out.reshape(H, W)


# --------------------------------------------------------------------------
# Shape metrics: the reference's Hu and phase-correlation kernels
# (cl/kernelGetPatchHu2D.cl, cl/kernelGetHuMap.cl,
# cl/kernelGetPhaseCorrelationMap.cl; shipped, never loaded by its Java code)
# --------------------------------------------------------------------------

def _shape_refshim(name, W, H, bw, bh, patch_size, bufs):
    R = refshim()
    if R is None:
        raise RuntimeError("refshim not built")
    pix = np.arange(W * H, dtype=np.int32)
    fn = getattr(R, f"rs_{name}")
    args = [C.c_int(W), C.c_int(H), C.c_int(bw), C.c_int(bh), C.c_int(patch_size), C.c_float(EPSILON),
            pix.ctypes.data_as(C.c_void_p), C.c_int(pix.size)]
    args += [None if b is None else b.ctypes.data_as(C.c_void_p) for b in bufs]
    if fn(*args) != 0:
        raise ValueError(f"refshim has no {name} instantiation for {bw}x{bh}")


def patch_hu_map(patch, img, bw, bh, patch_size=None, use_refshim=False):
    """cl/kernelGetPatchHu2D.cl over every pixel: interior pixels get
    sqrt(hu1(patch) * hu1(comparison patch)); border pixels stay 0.
    ``patch`` is the bw x bh grid the kernel reads (at the ellipse positions)."""
    img = _f32(img)
    H, W = img.shape
    patch = _f32(patch).ravel()
    ps = block_size(bw, bh) if patch_size is None else patch_size
    out = np.zeros(W * H, np.float32)
    if use_refshim:
        _shape_refshim("kernelGetPatchHu2D", W, H, bw, bh, ps, [patch, img, np.zeros_like(img), out])
    else:
        lib().orc_patch_hu(patch, img, W, H, bw, bh, ps, out)
    return out.reshape(H, W)


def patch_hu1(patch, bw, bh) -> float:
    return float(lib().orc_patch_hu1_ref(_f32(patch).ravel(), bw, bh))


def hu_prepare_patch(ref_pixels, bw, bh) -> np.ndarray:
    """bw x bh reference patch of the block-map Hu metric (see orc_hu_prepare_patch)."""
    g = np.zeros(bw * bh, np.float32)
    lib().orc_hu_prepare_patch(_f32(ref_pixels), bw, bh, g)
    return g.reshape(bh, bw)


def hu_map(img, bw, bh, means=None, stds=None, precision="f32", use_refshim=False):
    """cl/kernelGetHuMap.cl over every interior pixel (raw sums)."""
    img = _f32(img)
    H, W = img.shape
    if means is None:
        means, stds = local_stats(img, bw, bh)
    if use_refshim:
        out = np.zeros(W * H, np.float32)
        _shape_refshim("kernelGetHuMap", W, H, bw, bh, bw * bh, [img, _f32(means), _f32(stds), None, out])
        return out.reshape(H, W).astype(np.float64)
    out = np.zeros(W * H, np.float64)
    lib().orc_hu_map(img, _f32(means), _f32(stds), W, H, bw, bh, int(precision == "f64"), out)
    return out.reshape(H, W)


def phase_map(img, bw, bh, means=None, stds=None, precision="f32", use_refshim=False):
    """cl/kernelGetPhaseCorrelationMap.cl (three repairs, see orc_phase_map)
    over every interior pixel (raw sums)."""
    img = _f32(img)
    H, W = img.shape
    if means is None:
        means, stds = local_stats(img, bw, bh)
    if use_refshim:
        out = np.zeros(W * H, np.float32)
        _shape_refshim("kernelGetPhaseCorrelationMap", W, H, bw, bh, bw * bh,
                       [img, _f32(means), _f32(stds), None, out])
        return out.reshape(H, W).astype(np.float64)
    out = np.zeros(W * H, np.float64)
    if lib().orc_phase_map(img, _f32(means), _f32(stds), W, H, bw, bh, int(precision == "f64"), out):
        raise ValueError("phase correlation supports blocks up to 15x15")
    return out.reshape(H, W)


def block_phase_raw(img, ref_pixels, bw, bh, ref_std, means=None, stds=None):
    """Block-map phase correlation before post-processing (FP64)."""
    img = _f32(img)
    H, W = img.shape
    if means is None:
        means, stds = local_stats(img, bw, bh)
    out = np.zeros(W * H, np.float64)
    if lib().orc_block_phase(img, _f32(means), _f32(stds), W, H, bw, bh, _f32(ref_pixels),
                             C.c_float(ref_std), out):
        raise ValueError("phase correlation supports blocks up to 15x15")
    return out.reshape(H, W)


def block_hu7_raw(img, ref_pixels, bw, bh):
    """Block-map Hu distance before post-processing (FP64): the L2 distance of
    each block's seven Hu invariants to the reference block's; returns (map,
    reference 7-vector)."""
    img = _f32(img)
    H, W = img.shape
    out = np.zeros(W * H, np.float64)
    ref_h = np.zeros(7, np.float64)
    lib().orc_block_hu7(img, W, H, bw, bh, _f32(ref_pixels), ref_h, out)
    return out.reshape(H, W), ref_h


# --------------------------------------------------------------------------
# Variance stabilisation (java/VarianceStabilisingTransform2D_.java,
# java/GATMinimizer2D.java)
# --------------------------------------------------------------------------

def gat(img, gain, sigma, offset) -> np.ndarray:
    a = _f32(img).copy()
    lib().orc_gat(a.ravel(), a.size, float(gain), float(sigma), float(offset))
    return a


def gat_objective(img, gain, sigma, offset) -> float:
    a = _f32(img)
    H, W = a.shape
    return float(lib().orc_gat_objective(a.ravel(), W, H, float(gain), float(sigma), float(offset)))


# --------------------------------------------------------------------------
# 3D block repetition maps (cl/kernelGet*3D.cl, java/CLUtils.java:1030-1653)
# Volumes are float32 [D, H, W].
# --------------------------------------------------------------------------

BLOCK_METRICS_3D = {"Pearson's R": 0, "SSIM": 1, "NRMSE (inverted)": 2, "Abs. Diff. of StdDevs.": 3}


def block_size3d(bw, bh, bd) -> int:
    return lib().orc_block_size3d(bw, bh, bd)


def local_stats3d(vol, bw, bh, bd, use_refshim=False):
    v = _f32(vol)
    D, H, W = v.shape
    m = np.zeros_like(v)
    s = np.zeros_like(v)
    if use_refshim:
        R = refshim()
        pix = np.arange(v.size, dtype=np.int32)
        rc = R.rs_kernelGetLocalStatistics3D(C.c_int(block_size3d(bw, bh, bd)), W, H, D, bw, bh, bd,
                                             C.c_float(EPSILON), C.c_float(0), C.c_float(0),
                                             pix.ctypes.data_as(C.c_void_p), C.c_int(pix.size),
                                             v.ctypes.data_as(C.c_void_p), m.ctypes.data_as(C.c_void_p),
                                             s.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise ValueError("refshim has no instantiation for this block")
    else:
        lib().orc_local_stats3d_f32(v.ravel(), W, H, D, bw, bh, bd, m.ravel(), s.ravel())
    return m, s


def reference_block3d(block):
    b = _f32(block)
    bd, bh, bw = b.shape
    px = np.zeros(b.size, np.float32)
    m, s = C.c_float(), C.c_float()
    K = lib().orc_reference_block3d(b.ravel(), bw, bh, bd, px, C.byref(m), C.byref(s))
    return px[:K].copy(), np.float32(m.value), np.float32(s.value)


def block_map3d(metric, vol, ref_pixels, bw, bh, bd, ref_mean, ref_std, relevance_constant=0.0, normalize=True,
                use_refshim=False):
    """3D block map: the kernel (reference FP32 order) and the host steps."""
    v = _f32(vol)
    D, H, W = v.shape
    means, stds = local_stats3d(v, bw, bh, bd, use_refshim)
    ref = _f32(ref_pixels)
    K = ref.size
    m = BLOCK_METRICS_3D[metric]
    out = np.zeros(v.size, np.float32)
    if use_refshim:
        name = ["kernelGetBlockPearson3D", "kernelGetBlockSsim3D", "kernelGetBlockNrmse3D",
                "kernelGetBlockAbsDiffStds3D"][m]
        bufs = {"ref": ref, "img": v, "means": means, "stds": stds, "map": out}
        args = {0: ["ref", "img", "means", "stds", "map"], 1: ["ref", "img", "means", "stds", "map"],
                2: ["ref", "img", "means", "map"], 3: ["stds", "map"]}[m]
        pix = np.arange(v.size, dtype=np.int32)
        rc = getattr(refshim(), f"rs_{name}")(C.c_int(K), W, H, D, bw, bh, bd, C.c_float(EPSILON),
                                              C.c_float(ref_std), C.c_float(ref_mean),
                                              pix.ctypes.data_as(C.c_void_p), C.c_int(pix.size),
                                              *[bufs[a].ctypes.data_as(C.c_void_p) for a in args])
        if rc != 0:
            raise ValueError("refshim has no instantiation for this block")
    else:
        lib().orc_block3d_kernel_f32(m, v.ravel(), W, H, D, bw, bh, bd, means.ravel(), stds.ravel(), ref, K,
                                     C.c_float(ref_mean), C.c_float(ref_std), out)
    raw = out.copy()
    lib().orc_block3d_postprocess_f32(m, out, W, H, D, bw // 2, bh // 2, bd // 2, stds.ravel(),
                                      C.c_float(relevance_constant), int(normalize))
    return {"map": out.reshape(D, H, W), "raw": raw.reshape(D, H, W), "means": means, "stds": stds}


def relevance_mask3d(stds, bw, bh, bd, c):
    s = _f32(stds)
    D, H, W = s.shape
    mask = np.zeros(s.size, np.float32)
    nv = lib().orc_relevance_mask3d(W, H, D, bw // 2, bh // 2, bd // 2, s.ravel(), C.c_float(c), mask)
    return mask.reshape(D, H, W), np.float32(nv)


# --------------------------------------------------------------------------
# 3D global repetition maps (cl/kernelGetGlobal*3D.cl, java/CLUtils.java:2225-2816,
# java/GlobalRepetition3D_.java:97-158), with the relevance mask of the 3D
# block command (getRelevanceMask3D) in place of the 2D mask the 3D global
# command passes (java/GlobalRepetition3D_.java:126-128, which makes the
# command fail on its first interior slice).
# --------------------------------------------------------------------------

def _pix3(W, H, D, rw, rh, rd):
    zs, ys, xs = np.mgrid[rd:D - rd, rh:H - rh, rw:W - rw]
    return np.ascontiguousarray((zs * (W * H) + ys * W + xs).ravel(), dtype=np.int32)


def global3d_sums_f32(metric, vol, bw, bh, bd, means, stds, filter_param, threshold, pix=None,
                      use_refshim=False):
    """(num, den) per listed reference voxel, FP32 reference semantics."""
    v = _f32(vol)
    D, H, W = v.shape
    pix = _pix3(W, H, D, bw // 2, bh // 2, bd // 2) if pix is None else np.ascontiguousarray(pix, np.int32)
    m = GLOBAL_METRICS[metric]
    if use_refshim:
        R = refshim()
        if R is None:
            raise RuntimeError("refshim not built (no reference checkout at build time)")
        K = block_size3d(bw, bh, bd)
        num = np.zeros(v.size, np.float32)
        den = np.zeros(v.size, np.float32)
        name = ["kernelGetGlobalPearson3D", "kernelGetGlobalSsim3D", "kernelGetGlobalNrmse3D",
                "kernelGetGlobalAbsDiffStds3D"][m]
        args = [C.c_int(K), W, H, D, bw, bh, bd, C.c_float(filter_param), C.c_float(threshold),
                C.c_float(EPSILON), pix.ctypes.data_as(C.c_void_p), C.c_int(pix.size),
                v.ctypes.data_as(C.c_void_p)]
        if m != 3:
            args.append(_f32(means).ctypes.data_as(C.c_void_p))
        args += [_f32(stds).ctypes.data_as(C.c_void_p), den.ctypes.data_as(C.c_void_p),
                 num.ctypes.data_as(C.c_void_p)]
        if getattr(R, f"rs_{name}")(*args) != 0:
            raise ValueError(f"refshim has no instantiation for K={K}")
        return num[pix], den[pix]
    num = np.zeros(pix.size, np.float32)
    den = np.zeros(pix.size, np.float32)
    lib().orc_global3d_f32(m, v.ravel(), W, H, D, bw, bh, bd, _f32(means).ravel(), _f32(stds).ravel(),
                           C.c_float(filter_param), C.c_float(threshold), pix, pix.size, num, den)
    return num, den


def global3d_sums_f64(metric, vol, bw, bh, bd, stds, filter_param, threshold, pix=None):
    """(num, den) per listed reference voxel, FP64 judge."""
    v = _f32(vol)
    D, H, W = v.shape
    pix = _pix3(W, H, D, bw // 2, bh // 2, bd // 2) if pix is None else np.ascontiguousarray(pix, np.int32)
    num = np.zeros(pix.size, np.float64)
    den = np.zeros(pix.size, np.float64)
    lib().orc_global3d_f64(GLOBAL_METRICS[metric], v.ravel(), W, H, D, bw, bh, bd, _f32(stds).ravel(),
                           C.c_float(filter_param), C.c_float(threshold), pix, pix.size, num, den)
    return num, den


def global_map3d(metric, vol, bw, bh, bd, relevance_constant, normalize=True, precision="f32",
                 use_refshim=False):
    """Full 3D global repetition map; a dict with the map and every intermediate."""
    v = _f32(vol)
    D, H, W = v.shape
    rw, rh, rd = bw // 2, bh // 2, bd // 2
    means, stds = local_stats3d(v, bw, bh, bd, use_refshim)
    mask, nv = relevance_mask3d(stds, bw, bh, bd, relevance_constant)
    thr = np.float32(nv * np.float32(relevance_constant))
    npx = np.float32(lib().orc_n_pixels3d(mask.ravel(), W, H, D, rw, rh, rd))
    pix = _pix3(W, H, D, rw, rh, rd)
    m = GLOBAL_METRICS[metric]
    if precision == "f32":
        num, den = global3d_sums_f32(metric, v, bw, bh, bd, means, stds, nv, thr, pix, use_refshim)
        nf = np.zeros(v.size, np.float32)
        df = np.zeros(v.size, np.float32)
        nf[pix] = num
        df[pix] = den
        out = np.zeros(v.size, np.float32)
        lib().orc_global3d_finalize_f32(m, nf, df, W, H, D, rw, rh, rd, mask.ravel().copy(),
                                        C.c_float(relevance_constant), C.c_float(npx), int(normalize), out)
    else:
        num, den = global3d_sums_f64(metric, v, bw, bh, bd, stds, nv, thr, pix)
        nf = np.zeros(v.size, np.float64)
        df = np.zeros(v.size, np.float64)
        nf[pix] = num
        df[pix] = den
        out = np.zeros(v.size, np.float64)
        lib().orc_global3d_finalize_f64(m, nf, df, W, H, D, rw, rh, rd, mask.ravel().copy(),
                                        C.c_float(relevance_constant), C.c_double(float(npx)), int(normalize), out)
    sh = (D, H, W)
    return {"map": out.reshape(sh), "num": nf.reshape(sh), "den": df.reshape(sh), "means": means,
            "stds": stds, "mask": mask, "threshold": thr, "noise_var": nv, "n_pixels": npx}


# --------------------------------------------------------------------------
# Relevance-mask tools (java/RelevanceMask2D_.java, RelevanceMaskStack2D_.java,
# OptimiseRelevanceMask_.java)
# --------------------------------------------------------------------------

def local_var2d(img, bw, bh, take_sqrt, use_refshim=False):
    """cl/kernelGetRelevanceMask2D.cl (variance) or cl/kernelGetLocalMeans.cl (std)."""
    a = _f32(img)
    H, W = a.shape
    out = np.zeros(W * H, np.float32)
    if use_refshim:
        R = refshim()
        K = block_size(bw, bh)
        ys, xs = np.mgrid[bh // 2:H - bh // 2, bw // 2:W - bw // 2]
        pix = np.ascontiguousarray((ys * W + xs).ravel(), np.int32)
        if take_sqrt:
            means = np.zeros(W * H, np.float32)
            rc = R.rs_kernelGetLocalMeans(C.c_int(K), W, H, bw, bh, C.c_float(0), C.c_float(0), C.c_float(EPSILON),
                                          C.c_float(0), C.c_float(0), pix.ctypes.data_as(C.c_void_p),
                                          C.c_int(pix.size), a.ctypes.data_as(C.c_void_p),
                                          means.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
        else:
            rc = R.rs_kernelGetRelevanceMask2D(C.c_int(K), W, H, bw, bh, C.c_float(0), C.c_float(0),
                                               C.c_float(EPSILON), C.c_float(0), C.c_float(0),
                                               pix.ctypes.data_as(C.c_void_p), C.c_int(pix.size),
                                               a.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise ValueError(f"refshim has no instantiation for K={K}")
    else:
        lib().orc_local_var2d(a.ravel(), W, H, bw, bh, int(take_sqrt), out)
    return out.reshape(H, W)


def tool_noise_var(img, fp64):
    a = _f32(img)
    H, W = a.shape
    v = C.c_float()
    if lib().orc_tool_noise_var(a.ravel(), W, H, int(fp64), C.byref(v)) != 0:
        raise ValueError("image smaller than one noise-variance tile")
    return np.float32(v.value)


def tool_mask(stat, bw, bh, nv, c):
    s = _f32(stat)
    H, W = s.shape
    m = np.zeros(W * H, np.float32)
    lib().orc_tool_mask(s.ravel(), W, H, bw // 2, bh // 2, C.c_float(nv), C.c_float(c), m)
    return m.reshape(H, W)


def tool_range(stat, bw, bh, nv, step, max_iter=100000):
    s = _f32(stat)
    H, W = s.shape
    a, b = C.c_float(), C.c_float()
    rc = lib().orc_tool_range(s.ravel(), W, H, bw // 2, bh // 2, C.c_float(nv), C.c_float(step), max_iter,
                              C.byref(a), C.byref(b))
    if rc != 0:
        raise ValueError("the step never reaches an all-zero mask")
    return np.float32(a.value), np.float32(b.value)


def gat_objective3d(vol, gain, sigma, offset) -> float:
    """GATMinimizer3D.userFunction (java/GATMinimizer3D.java)."""
    v = _f32(vol)
    D, H, W = v.shape
    return float(lib().orc_gat_objective3d(v.ravel(), W, H, D, float(gain), float(sigma), float(offset)))


def classify_redundancy(redundancy_map, border=1, k=3, optimal_k=False, max_k=10, seed=0):
    """ClassifyRedundancy_.run (java/ClassifyRedundancy_.java) restated:
    (class map, classes used, WCSS)."""
    m = _f32(redundancy_map)
    H, W = m.shape
    out = np.zeros(W * H, np.float32)
    w = C.c_double()
    kc = lib().orc_classify_redundancy(m.ravel(), W, H, border, k, int(optimal_k), max_k, seed, out, C.byref(w))
    return out.reshape(H, W), kc, w.value


def java_random_next(seed, bits, n):
    out = np.zeros(n, np.int32)
    lib().orc_java_random_next(seed, bits, n, out)
    return out


def java_random_doubles(seed, n):
    out = np.zeros(n, np.float64)
    lib().orc_java_random_doubles(seed, n, out)
    return out


def f_quantile(p, df):
    return float(lib().orc_f_quantile(float(p), float(df)))


def gat_tree(img, octree=False, min_size=4, alpha=0.01, max_iter=50, frac=0.75, max_leaves=1 << 20):
    """QuadTree_ / OcTree_ variance stabilisation restated (FP32 reference
    order): dict with the transformed image, g0, eDC and the leaves."""
    a = _f32(img).copy()
    if octree:
        D, H, W = a.shape
    else:
        (H, W), D = a.shape, 1
    g0, edc = C.c_double(), C.c_double()
    boxes = np.zeros(6 * max_leaves, np.int32)
    means = np.zeros(max_leaves, np.float32)
    var = np.zeros(max_leaves, np.float32)
    nl = lib().orc_gat_tree(a.ravel(), W, H, D, int(octree), min_size, C.c_float(alpha), max_iter, C.c_float(frac),
                            C.byref(g0), C.byref(edc), boxes, means, var, max_leaves)
    if nl < 0:
        raise ValueError("the regression has no slope")
    return {"image": a, "g0": g0.value, "edc": edc.value, "boxes": boxes[:6 * nl].reshape(nl, 6),
            "means": means[:nl], "vars": var[:nl]}
