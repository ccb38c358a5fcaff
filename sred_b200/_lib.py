"""ctypes binding of libsred.so (the C ABI declared in include/sred.h).

The library is the only compute path: if it is missing or no CUDA device is
present, calls raise instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import threading
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libsred.so"

OK, ERR_ARG, ERR_UNKNOWN_METRIC, ERR_NODEV, ERR_OOM, ERR_LAUNCH, ERR_TIMEOUT, ERR_INTERNAL, ERR_INVALID_INPUT = range(9)
ENGINE_TC, ENGINE_FP32 = 0, 1

# Every symbol include/sred.h declares.
EXPORTS = [
    "sred_create", "sred_destroy", "sred_set_engine", "sred_status_string", "sred_last_error",
    "sred_block_size", "sred_local_statistics_2d", "sred_mean_noise_var_2d", "sred_relevance_mask_2d",
    "sred_calculate_global_repetition_map_2d", "sred_global_map_2d", "sred_global_map_2d_device",
    "sred_calculate_block_repetition_map_2d", "sred_block_map_2d_device", "sred_block_map_2d_stack",
    "sred_reference_block_2d",
    "sred_normalize_image_2d", "sred_debug_gram_rowdot", "sred_block_map_2d_device_noalloc",
    "sred_patch_hu_map_2d", "sred_hu_map_2d", "sred_phase_correlation_map_2d", "sred_global_map_2d_batch",
    "sred_global_map_2d_shard_sums", "sred_global_map_2d_shard_finish", "sred_set_log_callback",
    "sred_gat_2d", "sred_gat_objective_2d", "sred_gat_fit_2d", "sred_block_size_3d", "sred_reference_block_3d",
    "sred_local_statistics_3d", "sred_relevance_mask_3d", "sred_calculate_block_repetition_map_3d",
    "sred_block_map_3d_device", "sred_calculate_global_repetition_map_3d", "sred_global_map_3d_device",
    "sred_relevance_mask_tool_2d", "sred_relevance_mask_sweep_2d", "sred_relevance_constant_range_2d",
    "sred_gat_3d", "sred_gat_objective_3d", "sred_gat_fit_3d", "sred_classify_redundancy_2d",
    "sred_debug_divide_fixed", "sred_debug_divide_fixed64", "sred_gat_quadtree_2d", "sred_gat_octree_3d", "sred_f_quantile",
    "sred_global_map_3d_shard_sums", "sred_global_map_3d_shard_finish", "sred_debug_set_tc_wait",
    "sred_set_gram_tuning", "sred_gram_tuning_entries", "sred_gram_tuning_set", "sred_gram_tuning_clear",
]


class RunInfo(C.Structure):
    _fields_ = [("n_blocks", C.c_int64), ("n_relevant", C.c_int64), ("n_flat", C.c_int64),
                ("pairs", C.c_double), ("noise_var", C.c_float), ("threshold", C.c_float),
                ("n_pixels", C.c_float), ("k", C.c_int), ("engine", C.c_int),
                ("ms_moments", C.c_double), ("ms_gram", C.c_double), ("ms_finalize", C.c_double),
                ("ms_total", C.c_double), ("launches", C.c_int)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class SredJob(C.Structure):
    """sred_job: one map of sred_global_map_2d_batch."""
    _fields_ = [("metric", C.c_char_p), ("img", C.c_void_p), ("w", C.c_int), ("h", C.c_int), ("bw", C.c_int),
                ("bh", C.c_int), ("relevance_constant", C.c_float), ("normalize_output", C.c_int),
                ("out", C.c_void_p), ("info", C.POINTER(RunInfo)), ("status", C.c_int)]


class SredError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
LOG_CB = C.CFUNCTYPE(None, C.c_char_p, C.c_void_p)
_fp = C.POINTER(C.c_float)
_vp = C.c_void_p
_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load libsred.so, declaring every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise SredError(ERR_INTERNAL, f"{LIB_PATH} is not built; run `python -m sred_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        s = C.c_int
        L.sred_status_string.restype = C.c_char_p
        L.sred_status_string.argtypes = [s]
        L.sred_last_error.restype = C.c_char_p
        L.sred_last_error.argtypes = [_vp]
        L.sred_create.argtypes = [s, C.POINTER(_vp)]
        L.sred_destroy.argtypes = [_vp]
        L.sred_set_engine.argtypes = [_vp, s]
        L.sred_set_log_callback.argtypes = [_vp, LOG_CB, _vp]
        _dp = C.POINTER(C.c_double)
        L.sred_gat_2d.argtypes = [_vp, _f32p, s, s, C.c_double, C.c_double, C.c_double]
        L.sred_gat_objective_2d.argtypes = [_vp, _f32p, s, s, C.c_double, C.c_double, C.c_double, _dp]
        L.sred_gat_fit_2d.argtypes = [_vp, _f32p, s, s, s, _dp, _dp, _dp, _dp]
        L.sred_gat_3d.argtypes = [_vp, _f32p, s, s, s, C.c_double, C.c_double, C.c_double]
        L.sred_gat_objective_3d.argtypes = [_vp, _f32p, s, s, s, C.c_double, C.c_double, C.c_double, _dp]
        L.sred_gat_fit_3d.argtypes = [_vp, _f32p, s, s, s, s, _dp, _dp, _dp, _dp]
        L.sred_block_size.argtypes = [s, s]
        L.sred_local_statistics_2d.argtypes = [_vp, _f32p, s, s, s, s, _f32p, _f32p]
        L.sred_mean_noise_var_2d.argtypes = [_vp, _f32p, s, s, _fp]
        L.sred_relevance_mask_2d.argtypes = [_vp, _f32p, s, s, s, s, _f32p, C.c_float, _f32p, _fp, _fp]
        L.sred_calculate_global_repetition_map_2d.argtypes = [
            _vp, C.c_char_p, _f32p, s, s, s, s, s, _f32p, _f32p, _f32p, C.c_float, C.c_float, C.c_float,
            C.c_float, s, _f32p, C.POINTER(RunInfo)]
        L.sred_global_map_2d.argtypes = [_vp, C.c_char_p, _vp, s, s, s, s, C.c_float, s, _vp,
                                         C.POINTER(RunInfo)]
        L.sred_global_map_2d_device.argtypes = [_vp, C.c_char_p, _vp, s, s, s, s, C.c_float, s, _vp, _vp,
                                                C.POINTER(RunInfo)]
        L.sred_calculate_block_repetition_map_2d.argtypes = [
            _vp, C.c_char_p, _f32p, s, s, _f32p, s, s, s, C.c_float, C.c_float, C.c_float, s, _f32p]
        L.sred_block_map_2d_device.argtypes = [_vp, C.c_char_p, _vp, s, s, s, _f32p, s, s, s, C.c_float,
                                               C.c_float, C.c_float, s, _vp, _vp]
        L.sred_block_map_2d_stack.argtypes = [_vp, C.c_char_p, _f32p, s, s, s, _f32p, s, s, s, C.c_float,
                                              C.c_float, C.c_float, s, s, _f32p]
        L.sred_reference_block_2d.argtypes = [_f32p, s, s, _f32p, C.POINTER(C.c_int), _fp, _fp]
        L.sred_normalize_image_2d.argtypes = [_f32p, s, s, s, s, _vp]
        f = C.c_float
        L.sred_block_size_3d.argtypes = [s, s, s]
        L.sred_reference_block_3d.argtypes = [_f32p, s, s, s, _f32p, C.POINTER(C.c_int), _fp, _fp]
        L.sred_local_statistics_3d.argtypes = [_vp, _f32p, s, s, s, s, s, s, _f32p, _f32p]
        L.sred_relevance_mask_3d.argtypes = [_vp, s, s, s, s, s, s, _f32p, f, _f32p, _fp]
        L.sred_calculate_block_repetition_map_3d.argtypes = [_vp, C.c_char_p, _f32p, s, s, s, _f32p, s, s, s, s,
                                                             f, f, f, s, _f32p]
        L.sred_block_map_3d_device.argtypes = [_vp, C.c_char_p, _vp, s, s, s, _f32p, s, s, s, s, f, f, f, s, _vp,
                                               _vp]
        L.sred_calculate_global_repetition_map_3d.argtypes = [_vp, C.c_char_p, _f32p, s, s, s, s, s, s, f, s, _f32p,
                                                              C.POINTER(RunInfo)]
        L.sred_global_map_3d_device.argtypes = [_vp, C.c_char_p, _vp, s, s, s, s, s, s, f, s, _vp, _vp,
                                                C.POINTER(RunInfo)]
        L.sred_classify_redundancy_2d.argtypes = [_vp, _f32p, s, s, s, s, s, s, C.c_int64, _f32p,
                                                  C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.sred_debug_divide_fixed.argtypes = [_vp, _f32p, C.c_size_t, f, _f32p]
        _f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.sred_debug_divide_fixed64.argtypes = [_vp, _f64p, C.c_size_t, C.c_double, _f64p]
        L.sred_gat_quadtree_2d.argtypes = [_vp, _f32p, s, s, s, f, s, f, _dp, _dp, C.POINTER(C.c_int)]
        L.sred_gat_octree_3d.argtypes = [_vp, _f32p, s, s, s, s, f, s, f, _dp, _dp, C.POINTER(C.c_int)]
        L.sred_f_quantile.restype = C.c_double
        L.sred_f_quantile.argtypes = [C.c_double, C.c_double]
        L.sred_global_map_3d_shard_sums.argtypes = [_vp, C.c_char_p, _vp, s, s, s, s, s, s, f, s, s, _vp, C.c_size_t,
                                                    _vp, C.POINTER(RunInfo)]
        L.sred_global_map_3d_shard_finish.argtypes = [_vp, _vp, s, _vp, _vp, C.POINTER(RunInfo)]
        L.sred_relevance_mask_tool_2d.argtypes = [_vp, _f32p, s, s, s, s, f, _f32p, _fp, _fp]
        L.sred_relevance_mask_sweep_2d.argtypes = [_vp, _f32p, s, s, s, s, f, f, s, _f32p, _f32p, _fp]
        L.sred_relevance_constant_range_2d.argtypes = [_vp, _f32p, s, s, s, s, f, _fp, _fp, _fp]
        _f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.sred_debug_gram_rowdot.argtypes = [_vp, s, _f32p, _f32p, _f32p, s, s, _f64p, _f64p]
        L.sred_debug_set_tc_wait.argtypes = [_vp, C.c_ulonglong, C.c_longlong]
        L.sred_set_gram_tuning.argtypes = [_vp, s]
        L.sred_gram_tuning_entries.argtypes = [_vp, _vp, s]
        L.sred_gram_tuning_set.argtypes = [s, s, s, s, s, s, C.c_float]
        L.sred_gram_tuning_clear.argtypes = []
        L.sred_gram_tuning_entries.restype = s
        L.sred_block_map_2d_device_noalloc.argtypes = [C.c_char_p, _vp, s, s, s, _f32p, s, s, s, C.c_float,
                                                       C.c_float, s, _vp, _vp]
        L.sred_global_map_2d_batch.argtypes = [_vp, C.POINTER(SredJob), s, s]
        L.sred_global_map_2d_shard_sums.argtypes = [_vp, C.c_char_p, _vp, s, s, s, s, C.c_float, s, s, _vp,
                                                    C.c_size_t, _vp, C.POINTER(RunInfo)]
        L.sred_global_map_2d_shard_finish.argtypes = [_vp, _vp, s, _vp, _vp, C.POINTER(RunInfo)]
        L.sred_patch_hu_map_2d.argtypes = [_vp, _f32p, _f32p, s, s, s, s, s, _f32p]
        L.sred_hu_map_2d.argtypes = [_vp, _f32p, _f32p, _f32p, s, s, s, s, _f32p]
        L.sred_phase_correlation_map_2d.argtypes = [_vp, _f32p, _f32p, _f32p, s, s, s, s, _f32p]
        _lib = L
    path = tuning_path()
    if path is not None and path.exists():
        gram_tuning_load(path)
    return _lib


def status_string(st: int) -> str:
    return load().sred_status_string(st).decode()


class Context:
    """Owns a libsred context (device, stream, workspaces)."""

    def __init__(self, device: int = 0, engine: str = "fp32"):
        self._L = load()
        h = _vp()
        st = self._L.sred_create(device, C.byref(h))
        if st != OK:
            raise SredError(st, f"sred_create({device}): {status_string(st)}")
        self.h = h
        self.set_engine(engine)

    def set_engine(self, engine: str) -> None:
        e = {"tc": ENGINE_TC, "fp32": ENGINE_FP32}[engine]
        self.check(self._L.sred_set_engine(self.h, e), "sred_set_engine")
        self.engine = engine

    def set_gram_tuning(self, on: bool) -> None:
        """Time the tensor-core launch shapes of maps whose key the process
        table lacks (sred_set_gram_tuning)."""
        self.check(self._L.sred_set_gram_tuning(self.h, int(bool(on))), "sred_set_gram_tuning")

    def set_log_callback(self, fn) -> None:
        """fn(message: str) receives the context's messages; None turns logging off."""
        self._log_cb = LOG_CB(lambda msg, user: fn(msg.decode())) if fn else LOG_CB()
        self.check(self._L.sred_set_log_callback(self.h, self._log_cb, None), "sred_set_log_callback")

    def check(self, st: int, what: str) -> None:
        if st != OK:
            msg = self._L.sred_last_error(self.h).decode() if self.h else ""
            raise SredError(st, f"{what}: {status_string(st)} ({msg})")

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.sred_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Launch-shape table of the tensor-core engine (sred_set_gram_tuning)
# ---------------------------------------------------------------------------

# Metric codes of the table's keys.
TUNING_METRICS = {0: "Pearson's R", 1: "SSIM", 2: "NRMSE", 8: "NRMSE (3D, weighted terms)"}


def tuning_path() -> Path | None:
    """The table file next to the library, or the path in SRED_GRAM_TUNING
    ("off" or "0": none). load() reads it when it exists."""
    v = os.environ.get("SRED_GRAM_TUNING")
    if v in ("off", "0"):
        return None
    return Path(v) if v else PKG / "gram_tuning.json"


def gram_tuning_entries() -> list[dict]:
    """The process's table: one dict per (K', metric, size class) key."""
    L = load()
    n = L.sred_gram_tuning_entries(None, None, 0)
    e = np.zeros(6 * max(n, 1), np.int32)
    ms = np.zeros(max(n, 1), np.float32)
    n = min(n, L.sred_gram_tuning_entries(e.ctypes.data, ms.ctypes.data, n))
    out = []
    for i in range(n):
        kq, metric, ncls, bn, tr, ml = (int(v) for v in e[6 * i:6 * i + 6])
        out.append({"kq": kq, "metric": metric, "metric_name": TUNING_METRICS.get(metric, str(metric)),
                    "size_class": ncls, "bn": bn, "a_resident": bool(tr), "max_l": ml, "ms": float(ms[i])})
    return out


def gram_tuning_set(entries: list[dict]) -> int:
    """Stores entries (as gram_tuning_entries returns them); returns how many
    the library accepted (shapes that do not fit their K' are skipped)."""
    L = load()
    ok = 0
    for t in entries:
        st = L.sred_gram_tuning_set(int(t["kq"]), int(t["metric"]), int(t["size_class"]), int(t["bn"]),
                                    int(bool(t["a_resident"])), int(t["max_l"]), float(t.get("ms", 0.0)))
        ok += st == OK
    return ok


def gram_tuning_load(path: Path | str) -> int:
    """Reads a table file written by gram_tuning_save into the process table."""
    with open(path) as f:
        data = json.load(f)
    return gram_tuning_set(data.get("entries", []))


def gram_tuning_save(path: Path | str | None = None, device: str = "") -> Path:
    """Writes the process table (merged over the file's existing entries) as
    JSON; `device` names the GPU the shapes were timed on."""
    path = Path(path) if path is not None else (tuning_path() or PKG / "gram_tuning.json")
    entries = {}
    if path.exists():
        with open(path) as f:
            for t in json.load(f).get("entries", []):
                entries[(t["kq"], t["metric"], t["size_class"])] = t
    for t in gram_tuning_entries():
        entries[(t["kq"], t["metric"], t["size_class"])] = t
    tmp = path.with_suffix(".tmp")
    with open(tmp, "w") as f:
        json.dump({"device": device, "entries": sorted(entries.values(), key=lambda t: (t["kq"], t["metric"],
                                                                                       t["size_class"]))},
                  f, indent=1)
    os.replace(tmp, path)
    return path


def gram_tuning_clear() -> None:
    load().sred_gram_tuning_clear()


_default: Context | None = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default
