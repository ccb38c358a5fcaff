"""Build recipe for the oracle: the C restatement and the reference's own kernels.

TEST INFRASTRUCTURE ONLY.

1. ``oracle/liboracle.so`` from ``oracle/sred_oracle.c`` (committed source).
2. ``oracle/_ref/librefshim.so``: the reference's OpenCL C kernels, read from a
   SReD checkout (default ``/root/reference``), with their ``$PLACEHOLDER$``
   tokens substituted the way the reference's host code substitutes them
   (``java/CLUtils.java:325-339``, first occurrence only) and compiled as C++
   against ``oracle/refshim/shim.h``. The substituted kernel text is written
   only under ``oracle/_ref/`` (git-ignored); nothing of the reference's source
   is committed. Step 2 is skipped when the checkout is absent.

Usage: ``python oracle/refshim/build.py [--reference PATH] [--force]``
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE = HERE.parent
REF_OUT = ORACLE / "_ref"
CFLAGS = ["-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-fast-math"]

# Kernels the hot path uses (cl/ = src/main/resources/), with the argument
# lists of their entry points: g = global-map kernel, b = block-map kernel,
# s = local statistics.
KERNELS = {
    "kernelGetLocalStatistics2D": ("s", ["img", "means", "stds"]),
    "kernelGetGlobalPearson2D": ("g", ["img", "means", "stds", "den", "num"]),
    "kernelGetGlobalSsim2D": ("g", ["img", "means", "stds", "den", "num"]),
    "kernelGetGlobalNrmse2D": ("g", ["img", "means", "stds", "den", "num"]),
    "kernelGetGlobalAbsDiffStds2D": ("g", ["img", "stds", "den", "num"]),
    "kernelGetBlockPearson2D": ("b", ["ref", "img", "means", "stds", "map"]),
    "kernelGetBlockSsim2D": ("b", ["ref", "img", "means", "stds", "map"]),
    "kernelGetBlockNrmse2D": ("b", ["ref", "img", "means", "map"]),
    "kernelGetBlockAbsDiffStds2D": ("b", ["stds", "map"]),
    # relevance-mask tools: local variance and local std of the ellipse block
    "kernelGetRelevanceMask2D": ("s", ["img", "stds"]),
    "kernelGetLocalMeans": ("s", ["img", "means", "stds"]),
}

PLACEHOLDERS = {
    "$WIDTH$": "RS_W", "$HEIGHT$": "RS_H", "$BLOCK_SIZE$": "RS_KT",
    "$BW$": "RS_BW", "$BH$": "RS_BH", "$BRW$": "RS_BRW", "$BRH$": "RS_BRH",
    "$FILTER_PARAM$": "RS_FILTER", "$THRESHOLD$": "RS_THRESHOLD",
    "$EPSILON$": "RS_EPSILON", "$BLOCK_STD$": "RS_BLOCK_STD",
    "$BLOCK_MEAN$": "RS_BLOCK_MEAN", "$PATCH_SIZE$": "RS_KT",
}
MACROS = ["image_width", "image_height", "block_size", "bW", "bH", "bRW", "bRH",
          "filter_param", "threshold", "EPSILON", "w", "h", "ref_std", "ref_mean", "kernel", "patch_size"]

MAX_BLOCK = 15  # every odd block width/height 3..15 is instantiated

# Shape-metric kernels (shipped by the reference, never loaded by its Java
# code). Their block width and height are template parameters; $PATCH_SIZE$
# is the ellipse count K for the Hu patch kernel (the Java convention of
# java/RelevanceMask2D_.java:161-167) and bw*bh for the two all-pairs kernels,
# whose private arrays hold the whole square block.
SHAPE_KERNELS = {
    "kernelGetPatchHu2D": (["patch", "img", "means", "map"], "RS_PS"),
    "kernelGetHuMap": (["img", "means", "stds", "uniq", "map"], "(RS_TBW*RS_TBH)"),
    "kernelGetPhaseCorrelationMap": (["img", "means", "stds", "uniq", "map"], "(RS_TBW*RS_TBH)"),
}
# The phase kernel does not compile as shipped; these text repairs make it
# the intended computation (each is documented in oracle/sred_oracle.c):
#   nUnique is never defined (:27) -> the unique-coordinate pre-filter is off;
#   (1*i*ii/bW) divides integers (:66, :101, :138) -> real-valued phases;
#   cross_corr_real[j*w+i] reads past the block (:150) -> block width.
PHASE_REPAIRS = [("(1*i*ii/bW)", "(1.0*i*ii/bW)"), ("(1*j*jj/bH)", "(1.0*j*jj/bH)"),
                 ("cross_corr_real[j*w+i]", "cross_corr_real[j*bW+i]")]
# 3D kernels (block maps and local statistics): same scheme with a depth.
KERNELS_3D = {
    "kernelGetLocalStatistics3D": ["img", "means", "stds"],
    "kernelGetBlockPearson3D": ["ref", "img", "means", "stds", "map"],
    "kernelGetBlockSsim3D": ["ref", "img", "means", "stds", "map"],
    "kernelGetBlockNrmse3D": ["ref", "img", "means", "map"],
    "kernelGetBlockAbsDiffStds3D": ["stds", "map"],
}
PLACEHOLDERS_3D = {"$DEPTH$": "RS_D", "$BZ$": "RS_BZ", "$BRZ$": "RS_BRZ"}
MACROS_3D = ["image_depth", "bZ", "bRZ", "imageWidth", "imageHeight", "imageDepth"]
SIZES_3D = [(a, b, c) for a in (3, 5, 7) for b in (3, 5, 7) for c in (3, 5)]


# 3D global-map kernels. Two repairs (documented in oracle/sred_oracle.c,
# orc_global3d_f32): the reference block is gathered over all bd slices
# (the kernels stop one slice short), and SSIM's below-threshold branch names
# its own map (the shipped kernel names an undeclared pearson_map).
KERNELS_3D_GLOBAL = {
    "kernelGetGlobalPearson3D": ["img", "means", "stds", "den", "num"],
    "kernelGetGlobalSsim3D": ["img", "means", "stds", "den", "num"],
    "kernelGetGlobalNrmse3D": ["img", "means", "stds", "den", "num"],
    "kernelGetGlobalAbsDiffStds3D": ["img", "stds", "den", "num"],
}
GLOBAL_3D_REPAIRS = {
    "kernelGetGlobalPearson3D": [("z<gz+bRZ", "z<=gz+bRZ")],
    "kernelGetGlobalSsim3D": [("z<gz+bRZ", "z<=gz+bRZ"), ("pearson_map[ref_index] += 0.0f;",
                                                          "ssim_map[ref_index] += 0.0f;")],
    "kernelGetGlobalNrmse3D": [("z<gz+bRZ", "z<=gz+bRZ")],
    "kernelGetGlobalAbsDiffStds3D": [],
}


def ellipsoid_k(bw: int, bh: int, bd: int) -> int:
    f = np.float32
    rw, rh, rd = bw // 2, bh // 2, bd // 2
    k = 0
    for z in range(bd):
        for y in range(bh):
            for x in range(bw):
                dx, dy, dz = f(x - rw), f(y - rh), f(z - rd)
                if (dx * dx) / f(rw * rw) + (dy * dy) / f(rh * rh) + (dz * dz) / f(rd * rd) <= f(1):
                    k += 1
    return k


def gen_unit_3d(ref: Path, name: str) -> str:
    args = KERNELS_3D[name]
    src = (ref / "src/main/resources" / f"{name}.cl").read_text()
    for tok, repl in {**PLACEHOLDERS, **PLACEHOLDERS_3D}.items():
        src = replace_first(src, tok, repl)
    ks = sorted({ellipsoid_k(*s) for s in SIZES_3D})
    call = ", ".join(f"(float*){a}" for a in args)
    params = ", ".join(f"const float* {a}" if a in ("img", "means", "stds", "ref") else f"float* {a}"
                       for a in args)
    cases = "\n".join(f"    case {k}: rs_loop<{k}>(pix, npix, {', '.join(args)}); break;" for k in ks)
    undef = "".join(f"#undef {m}\n" for m in MACROS + MACROS_3D)
    return f"""#include "shim.h"
#include <cfloat>
using std::fmax;
using std::max;
using std::min;
namespace rsns_{name} {{
#define kernel template <int RS_KT> static inline
{src}
{undef}
template <int KT>
static void rs_loop(const int* pix, int npix, {params}) {{
  #pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < npix; i++) {{
    rs_gid[0] = pix[i] % RS_W;
    rs_gid[1] = (pix[i] / RS_W) % RS_H;
    rs_gid[2] = pix[i] / (RS_W * RS_H);
    {name}<KT>({call});
  }}
}}
}}  // namespace rsns_{name}

extern "C" int rs_{name}(int K, int W, int H, int D, int bw, int bh, int bd, float eps, float block_std,
                       float block_mean, const int* pix, int npix, {params}) {{
  using namespace rsns_{name};
  RS_W = W; RS_H = H; RS_D = D; RS_BW = bw; RS_BH = bh; RS_BZ = bd;
  RS_BRW = bw / 2; RS_BRH = bh / 2; RS_BRZ = bd / 2;
  RS_EPSILON = eps; RS_BLOCK_STD = block_std; RS_BLOCK_MEAN = block_mean;
  switch (K) {{
{cases}
    default: return -1;
  }}
  return 0;
}}
"""


def gen_unit_3d_global(ref: Path, name: str) -> str:
    args = KERNELS_3D_GLOBAL[name]
    src = (ref / "src/main/resources" / f"{name}.cl").read_text()
    for tok, repl in {**PLACEHOLDERS, **PLACEHOLDERS_3D}.items():
        src = replace_first(src, tok, repl)
    for a, b in GLOBAL_3D_REPAIRS[name]:
        if a not in src:
            raise RuntimeError(f"repair target {a!r} not found in {name}.cl")
        src = src.replace(a, b)
    ks = sorted({ellipsoid_k(*s) for s in SIZES_3D})
    call = ", ".join(f"(float*){a}" for a in args)
    params = ", ".join(f"const float* {a}" if a in ("img", "means", "stds") else f"float* {a}" for a in args)
    cases = "\n".join(f"    case {k}: rs_loop<{k}>(pix, npix, {', '.join(args)}); break;" for k in ks)
    undef = "".join(f"#undef {m}\n" for m in MACROS + MACROS_3D)
    return f"""#include "shim.h"
#include <cfloat>
using std::fmax;
namespace rsns_{name} {{
#define kernel template <int RS_KT> static inline
{src}
{undef}
template <int KT>
static void rs_loop(const int* pix, int npix, {params}) {{
  #pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < npix; i++) {{
    rs_gid[0] = pix[i] % RS_W;
    rs_gid[1] = (pix[i] / RS_W) % RS_H;
    rs_gid[2] = pix[i] / (RS_W * RS_H);
    {name}<KT>({call});
  }}
}}
}}  // namespace rsns_{name}

extern "C" int rs_{name}(int K, int W, int H, int D, int bw, int bh, int bd, float filter, float threshold,
                       float eps, const int* pix, int npix, {params}) {{
  using namespace rsns_{name};
  RS_W = W; RS_H = H; RS_D = D; RS_BW = bw; RS_BH = bh; RS_BZ = bd;
  RS_BRW = bw / 2; RS_BRH = bh / 2; RS_BRZ = bd / 2;
  RS_FILTER = filter; RS_THRESHOLD = threshold; RS_EPSILON = eps;
  switch (K) {{
{cases}
    default: return -1;
  }}
  return 0;
}}
"""


SHAPE_SIZES = sorted({(a, b) for a in (3, 5, 7, 9) for b in (3, 5, 7, 9)} | {(11, 11), (13, 13), (15, 15)})


def ellipse_k(bw: int, bh: int) -> int:
    f = np.float32
    rw, rh = bw // 2, bh // 2
    k = 0
    for y in range(bh):
        for x in range(bw):
            dx, dy = f(x - rw), f(y - rh)
            if (dx * dx) / f(rw * rw) + (dy * dy) / f(rh * rh) <= f(1):
                k += 1
    return k


def k_list() -> list[int]:
    return sorted({ellipse_k(a, b) for a in range(3, MAX_BLOCK + 1, 2)
                   for b in range(3, MAX_BLOCK + 1, 2)})


def replace_first(src: str, target: str, repl: str) -> str:
    i = src.find(target)
    return src if i < 0 else src[:i] + repl + src[i + len(target):]


def entry_code(name: str, kind: str, args: list[str], ks: list[int]) -> str:
    call = ", ".join(f"(float*){a}" for a in args)
    cases = "\n".join(f"    case {k}: rs_loop<{k}>(pix, npix, {', '.join(args)}); break;" for k in ks)
    params = ", ".join(f"const float* {a}" if a in ("img", "means", "stds", "ref") else f"float* {a}"
                       for a in args)
    return f"""
{''.join(f'#undef {m}' + chr(10) for m in MACROS)}
template <int KT>
static void rs_loop(const int* pix, int npix, {params}) {{
  #pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < npix; i++) {{
    rs_gid[0] = pix[i] % RS_W;
    rs_gid[1] = pix[i] / RS_W;
    {name}<KT>({call});
  }}
}}

extern "C" int rs_{name}(int K, int W, int H, int bw, int bh, float filter, float threshold,
                       float eps, float block_std, float block_mean, const int* pix, int npix,
                       {params}) {{
  RS_W = W; RS_H = H; RS_BW = bw; RS_BH = bh; RS_BRW = bw / 2; RS_BRH = bh / 2;
  RS_FILTER = filter; RS_THRESHOLD = threshold; RS_EPSILON = eps;
  RS_BLOCK_STD = block_std; RS_BLOCK_MEAN = block_mean;
  switch (K) {{
{cases}
    default: return -1;
  }}
  return 0;
}}
"""


def gen_unit(ref: Path, name: str, ks: list[int]) -> str:
    kind, args = KERNELS[name]
    src = (ref / "src/main/resources" / f"{name}.cl").read_text()
    for tok, repl in PLACEHOLDERS.items():
        src = replace_first(src, tok, repl)
    head = ('#include "shim.h"\n'
            "#define kernel template <int RS_KT> static inline\n")
    return head + src + "\n" + entry_code(name, kind, args, ks)


def gen_shape_unit(ref: Path, name: str) -> str:
    args, psize = SHAPE_KERNELS[name]
    src = (ref / "src/main/resources" / f"{name}.cl").read_text()
    reps = {"$WIDTH$": "RS_W", "$HEIGHT$": "RS_H", "$PATCH_SIZE$": psize, "$BW$": "RS_TBW",
            "$BH$": "RS_TBH", "$BRW$": "(RS_TBW/2)", "$BRH$": "(RS_TBH/2)", "$EPSILON$": "RS_EPSILON",
            "$NUNIQUE$": "0", "$SPEEDUP$": "0"}
    for tok, repl in reps.items():
        src = replace_first(src, tok, repl)
    if name == "kernelGetPhaseCorrelationMap":
        src = "#define nUnique 0\n" + src
        for a, b in PHASE_REPAIRS:
            if a not in src:
                raise RuntimeError(f"repair target {a!r} not found in {name}.cl")
            src = src.replace(a, b)
    ptypes = {"patch": "const float*", "img": "const float*", "means": "const float*",
              "stds": "const float*", "uniq": "void*", "map": "float*"}
    params = ", ".join(f"{ptypes[a]} {a}" for a in args)
    call = ", ".join(f"(int*){a}" if (a == "uniq" and name == "kernelGetHuMap") else
                     f"(float*){a}" for a in args)
    cases = "\n".join(f"    case {a * 100 + b}: rs_loop<{a}, {b}>(pix, npix, {', '.join(args)}); break;"
                      for a, b in SHAPE_SIZES)
    undef = "".join(f"#undef {m}\n" for m in MACROS + ["patch_size", "nUnique", "speedUp"])
    return f"""#include "shim_shape.h"
namespace rsns_{name} {{
#define kernel template <int RS_TBW, int RS_TBH> static inline
{src}
{undef}
template <int TBW, int TBH>
static void rs_loop(const int* pix, int npix, {params}) {{
  #pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < npix; i++) {{
    rs_gid[0] = pix[i] % RS_W;
    rs_gid[1] = pix[i] / RS_W;
    {name}<TBW, TBH>({call});
  }}
}}
}}  // namespace rsns_{name}

extern "C" int rs_{name}(int W, int H, int bw, int bh, int patch_size, float eps, const int* pix,
                       int npix, {params}) {{
  using namespace rsns_{name};
  RS_W = W; RS_H = H; RS_BW = bw; RS_BH = bh; RS_BRW = bw / 2; RS_BRH = bh / 2;
  RS_PS = patch_size; RS_EPSILON = eps;
  switch (bw * 100 + bh) {{
{cases}
    default: return -1;
  }}
  return 0;
}}
"""


def run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build_oracle(force: bool = False) -> Path:
    out = ORACLE / "liboracle.so"
    src = ORACLE / "sred_oracle.c"
    if force or not out.exists() or out.stat().st_mtime < src.stat().st_mtime:
        run(["gcc", *CFLAGS, "-shared", str(src), "-o", str(out), "-lm"])
    return out


def build_refshim(ref: Path, force: bool = False) -> Path | None:
    if not (ref / "src/main/resources/kernelGetGlobalPearson2D.cl").exists():
        return None
    out = REF_OUT / "librefshim.so"
    ks = k_list()
    units = {n: gen_unit(ref, n, ks) for n in KERNELS}
    units.update({n: gen_shape_unit(ref, n) for n in SHAPE_KERNELS})
    units.update({n: gen_unit_3d(ref, n) for n in KERNELS_3D})
    units.update({n: gen_unit_3d_global(ref, n) for n in KERNELS_3D_GLOBAL})
    digest = hashlib.sha256(("".join(units.values()) + (HERE / "shim.h").read_text()
                             + (HERE / "shim_shape.h").read_text()).encode()).hexdigest()
    stamp = REF_OUT / "build.sha256"
    if not force and out.exists() and stamp.exists() and stamp.read_text() == digest:
        return out
    gen = REF_OUT / "gen"
    gen.mkdir(parents=True, exist_ok=True)
    objs = []
    jobs = []
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        for n, text in units.items():
            cpp = gen / f"{n}.cpp"
            cpp.write_text(text)
            obj = gen / f"{n}.o"
            objs.append(str(obj))
            jobs.append(ex.submit(run, ["g++", "-std=c++17", *CFLAGS, "-w", f"-I{HERE}", "-c",
                                        str(cpp), "-o", str(obj)]))
        for j in jobs:
            j.result()
    run(["g++", "-shared", "-fopenmp", *objs, "-o", str(out)])
    stamp.write_text(digest)
    return out


def reference_root() -> Path:
    """The SReD checkout the recipe reads: $SRED_REFERENCE, else the default
    location of this build's reference checkout."""
    return Path(os.environ.get("SRED_REFERENCE", "/root/reference"))


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(reference_root()))
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print("oracle:", build_oracle(a.force))
    r = build_refshim(Path(a.reference), a.force)
    print("refshim:", r if r else "skipped (no reference checkout)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
