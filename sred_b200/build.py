"""Build libsred.so (sm_100a) in-tree from sred_b200/csrc with nvcc.

Usage: python -m sred_b200.build [--force]
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "libsred.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
         "--expt-relaxed-constexpr", "-Xptxas", "-v"]
SOURCES = ["sred_api.cu", "moments.cu", "block_map.cu", "global_fp32.cu", "global_tc.cu", "noalloc.cu", "shape.cu", "gat.cu", "volume.cu", "relevance.cu", "cluster.cu", "gat_tree.cu"]
# shape.cu, gat.cu, volume.cu, relevance.cu and gat_tree.cu restate the reference's FP32/FP64 evaluation order: no fused multiply-add.
FILE_FLAGS = {"shape.cu": ["-fmad=false"], "gat.cu": ["-fmad=false"], "volume.cu": ["-fmad=false"],
              "relevance.cu": ["-fmad=false"], "gat_tree.cu": ["-fmad=false"]}


def _digest() -> str:
    h = hashlib.sha256()
    for p in sorted(CSRC.glob("*")) + [ROOT / "include" / "sred.h"]:
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(" ".join(ARCH + FLAGS).encode())
    h.update(repr(sorted(FILE_FLAGS.items())).encode())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> Path:
    stamp = PKG / ".libsred.sha256"
    d = _digest()
    if not force and OUT.exists() and stamp.exists() and stamp.read_text() == d:
        return OUT
    objdir = ROOT / "_build" / "sred"
    objdir.mkdir(parents=True, exist_ok=True)
    procs, objs, logs = [], [], []
    for s in SOURCES:
        o = objdir / (s + ".o")
        objs.append(str(o))
        cmd = [NVCC, *ARCH, *FLAGS, *FILE_FLAGS.get(s, []), f"-I{ROOT / 'include'}", "-c", str(CSRC / s),
               "-o", str(o)]
        procs.append((s, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for s, p in procs:
        out, _ = p.communicate()
        logs.append(f"== {s}\n{out}")
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s}:\n{out}")
    link = [NVCC, *ARCH, "-shared", *objs, "-o", str(OUT), "-lcudart"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    (ROOT / "_build" / "ptxas.log").write_text("\n".join(logs))
    stamp.write_text(d)
    if verbose:
        print("\n".join(logs))
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
