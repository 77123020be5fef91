"""Builds libpwa_b200.so in-tree for sm_100a (nvcc cross-compiles without a GPU)."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "pwa_b200" / "libpwa_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["pwa_kernels.cu", "pwa_batch.cu", "pwa_batch_s20.cu", "pwa_batch_s30.cu", "pwa_batch_s150.cu",
           "pwa_batch_grid.cu", "pwa_abi.cu", "pwa_generate.cu", "pwa_noalloc.cu", "pwa_lineshape_diag.cu", "pwa_flow.cu",
           "pwa_ensemble.cu",
           "kernel_calEva_compat.cpp"]


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    deps = list(CSRC.glob("*")) + list((HERE.parent / "include").glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the translation units in parallel (the batched kernels' unit dominates), then links."""
    if not force and not needs_build():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    objdir = HERE / "_build"
    objdir.mkdir(exist_ok=True)
    common = [nvcc, "-std=c++17", *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-v" if verbose else "-O3"]

    def compile_one(src):
        obj = objdir / (src + ".o")
        cmd = common + ["-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for src, _, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr[-6000:]}")
        if verbose:
            print(r.stderr)
    link = [nvcc, *ARCH, "-shared", "-o", str(OUT)] + [str(o) for _, o, _ in results]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-6000:]}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
