"""TEST INFRASTRUCTURE ONLY -- builds the reference's own likelihood code for host cores.

Recipe (no reference source is copied into the repository; all output goes to oracle/_ref/):

* ``src/cu_DPFPropogator.cu`` is compiled by g++ exactly where it lies in the reference tree, with
  ``oracle/ref_host/shim.h`` pre-included (CUDA qualifiers and runtime calls become host code).
* ``src/kernel_calEva.cu`` is compiled from a generated translation unit in ``oracle/_ref/``.  The
  generator changes only two things, textually: each ``K<<<g, b>>>(args)`` launch becomes
  ``ref_host::launch(g, b, K)(args)`` (g++ cannot parse the launch syntax), and each
  ``make_cuFloatComplex(_constant_paraList[ampcount++], _constant_paraList[ampcount++])`` becomes an
  explicitly ordered read (g++ evaluates those two arguments right to left, which would swap the
  real and imaginary parts of every coupling; nvcc device code reads them left to right).
  The model sizes of ``RooTDalitz/NDefine.h`` are compile-time constants in the reference, so each
  (NR, NZ, NX, max_ikmcount) bucket gets its own generated NDefine.h; every other reference header
  is used in place through symlinks.  The generated source is deleted after compilation.
* The isospin-split K-matrix is the reference's compile-time switch ``ISOSPIN_SIGMACD``
  (``RooTDalitz/Resonances.h:17``): its buckets (``libref_iso_*.so``) get a generated Resonances.h with
  the switch on, and ``cu_DPFPropogator.cu`` is then compiled from a generated translation unit beside
  it (same text) so that its relative includes find that header.
* ``oracle/ref_host/driver.cpp`` (this repository's code) adds C entry points.

The result, ``oracle/_ref/libref_<NR>_<NZ>_<NX>_<IKM>.so``, runs the reference's FP32 arithmetic
on host cores (OpenMP over thread blocks).  It is the parity anchor for the FP64 oracle and the
CPU baseline of bench.py.  It needs the reference tree, named by the environment variable
``PWA_REFERENCE_TREE`` (the build entry point sets it where the tree is mounted), so it is built
where that tree exists and shipped prebuilt.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
REF = Path(os.environ["PWA_REFERENCE_TREE"]) if os.environ.get("PWA_REFERENCE_TREE") else None


def reference_tree() -> Path:
    """The reference tree named by PWA_REFERENCE_TREE; a clear error when it is unset or missing."""
    if REF is None:
        raise FileNotFoundError("PWA_REFERENCE_TREE is not set: it must name the reference source tree")
    if not (REF / "src" / "kernel_calEva.cu").is_file():
        raise FileNotFoundError(f"PWA_REFERENCE_TREE={REF} holds no src/kernel_calEva.cu")
    return REF
CUDA_INC = "/usr/local/cuda/include"

# Model-size buckets used by the tests and the bench (NR, NZ, NX, max_ikmcount).
DEFAULT_BUCKETS = [(6, 0, 0, 6), (6, 12, 0, 6), (14, 3, 0, 6), (3, 4, 0, 6), (2, 2, 0, 6), (2, 1, 2, 6),
                   (5, 5, 0, 6)]

# The isospin-split K-matrix variant is built for the small K-matrix test model's bucket.
ISOSPIN_BUCKETS = [(3, 4, 0, 6)]

LAUNCH_RE = re.compile(r"(\b\w+)<<<\s*([^,>]+?)\s*,\s*([^>]+?)\s*>>>\s*\(")
COUPLING_RE = re.compile(
    r"make_cuFloatComplex\(\s*_constant_paraList\[ampcount\+\+\]\s*,\s*_constant_paraList\[ampcount\+\+\]\s*\)")


def lib_name(nr: int, nz: int, nx: int, ikm: int, isospin: bool = False) -> str:
    return f"libref_{'iso_' if isospin else ''}{nr}_{nz}_{nx}_{ikm}.so"


def lib_path(nr: int, nz: int, nx: int, ikm: int = 6, isospin: bool = False) -> Path:
    return OUT / lib_name(nr, nz, nx, ikm, isospin)


ISOSPIN_RE = re.compile(r"constexpr\s+bool\s+ISOSPIN_SIGMACD\s*=\s*false\s*;")


def available() -> bool:
    return REF is not None and (REF / "src" / "kernel_calEva.cu").is_file()


def _ndefine(nr: int, nz: int, nx: int, ikm: int) -> str:
    # Same declarations as RooTDalitz/NDefine.h with this bucket's sizes.
    return f"""#pragma once
namespace Constant {{
static constexpr unsigned number_of_Lz = {nr};
static constexpr unsigned number_of_Pc = {nz};
static constexpr unsigned number_of_Zcs = {nx};
static constexpr unsigned number_of_resonances = number_of_Lz + number_of_Pc + number_of_Zcs;
static constexpr unsigned max_ikmcount = {ikm};
}};
static constexpr unsigned MYRN = Constant::number_of_Lz;
static constexpr unsigned MYZN = Constant::number_of_Pc;
static constexpr unsigned MYXN = Constant::number_of_Zcs;
"""


def build_bucket(nr: int, nz: int, nx: int, ikm: int = 6, verbose: bool = False, isospin: bool = False) -> Path:
    """One model-size bucket.  isospin: the reference's ISOSPIN_SIGMACD build (RooTDalitz/Resonances.h:17
    set to true in a generated copy of that header, and cu_DPFPropogator.cu compiled from a generated
    translation unit next to it so that its relative includes find the copy)."""
    reference_tree()
    OUT.mkdir(parents=True, exist_ok=True)
    target = lib_path(nr, nz, nx, ikm, isospin)
    work = OUT / f"b_{'iso_' if isospin else ''}{nr}_{nz}_{nx}_{ikm}"
    if work.exists():
        shutil.rmtree(work)
    (work / "src").mkdir(parents=True)
    hdr = work / "RooTDalitz"
    hdr.mkdir()
    for f in (REF / "RooTDalitz").iterdir():
        if f.name != "NDefine.h" and not (isospin and f.name == "Resonances.h"):
            (hdr / f.name).symlink_to(f)
    (hdr / "NDefine.h").write_text(_ndefine(nr, nz, nx, ikm))
    prop_src = REF / "src" / "cu_DPFPropogator.cu"
    if isospin:
        res, n_iso = ISOSPIN_RE.subn("constexpr bool ISOSPIN_SIGMACD = true;", (REF / "RooTDalitz" / "Resonances.h").read_text())
        if n_iso != 1:
            raise RuntimeError("ISOSPIN_SIGMACD switch not found in Resonances.h; recipe out of date")
        (hdr / "Resonances.h").write_text(f'#line 1 "{REF / "RooTDalitz" / "Resonances.h"}"\n' + res)
        prop_src = work / "src" / "cu_DPFPropogator_host.cpp"
        prop_src.write_text(f'#line 1 "{REF / "src" / "cu_DPFPropogator.cu"}"\n' +
                            (REF / "src" / "cu_DPFPropogator.cu").read_text())

    text = (REF / "src" / "kernel_calEva.cu").read_text()
    text, n_launch = LAUNCH_RE.subn(lambda m: f"ref_host::launch(({m.group(2)}), ({m.group(3)}), {m.group(1)})(", text)
    text, n_coup = COUPLING_RE.subn("ref_host::ordered_pair(_constant_paraList, ampcount)", text)
    if n_coup < 3:
        raise RuntimeError("coupling reads not found in kernel_calEva.cu; recipe out of date")
    gen = work / "src" / "kernel_calEva_host.cpp"
    gen.write_text(f'#line 1 "{REF / "src" / "kernel_calEva.cu"}"\n' + text)

    flags = ["-std=c++17", "-O2", "-fopenmp", "-fPIC", "-w", "-fpermissive", f"-I{CUDA_INC}",
             "-DiDevice=0", "-DDEVICE_NUM=1", "-DNLL_SHIFT=10000000",
             "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_CPP", "-include", str(HERE / "ref_host" / "shim.h")]
    objs = []
    cmds = [
        (["g++", *flags, "-x", "c++", "-c", str(prop_src), "-o", str(work / "prop.o")], work / "prop.o"),
        (["g++", *flags, "-x", "c++", "-c", str(gen), "-o", str(work / "kern.o")], work / "kern.o"),
        (["g++", "-std=c++17", "-O2", "-fPIC", f"-I{CUDA_INC}", "-c", str(HERE / "ref_host" / "driver.cpp"),
          "-o", str(work / "drv.o")], work / "drv.o"),
    ]
    for cmd, obj in cmds:
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference host build failed:\n{' '.join(cmd)}\n{r.stderr[-4000:]}")
        objs.append(str(obj))
    r = subprocess.run(["g++", "-shared", "-fopenmp", "-o", str(target), *objs], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-4000:])
    shutil.rmtree(work)
    return target


AUX_LIB = "libref_aux.so"
DFUN_START = "inline Double_t dfunhalf("
DFUN_END = "// parital angluar depdent part"


def build_aux(verbose: bool = False) -> Path:
    """Clebsch-Gordan tables (src/EvtCGCoefSingle.cpp, src/EvtOrthogVector.cpp, compiled in place) and
    the Wigner d-functions of src/RooDalitzAmplitude.cxx (the block from ``dfunhalf`` to the end of
    ``dfun``, extracted at build time and renamed with an ``_impl`` suffix)."""
    reference_tree()
    OUT.mkdir(parents=True, exist_ok=True)
    work = OUT / "b_aux"
    if work.exists():
        shutil.rmtree(work)
    work.mkdir(parents=True)
    text = (REF / "src" / "RooDalitzAmplitude.cxx").read_text()
    i, j = text.index(DFUN_START), text.index(DFUN_END)
    line0 = text[:i].count("\n") + 1
    block = text[i:j]
    for f in ("dfunhalf", "dfunone", "dfun"):
        block = re.sub(rf"\binline Double_t {f}\(", f"Double_t ref_{f}_impl(", block)
    gen = work / "dfun_host.cpp"
    gen.write_text(f'#include "{HERE / "ref_host" / "tmath_shim.h"}"\n#line {line0} "{REF / "src" / "RooDalitzAmplitude.cxx"}"\n'
                   + block)
    target = OUT / AUX_LIB
    cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-w", f"-I{REF}", str(gen),
           str(REF / "src" / "EvtCGCoefSingle.cpp"), str(REF / "src" / "EvtOrthogVector.cpp"),
           str(HERE / "ref_host" / "aux_driver.cpp"), "-o", str(target)]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-4000:])
    shutil.rmtree(work)
    return target


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--bucket", action="append", default=[], help="NR,NZ,NX[,IKM]")
    ap.add_argument("--isospin", action="store_true", help="also build the ISOSPIN_SIGMACD variant of the K-matrix bucket")
    ap.add_argument("-v", action="store_true")
    args = ap.parse_args(argv)
    if not available():
        print(f"reference tree not available (PWA_REFERENCE_TREE={REF}); nothing built")
        return 0
    buckets = [tuple(int(x) for x in b.split(",")) for b in args.bucket] or DEFAULT_BUCKETS
    for b in buckets:
        b = tuple(b) + ((6,) if len(b) == 3 else ())
        print("built", build_bucket(*b, verbose=args.v))
    for b in ISOSPIN_BUCKETS if (args.isospin or not args.bucket) else []:
        print("built", build_bucket(*b, verbose=args.v, isospin=True))
    print("built", build_aux(verbose=args.v))
    return 0


if __name__ == "__main__":
    sys.exit(main())
