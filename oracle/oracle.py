"""TEST INFRASTRUCTURE ONLY -- Python bindings of the FP64 oracle (oracle/pwa_oracle.cpp) and of the
reference's own code built for host cores (oracle/build_ref.py).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, as the
checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
NLL_SHIFT = 10000000.0

_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)


def build(force: bool = False) -> Path:
    src = HERE / "pwa_oracle.cpp"
    if force or not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared", str(src), "-o", str(LIB)],
                       check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.oracle_eval_fx.restype = C.c_int
        L.oracle_eval_fx.argtypes = [_fp, _fp, _fp, C.c_long, C.c_long, C.c_long, C.c_long, _fp, C.c_int, C.c_int,
                                     C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_int, _dp, _dp,
                                     C.c_int]
        L.oracle_amp2.restype = C.c_int
        L.oracle_amp2.argtypes = [_fp, _fp, _fp, C.c_long, C.c_long, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_int, C.c_float, C.c_float, _dp, C.c_int]
        L.oracle_eval_fx_x.restype = C.c_int
        L.oracle_eval_fx_x.argtypes = [_fp, _fp, _fp, _fp, _fp, C.c_long, C.c_long, C.c_long, C.c_long, _fp,
                                       C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                       C.c_int, _dp, _dp, C.c_int]
        L.oracle_eval_fx_grid.restype = C.c_int
        L.oracle_eval_fx_grid.argtypes = [_fp, _fp, _fp, _fp, _fp, C.c_long, C.c_long, C.c_int, _dp, _dp, _fp,
                                          C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                          C.c_float, _dp, _dp, C.c_int]
        L.oracle_amp2_x.restype = C.c_int
        L.oracle_amp2_x.argtypes = [_fp, _fp, _fp, _fp, _fp, C.c_long, C.c_long, _fp, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _dp, C.c_int]
        L.oracle_set_kmatrix_isospin.argtypes = [C.c_int]
        L.oracle_assemble_nll.restype = C.c_double
        L.oracle_assemble_nll.argtypes = [_dp, _dp, _fp, C.c_long, C.c_long, C.c_double, C.c_double, C.c_double, _dp]
        for f in ("oracle_bw_lstar", "oracle_bw_pc"):
            getattr(L, f).argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_double, _dp]
        for f in ("oracle_barrier_lb_lstar", "oracle_barrier_lb_pc"):
            getattr(L, f).restype = C.c_double
            getattr(L, f).argtypes = [C.c_double] * 4
        L.oracle_lineshapes.restype = C.c_int
        L.oracle_lineshapes.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                        C.c_double, C.c_double, _dp, _dp]
        L.oracle_lineshapes_lstar_km.restype = C.c_int
        L.oracle_lineshapes_lstar_km.argtypes = [_fp, C.c_int, C.c_int, C.c_float, _fp, _dp, _dp, _dp, _dp]
        L.oracle_kmatrix.restype = C.c_int
        L.oracle_kmatrix.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                     C.c_int, _dp]
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data_as(_fp)


def _planes_x(sample):
    """Zcs chain planes of a sample (null pointers when the sample has none)."""
    p3, p4 = getattr(sample, "pp3", None), getattr(sample, "pp4", None)
    if p3 is None:
        return None, None, None
    a3 = np.ascontiguousarray(p3, np.float32)
    a4 = np.ascontiguousarray(p4, np.float32)
    return a3.ctypes.data_as(_fp), a4.ctypes.data_as(_fp), (a3, a4)


def eval_fx(sample, block, nda_smr: int, nda_fine: int, swap_coupling_parts: bool = False,
            threads: int | None = None):
    """Per-event |A|^2 (fx) and non-interfering w|A|^2 with the reference's band dispatch."""
    fx = np.zeros(sample.n, np.float64)
    fxn = np.zeros(sample.n, np.float64)
    pl = np.ascontiguousarray(block.data, np.float32)
    p3, p4, kx = _planes_x(sample)
    keep = (sample.pp, sample.pp1, sample.pp2, pl, kx)
    rc = lib().oracle_eval_fx_x(_f(sample.pp), _f(sample.pp1), _f(sample.pp2), p3, p4, sample.n_size, sample.n,
                                nda_smr, nda_fine, pl.ctypes.data_as(_fp), block.para_size, block.vamp_size,
                                block.spline_size, block.NR, block.NZ, block.NX, block.ffr, block.ffb,
                                int(swap_coupling_parts), fx.ctypes.data_as(_dp), fxn.ctypes.data_as(_dp),
                                threads or os.cpu_count())
    del keep
    if rc != 0:
        raise RuntimeError(f"oracle_eval_fx failed: {rc}")
    return fx, fxn


def gauss_grid(sigma: float, step: float, half_bins: int) -> tuple:
    """Offsets (GeV) and weights of the fixed-width Gaussian resolution on a mass grid:
    offset_b = (b - half_bins) * step, w_b proportional to exp(-offset_b^2 / (2 sigma^2)), sum w_b = 1."""
    off = (np.arange(2 * half_bins + 1) - half_bins) * float(step)
    w = np.exp(-0.5 * (off / float(sigma)) ** 2)
    return off, w / w.sum()


def eval_fx_grid(sample, block, sigma: float, step: float, half_bins: int, threads: int | None = None):
    """Per-event fx and non-interfering w|A|^2 with every event smeared by the Gaussian grid."""
    off, wt = gauss_grid(sigma, step, half_bins)
    fx = np.zeros(sample.n, np.float64)
    fxn = np.zeros(sample.n, np.float64)
    pl = np.ascontiguousarray(block.data, np.float32)
    p3, p4, kx = _planes_x(sample)
    keep = (sample.pp, sample.pp1, sample.pp2, pl, kx, off, wt)
    rc = lib().oracle_eval_fx_grid(_f(sample.pp), _f(sample.pp1), _f(sample.pp2), p3, p4, sample.n_size, sample.n,
                                   len(off), off.ctypes.data_as(_dp), wt.ctypes.data_as(_dp), pl.ctypes.data_as(_fp),
                                   block.para_size, block.vamp_size, block.spline_size, block.NR, block.NZ, block.NX,
                                   block.ffr, block.ffb, fx.ctypes.data_as(_dp), fxn.ctypes.data_as(_dp),
                                   threads or os.cpu_count())
    del keep
    if rc != 0:
        raise RuntimeError(f"oracle_eval_fx_grid failed: {rc}")
    return fx, fxn


def amp2(sample, block, threads: int | None = None) -> np.ndarray:
    """Unsmeared, unweighted coherent |A|^2 per event (host_store_amp2s semantics)."""
    out = np.zeros(sample.n, np.float64)
    pl = np.ascontiguousarray(block.data, np.float32)
    p3, p4, kx = _planes_x(sample)
    rc = lib().oracle_amp2_x(_f(sample.pp), _f(sample.pp1), _f(sample.pp2), p3, p4, sample.n_size, sample.n,
                             pl.ctypes.data_as(_fp), block.para_size, block.vamp_size, block.spline_size, block.NR,
                             block.NZ, block.NX, block.ffr, block.ffb, out.ctypes.data_as(_dp),
                             threads or os.cpu_count())
    del kx
    if rc != 0:
        raise RuntimeError(f"oracle_amp2 failed: {rc}")
    return out


def lineshapes(block, mkp: float, mz: float) -> tuple:
    """Every Lambda* lineshape times its production barrier at mkp and every Pc lineshape times its
    barrier at mz (complex arrays of NR and NZ), as the amplitude uses them."""
    pl = np.ascontiguousarray(block.data, np.float32)
    ls = np.zeros(2 * max(block.NR, 1))
    pc = np.zeros(2 * max(block.NZ, 1))
    rc = lib().oracle_lineshapes(pl.ctypes.data_as(_fp), block.para_size, block.vamp_size, block.spline_size,
                                 block.NR, block.NZ, block.ffr, block.ffb, mkp, mz, ls.ctypes.data_as(_dp),
                                 pc.ctypes.data_as(_dp))
    if rc != 0:
        raise RuntimeError(f"oracle_lineshapes failed: {rc}")
    return ls[0::2][:block.NR] + 1j * ls[1::2][:block.NR], pc[0::2][:block.NZ] + 1j * pc[1::2][:block.NZ]


def lineshapes_lstar_km(block, mkp) -> tuple:
    """host_store_lineshapeLsKM's outputs (revised K-matrix and Breit-Wigner lineshape of every Lambda*
    entry, each times the Lambda_b barrier with radius FFR) as complex [NR, n] arrays."""
    m = np.ascontiguousarray(mkp, np.float32)
    n, nr = len(m), block.NR
    out = [np.zeros(n * nr) for _ in range(4)]
    pl = np.ascontiguousarray(block.data, np.float32)
    lib().oracle_lineshapes_lstar_km(m.ctypes.data_as(_fp), n, nr, block.ffr, pl.ctypes.data_as(_fp),
                                     *[o.ctypes.data_as(_dp) for o in out])
    return (out[0] + 1j * out[1]).reshape(nr, n), (out[2] + 1j * out[3]).reshape(nr, n)


def assemble_nll(sample, fx, fxn) -> tuple:
    out = C.c_double()
    sw = np.ascontiguousarray(sample.sw, np.float32)
    s = lib().oracle_assemble_nll(fx.ctypes.data_as(_dp), fxn.ctypes.data_as(_dp), sw.ctypes.data_as(_fp),
                                  sample.nda, sample.n, sample.sum_w_mc, sample.sum_w_data, NLL_SHIFT, C.byref(out))
    return out.value, s


def nll(sample, block, swap_coupling_parts: bool = False) -> tuple:
    """(NLL, MC normalisation sum, fx, fx_noint) as host_store_fx would return them, for the band
    arguments RooDalitzAmplitude::IntegralMethod2 passes."""
    a, b = sample.reference_band_args()
    fx, fxn = eval_fx(sample, block, a, b, swap_coupling_parts)
    v, s = assemble_nll(sample, fx, fxn)
    return v, s, fx, fxn


# ------------------------------------------------------------------ reference built for host cores
_ref_libs = {}


def set_kmatrix_isospin(on: bool):
    """The 7-channel isospin-split K-matrix of the reference's ISOSPIN_SIGMACD build (Isospin_KMatrix,
    src/cu_DPFPropogator.cu:384-586) instead of the 4-channel default, for every later oracle call."""
    lib().oracle_set_kmatrix_isospin(int(bool(on)))


def ref_lib(NR: int, NZ: int, NX: int = 0, ikm: int = 6, build_if_missing: bool = True, isospin: bool = False):
    import importlib.util
    spec = importlib.util.spec_from_file_location("pwa_build_ref", HERE / "build_ref.py")
    br = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(br)
    path = br.lib_path(NR, NZ, NX, ikm, isospin)
    if not path.exists():
        if not (build_if_missing and br.available()):
            return None
        br.build_bucket(NR, NZ, NX, ikm, isospin=isospin)
    key = str(path)
    if key not in _ref_libs:
        L = C.CDLL(key)
        L.ref_configure.argtypes = [_fp, C.c_int]
        L.ref_reset.argtypes = []
        L.ref_host_store_fx.restype = C.c_double
        L.ref_host_store_fx.argtypes = [_fp, _fp, _fp, _fp, _fp, _fp, _fp, C.c_int, C.c_int, C.c_int, _dp, C.c_int,
                                        C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _dp,
                                        C.c_double, C.c_double, C.c_float, C.c_float, C.c_int, C.c_int]
        L.ref_host_store_amp2s.argtypes = [_fp, _fp, _fp, _fp, _fp, _fp, C.c_int, C.c_int, C.c_int, _dp, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_float, C.c_float]
        L.ref_host_store_lineshapeLsKM.argtypes = [_fp, _fp, _fp, _fp, _fp, C.c_int, C.c_int, C.c_int, C.c_float,
                                                   _fp, C.c_int, C.c_int, C.c_int]
        _ref_libs[key] = L
    return _ref_libs[key]


class RefHost:
    """The reference's host_store_fx on host cores for one sample (SoA buffers set once)."""

    def __init__(self, sample, block, isospin: bool = False):
        self.L = ref_lib(block.NR, block.NZ, block.NX, isospin=isospin)
        if self.L is None:
            raise FileNotFoundError("reference host build unavailable")
        self.s = sample
        self.pp = np.ascontiguousarray(sample.pp, np.float32)
        self.pp1 = np.ascontiguousarray(sample.pp1, np.float32)
        self.pp2 = np.ascontiguousarray(sample.pp2, np.float32)
        p3, p4 = getattr(sample, "pp3", None), getattr(sample, "pp4", None)
        self.pp3 = np.ascontiguousarray(p3, np.float32) if p3 is not None else np.zeros(16, np.float32)
        self.pp4 = np.ascontiguousarray(p4, np.float32) if p4 is not None else np.zeros(16, np.float32)
        self.sw = np.ascontiguousarray(sample.sw, np.float32)
        self.L.ref_reset()
        pl = np.ascontiguousarray(block.data, np.float32)
        self.L.ref_configure(pl.ctypes.data_as(_fp), block.para_size)
        self.fx = np.zeros(sample.n, np.float64)

    def store_fx(self, block, store_h_fx: bool = True) -> tuple:
        s = self.s
        pl = np.ascontiguousarray(block.data, np.float32)
        out = C.c_double()
        a, b = s.reference_band_args()
        sumint = self.L.ref_host_store_fx(_f(self.pp), _f(self.pp1), _f(self.pp2), _f(self.pp3), _f(self.pp4),
                                          _f(self.sw), pl.ctypes.data_as(_fp), block.para_size, block.vamp_size,
                                          block.spline_size, self.fx.ctypes.data_as(_dp), s.n, 0, s.nda, a, b,
                                          block.NR, block.NZ, block.NX, C.byref(out), s.sum_w_mc, s.sum_w_data,
                                          block.ffr, block.ffb, int(store_h_fx), 1)
        return out.value, sumint

    def amp2s(self, block) -> np.ndarray:
        out = np.zeros(self.s.n, np.float64)
        pl = np.ascontiguousarray(block.data, np.float32)
        self.L.ref_host_store_amp2s(_f(self.pp), _f(self.pp1), _f(self.pp2), _f(self.pp3), _f(self.pp4),
                                    pl.ctypes.data_as(_fp), block.para_size, block.vamp_size, block.spline_size,
                                    out.ctypes.data_as(_dp), self.s.n, block.NR, block.NZ, block.NX, block.ffr,
                                    block.ffb)
        return out


def ref_lineshapes_lstar_km(block, mkp) -> tuple:
    """The reference's own host_store_lineshapeLsKM (FP32, host build) as complex [NR, n] arrays; n must
    be a multiple of 32 (its kernel has no bounds check)."""
    L = ref_lib(block.NR, block.NZ, block.NX)
    if L is None:
        raise FileNotFoundError("reference host build unavailable")
    m = np.ascontiguousarray(mkp, np.float32)
    n, nr = len(m), block.NR
    if n % 32:
        raise ValueError("n must be a multiple of 32")
    out = [np.zeros(n * nr, np.float32) for _ in range(4)]
    pl = np.ascontiguousarray(block.data, np.float32).copy()
    L.ref_configure(pl.ctypes.data_as(_fp), block.para_size)
    L.ref_host_store_lineshapeLsKM(m.ctypes.data_as(_fp), *[o.ctypes.data_as(_fp) for o in out], n, nr, nr,
                                   block.ffr, pl.ctypes.data_as(_fp), block.para_size, block.vamp_size,
                                   block.spline_size)
    return ((out[0] + 1j * out[1]).reshape(nr, n).astype(complex),
            (out[2] + 1j * out[3]).reshape(nr, n).astype(complex))
