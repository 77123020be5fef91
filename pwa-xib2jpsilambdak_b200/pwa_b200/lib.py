"""ctypes bindings of libpwa_b200.so (include/pwa_b200.h).

The library is the only compute path: there is no CPU fallback, and loading fails loudly if the
shared object is missing.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

import os

# The in-tree build; PWA_B200_LIB may name another build of the same library (A/B comparisons).
LIB_PATH = Path(os.environ.get("PWA_B200_LIB", str(Path(__file__).resolve().parent / "libpwa_b200.so")))

EXPORTED = ["pwa_ctx_create", "pwa_ctx_destroy", "pwa_ctx_upload_events", "pwa_ctx_upload_events_unsorted", "pwa_band_order", "pwa_ctx_set_device_events",
            "pwa_ctx_upload_zcs_events", "pwa_ctx_set_device_zcs_events", "pwa_ctx_set_smearing", "pwa_ctx_select_data",
            "pwa_ctx_eval_nll", "pwa_ctx_eval_nll_batch", "pwa_ctx_last_batch_ms", "pwa_ctx_batch_segment_ms", "pwa_ctx_amp2", "pwa_ctx_mc_integral", "pwa_ctx_last_kernel_ms", "pwa_ctx_last_launches", "pwa_ctx_stream",
            "pwa_ctx_set_timing", "pwa_ctx_set_lineshape_tables", "pwa_ctx_set_event_order", "pwa_ctx_set_kmatrix", "pwa_ctx_set_batch_waves", "pwa_ctx_segment_count", "pwa_ctx_segment_info", "pwa_ctx_segment_deferred", "pwa_point_table_bytes",
            "pwa_host_lineshapes", "pwa_host_lineshapes_km", "pwa_lineshapes_lstar_km", "pwa_generate_events", "pwa_events_from_unit",
            "pwa_unit_flat", "pwa_flow_create", "pwa_flow_destroy", "pwa_flow_param_count", "pwa_flow_get_params",
            "pwa_flow_set_params", "pwa_flow_train_step", "pwa_flow_gradients", "pwa_flow_log_density",
            "pwa_flow_sample", "pwa_flow_fit_premap", "pwa_flow_get_premap", "pwa_flow_set_premap",
            "pwa_basis_from_angles", "pwa_angles_from_vectors",
            "pwa_ens_create", "pwa_ens_destroy", "pwa_ens_slot_count", "pwa_ens_slots", "pwa_ens_gram",
            "pwa_ens_set_launch", "pwa_ens_eval", "pwa_ens_last_ms", "pwa_ens_setup_ms",
            "pwa_error_string", "pwa_last_cuda_error"]

_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)


def band_order(mz) -> tuple:
    """(order, band-1 count, band-2 count) of data masses as the library sorts them (pwa_band_order)."""
    L = load()
    m = np.ascontiguousarray(mz, np.float32)
    order = np.zeros(len(m), np.int32)
    n1, n2 = C.c_int64(), C.c_int64()
    check(L.pwa_band_order(_f(m), len(m), order.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(n1), C.byref(n2)),
          "pwa_band_order")
    return order, n1.value, n2.value


class PwaResult(C.Structure):
    _fields_ = [("nll", C.c_double), ("sumint", C.c_double), ("sum_noint", C.c_double),
                ("data_term", C.c_double), ("n_nonpos", C.c_int64)]


class PwaError(RuntimeError):
    pass


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise PwaError(f"{LIB_PATH} is missing: build it with pwa-xib2jpsilambdak_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        L.pwa_ctx_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.pwa_ctx_destroy.argtypes = [C.c_void_p]
        L.pwa_ctx_upload_events.argtypes = [C.c_void_p, _fp, _fp, _fp, _fp] + [C.c_int64] * 5
        L.pwa_ctx_set_device_events.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p] + \
            [C.c_int64] * 5
        L.pwa_ctx_eval_nll.argtypes = [C.c_void_p, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_float, C.c_float, C.c_double, C.c_double, C.c_double,
                                       C.POINTER(PwaResult), _dp]
        L.pwa_ctx_amp2.argtypes = [C.c_void_p, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_float, C.c_float, _dp]
        L.pwa_ctx_upload_events_unsorted.argtypes = [C.c_void_p, _fp, _fp, _fp, _fp] + [C.c_int64] * 3
        L.pwa_ctx_upload_zcs_events.argtypes = [C.c_void_p, _fp, _fp]
        L.pwa_ctx_set_device_zcs_events.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.pwa_ctx_set_smearing.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_int]
        L.pwa_ctx_select_data.argtypes = [C.c_void_p] + [C.c_int64] * 4
        L.pwa_band_order.argtypes = [_fp, C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64)]
        L.pwa_ctx_mc_integral.argtypes = [C.c_void_p, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_float, C.c_float, _dp]
        L.pwa_ctx_eval_nll_batch.argtypes = [C.c_void_p, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                             C.c_int, C.c_int, C.c_float, C.c_float, C.c_double, C.c_double,
                                             C.c_double, C.POINTER(PwaResult), C.POINTER(C.c_int)]
        L.pwa_ctx_last_batch_ms.restype = C.c_double
        L.pwa_ctx_last_batch_ms.argtypes = [C.c_void_p]
        L.pwa_ctx_batch_segment_ms.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double)]
        L.pwa_ctx_last_kernel_ms.restype = C.c_double
        L.pwa_ctx_last_kernel_ms.argtypes = [C.c_void_p]
        L.pwa_ctx_last_launches.argtypes = [C.c_void_p]
        L.pwa_ctx_set_timing.argtypes = [C.c_void_p, C.c_int]
        L.pwa_ctx_set_lineshape_tables.argtypes = [C.c_void_p, C.c_int]
        L.pwa_ctx_segment_count.argtypes = [C.c_void_p]
        L.pwa_ctx_segment_deferred.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]
        L.pwa_ctx_segment_info.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                           C.POINTER(C.c_double)]
        L.pwa_point_table_bytes.restype = C.c_int64
        L.pwa_ctx_stream.restype = C.c_void_p
        L.pwa_ctx_stream.argtypes = [C.c_void_p]
        L.pwa_host_lineshapes.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                          C.c_float, C.c_double, C.c_double, _dp, _dp]
        L.pwa_host_lineshapes_km.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                             C.c_float, C.c_int, C.c_double, C.c_double, _dp, _dp]
        L.pwa_lineshapes_lstar_km.argtypes = [C.c_int, _fp, C.c_int, C.c_int, C.c_float, _fp, C.c_int, _dp, _dp,
                                              _dp, _dp]
        L.pwa_generate_events.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64, C.c_int64,
                                          C.c_uint64, C.c_uint64, C.c_float, C.c_float, C.c_int, C.c_void_p]
        L.pwa_basis_from_angles.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                            C.c_void_p]
        L.pwa_angles_from_vectors.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        L.pwa_error_string.restype = C.c_char_p
        L.pwa_last_cuda_error.restype = C.c_char_p
        _lib = L
    return _lib


def check(rc: int, what: str):
    if rc != 0:
        L = load()
        raise PwaError(f"{what}: {L.pwa_error_string(rc).decode()} ({L.pwa_last_cuda_error().decode()})")


def _f(a):
    return a.ctypes.data_as(_fp)


class Context:
    """One device context holding an uploaded event sample."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        check(self.L.pwa_ctx_create(device, C.byref(h)), "pwa_ctx_create")
        self.h = h
        self.device = device
        self.sample = None
        self.n = 0

    def close(self):
        if self.h:
            self.L.pwa_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, sample, nda_smr: int | None = None, nda_fine: int | None = None):
        """Upload a Sample (reference layout).  Band arguments default to what
        RooDalitzAmplitude::IntegralMethod2 passes (first count minus one)."""
        a, b = sample.reference_band_args()
        a = a if nda_smr is None else nda_smr
        b = b if nda_fine is None else nda_fine
        pp = np.ascontiguousarray(sample.pp, np.float32)
        pp1 = np.ascontiguousarray(sample.pp1, np.float32)
        pp2 = np.ascontiguousarray(sample.pp2, np.float32)
        sw = np.ascontiguousarray(sample.sw, np.float32)
        check(self.L.pwa_ctx_upload_events(self.h, _f(pp), _f(pp1), _f(pp2), _f(sw), sample.n, sample.n_size,
                                           sample.nda, a, b), "pwa_ctx_upload_events")
        self._upload_zcs(sample)
        self.sample = sample
        self.n = sample.n

    def _upload_zcs(self, sample):
        """Zcs chain planes of a sample that has them (pwa_ctx_upload_zcs_events)."""
        if getattr(sample, "pp3", None) is None:
            return
        pp3 = np.ascontiguousarray(sample.pp3, np.float32)
        pp4 = np.ascontiguousarray(sample.pp4, np.float32)
        check(self.L.pwa_ctx_upload_zcs_events(self.h, _f(pp3), _f(pp4)), "pwa_ctx_upload_zcs_events")

    def set_smearing(self, mode: str = "reference", sigma: float = 0.0027, step: float = 0.0005,
                     half_bins: int = 17):
        """Resolution model of m(J/psi p) (pwa_ctx_set_smearing): "reference" (the reference's bands
        and quantile schemes) or "gauss" (every event, Gaussian of width sigma GeV on a grid of
        2 half_bins + 1 offsets spaced step GeV)."""
        modes = {"reference": 0, "gauss": 1}
        check(self.L.pwa_ctx_set_smearing(self.h, modes[mode], sigma, step, half_bins), "pwa_ctx_set_smearing")

    def select_data(self, first: int, n_data: int, nda_smr: int, nda_fine: int):
        """Evaluate only the data events [first, first + n_data) with all MC (pwa_ctx_select_data);
        n_data < 0 selects all data again."""
        check(self.L.pwa_ctx_select_data(self.h, first, n_data, nda_smr, nda_fine), "pwa_ctx_select_data")

    def upload_unsorted(self, sample):
        """Upload a Sample whose data events are in any order (pwa_ctx_upload_events_unsorted): the
        library sorts them into the m(J/psi p) bands and derives the band arguments itself."""
        pp = np.ascontiguousarray(sample.pp, np.float32)
        pp1 = np.ascontiguousarray(sample.pp1, np.float32)
        pp2 = np.ascontiguousarray(sample.pp2, np.float32)
        sw = np.ascontiguousarray(sample.sw, np.float32)
        check(self.L.pwa_ctx_upload_events_unsorted(self.h, _f(pp), _f(pp1), _f(pp2), _f(sw), sample.n,
                                                    sample.n_size, sample.nda), "pwa_ctx_upload_events_unsorted")
        self._upload_zcs(sample)
        self.sample = sample
        self.n = sample.n

    def bind_device(self, dsample, nda_smr: int | None = None, nda_fine: int | None = None):
        """Use a DeviceSample's torch-owned planes (borrowed; the sample must outlive the binding)."""
        a, b = dsample.reference_band_args()
        a = a if nda_smr is None else nda_smr
        b = b if nda_fine is None else nda_fine
        check(self.L.pwa_ctx_set_device_events(self.h, dsample.pp.data_ptr(), dsample.pp1.data_ptr(),
                                               dsample.pp2.data_ptr(), dsample.sw.data_ptr(), dsample.n,
                                               dsample.n_size, dsample.nda, a, b), "pwa_ctx_set_device_events")
        self.sample = dsample
        self.n = dsample.n

    def bind_planes(self, pp, pp1, pp2, sw, n: int, n_size: int, nda: int = 0, nda_smr: int = -1, nda_fine: int = 0):
        """Use device planes given as torch tensors (borrowed)."""
        check(self.L.pwa_ctx_set_device_events(self.h, pp.data_ptr(), pp1.data_ptr(), pp2.data_ptr(), sw.data_ptr(),
                                               n, n_size, nda, nda_smr, nda_fine), "pwa_ctx_set_device_events")
        self.sample = None
        self.n = n

    def eval_nll(self, block, nll_shift: float = 1e7, want_fx: bool = False):
        s = self.sample
        pl = np.ascontiguousarray(block.data, np.float32)
        r = PwaResult()
        fx = np.zeros(s.n, np.float64) if want_fx else None
        check(self.L.pwa_ctx_eval_nll(self.h, _f(pl), block.para_size, block.vamp_size, block.spline_size, block.NR,
                                      block.NZ, block.NX, block.ffr, block.ffb, s.sum_w_mc, s.sum_w_data, nll_shift,
                                      C.byref(r), fx.ctypes.data_as(_dp) if want_fx else None), "pwa_ctx_eval_nll")
        return (r, fx) if want_fx else r

    def eval_nll_batch(self, blocks, nll_shift: float = 1e7):
        """Likelihood at several parameter points of one model in one call (pwa_ctx_eval_nll_batch).
        blocks: ParamBlocks with equal sizes; returns (results, number of points evaluated together
        from the first point's per-event terms)."""
        s = self.sample
        b0 = blocks[0]
        stride = len(b0.data)
        for b in blocks:
            if len(b.data) != stride or (b.para_size, b.vamp_size, b.NR, b.NZ) != (b0.para_size, b0.vamp_size,
                                                                                    b0.NR, b0.NZ):
                raise PwaError("eval_nll_batch: parameter blocks of different models")
        pl = np.ascontiguousarray(np.stack([np.asarray(b.data, np.float32) for b in blocks]))
        res = (PwaResult * len(blocks))()
        ns = C.c_int()
        check(self.L.pwa_ctx_eval_nll_batch(self.h, _f(pl), len(blocks), stride, b0.para_size, b0.vamp_size,
                                            b0.spline_size, b0.NR, b0.NZ, b0.NX, b0.ffr, b0.ffb, s.sum_w_mc,
                                            s.sum_w_data, nll_shift, res, C.byref(ns)), "pwa_ctx_eval_nll_batch")
        return list(res), ns.value

    def last_batch_ms(self) -> float:
        return self.L.pwa_ctx_last_batch_ms(self.h)

    def mc_integral(self, block) -> float:
        """Sum over the MC events of w * unsmeared |A|^2 (pwa_ctx_mc_integral)."""
        pl = np.ascontiguousarray(block.data, np.float32)
        out = C.c_double()
        check(self.L.pwa_ctx_mc_integral(self.h, _f(pl), block.para_size, block.vamp_size, block.spline_size,
                                         block.NR, block.NZ, block.NX, block.ffr, block.ffb, C.byref(out)),
              "pwa_ctx_mc_integral")
        return out.value

    def amp2(self, block) -> np.ndarray:
        pl = np.ascontiguousarray(block.data, np.float32)
        out = np.zeros(self.n, np.float64)
        check(self.L.pwa_ctx_amp2(self.h, _f(pl), block.para_size, block.vamp_size, block.spline_size, block.NR,
                                  block.NZ, block.NX, block.ffr, block.ffb, out.ctypes.data_as(_dp)), "pwa_ctx_amp2")
        return out

    def set_batch_waves(self, kind: int, waves: int):
        """Waves of resident blocks for the batched passes over event class `kind`."""
        check(self.L.pwa_ctx_set_batch_waves(self.h, int(kind), int(waves)), "pwa_ctx_set_batch_waves")

    def set_kmatrix(self, isospin: bool):
        """Coupled-channel K-matrix: the 7-channel isospin split (True) or the 4-channel default."""
        check(self.L.pwa_ctx_set_kmatrix(self.h, int(bool(isospin))), "pwa_ctx_set_kmatrix")

    def set_event_order(self, by_mass: bool):
        """Walk each MC event class by m(J/psi p) (True) or by event index (False, the default)."""
        check(self.L.pwa_ctx_set_event_order(self.h, int(bool(by_mass))), "pwa_ctx_set_event_order")

    def set_lineshape_tables(self, on: bool = True):
        check(self.L.pwa_ctx_set_lineshape_tables(self.h, int(on)), "pwa_ctx_set_lineshape_tables")

    def set_timing(self, on: bool = True):
        check(self.L.pwa_ctx_set_timing(self.h, int(on)), "pwa_ctx_set_timing")

    def segments(self) -> list:
        """[(kind, events, last_ms)] of the event-class kernels of the last evaluation."""
        out = []
        for i in range(self.L.pwa_ctx_segment_count(self.h)):
            k, n, ms = C.c_int(), C.c_int64(), C.c_double()
            check(self.L.pwa_ctx_segment_info(self.h, i, C.byref(k), C.byref(n), C.byref(ms)), "segment_info")
            out.append((k.value, n.value, ms.value))
        return out

    def batch_segment_ms(self) -> list:
        """Device time (ms) per segment of the last batched evaluation with timing on."""
        out = []
        for i in range(self.L.pwa_ctx_segment_count(self.h)):
            ms = C.c_double()
            check(self.L.pwa_ctx_batch_segment_ms(self.h, i, C.byref(ms)), "batch_segment_ms")
            out.append(ms.value)
        return out

    def segments_deferred(self) -> list:
        """Events per segment the last timed evaluation deferred to the exact pass."""
        out = []
        for i in range(self.L.pwa_ctx_segment_count(self.h)):
            d = C.c_int64()
            check(self.L.pwa_ctx_segment_deferred(self.h, i, C.byref(d)), "segment_deferred")
            out.append(d.value)
        return out

    def stream(self) -> int:
        return self.L.pwa_ctx_stream(self.h) or 0

    def last_kernel_ms(self) -> float:
        return self.L.pwa_ctx_last_kernel_ms(self.h)

    def last_launches(self) -> int:
        return self.L.pwa_ctx_last_launches(self.h)


def host_lineshapes(block, mkp: float, mz: float, isospin: bool = False):
    """Decoded Lambda* and Pc lineshapes (times production barriers) evaluated on the host; isospin: the
    7-channel isospin-split K-matrix."""
    L = load()
    pl = np.ascontiguousarray(block.data, np.float32)
    ls = np.zeros(2 * max(block.NR, 1))
    pc = np.zeros(2 * max(block.NZ, 1))
    check(L.pwa_host_lineshapes_km(_f(pl), block.para_size, block.vamp_size, block.spline_size, block.NR, block.NZ,
                                   block.NX, block.ffr, block.ffb, int(bool(isospin)), mkp, mz,
                                   ls.ctypes.data_as(_dp), pc.ctypes.data_as(_dp)), "pwa_host_lineshapes_km")
    return ls[0::2][:block.NR] + 1j * ls[1::2][:block.NR], pc[0::2][:block.NZ] + 1j * pc[1::2][:block.NZ]


def lineshapes_lstar_km(block, mkp, device: int = 0) -> tuple:
    """pwa_lineshapes_lstar_km (the reference's host_store_lineshapeLsKM on the device): revised K-matrix
    and Breit-Wigner lineshape of every Lambda* entry, each times the Lambda_b barrier with radius FFR,
    as complex [NR, n] arrays."""
    L = load()
    m = np.ascontiguousarray(mkp, np.float32)
    n, nr = len(m), block.NR
    out = [np.zeros(n * nr) for _ in range(4)]
    pl = np.ascontiguousarray(block.data, np.float32)
    check(L.pwa_lineshapes_lstar_km(device, _f(m), n, nr, block.ffr, _f(pl), block.para_size,
                                    *[o.ctypes.data_as(_dp) for o in out]), "pwa_lineshapes_lstar_km")
    return (out[0] + 1j * out[1]).reshape(nr, n), (out[2] + 1j * out[3]).reshape(nr, n)
