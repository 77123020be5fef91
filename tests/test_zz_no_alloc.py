"""The allocation-free entry point pwa_eval_nll_noalloc against the context entry point.

pwa_eval_nll_noalloc serves callers that must not allocate device memory during a fit (their
process's GPU memory belongs to another framework's caching allocator, or they run under a fixed
device-memory budget): all of its scratch is a fixed array inside the library.  This file runs last
so that a failure here leaves every other test already run; it passes in a fresh process too."""
import ctypes as C

import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu

NLL_TOL = 1e-6  # the FP64 parity tolerance of the GPU tests


def _noalloc(L, planes, smp, blk, band, stream=None):
    import torch  # noqa: F401
    from pwa_b200 import lib
    pp, pp1, pp2, sw = planes
    r = lib.PwaResult()
    pl = np.ascontiguousarray(blk.data, np.float32)
    rc = L.pwa_eval_nll_noalloc(0, C.c_void_p(pp.data_ptr()), C.c_void_p(pp1.data_ptr()),
                                C.c_void_p(pp2.data_ptr()), C.c_void_p(sw.data_ptr()), smp.n, smp.n_size, smp.nda,
                                band[0], band[1], pl.ctypes.data_as(C.POINTER(C.c_float)), blk.para_size,
                                blk.vamp_size, blk.spline_size, blk.NR, blk.NZ, blk.NX, C.c_float(blk.ffr),
                                C.c_float(blk.ffb), C.c_double(smp.sum_w_mc), C.c_double(smp.sum_w_data),
                                C.c_double(1e7), stream, C.byref(r))
    return rc, r


def _bind(L):
    from pwa_b200 import lib
    L.pwa_eval_nll_noalloc.restype = C.c_int
    L.pwa_eval_nll_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int64,
                                       C.c_int64, C.c_int64, C.c_int64, C.POINTER(C.c_float), C.c_int, C.c_int,
                                       C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_double,
                                       C.c_double, C.c_double, C.c_void_p, C.POINTER(lib.PwaResult)]
    return L


@pytest.mark.parametrize("name,nd,nm", [("small_kmatrix", 1500, 15000), ("kmatrix", 1200, 12000)])
def test_noalloc_matches_context_entry_point_twice(name, nd, nm):
    import torch
    from pwa_b200 import lib
    L = _bind(lib.load())
    mdl, vals, blk, smp = make_test_sample(name, nd, nm)
    planes = [torch.as_tensor(a, device="cuda") for a in (smp.pp, smp.pp1, smp.pp2, smp.sw)]
    band = smp.reference_band_args()
    ctx = lib.Context(0)
    ctx.upload(smp)
    want = ctx.eval_nll(blk)
    ctx.close()
    torch.cuda.synchronize()
    for i in range(2):  # consecutive calls share the library's scratch array
        free0 = torch.cuda.mem_get_info()[0]
        rc, got = _noalloc(L, planes, smp, blk, band)
        assert rc == 0, lib.load().pwa_error_string(rc)
        if i == 1:  # after the first call (which loads the module on this device) no memory is taken
            assert torch.cuda.mem_get_info()[0] == free0
        assert abs(got.nll - want.nll) < NLL_TOL
        assert abs(got.sumint / want.sumint - 1) < 1e-12 and abs(got.sum_noint / want.sum_noint - 1) < 1e-12
        assert got.n_nonpos == want.n_nonpos


def test_noalloc_on_a_torch_stream_and_empty_sample():
    """Work queued on a caller's stream gives the same result; an empty sample after a full one
    returns zero sums, not the previous call's partials left in the shared array."""
    import copy
    import torch
    from pwa_b200 import lib
    L = _bind(lib.load())
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    planes = [torch.as_tensor(a, device="cuda") for a in (smp.pp, smp.pp1, smp.pp2, smp.sw)]
    band = smp.reference_band_args()
    rc, want = _noalloc(L, planes, smp, blk, band)
    assert rc == 0
    s = torch.cuda.Stream()
    rc, got = _noalloc(L, planes, smp, blk, band, stream=C.c_void_p(s.cuda_stream))
    assert rc == 0, lib.load().pwa_error_string(rc)
    assert abs(got.nll - want.nll) < NLL_TOL and abs(got.sumint / want.sumint - 1) < 1e-12
    empty = copy.copy(smp)
    empty.n, empty.nda = 0, 0
    rc, got = _noalloc(L, planes, empty, blk, (-1, 0))
    assert rc == 0, lib.load().pwa_error_string(rc)
    assert got.sumint == 0.0 and got.sum_noint == 0.0 and got.data_term == 0.0


def test_noalloc_rejects_oversize_sample():
    import torch
    from pwa_b200 import lib
    L = _bind(lib.load())
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    planes = [torch.as_tensor(a, device="cuda") for a in (smp.pp, smp.pp1, smp.pp2, smp.sw)]
    import copy
    big = copy.copy(smp)
    big.n = (1 << 20) + 1
    big.n_size = big.n + 31
    rc, _ = _noalloc(L, planes, big, blk, (-1, 0))
    assert rc == 4  # PWA_E_SIZE, before any device work
