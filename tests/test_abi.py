"""The C ABI library: loads, exports every symbol the headers declare, host-side diagnostics."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT
from pwa_b200 import configs, lib, model as M


def _declared(header):
    txt = (ROOT / "include" / header).read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return set(re.findall(r"\b(pwa_\w+)\s*\(", txt))


def test_exports_every_declared_symbol():
    L = lib.load()
    names = _declared("pwa_b200.h")
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib.LIB_PATH)], capture_output=True, text=True).stdout
    for mangled in ("_Z13host_store_fxSt6vectorIPfSaIS0_EES2_S2_S2_S2_S2_S0_iiiPdiiiiiiiiRdddffb",
                    "_Z14cu_malloc_h_ppPfRS_ii", "_Z10cu_Free_ppSt6vectorIPfSaIS0_EES2_S2_S2_S2_",
                    "_Z25cuda_configure_Pc_KMatrixPKf", "_Z23cuda_configure_ampcountPKfi", "_Z20cuda_configure_smearv",
                    "_Z16host_store_amp2sSt6vectorIPfSaIS0_EES2_S2_S2_S2_S0_iiiPdiiiiiff",
                    "_Z24host_store_lineshapeLsKMPKfPfS1_S1_S1_iiifS1_iii"):
        assert mangled in out, mangled


@pytest.mark.parametrize("name", ["kmatrix", "small_kmatrix", "full_bw"])
def test_host_lineshapes_match_oracle(name, oracle_mod):
    mdl, vals = configs.MODELS[name]()
    b = M.build_param_block(mdl, vals)
    O = oracle_mod.lib()
    dp = C.POINTER(C.c_double)
    for mkp, mz in [(1.52, 4.312), (1.8, 4.4401), (2.2, 4.52), (1.6, 4.4575), (2.0, 4.3206), (1.9, 4.462)]:
        ls, pc = lib.host_lineshapes(b, mkp, mz)
        slots = [0, 0, 0, 0]
        for r in range(b.NR):
            q = b.data[6 * r:6 * r + 6]
            o = np.zeros(2)
            O.oracle_bw_lstar(float(q[0]), float(q[1]), mkp, int(q[3]), b.ffr, o.ctypes.data_as(dp))
            ref = complex(*o) * O.oracle_barrier_lb_lstar(0.5 * q[2], mkp, float(q[0]), b.ffb)
            assert abs(ls[r] - ref) <= 1e-12 * abs(ref)
        for i in range(b.NZ):
            q = b.data[6 * (b.NR + i):6 * (b.NR + i) + 6]
            if int(q[4]) == 240:
                ik = (3 if q[2] == 3 else 2) if q[3] > 0 else (1 if q[2] == 3 else 0)
                o = np.zeros(16)
                O.oracle_kmatrix(oracle_mod._f(b.data), b.para_size, b.vamp_size, 0, b.NR, b.NZ, b.ffb, mz, ik,
                                 o.ctypes.data_as(dp))
                v = complex(o[2 * slots[ik]], o[2 * slots[ik] + 1])
                slots[ik] += 1
            else:
                o = np.zeros(2)
                O.oracle_bw_pc(float(q[0]), float(q[1]), mz, int(q[3]), b.ffr, o.ctypes.data_as(dp))
                v = complex(*o)
            ref = v * O.oracle_barrier_lb_pc(0.5 * q[2], mz, float(q[0]), b.ffb)
            assert abs(pc[i] - ref) <= 1e-12 * abs(ref)


def test_error_codes():
    mdl, vals = configs.small_kmatrix()
    b = M.build_param_block(mdl, vals)
    L = lib.load()
    d = np.zeros(64)
    dp = C.POINTER(C.c_double)
    pl = np.ascontiguousarray(b.data)
    args = (b.para_size, b.vamp_size, 0, b.NR, b.NZ)
    f = lib._f(pl)
    bad = pl.copy()
    bad[4] = 2  # Flatte Lambda* lineshape: the reference kernels have no case for it
    assert L.pwa_host_lineshapes(lib._f(bad), *args, 0, b.ffr, b.ffb, 1.5, 4.4, d.ctypes.data_as(dp),
                                 d.ctypes.data_as(dp)) == 5
    bad[4] = 3  # a spline wave without its spline block
    assert L.pwa_host_lineshapes(lib._f(bad), *args, 0, b.ffr, b.ffb, 1.5, 4.4, d.ctypes.data_as(dp),
                                 d.ctypes.data_as(dp)) == 3
    assert L.pwa_host_lineshapes(f, *args, 1, b.ffr, b.ffb, 1.5, 4.4, d.ctypes.data_as(dp),
                                 d.ctypes.data_as(dp)) == 3  # a Zcs entry without its table row
    mz_, vz = configs.small_zcs()
    bz = M.build_param_block(mz_, vz)
    pz = np.ascontiguousarray(bz.data)
    assert L.pwa_host_lineshapes(lib._f(pz), bz.para_size, bz.vamp_size, 0, bz.NR, bz.NZ, bz.NX, bz.ffr, bz.ffb,
                                 1.5, 4.4, d.ctypes.data_as(dp), d.ctypes.data_as(dp)) == 0
    assert L.pwa_host_lineshapes(f, b.para_size + 6, b.vamp_size, 0, b.NR, b.NZ, 0, b.ffr, b.ffb, 1.5, 4.4,
                                 d.ctypes.data_as(dp), d.ctypes.data_as(dp)) == 3  # layout
    assert L.pwa_host_lineshapes(f, b.para_size, b.vamp_size - 2, 0, b.NR, b.NZ, 0, b.ffr, b.ffb, 1.5, 4.4,
                                 d.ctypes.data_as(dp), d.ctypes.data_as(dp)) == 3
    assert L.pwa_host_lineshapes(None, *args, 0, b.ffr, b.ffb, 1.5, 4.4, d.ctypes.data_as(dp),
                                 d.ctypes.data_as(dp)) == 2
    assert lib.load().pwa_error_string(5).decode().startswith("lineshape")


def test_band_order_matches_reorder_semantics():
    """pwa_band_order (host, no GPU) against the numpy restatement of reOrder.C."""
    import numpy as np
    from pwa_b200 import basis as B, lib
    rng = np.random.default_rng(3)
    mz = rng.uniform(4.05, 4.9, 5000).astype(np.float32)
    order, n1, n2 = lib.band_order(mz)
    ref = B.order_data_by_band(mz)
    assert np.array_equal(order, ref)
    b = B.band_of(mz)
    assert n1 == int(np.sum(b == 1)) and n2 == int(np.sum(b == 2))


def test_decoded_lineshapes_of_every_type_match_oracle(oracle_mod):
    """The decoded point table's lineshapes (spline waves, revised K-matrices, the triangle cusp, next to
    Breit-Wigners), evaluated on the host by the same functions the kernels use, against the FP64
    oracle over the kinematic ranges (cusp masses away from its branch jumps: both are FP64, so they
    only differ where one side rounds across a jump, which a scan does not hit)."""
    mdl, vals = configs.lineshapes()
    b = M.build_param_block(mdl, vals)
    for mkp, mz in zip(np.linspace(1.433, 2.52, 97), np.linspace(4.036, 5.125, 97)):
        ls, pc = lib.host_lineshapes(b, float(mkp), float(mz))
        ols, opc = oracle_mod.lineshapes(b, float(mkp), float(mz))
        assert np.allclose(ls, ols, rtol=1e-12, atol=1e-300), (mkp, ls, ols)
        assert np.allclose(pc, opc, rtol=1e-11, atol=1e-300), (mz, pc, opc)
