"""The 7-channel isospin-split K-matrix (Isospin_KMatrix, src/cu_DPFPropogator.cu:384-586, the
reference's ISOSPIN_SIGMACD build), no GPU: the FP64 oracle's restatement against the reference's own
FP32 code built with the switch on, and the library's decoded lineshapes (the device code run on the
host) against the oracle."""
import numpy as np
import pytest

from conftest import make_test_sample


@pytest.fixture
def isospin(oracle_mod):
    oracle_mod.set_kmatrix_isospin(True)
    yield
    oracle_mod.set_kmatrix_isospin(False)


def test_oracle_vs_reference_isospin_build(oracle_mod, isospin):
    L = oracle_mod.ref_lib(3, 4, 0, build_if_missing=True, isospin=True)
    if L is None:
        pytest.skip("reference host build unavailable")
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 600, 6000, seed=31)
    v, s, fx, _ = oracle_mod.nll(smp, blk)
    ref = oracle_mod.RefHost(smp, blk, isospin=True)
    rv, rs = ref.store_fx(blk)
    rel = np.abs(ref.fx - fx) / np.abs(fx)
    # the reference computes in FP32 (its solve in FP64): float rounding, with the larger deviations on
    # the steep structures near the channel thresholds, as for the 4-channel K-matrix
    assert np.median(rel) < 1e-5 and np.max(rel) < 2e-3, (np.median(rel), np.max(rel))
    assert abs(rv - v) < 0.05
    # and the isospin split is a different model: the default K-matrix is far off both
    oracle_mod.set_kmatrix_isospin(False)
    v0, _, _, _ = oracle_mod.nll(smp, blk)
    assert abs(v0 - rv) > 100 * abs(rv - v)


def test_library_lineshapes_match_oracle(oracle_mod, isospin):
    """Pc lineshapes of the decoded point table (pole shifts of channels 1 and 3, the 7 x 7 solve, the
    folding onto the production channels) at masses across the thresholds of all seven channels."""
    from pwa_b200 import configs, lib, model as M
    mdl, vals = configs.small_kmatrix()
    blk = M.build_param_block(mdl, vals)
    worst = 0.0
    for mz in np.linspace(4.05, 5.1, 211):
        _, pc = lib.host_lineshapes(blk, 1.6, float(mz), isospin=True)
        _, po = oracle_mod.lineshapes(blk, 1.6, float(mz))
        worst = max(worst, float(np.max(np.abs(pc - po) / (np.abs(po) + 1e-300))))
        _, p0 = lib.host_lineshapes(blk, 1.6, float(mz), isospin=False)
        if mz > 4.3:
            assert np.max(np.abs(p0 - po)) > 1e-6 * np.max(np.abs(po))
    assert worst < 1e-11, worst


def test_unacceptable_pole_channel_is_refused():
    """A K-matrix pole of channel 2 has no near-threshold shift in the isospin split: the reference prints
    an error and reads an unset mass; the decoder refuses the block."""
    from pwa_b200 import configs, lib, model as M
    mdl, vals = configs.small_kmatrix()
    for r in mdl.resonances:
        if r.name == "Pc4457":
            r.width = 2.0  # the WIDTH slot holds iChannel for a K-matrix pole
    blk = M.build_param_block(mdl, vals)
    with pytest.raises(Exception):
        lib.host_lineshapes(blk, 1.6, 4.4, isospin=True)
    lib.host_lineshapes(blk, 1.6, 4.4, isospin=False)
