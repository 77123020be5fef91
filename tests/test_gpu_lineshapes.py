"""Spline waves, revised K-matrices and the triangle cusp on the GPU (model `lineshapes`) against the
FP64 oracle: the likelihood, per-event |A|^2, gradient batches whose points move those lineshapes'
parameters, and the Lambda* lineshape diagnostic (host_store_lineshapeLsKM)."""
import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu

NLL_TOL = 1e-6  # FP64 GPU vs FP64 oracle


def _per_event_agreement(g, o):
    """FP64 against FP64.  The triangle cusp reaches every event and sets the level: its integrand
    (t1 - t2) / sqrt(4c - b^2) is a difference of two arctangents of nearly equal arguments, so the
    last-bit differences between the host's and the device's acos and log grow to ~1e-10 relative
    (1e-12 for the other lineshapes), and to a few 1e-6 where one of its 100 bins has 4c - b^2 close
    to zero; those events are few and stay within 1e-3."""
    rel = np.abs(g - o) / np.abs(o)
    assert np.median(rel) < 1e-8 and np.percentile(rel, 99) < 1e-6 and np.max(rel) < 1e-3, (
        np.median(rel), np.percentile(rel, 99), np.max(rel))


@pytest.fixture(scope="module")
def sample():
    return make_test_sample("lineshapes", 1200, 12000, seed=17)


def test_nll_and_fx_match_oracle(sample, oracle_mod):
    from pwa_b200 import lib
    mdl, vals, blk, smp = sample
    v, s, fx, _ = oracle_mod.nll(smp, blk)
    ctx = lib.Context(0)
    try:
        ctx.upload(smp)
        r, gfx = ctx.eval_nll(blk, want_fx=True)
        assert abs(r.nll - v) < NLL_TOL and abs(r.sumint / s - 1) < 1e-8
        _per_event_agreement(gfx, fx)
        ctx.set_lineshape_tables(False)  # exact lineshapes at every lookup give the same
        assert abs(ctx.eval_nll(blk).nll - v) < NLL_TOL
    finally:
        ctx.close()


def test_amp2_matches_oracle(sample, oracle_mod):
    from pwa_b200 import lib
    mdl, vals, blk, smp = sample
    ctx = lib.Context(0)
    try:
        ctx.upload(smp)
        a = ctx.amp2(blk)
    finally:
        ctx.close()
    o = oracle_mod.amp2(smp, blk)
    nz = o != 0
    assert np.all(a[~nz] == 0)
    _per_event_agreement(a[nz], o[nz])


def test_gradient_batch_over_new_lineshapes(sample, oracle_mod):
    """Points that move a Lambda* spline knot, a Pc spline knot, a Lambda* and a Pc revised K-matrix
    mass (which moves the whole set's lineshapes), the cusp's loop mass and couplings of each entry:
    batched vs one by one, and a subset against the oracle."""
    from pwa_b200 import gradient, lib
    mdl, vals, blk, smp = sample
    names = ["SR_S01_05", "SI_S01_12", "SR_ZS01_04", "m0_1405", "width_1670", "m0_Z4440", "width_Z4457",
             "m0_T4337", "a_p1p1_1670", "a_L0_Z4440", "a_L0_T4337", "a_Bp_ZS01", "scRe"]
    labels, blocks = gradient.gradient_blocks(mdl, vals, names=names)
    ctx = lib.Context(0)
    try:
        ctx.upload(smp)
        res, nstruct = ctx.eval_nll_batch(blocks)
        single = [ctx.eval_nll(b).nll for b in blocks]
    finally:
        ctx.close()
    assert nstruct >= len(blocks) // 2  # most points are formed from the centre's per-event terms
    assert np.max(np.abs(np.array([r.nll for r in res]) - np.array(single))) < NLL_TOL
    for i in (0, 1, 5, 7, 11, 15):
        assert abs(res[i].nll - oracle_mod.nll(smp, blocks[i])[0]) < NLL_TOL, labels[i]


def test_lineshape_diagnostic_on_device(oracle_mod):
    """pwa_lineshapes_lstar_km (the reference's host_store_lineshapeLsKM) against the oracle's FP64
    restatement, and against the reference's own FP32 function where its host build is present."""
    from pwa_b200 import configs, lib, model as M
    mdl, vals = configs.lineshapes()
    blk = M.build_param_block(mdl, vals)
    m = np.linspace(1.44, 2.5, 96).astype(np.float32)
    km, bw = lib.lineshapes_lstar_km(blk, m)
    km_o, bw_o = oracle_mod.lineshapes_lstar_km(blk, m)
    for g, o in ((km, km_o), (bw, bw_o)):
        fin = np.isfinite(o)
        assert np.array_equal(fin, np.isfinite(g))
        assert np.allclose(g[fin], o[fin], rtol=1e-12, atol=0)
    if oracle_mod.ref_lib(blk.NR, blk.NZ, blk.NX, build_if_missing=False) is not None:
        km_r, _ = oracle_mod.ref_lineshapes_lstar_km(blk, m)
        fin = np.isfinite(km_o)
        assert np.max(np.abs(km_r[fin] - km[fin]) / np.abs(km[fin])) < 2e-5
