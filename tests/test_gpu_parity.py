"""GPU likelihood vs the FP64 oracle on identical seeded inputs (calls through the C ABI)."""
import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu

# FP64 on both sides: the tolerance covers summation-order differences only.
NLL_TOL = 1e-6
FX_RTOL = 1e-9

CASES = [("small_kmatrix", 1500, 15000), ("small_bw", 1500, 15000), ("lstar_only", 1000, 10000),
         ("kmatrix", 1200, 12000), ("full_bw", 800, 8000), ("small_zcs", 1500, 15000)]


@pytest.fixture(scope="module")
def ctx():
    from pwa_b200 import lib
    c = lib.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name,nd,nm", CASES)
def test_nll_and_fx_match_oracle(ctx, oracle_mod, name, nd, nm):
    mdl, vals, blk, smp = make_test_sample(name, nd, nm)
    ctx.upload(smp)
    r, fx = ctx.eval_nll(blk, want_fx=True)
    v, s, ofx, ofxn = oracle_mod.nll(smp, blk)
    rel = np.abs(fx - ofx) / np.maximum(np.abs(ofx), 1e-300)
    assert np.max(rel) < FX_RTOL, (name, np.max(rel), int(np.argmax(rel)))
    assert abs(r.nll - v) < NLL_TOL, (name, r.nll, v)
    assert abs(r.sumint / s - 1) < 1e-12
    assert r.n_nonpos == 0


@pytest.mark.parametrize("name", ["small_kmatrix", "small_zcs"])
def test_amp2_matches_oracle(ctx, oracle_mod, name):
    mdl, vals, blk, smp = make_test_sample(name, 1500, 15000)
    ctx.upload(smp)
    a = ctx.amp2(blk)
    o = oracle_mod.amp2(smp, blk)
    assert np.max(np.abs(a - o) / o) < FX_RTOL


def test_band_edges_and_ragged_sizes(ctx, oracle_mod):
    """Band arguments at the edges (no band-1 events, -1 shift, bands covering everything) and
    sizes not multiple of the tile/warp widths."""
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 700, 5013, seed=5)
    for a, b in [(-1, 0), (0, 0), (smp.nda_smr1 - 1, smp.nda_fine), (smp.nda_smr1, smp.nda_fine),
                 (smp.nda, 0), (-1, smp.nda_fine + 3), (37, 1)]:
        ctx.upload(smp, a, b)
        r, fx = ctx.eval_nll(blk, want_fx=True)
        ofx, ofxn = oracle_mod.eval_fx(smp, blk, a, b)
        v, s = oracle_mod.assemble_nll(smp, ofx, ofxn)
        assert np.max(np.abs(fx - ofx) / np.abs(ofx)) < FX_RTOL, (a, b)
        assert abs(r.nll - v) < NLL_TOL, (a, b)


def test_repeated_calls_identical(ctx):
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    ctx.upload(smp)
    a = ctx.eval_nll(blk).nll
    b = ctx.eval_nll(blk).nll
    assert a == b


def test_lineshape_tables_match_exact_solves(ctx, oracle_mod):
    """K-matrix tables (interpolated) against solving the K-matrix for every lookup, and the oracle."""
    mdl, vals, blk, smp = make_test_sample("kmatrix", 3000, 40000, seed=17)
    ctx.upload(smp)
    ctx.set_lineshape_tables(False)
    r0, fx0 = ctx.eval_nll(blk, want_fx=True)
    ctx.set_lineshape_tables(True)
    r1, fx1 = ctx.eval_nll(blk, want_fx=True)
    assert np.max(np.abs(fx1 - fx0) / np.abs(fx0)) < 1e-10
    assert abs(r1.nll - r0.nll) < 1e-7
    v, s, ofx, _ = oracle_mod.nll(smp, blk)
    assert abs(r1.nll - v) < NLL_TOL


@pytest.mark.parametrize("name", ["small_kmatrix", "small_zcs"])
def test_unsorted_upload_matches_sorted(ctx, name):
    """Data in shuffled order through pwa_ctx_upload_events_unsorted: same NLL as the band-sorted
    upload, per-event fx returned in the caller's order (Zcs planes permuted alike)."""
    import copy
    mdl, vals, blk, smp = make_test_sample(name, 1500, 15000)
    ctx.upload(smp)
    r0, fx0 = ctx.eval_nll(blk, want_fx=True)
    rng = np.random.default_rng(4)
    perm = rng.permutation(smp.nda)
    # the reference's caller passes the band-1 count minus one, so the last band-1 event by position is
    # evaluated with 150 offsets and the last band-2 event with 20 (tail window): keep both last in
    # their bands
    last1, last2 = smp.nda_smr1 - 1, smp.nda_smr1 + smp.nda_fine - 1
    perm = np.concatenate([perm[(perm != last1) & (perm != last2)], [last1, last2]])
    sh = copy.copy(smp)
    ns = smp.n_size
    for plane, planes in (("pp", 111), ("pp1", 96), ("pp2", 96), ("pp3", 97), ("pp4", 96)):
        if getattr(smp, plane, None) is None:
            continue
        a = np.array(getattr(smp, plane), np.float32).reshape(planes, ns).copy()
        a[:, :smp.nda] = a[:, perm]
        setattr(sh, plane, a.reshape(-1))
    sw = np.array(smp.sw, np.float32).copy()
    sw[:smp.nda] = sw[perm]
    sh.sw = sw
    ctx.upload_unsorted(sh)
    r1, fx1 = ctx.eval_nll(blk, want_fx=True)
    assert abs(r1.nll - r0.nll) < NLL_TOL
    assert np.array_equal(fx1[:smp.nda], fx0[perm])
    assert np.array_equal(fx1[smp.nda:], fx0[smp.nda:])
    ctx.upload(smp)


def test_zcs_terms_enter_and_need_their_planes(ctx, oracle_mod):
    """The Zcs chain changes the likelihood (same events, couplings of the Zcs entries zeroed), and a
    model with Zcs entries is refused when the events carry no Zcs planes."""
    import copy
    from pwa_b200 import lib, model as M
    mdl, vals, blk, smp = make_test_sample("small_zcs", 1500, 15000)
    ctx.upload(smp)
    r_on = ctx.eval_nll(blk)
    z = dict(vals)
    for res in mdl.zcs:
        for c in res.couplings:
            z[c] = 0.0
    blk0 = M.build_param_block(mdl, z)
    r_off = ctx.eval_nll(blk0)
    v_off, _, _, _ = oracle_mod.nll(smp, blk0)
    assert abs(r_off.nll - v_off) < NLL_TOL
    assert abs(r_on.nll - r_off.nll) > 1.0
    bare = copy.copy(smp)
    bare.pp3 = bare.pp4 = None
    ctx.upload(bare)
    with pytest.raises(lib.PwaError, match="no events"):
        ctx.eval_nll(blk)
    ctx.upload(smp)


@pytest.mark.parametrize("name", ["full_bw", "small_kmatrix", "small_zcs"])
def test_gaussian_grid_smearing_matches_oracle(ctx, oracle_mod, name):
    """Fixed-width Gaussian resolution (sigma 2.7 MeV on a 0.5 MeV grid, 35 offsets) on every event:
    per-event fx and NLL against the oracle's direct sum over offsets; back in reference mode the
    reference NLL returns unchanged."""
    mdl, vals, blk, smp = make_test_sample(name, 1000, 10000)
    ctx.upload(smp)
    r_ref = ctx.eval_nll(blk)
    ctx.set_smearing("gauss", 0.0027, 0.0005, 17)
    try:
        r, fx = ctx.eval_nll(blk, want_fx=True)
        ofx, ofxn = oracle_mod.eval_fx_grid(smp, blk, 0.0027, 0.0005, 17)
        v, s = oracle_mod.assemble_nll(smp, ofx, ofxn)
        rel = np.abs(fx - ofx) / np.abs(ofx)
        assert np.max(rel) < FX_RTOL, (name, np.max(rel), int(np.argmax(rel)))
        assert abs(r.nll - v) < NLL_TOL, (name, r.nll, v)
        assert abs(r.nll - r_ref.nll) > 1e-3  # the resolution model matters
    finally:
        ctx.set_smearing("reference")
    assert ctx.eval_nll(blk).nll == r_ref.nll


@pytest.mark.parametrize("name", ["small_kmatrix", "full_bw"])
def test_gaussian_grid_batch_and_arguments(ctx, name):
    """Gaussian resolution model: the batched gradient (every point formed from the centre) against
    one-by-one evaluation, and argument checks."""
    from pwa_b200 import gradient, lib
    mdl, vals, blk, smp = make_test_sample(name, 1500, 15000)
    ctx.upload(smp)
    ctx.set_smearing("gauss", 0.0027, 0.0005, 17)
    try:
        labels, blocks = gradient.gradient_blocks(mdl, vals)
        res, nstruct = ctx.eval_nll_batch(blocks)
        assert nstruct == len(blocks)  # the batched kernels take the weighted grid too
        for r, b in zip(res, blocks):
            assert abs(r.nll - ctx.eval_nll(b).nll) < NLL_TOL
        with pytest.raises(lib.PwaError):
            ctx.set_smearing("gauss", 0.0027, 0.0005, 64)  # 129 offsets
        with pytest.raises(lib.PwaError):
            ctx.set_smearing("gauss", -1.0, 0.0005, 17)
    finally:
        ctx.set_smearing("reference")
