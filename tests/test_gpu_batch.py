"""Batched evaluation at the 2N+1 points of Minuit's numerical gradient (pwa_ctx_eval_nll_batch)
against one-by-one evaluation of the same float parameter blocks, and against the FP64 oracle."""
import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu

# Both sides evaluate the same float parameter blocks in FP64; the batched path forms each point from
# the centre's per-event terms, so only the summation order differs.
NLL_TOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    from pwa_b200 import lib
    c = lib.Context(0)
    yield c
    c.close()


def _check_batch(ctx, name, nd, nm, tables=True, seed=0):
    from pwa_b200 import gradient
    mdl, vals, blk, smp = make_test_sample(name, nd, nm, seed=seed) if seed else make_test_sample(name, nd, nm)
    ctx.upload(smp)
    ctx.set_lineshape_tables(tables)
    labels, blocks = gradient.gradient_blocks(mdl, vals)
    res, nstruct = ctx.eval_nll_batch(blocks)
    one = [ctx.eval_nll(b).nll for b in blocks]
    diff = np.array([r.nll - o for r, o in zip(res, one)])
    worst = int(np.argmax(np.abs(diff)))
    assert np.max(np.abs(diff)) < NLL_TOL, (name, labels[worst], diff[worst])
    ctx.set_lineshape_tables(True)
    return labels, blocks, res, nstruct, smp


@pytest.mark.parametrize("name,nd,nm", [("small_kmatrix", 1500, 15000), ("small_bw", 1500, 15000),
                                        ("lstar_only", 1000, 8000), ("kmatrix", 1200, 12000),
                                        ("full_bw", 800, 8000)])
def test_gradient_batch_matches_single_points(ctx, name, nd, nm):
    labels, blocks, res, nstruct, smp = _check_batch(ctx, name, nd, nm)
    # every point of these models moves one part of the amplitude, and the points that move a Pc
    # lineshape (each with its own table, at most 128 per batch) are fewer than the table limit
    assert nstruct == len(blocks), (nstruct, len(blocks))


def test_gradient_batch_exact_lineshapes(ctx):
    """Tables off: every lineshape exact, no deferred pass."""
    _check_batch(ctx, "small_kmatrix", 1500, 15000, tables=False)


def test_batch_point_kinds_and_oracle(ctx, oracle_mod):
    """Points of every kind (Lambda* coupling and mass, Lambda* scale, Pc couplings shared by several
    K-matrix entries, K-matrix pole mass and coupling, scattering term) against the FP64 oracle, and a
    point that moves two parts at once (single-point path)."""
    from pwa_b200 import configs, model as M
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    ctx.upload(smp)
    moves = [{}, {"a_p1p1_1520": 0.01}, {"m0_1670": 1e-3}, {"scRe": 0.02}, {"a_L0_ZM1SC1": -0.02},
             {"g2_Pc4312": 0.01}, {"m0_Pc4457": 2e-4}, {"fsc_ZM1SC2": 0.05},
             {"a_p1p1_1520": 0.01, "m0_Pc4457": 2e-4}]
    blocks = []
    for mv in moves:
        v = dict(vals)
        for k, d in mv.items():
            v[k] = vals[k] + d
        blocks.append(M.build_param_block(mdl, v))
    res, nstruct = ctx.eval_nll_batch(blocks)
    assert nstruct == len(blocks) - 1
    for mv, b, r in zip(moves, blocks, res):
        o, _, _, _ = oracle_mod.nll(smp, b)
        assert abs(r.nll - o) < NLL_TOL, (mv, r.nll - o)


def test_batch_repeated_and_chunked(ctx):
    """More points than one launch takes (chunks), and identical results on a second call."""
    from pwa_b200 import model as M
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 600, 6000)
    ctx.upload(smp)
    rng = np.random.default_rng(7)
    names = [n for n in mdl.parameter_names() if n.startswith(("a_", "p_"))]
    blocks = [blk]
    for i in range(400):
        v = dict(vals)
        n = names[i % len(names)]
        v[n] = vals[n] + float(rng.normal(0, 0.01))
        blocks.append(M.build_param_block(mdl, v))
    r1, n1 = ctx.eval_nll_batch(blocks)
    r2, n2 = ctx.eval_nll_batch(blocks)
    assert n1 == n2 == len(blocks)
    assert [a.nll for a in r1] == [b.nll for b in r2]
    for i in (0, 1, 200, 399, 400):
        assert abs(r1[i].nll - ctx.eval_nll(blocks[i]).nll) < NLL_TOL


def test_gradient_batch_with_zcs_entries(ctx):
    """A model with Zcs entries: the centre's Lambda* amplitudes carry the Zcs terms, points that move a
    Lambda* or Pc parameter are formed from it, points that move a Zcs parameter go through the
    single-point path; every point matches one-by-one calls."""
    from pwa_b200 import configs
    labels, blocks, res, nstruct, smp = _check_batch(ctx, "small_zcs", 1500, 15000)
    mdl, _ = configs.small_zcs()
    zn = {ref for r in mdl.zcs for ref in (*r.couplings, *r.extra, r.mass, r.width) if isinstance(ref, str)}
    n_zcs = sum(1 for name, _ in labels if name in zn)
    # (a Zcs coupling that only fills slots the reference kernel does not read leaves the point equal to
    # the centre, so such points are formed from it as well)
    assert n_zcs > 0 and len(blocks) - n_zcs <= nstruct < len(blocks), (nstruct, len(blocks), n_zcs)


def test_mass_ordered_event_lists(ctx):
    """Walking the MC classes by m(J/psi p) (pwa_ctx_set_event_order) changes only the order of the
    sums: single points and the gradient batch equal the index-ordered results."""
    from pwa_b200 import gradient
    mdl, vals, blk, smp = make_test_sample("kmatrix", 1200, 12000)
    ctx.upload(smp)
    labels, blocks = gradient.gradient_blocks(mdl, vals)
    ref, _ = ctx.eval_nll_batch(blocks)
    ctx.set_event_order(True)
    try:
        res, _ = ctx.eval_nll_batch(blocks)
        assert np.max(np.abs(np.array([r.nll for r in res]) - [r.nll for r in ref])) < NLL_TOL
        assert abs(ctx.eval_nll(blk).nll - ref[0].nll) < NLL_TOL
    finally:
        ctx.set_event_order(False)


def test_batch_waves_and_tuner(ctx, tmp_path):
    """Wider grids (more waves of blocks per event class) only change the order of the sums; the batch
    tuner picks one per class, caches it, and a second call takes the cache."""
    from pwa_b200 import autotune, gradient
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    ctx.upload(smp)
    labels, blocks = gradient.gradient_blocks(mdl, vals)
    kinds = sorted({k for k, _, _ in ctx.segments()})
    ref, _ = ctx.eval_nll_batch(blocks)
    for w in (2, 4, 64):
        for k in kinds:
            ctx.set_batch_waves(k, w)
        res, _ = ctx.eval_nll_batch(blocks)
        diff = np.array([r.nll - o.nll for r, o in zip(res, ref)])
        assert np.max(np.abs(diff)) < NLL_TOL, (w, np.max(np.abs(diff)))
    with pytest.raises(Exception):
        ctx.set_batch_waves(kinds[0], 0)
    cache = tmp_path / "tune.json"
    first = autotune.tune_batch(ctx, blocks, cache=cache, reps=1)
    assert not first["cached"] and set(first["waves"]) == {str(k) for k in kinds}
    assert all(int(w) in autotune.BATCH_WAVES for w in first["waves"].values())
    second = autotune.tune_batch(ctx, blocks, cache=cache)
    assert second["cached"] and second["waves"] == first["waves"]
    res, _ = ctx.eval_nll_batch(blocks)
    assert max(abs(r.nll - o.nll) for r, o in zip(res, ref)) < NLL_TOL
    ctx.set_timing(False)
    for k in kinds:
        ctx.set_batch_waves(k, 1)
