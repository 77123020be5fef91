"""Toy ensembles fitted together (pwa_ens_*): every toy's NLL from the Gram matrix of the shared MC and
the ensemble kernel equals the single-point evaluator on that toy's window and the FP64 oracle on the
toy alone; the analytic gradient equals finite differences; the batched fit reaches the minima the
toy-by-toy fit (batched numerical gradient, Migrad-like) reaches; the autotuner caches its choice."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NLL_TOL = 1e-6  # FP64 against FP64


def _toys(model="small_kmatrix", sizes=(900, 2500, 400, 1600), n_mc=12000, seed=3):
    from pwa_b200 import configs, dataset as D, model as M, toys
    import oracle as O
    mdl, vals = getattr(configs, model)()
    blk = M.build_param_block(mdl, vals)

    def amp2(ang):
        s = D.build_sample({k: v[:0] for k, v in ang.items()}, ang, np.ones(len(ang["mLk"])))
        fx, _ = O.eval_fx(s, blk, -1, 0)
        return fx

    ens = toys.make_ensemble(list(sizes), n_mc, (0.2, 1.0), seed, amp2)
    return mdl, vals, blk, ens


@pytest.fixture(scope="module", params=["reference", "gauss"])
def setup(request):
    from pwa_b200 import ensemble, lib
    mdl, vals, blk, ens = _toys()
    ctx = lib.Context(0)
    ctx.upload(ens.sample)
    if request.param == "gauss":
        ctx.set_smearing("gauss", 0.0027, 0.0005, 17)
    names = ensemble.coupling_names(mdl)
    E = ensemble.Ensemble(ctx, ens, mdl, vals, names)
    yield request.param, mdl, vals, ens, ctx, E
    E.close()
    ctx.close()


def _random_points(E, scale, seed):
    rng = np.random.default_rng(seed)
    return E.x0[None, :] + rng.normal(0, scale, (E.n_toys, len(E.names)))


def test_nll_matches_single_point_per_toy(setup):
    from pwa_b200 import toys
    mode, mdl, vals, ens, ctx, E = setup
    X = _random_points(E, 0.2, 5)
    S = np.stack([E.exact_slots(x) for x in X])
    out, _, bad = E.eval_slots(S)
    assert np.all(bad == 0)
    for t in range(E.n_toys):
        toys.select(ctx, ens, t)
        r = ctx.eval_nll(E.builder.block(dict(zip(E.names, X[t]))))
        assert abs(out[t, 0] - r.nll) < NLL_TOL, (mode, t, out[t, 0], r.nll)
        assert abs(out[t, 1] - r.data_term) < NLL_TOL
        assert abs(out[t, 2] / r.sumint - 1) < 1e-10 and abs(out[t, 3] / r.sum_noint - 1) < 1e-10
    toys.select_all(ctx, ens)


def test_couplings_zero_at_the_set_up_point(setup):
    """Couplings that are zero where the ensemble is set up (so the set-up point's helicity masks leave
    their slots out) and move in the fit: still the single-point evaluator's NLL."""
    from pwa_b200 import ensemble, toys
    mode, mdl, vals, ens, ctx, E = setup
    v0 = dict(vals)
    zeroed = E.names[:4] + E.names[-4:]
    for n in zeroed:
        v0[n] = 0.0
    E0 = ensemble.Ensemble(ctx, ens, mdl, v0, E.names)
    try:
        X = _random_points(E0, 0.2, 9)
        out, _, bad = E0.eval_slots(np.stack([E0.exact_slots(x) for x in X]))
        assert np.all(bad == 0)
        for t in (1, 3):
            toys.select(ctx, ens, t)
            r = ctx.eval_nll(E0.builder.block(dict(zip(E0.names, X[t]))))
            assert abs(out[t, 0] - r.nll) < NLL_TOL, (mode, t, out[t, 0], r.nll)
        toys.select_all(ctx, ens)
    finally:
        E0.close()


def test_nll_matches_oracle_on_toy_alone(setup, oracle_mod):
    from pwa_b200 import dataset as D
    mode, mdl, vals, ens, ctx, E = setup
    if mode != "reference":
        pytest.skip("the oracle takes the reference's resolution scheme")
    s = ens.sample
    X = _random_points(E, 0.2, 6)
    out, _, bad = E.eval_slots(np.stack([E.exact_slots(x) for x in X]))
    assert np.all(bad == 0)
    for t in (0, 2):
        v = ens.view(t)
        cols = np.r_[v.first:v.first + v.nda, s.nda:s.n]
        n = len(cols)
        ns1 = (n // 32 + 1) * 32
        planes = []
        for p, k in ((s.pp, 111), (s.pp1, 96), (s.pp2, 96)):
            a = np.zeros((k, ns1), np.float32)
            a[:, :n] = np.asarray(p, np.float32).reshape(k, s.n_size)[:, cols]
            planes.append(a.reshape(-1))
        sw = np.zeros(ns1, np.float32)
        sw[:v.nda] = np.asarray(s.sw, np.float32)[v.first:v.first + v.nda]
        alone = D.Sample(planes[0], planes[1], planes[2], sw, n, ns1, v.nda, v.nda_smr1, v.nda_fine, s.sum_w_mc,
                         v.sum_w_data, v.sum_w2_data)
        o, _, _, _ = oracle_mod.nll(alone, E.builder.block(dict(zip(E.names, X[t]))))
        assert abs(out[t, 0] - o) < NLL_TOL, (t, out[t, 0], o)


def test_gradient_matches_finite_differences(setup):
    mode, mdl, vals, ens, ctx, E = setup
    X = _random_points(E, 0.2, 7)
    f0, g = E.fcn_grad(X)
    rng = np.random.default_rng(8)
    h = 1e-5
    for j in rng.choice(len(E.names), 6, replace=False):
        Xp, Xm = X.copy(), X.copy()
        Xp[:, j] += h
        Xm[:, j] -= h
        fd = (E.fcn_grad(Xp)[0] - E.fcn_grad(Xm)[0]) / (2 * h)
        assert np.allclose(g[:, j], fd, rtol=1e-5, atol=1e-4 * np.abs(g).max()), (E.names[j], g[:, j], fd)


def test_gram_matrices_are_hermitian_and_positive(setup):
    mode, mdl, vals, ens, ctx, E = setup
    M, Mn = E.gram()
    assert np.allclose(M, M.conj().T, rtol=0, atol=1e-12 * np.abs(M).max())
    J = E.J
    # restricted to the fit directions the normalisation is a positive quadratic form; its null space is
    # that of J (parameters, or combinations of them, that move no helicity coupling)
    H = np.real(J.conj().T @ M @ J)
    ev = np.linalg.eigvalsh(0.5 * (H + H.T))
    rank = np.linalg.matrix_rank(np.vstack([J.real, J.imag]))
    assert ev.min() > -1e-12 * ev.max()
    assert np.sum(ev > 1e-9 * ev.max()) == rank
    assert np.all(np.real(np.diag(Mn)) >= 0)


def test_ensemble_fit_matches_toy_by_toy_fit(setup):
    """A few couplings fitted to two toys: the ensemble's minimiser (analytic gradient, Gram-matrix
    normalisation, all toys in one launch) and the sequential Migrad-like fit of each toy (batched
    numerical gradient over the toy's window and the MC) agree within 0.05 sigma."""
    from pwa_b200 import ensemble, toys
    mode, mdl, vals, ens, ctx, E = setup
    names = ensemble.coupling_names(mdl)[:6]
    E6 = ensemble.Ensemble(ctx, ens, mdl, vals, names)
    try:
        fit = E6.fit(toys=[0, 1], tolerance=0.01)
        assert fit.converged[0] and fit.converged[1]
        seq = toys.fit_toys(ctx, ens, mdl, vals, names, toys=[0, 1], tolerance=0.01)
        for t in (0, 1):
            assert seq[t].converged
            dev = np.abs(fit.x[t] - seq[t].x) / seq[t].errors
            assert dev.max() < 0.05, (t, dev, fit.x[t], seq[t].x)
            assert abs(fit.fval[t] - (seq[t].fval)) < 1e-3
    finally:
        E6.close()


def test_autotune_picks_and_caches(setup, tmp_path):
    from pwa_b200 import ensemble
    mode, mdl, vals, ens, ctx, E = setup
    cache = tmp_path / "tune.json"
    c1 = ensemble.autotune(E, cache, reps=2)
    assert not c1["cached"] and (c1["warps"], c1["tile_events"]) in ensemble.CANDIDATES
    table = json.loads(cache.read_text())
    assert ensemble.tune_key(E) in table
    c2 = ensemble.autotune(E, cache)
    assert c2["cached"] and (c2["warps"], c2["tile_events"]) == (c1["warps"], c1["tile_events"])
    # the chosen shape evaluates the same numbers as another one
    S = np.repeat(E.s0[None, :], E.n_toys, axis=0)
    a, ga, _ = E.eval_slots(S)
    E.set_launch(4, 256)
    b, gb, _ = E.eval_slots(S)
    assert np.allclose(a, b, rtol=1e-12, atol=1e-9) and np.allclose(ga, gb, rtol=1e-9, atol=1e-9)
