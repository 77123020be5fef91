"""Toy ensemble on the GPU: each toy evaluated through its data window on one upload (shared MC)
equals the same toy uploaded alone with the same MC, and the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NLL_TOL = 1e-6


def _ensemble():
    from pwa_b200 import configs, dataset as D, model as M, toys
    import oracle as O
    mdl, vals = configs.small_kmatrix()
    blk = M.build_param_block(mdl, vals)

    def amp2(ang):
        s = D.build_sample({k: v[:0] for k, v in ang.items()}, ang, np.ones(len(ang["mLk"])))
        fx, _ = O.eval_fx(s, blk, -1, 0)
        return fx

    ens = toys.make_ensemble([600, 1500, 350], 8000, (0.2, 1.0), 3, amp2)
    return mdl, vals, blk, ens


def test_toy_windows_match_separate_uploads(oracle_mod):
    from pwa_b200 import dataset as D, lib, toys
    mdl, vals, blk, ens = _ensemble()
    s = ens.sample
    ns = s.n_size
    ctx, solo = lib.Context(0), lib.Context(0)
    try:
        ctx.upload(s)
        for t in range(ens.n_toys):
            v = toys.select(ctx, ens, t)
            r = ctx.eval_nll(blk)
            # the same toy alone: its data columns and the MC columns, repacked
            cols = np.r_[v.first:v.first + v.nda, s.nda:s.n]
            n = len(cols)
            ns1 = (n // 32 + 1) * 32
            planes = []
            for p, k in ((s.pp, 111), (s.pp1, 96), (s.pp2, 96)):
                a = np.zeros((k, ns1), np.float32)
                a[:, :n] = np.asarray(p, np.float32).reshape(k, ns)[:, cols]
                planes.append(a.reshape(-1))
            sw = np.zeros(ns1, np.float32)
            sw[:v.nda] = np.asarray(s.sw, np.float32)[v.first:v.first + v.nda]
            alone = D.Sample(planes[0], planes[1], planes[2], sw, n, ns1, v.nda, v.nda_smr1, v.nda_fine, s.sum_w_mc,
                             v.sum_w_data, v.sum_w2_data)
            solo.upload(alone)
            r1 = solo.eval_nll(blk)
            assert abs(r.nll - r1.nll) < NLL_TOL, (t, r.nll, r1.nll)
            assert abs(r.sumint / r1.sumint - 1) < 1e-12
            o, _, _, _ = oracle_mod.nll(alone, blk)
            assert abs(r.nll - o) < NLL_TOL, (t, r.nll, o)
        toys.select_all(ctx, ens)
        r_all = ctx.eval_nll(blk)
        assert r_all.n_nonpos == 0
    finally:
        ctx.close()
        solo.close()


def test_toy_batched_gradient_and_fit():
    """The batched gradient of a toy window equals single-point calls, and fitting two toys moves a
    coupling to each toy's own minimum (different toys, different minima)."""
    from pwa_b200 import gradient, lib, toys
    mdl, vals, blk, ens = _ensemble()
    ctx = lib.Context(0)
    try:
        ctx.upload(ens.sample)
        toys.select(ctx, ens, 1)
        labels, blocks = gradient.gradient_blocks(mdl, vals)
        res, nstruct = ctx.eval_nll_batch(blocks[:40])
        for r, b in zip(res, blocks[:40]):
            assert abs(r.nll - ctx.eval_nll(b).nll) < NLL_TOL
        names = ["a_p1p1_1520", "a_L0_Pc4312"]
        fits = toys.fit_toys(ctx, ens, mdl, vals, names, toys=[0, 1], tolerance=0.05)
        assert all(f.converged for f in fits)
        assert np.max(np.abs(fits[0].x - fits[1].x)) > 1e-4
    finally:
        ctx.close()


def test_toy_window_under_gaussian_resolution():
    """A toy window with the Gaussian resolution model (all events on the weighted grid) equals the same
    toy alone, and the batch segment timing reports the window's classes."""
    from pwa_b200 import dataset as D, lib, toys
    mdl, vals, blk, ens = _ensemble()
    s = ens.sample
    ctx, solo = lib.Context(0), lib.Context(0)
    try:
        ctx.upload(s)
        ctx.set_smearing("gauss", 0.0027, 0.0005, 17)
        v = toys.select(ctx, ens, 0)
        r = ctx.eval_nll(blk)
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
        solo.upload(alone)
        solo.set_smearing("gauss", 0.0027, 0.0005, 17)
        solo.sample = alone
        assert abs(r.nll - solo.eval_nll(blk).nll) < NLL_TOL
        # per-segment device time of a batched call
        from pwa_b200 import gradient
        labels, blocks = gradient.gradient_blocks(mdl, vals)
        ctx.set_timing(True)
        ctx.eval_nll_batch(blocks[:20])
        ms = ctx.batch_segment_ms()
        assert len(ms) == len(ctx.segments()) == 2 and all(m > 0 for m in ms)
        assert sum(ms) <= ctx.last_batch_ms() + 1e-3
    finally:
        ctx.close()
        solo.close()


def test_toy_ensemble_generated_on_gpu(oracle_mod):
    """Toys drawn on the GPU share one MC block; each toy's window is in its own band order and its
    NLL equals the FP64 oracle on a host copy of that toy with the MC."""
    from pwa_b200 import basis as B, configs, lib, model as M, toys
    mdl, vals = configs.small_kmatrix()
    blk = M.build_param_block(mdl, vals)
    sizes = toys.toy_sizes(3, lo=500, hi=3000, seed=7)
    ens = toys.make_ensemble_gpu(blk, sizes, 20000, seed=11)
    ds = ens.sample
    assert ds.nda == int(sizes.sum()) and list(ens.offsets[1:] - ens.offsets[:-1]) == list(sizes)
    ctx = lib.Context(0)
    try:
        ctx.bind_device(ds)
        for t in range(ens.n_toys):
            v = toys.select(ctx, ens, t)
            band = B.band_of(ds.pp[1, v.first:v.first + v.nda].cpu().numpy())
            assert np.all(np.diff(band) >= 0)
            r = ctx.eval_nll(blk)
            host = ds.to_host(data_idx=np.arange(v.first, v.first + v.nda))
            o, _, _, _ = oracle_mod.nll(host, blk)
            assert abs(r.nll - o) < NLL_TOL, (t, r.nll, o)
    finally:
        ctx.close()
