"""The learned proposal on the GPU: the tcgen05 forward kernels against a float32 restatement of the
network, the backward kernels (gradients) against a CPU float64 implementation, sampling consistent
with the density and normalised, and a trained proposal that is unbiased and cuts the amplitude
evaluations per accepted toy event relative to flat hit-or-miss."""
import numpy as np
import pytest

import flow_reference as R

pytestmark = pytest.mark.gpu


def _flow(max_batch=1024, seed=3):
    from pwa_b200 import flow
    f = flow.Flow(0, max_batch=max_batch, seed=seed)
    # non-trivial biases so every output block carries information
    rng = np.random.default_rng(seed)
    params = [(W, (b + 0.3 * rng.normal(size=b.shape)).astype(np.float32)) for W, b in f.params()]
    f.set_params(params)
    return f, f.params()


def test_log_density_matches_float32_reference():
    import torch
    f, params = _flow()
    x = torch.rand((7, 1024), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    lq = f.log_density(x).cpu().numpy()
    ref, _ = R.log_q(params, x.cpu().numpy(), torch.float32, emulate_bf16=True)
    # BF16 operands with FP32 accumulation on both sides: summation order differs, and now and then an
    # activation rounds to the other neighbouring BF16 value
    d = np.abs(lq - ref.numpy())
    assert np.median(d) < 1e-5 and np.max(d) < 1e-2, (np.median(d), np.max(d))
    f.close()


def _random_premap(seed):
    """Strictly increasing pre-map nodes with cells of widths varying over two decades."""
    from pwa_b200 import flow
    rng = np.random.default_rng(seed)
    dens = np.exp(rng.normal(0, 1.2, (flow.D, flow.PREMAP_NODES - 1)))
    cdf = np.concatenate([np.zeros((flow.D, 1)), np.cumsum(dens, axis=1)], axis=1)
    cdf /= cdf[:, -1:]
    cdf[:, -1] = 1.0
    return cdf


def test_log_density_with_premap_matches_reference():
    import torch
    f, params = _flow(seed=5)
    cdf = _random_premap(6)
    f.set_premap(cdf)
    assert np.array_equal(f.premap(), cdf)
    x = torch.rand((7, 1024), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
    lq = f.log_density(x).cpu().numpy()
    ref, _ = R.log_q(params, x.cpu().numpy(), torch.float32, emulate_bf16=True, cdf=cdf)
    d = np.abs(lq - ref.numpy())
    assert np.median(d) < 1e-5 and np.max(d) < 1e-2, (np.median(d), np.max(d))
    f.close()


def test_premap_fit_follows_the_marginals():
    """A weighted sample whose coordinate 0 piles up near 0.3: the fitted map's density there is the
    weighted histogram's (mixed with the uniform floor)."""
    import torch
    from pwa_b200 import flow
    f, _ = _flow()
    g = torch.Generator("cuda").manual_seed(8)
    x = torch.rand((7, 1 << 20), dtype=torch.float64, device="cuda", generator=g)
    w = 1.0 + 50.0 * torch.exp(-0.5 * ((x[0] - 0.3) / 0.01) ** 2)
    f.fit_premap(x, w, mix=0.1)
    c = f.premap()
    cells = flow.PREMAP_NODES - 1
    h = np.histogram(x[0].cpu().numpy(), bins=cells, range=(0, 1), weights=w.cpu().numpy())[0]
    want = 0.9 * h / h.sum() + 0.1 / cells
    assert np.allclose(np.diff(c[0]), want, rtol=1e-9, atol=1e-15)
    assert np.all(np.diff(c, axis=1) > 0) and np.all(c[:, 0] == 0) and np.all(c[:, -1] == 1)
    bad = c.copy()
    bad[3, 10] = bad[3, 9]
    with pytest.raises(Exception):
        f.set_premap(bad)
    f.close()


def test_gradients_match_cpu_float64():
    import torch
    f, params = _flow()
    g = torch.Generator("cuda").manual_seed(2)
    x = torch.rand((7, 1024), dtype=torch.float64, device="cuda", generator=g)
    w = torch.rand(1024, dtype=torch.float64, device="cuda", generator=g) + 0.1
    loss, grads = f.gradients(x, w)
    rloss, rgrads = R.loss_and_grads(params, x.cpu().numpy(), w.cpu().numpy(), emulate_bf16=True)
    assert abs(loss - rloss) < 1e-3 * abs(rloss) + 1e-4
    from pwa_b200 import flow
    for (gW, gb), (rW, rb), (mW, mb) in zip(grads, rgrads, flow.masks()):
        for a, b in ((gW * mW, rW * mW), (gb * mb, rb * mb)):
            a, b = a.ravel().astype(np.float64), b.ravel()
            if np.linalg.norm(b) == 0:
                assert np.linalg.norm(a) < 1e-6
                continue
            rel = np.linalg.norm(a - b) / np.linalg.norm(b)
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            # the GPU keeps the backward activations in BF16: a few 1e-3 relative
            assert rel < 3e-2 and cos > 0.9995, (rel, cos)
    f.close()


@pytest.mark.parametrize("premap", [False, True])
def test_sampling_matches_density_and_is_normalised(premap):
    import torch
    f, _ = _flow(max_batch=16384, seed=4)
    if premap:
        f.set_premap(_random_premap(10))
    x, lq = f.sample(65536, seed=9)
    assert float(x.min()) >= 0.0 and float(x.max()) < 1.0
    lq2 = f.log_density(x)
    assert float((lq - lq2).abs().max()) < 1e-4
    # the unit cube has volume 1: E_q[1 / q] = 1
    r = torch.exp(-lq.double())
    m, s = float(r.mean()), float(r.std()) / np.sqrt(r.numel())
    assert abs(m - 1.0) < 5 * s + 1e-3, (m, s)
    f.close()


def _amp2_at(ctx, blk, x):
    from pwa_b200 import flow
    import torch
    (pp, pp1, pp2, ns), flat = flow.events_from_unit(x)
    sw = torch.zeros(ns, dtype=torch.float32, device=x.device)
    ctx.bind_planes(pp, pp1, pp2, sw, x.shape[1], ns)
    return torch.as_tensor(ctx.amp2(blk), device=x.device), flat


def test_trained_proposal_is_unbiased_and_beats_hit_or_miss():
    import torch
    from pwa_b200 import configs, flow, lib, model as M
    mdl, vals = configs.small_kmatrix()
    blk = M.build_param_block(mdl, vals)
    ctx = lib.Context(0)
    n = 1 << 18
    xt = flow.flat_unit(1 << 21, seed=21)
    a2t, _ = _amp2_at(ctx, blk, xt)
    f = flow.Flow(0, max_batch=16384, seed=7)
    f.fit_premap(xt, a2t)
    hist = f.train(xt, a2t, epochs=6, batch=16384, lr=3e-3)
    assert np.mean(hist[-20:]) < np.mean(hist[:20])
    # flat hit-or-miss vs the learned proposal on fresh events
    xf = flow.flat_unit(n, seed=22)
    a2f, _ = _amp2_at(ctx, blk, xf)
    xq, lq = f.sample(n, seed=23)
    a2q, flat = _amp2_at(ctx, blk, xq)
    wq = a2q * flat / torch.exp(lq.double())
    i_f, s_f = float(a2f.mean()), float(a2f.std()) / np.sqrt(n)
    i_q, s_q = float(wq.mean()), float(wq.std()) / np.sqrt(n)
    assert abs(i_q - i_f) < 5 * np.hypot(s_f, s_q), (i_f, s_f, i_q, s_q)
    # amplitude evaluations per accepted toy event (hit-or-miss against the largest weight) and per
    # effective event of a weighted sample
    evals_flat = float(a2f.max()) / i_f
    evals_q = float(wq.max()) / i_q
    ess_flat = i_f ** 2 / float((a2f ** 2).mean())
    ess_q = i_q ** 2 / float((wq ** 2).mean())
    assert ess_q > 2 * ess_flat and evals_q < evals_flat / 2, (evals_flat, evals_q, ess_flat, ess_q)
    ctx.close()
    f.close()
