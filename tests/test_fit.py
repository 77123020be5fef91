"""The Migrad-like minimiser (pwa_b200.fit) on analytic functions (CPU) and on the amplitude FCN:
the same minimiser on the GPU batched evaluator and on the FP64 oracle must agree within 0.05 sigma."""
import numpy as np
import pytest

from conftest import make_test_sample


def _batch(f):
    return lambda X: np.array([f(x) for x in np.asarray(X)])


def test_migrad_quadratic_minimum_and_errors():
    from pwa_b200 import fit
    A = np.array([[4.0, 1.0, 0.0], [1.0, 3.0, 0.5], [0.0, 0.5, 2.0]])
    xm = np.array([1.0, -2.0, 0.5])
    f = _batch(lambda x: 0.5 * (x - xm) @ A @ (x - xm))
    r = fit.migrad(f, np.zeros(3), np.full(3, 0.1), up=0.5)
    assert r.converged
    # EDM < 0.002 * tolerance * up places the minimum within ~0.015 sigma
    assert np.max(np.abs(r.x - xm) / r.errors) < 0.02
    # FCN = chi2 / 2 style (up = 0.5): covariance = inverse of A
    assert np.allclose(r.cov, np.linalg.inv(A), rtol=0.1, atol=2e-3)


def test_migrad_rosenbrock():
    from pwa_b200 import fit
    f = _batch(lambda x: (1 - x[0]) ** 2 + 100 * (x[1] - x[0] ** 2) ** 2)
    r = fit.migrad(f, np.array([-1.2, 1.0]), np.array([0.01, 0.01]), tolerance=1e-3, max_iter=2000)
    assert r.converged
    # converged in Migrad's sense: the FCN is within a small fraction of `up` of its minimum (0)
    assert r.fval < 2e-3 * 0.5, r
    assert np.allclose(r.x, [1.0, 1.0], atol=0.05), r


@pytest.mark.gpu
def test_fit_gpu_matches_oracle_fit(oracle_mod):
    """Fit a few couplings, a Lambda* mass and a K-matrix pole coupling of the small K-matrix model
    on a seeded sample: GPU batched FCN vs FP64 oracle FCN, same minimiser and start."""
    from pwa_b200 import fit, lib
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    names = ["a_p1p1_1520", "p_p1p1_1520", "a_p100_1670", "m0_1690", "a_L0_Pc4312", "g2_Pc4457"]
    start = dict(vals)
    for i, n in enumerate(names):
        start[n] = vals[n] + (0.05 if "m0" not in n else 0.003) * (1 if i % 2 == 0 else -1)
    x0 = np.array([start[n] for n in names])
    step = np.array([1e-3] * len(names))
    ctx = lib.Context(0)
    try:
        ctx.upload(smp)
        rg = fit.migrad(fit.gpu_fcn(ctx, mdl, start, names), x0, step, tolerance=0.01)
    finally:
        ctx.close()
    ofcn = fit.oracle_fcn(oracle_mod, smp, mdl, start, names)
    ro = fit.migrad(ofcn, x0, step, tolerance=0.01)
    assert rg.converged and ro.converged
    pull = np.abs(rg.x - ro.x) / ro.errors
    assert np.max(pull) < 0.05, (pull, rg.x, ro.x, ro.errors)
    # the same FCN: the oracle at the GPU fit's minimum gives the GPU's value
    assert abs(float(ofcn(rg.x[None, :])[0]) - rg.fval) < 1e-4
    # both minimisations stop inside the region where the FCN is within that of a 0.05-sigma
    # displacement (0.5 x 0.05^2 for up = 0.5) of each other
    assert abs(rg.fval - ro.fval) < 0.5 * 0.05**2, (rg.fval, ro.fval)


@pytest.mark.gpu
def test_config1_fit_all_couplings_within_005_sigma(oracle_mod):
    """Lambda*-only workload: 6 Lambda* Breit-Wigners, every helicity coupling free except the
    reference coupling of the Lambda(1520) (70 parameters), 20k data drawn from the model by
    hit-or-miss and 200k flat MC with w = 1, one Migrad-like fit on the GPU batched FCN.  An FP64
    oracle fit of 70 parameters takes too long for a test, so the oracle is checked at the GPU
    minimum: its gradient there, through the fit's inverse Hessian, must not move any parameter by
    more than 0.05 sigma (the Newton step to the oracle's minimum), and its FCN must agree with the
    GPU's to 1e-4."""
    from pwa_b200 import configs, fit, gpu_sample, lib, model as M
    mdl, vals = configs.lstar_only()
    blk = M.build_param_block(mdl, vals)
    ds = gpu_sample.generate(blk, 20_000, 200_000, (1.0, 1.0), seed=77, device=0)
    names = [n for n in mdl.parameter_names() if n[:2] in ("a_", "p_") and n not in ("a_p1p1_1520", "p_p1p1_1520")]
    assert len(names) == 70
    rng = np.random.default_rng(5)
    start = dict(vals)
    for n in names:
        start[n] = vals[n] + (0.05 * abs(vals[n]) + 0.01) * rng.choice([-1.0, 1.0])
    x0 = np.array([start[n] for n in names])
    ctx = lib.Context(0)
    try:
        ctx.bind_device(ds)
        rg = fit.migrad(fit.gpu_fcn(ctx, mdl, start, names), x0, np.full(len(names), 1e-3), tolerance=0.1,
                        max_iter=400)
        assert rg.converged, rg
        h = np.clip(0.02 * rg.errors, 1e-7, None)
        X = fit._grad_points(rg.x, h)
        f_gpu = fit.gpu_fcn(ctx, mdl, start, names)(X)
    finally:
        ctx.close()
    host = ds.to_host()
    f_or = fit.oracle_fcn(oracle_mod, host, mdl, start, names)(X)
    assert abs(f_or[0] - f_gpu[0]) < 1e-4
    _, g_or, _ = fit._grad_from(f_or, h)
    _, g_gpu, _ = fit._grad_from(f_gpu, h)
    V = rg.cov / (2 * 0.5)  # inverse Hessian of the FCN (up = 0.5)
    shift = np.abs(V @ g_or) / rg.errors
    assert np.max(shift) < 0.05, (np.max(shift), names[int(np.argmax(shift))])
    # the two evaluators' gradients agree to far below the 0.05-sigma scale
    assert np.max(np.abs(V @ (g_or - g_gpu)) / rg.errors) < 1e-3
