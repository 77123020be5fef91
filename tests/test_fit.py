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
    ro = fit.migrad(fit.oracle_fcn(oracle_mod, smp, mdl, start, names), x0, step, tolerance=0.01)
    assert rg.converged and ro.converged
    pull = np.abs(rg.x - ro.x) / ro.errors
    assert np.max(pull) < 0.05, (pull, rg.x, ro.x, ro.errors)
    assert abs(rg.fval - ro.fval) < 1e-4
