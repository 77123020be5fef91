"""A Migrad-like minimiser for the amplitude fit, fed by batched likelihood evaluations.

The reference fits with RooMinuit / Minuit2 Migrad (src/fit.cpp:222-288) on the FCN
(NLL - NLL_SHIFT) * alpha + constraints (src/fit.cpp:312-317).  ROOT is not part of this project, so
the minimiser here follows Migrad's scheme in plain numpy: a variable-metric (BFGS) iteration whose
gradient and diagonal second derivatives come from central differences over the 2N+1 points
(centre, +-h per parameter), evaluated in one batch; the line search evaluates its trial steps in
one batch too; convergence on the estimated distance to minimum EDM = g^T V g / 2 below
0.002 * tolerance * up (Minuit2's criterion); parameter errors sqrt(2 up V_ii) from the final
inverse-Hessian estimate V.

`fcn_batch(X) -> values` takes an (P, N) array of parameter vectors; `gpu_fcn` and `oracle_fcn`
build it from the GPU context and from the FP64 oracle so that the same minimiser can run on both.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .model import BlockBuilder, fcn as ref_fcn


@dataclasses.dataclass
class FitResult:
    x: np.ndarray
    fval: float
    errors: np.ndarray
    edm: float
    iterations: int
    evaluations: int
    converged: bool
    cov: np.ndarray


def _grad_points(x: np.ndarray, h: np.ndarray) -> np.ndarray:
    n = len(x)
    X = np.repeat(x[None, :], 2 * n + 1, axis=0)
    for i in range(n):
        X[1 + 2 * i, i] += h[i]
        X[2 + 2 * i, i] -= h[i]
    return X


def _grad_from(F: np.ndarray, h: np.ndarray) -> tuple:
    f0 = F[0]
    fp, fm = F[1::2], F[2::2]
    g = (fp - fm) / (2 * h)
    g2 = (fp + fm - 2 * f0) / (h * h)
    return f0, g, g2


def migrad(fcn_batch, x0, step0, tolerance: float = 0.1, up: float = 0.5, max_iter: int = 200,
           alphas=(1.0, 0.5, 0.25, 0.1, 2.0)) -> FitResult:
    x = np.asarray(x0, float).copy()
    n = len(x)
    h = np.asarray(step0, float).copy()
    nev = 0
    F = np.asarray(fcn_batch(_grad_points(x, h)))
    nev += len(F)
    f, g, g2 = _grad_from(F, h)
    V = np.diag(1.0 / np.where(g2 > 0, g2, 1.0 / np.maximum(h * h, 1e-300)))
    edm = 0.5 * g @ V @ g
    it = 0
    converged = edm < 0.002 * tolerance * up
    just_reset = True

    def diag_metric():
        return np.diag(1.0 / np.where(g2 > 0, g2, 1.0 / np.maximum(h * h, 1e-300)))

    while not converged and it < max_iter:
        it += 1
        d = -V @ g
        if g @ d >= 0:  # not a descent direction: restart from the diagonal
            V = diag_metric()
            just_reset = True
            d = -V @ g
        trial = np.array([x + a * d for a in alphas])
        Ft = np.asarray(fcn_batch(trial))
        nev += len(Ft)
        k = int(np.argmin(Ft))
        if not Ft[k] < f:
            # shrink until the step lowers the FCN (Migrad's line search would too)
            a = min(alphas) * 0.1
            while a > 1e-8:
                ft = float(np.asarray(fcn_batch((x + a * d)[None, :]))[0])
                nev += 1
                if ft < f:
                    break
                a *= 0.1
            else:
                if just_reset:  # no descent even along the diagonal metric: at the precision limit
                    break
                V = diag_metric()  # the metric has gone stale: restart from the diagonal
                just_reset = True
                continue
            xn = x + a * d
        else:
            xn = trial[k]
        # step sizes for the next gradient: a fraction of the current error estimate
        err = np.sqrt(np.maximum(2 * up * np.diag(V), 0))
        h = np.clip(0.02 * err, 1e-7, None)
        Fn = np.asarray(fcn_batch(_grad_points(xn, h)))
        nev += len(Fn)
        fn, gn, g2 = _grad_from(Fn, h)
        s, y = xn - x, gn - g
        sy = s @ y
        if sy > 1e-300:  # BFGS update of the inverse Hessian
            rho = 1.0 / sy
            I = np.eye(n)
            V = (I - rho * np.outer(s, y)) @ V @ (I - rho * np.outer(y, s)) + rho * np.outer(s, s)
        x, f, g = xn, fn, gn
        just_reset = False
        edm = 0.5 * g @ V @ g
        converged = edm < 0.002 * tolerance * up
    err = np.sqrt(np.maximum(2 * up * np.diag(V), 0))
    return FitResult(x, float(f), err, float(edm), it, nev, bool(converged), 2 * up * V)


def gpu_fcn(ctx, model, vals: dict, names: list, constraints=(), alpha: float = 1.0, nll_shift: float = 1e7):
    """fcn_batch on a GPU context (pwa_b200.lib.Context with events uploaded): one
    pwa_ctx_eval_nll_batch per call."""
    builder = BlockBuilder(model, vals)

    def f(X):
        blocks = [builder.block(dict(zip(names, map(float, x)))) for x in X]
        res, _ = ctx.eval_nll_batch(blocks, nll_shift)
        out = []
        for r, x in zip(res, X):
            v = dict(vals)
            v.update(zip(names, map(float, x)))
            out.append(ref_fcn(r.nll, nll_shift, alpha, list(constraints), v))
        return np.array(out)

    return f


def oracle_fcn(oracle_mod, sample, model, vals: dict, names: list, constraints=(), alpha: float = 1.0,
               nll_shift: float = 1e7):
    """The same FCN on the FP64 oracle (one evaluation per point, host cores)."""
    builder = BlockBuilder(model, vals)

    def f(X):
        out = []
        for x in X:
            v = dict(vals)
            v.update(zip(names, map(float, x)))
            nll, _, _, _ = oracle_mod.nll(sample, builder.block(dict(zip(names, map(float, x)))))
            out.append(ref_fcn(nll, nll_shift, alpha, list(constraints), v))
        return np.array(out)

    return f
