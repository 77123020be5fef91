"""Fit and interference fractions (getIFandFF semantics) from the GPU MC integral against the same
matrix from the FP64 oracle's per-event |A|^2."""
import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu


def _oracle_integral(oracle_mod, smp):
    w = np.asarray(smp.pp[2 * smp.n_size: 2 * smp.n_size + smp.n], np.float64)

    def integral(block):
        a = oracle_mod.amp2(smp, block)
        return float(np.sum(a[smp.nda:] * w[smp.nda:]))

    return integral


@pytest.mark.parametrize("name", ["small_kmatrix", "small_bw"])
def test_interference_matrix_matches_oracle(oracle_mod, name):
    from pwa_b200 import fractions, lib
    mdl, vals, blk, smp = make_test_sample(name, 1000, 10000)
    ctx = lib.Context(0)
    try:
        ctx.upload(smp)
        Mg = fractions.interference_matrix(ctx.mc_integral, mdl, vals)
        ff = fractions.fit_fractions(ctx.mc_integral, mdl, vals)
    finally:
        ctx.close()
    Mo = fractions.interference_matrix(_oracle_integral(oracle_mod, smp), mdl, vals)
    assert abs(Mg.sum() - 100.0) < 1e-9
    assert np.max(np.abs(Mg - Mo)) < 1e-8, np.max(np.abs(Mg - Mo))
    names = [r.name for r in mdl.resonances]
    for i, n in enumerate(names):
        assert abs(ff[n] - Mg[i, i]) < 1e-9


def test_mc_integral_equals_weighted_amp2(oracle_mod):
    from pwa_b200 import lib
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    ctx = lib.Context(0)
    try:
        ctx.upload(smp)
        I = ctx.mc_integral(blk)
        a = ctx.amp2(blk)
    finally:
        ctx.close()
    w = np.asarray(smp.pp[2 * smp.n_size: 2 * smp.n_size + smp.n], np.float64)
    ref = float(np.sum(a[smp.nda:] * w[smp.nda:]))
    assert abs(I / ref - 1) < 1e-12
