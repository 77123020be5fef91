"""The isospin-split K-matrix on the GPU (pwa_ctx_set_kmatrix): the likelihood with and without the
lineshape tables, and the gradient batch, against the FP64 oracle's restatement."""
import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu

NLL_TOL = 1e-6


def test_isospin_kmatrix_nll_and_batch(oracle_mod):
    from pwa_b200 import gradient, lib
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 1500, 15000)
    ctx = lib.Context(0)
    oracle_mod.set_kmatrix_isospin(True)
    try:
        ctx.upload(smp)
        ctx.set_kmatrix(True)
        v, s, fx, _ = oracle_mod.nll(smp, blk)
        r, gfx = ctx.eval_nll(blk, want_fx=True)
        assert abs(r.nll - v) < NLL_TOL and abs(r.sumint / s - 1) < 1e-9
        rel = np.abs(gfx - fx) / np.abs(fx)
        assert np.max(rel) < 1e-8, np.max(rel)
        ctx.set_lineshape_tables(False)
        assert abs(ctx.eval_nll(blk).nll - v) < NLL_TOL
        ctx.set_lineshape_tables(True)
        labels, blocks = gradient.gradient_blocks(mdl, vals)
        res, _ = ctx.eval_nll_batch(blocks)
        single = [ctx.eval_nll(b).nll for b in blocks]
        assert np.max(np.abs(np.array([x.nll for x in res]) - single)) < NLL_TOL
        for i in (0, 1, len(blocks) - 2):
            assert abs(res[i].nll - oracle_mod.nll(smp, blocks[i])[0]) < NLL_TOL, labels[i]
        # back to the 4-channel default
        ctx.set_kmatrix(False)
        oracle_mod.set_kmatrix_isospin(False)
        assert abs(ctx.eval_nll(blk).nll - oracle_mod.nll(smp, blk)[0]) < NLL_TOL
    finally:
        oracle_mod.set_kmatrix_isospin(False)
        ctx.close()
