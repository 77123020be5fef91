"""Event shards through the library (pwa_b200.dist.ShardedLikelihood): contexts that each evaluate one
contiguous shard of one device sample (the reference's multi-device split, kernel_calEva.cu:1237-1243)
give, combined, the NLL of the whole sample, for a single point and for a gradient batch.  One GPU
holds all shards here; across GPUs the same shard sums are all-reduced (tests/test_dist_gloo.py)."""
import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_shards_on_contexts_match_whole_sample(world):
    from pwa_b200 import dist as D, gpu_sample, gradient, lib
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 3000, 4000, seed=13)
    ds = gpu_sample.DeviceSample.from_host(smp, 0)
    whole = lib.Context(0)
    whole.bind_device(ds)
    labels, blocks = gradient.gradient_blocks(mdl, vals, names=["a_p1p1_1670", "m0_1690", "a_L0_Pc4312",
                                                                 "g2_Pc4457", "fsc_ZM1SC2"])
    want = whole.eval_nll(blk).nll
    want_b = [r.nll for r in whole.eval_nll_batch(blocks)[0]]
    ctxs = [lib.Context(0) for _ in range(world)]
    try:
        shards = [D.ShardedLikelihood(c, ds, r, world, distributed=False) for r, c in enumerate(ctxs)]
        got = D.combine([s.nll(blk) for s in shards], D.NLL_SHIFT, ds.sum_w_mc, ds.sum_w_data)
        assert abs(got - want) < 1e-6
        got_b = D.combine_batch([s.nll_batch(blocks) for s in shards], D.NLL_SHIFT, ds.sum_w_mc, ds.sum_w_data)
        assert np.max(np.abs(np.array(got_b) - np.array(want_b))) < 1e-6
    finally:
        for c in ctxs:
            c.close()
        whole.close()
