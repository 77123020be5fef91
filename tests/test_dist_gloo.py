"""Event-sharded NLL across 2 ranks (gloo, CPU): the all-reduced shard sums reproduce the NLL of the
whole sample.  The per-shard sums come from the oracle; the reduction and assembly are the product's."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import make_test_sample


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, shards, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from pwa_b200 import dist as D
    out[rank] = D.sharded_nll(shards[rank])
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_nll_two_ranks(oracle_mod):
    mdl, vals, blk, smp = make_test_sample("small_bw", 800, 8000, seed=9)
    ofx, ofxn = oracle_mod.eval_fx(smp, blk, *smp.reference_band_args())
    full, _ = oracle_mod.assemble_nll(smp, ofx, ofxn)
    sw = smp.sw[:smp.nda].astype(np.float64)
    w = smp.pp.reshape(111, smp.n_size)[2, smp.nda:smp.n].astype(np.float64)
    # two shards: each takes half of the data and half of the MC
    shards = []
    for r in range(2):
        d = slice(r * smp.nda // 2, (r + 1) * smp.nda // 2)
        m = slice(smp.nda + r * smp.nmc // 2, smp.nda + (r + 1) * smp.nmc // 2)
        mw = slice(r * smp.nmc // 2, (r + 1) * smp.nmc // 2)
        shards.append({"data_term": float(np.sum(np.log(ofx[d]) * sw[d])), "sumint": float(ofx[m].sum()),
                       "sum_noint": float(ofxn[m].sum()), "sum_w_mc": float(w[mw].sum()),
                       "sum_w_data": float(sw[d].sum())})
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    mp.spawn(_worker, args=(2, port, shards, out), nprocs=2, join=True)
    assert out[0] == pytest.approx(full, abs=1e-6) and out[1] == out[0]


def _oracle_sums(oracle_mod, smp, blk):
    """(data_term, sumint, sum_noint) of a sample with its own band arguments."""
    fx, fxn = oracle_mod.eval_fx(smp, blk, *smp.reference_band_args())
    sw = smp.sw[:smp.nda].astype(np.float64)
    return float(np.sum(np.log(fx[:smp.nda]) * sw)), float(fx[smp.nda:smp.n].sum()), float(fxn[smp.nda:smp.n].sum())


@pytest.mark.parametrize("world", [2, 3, 4])
def test_shards_keep_every_event_in_its_class(world, oracle_mod):
    """The reference's contiguous split (kernel_calEva.cu:1237-1243) over a sample with more data than
    one shard holds: shards evaluated as samples of their own, with shard_band_args, add up to the
    whole sample's sums, so every event keeps its smearing class (including the reference's
    last-event shift of the first band)."""
    from pwa_b200 import dist as D
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 3000, 4000, seed=13)
    whole = _oracle_sums(oracle_mod, smp, blk)
    parts = [_oracle_sums(oracle_mod, smp.shard(b, e), blk) for b, e in D.shard_bounds(smp.n, world)]
    for k in range(3):
        assert sum(p[k] for p in parts) == pytest.approx(whole[k], rel=1e-12, abs=1e-9)
    bounds = D.shard_bounds(smp.n, world)
    assert bounds[0][0] == 0 and bounds[-1][1] == smp.n and all(a[1] == b[0] for a, b in zip(bounds, bounds[1:]))


def _batch_worker(rank, world, port, local, out, sum_w_mc, sum_w_data):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from pwa_b200 import dist as D
    g = D.allreduce_point_sums(np.asarray(local[rank]))
    out[rank] = D.nll_from_point_sums(g, sum_w_mc, sum_w_data)
    dist.barrier()
    dist.destroy_process_group()


def test_batched_point_sums_two_ranks(oracle_mod):
    """The P x 3 all-reduce of a batched evaluation (gloo, 2 ranks): per-point global NLLs equal the
    whole sample's, point by point."""
    from pwa_b200 import dist as D, gradient
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 3000, 4000, seed=13)
    labels, blocks = gradient.gradient_blocks(mdl, vals, names=["a_p1p1_1670", "m0_1690", "g2_Pc4457"])
    local = []
    for b, e in D.shard_bounds(smp.n, 2):
        sh = smp.shard(b, e)
        local.append([list(_oracle_sums(oracle_mod, sh, bk)) for bk in blocks])
    want = [oracle_mod.nll(smp, bk)[0] for bk in blocks]
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_batch_worker, args=(2, _free_port(), local, out, smp.sum_w_mc, smp.sum_w_data), nprocs=2, join=True)
    assert out[0] == out[1]
    assert np.max(np.abs(np.array(out[0]) - np.array(want))) < 1e-6
