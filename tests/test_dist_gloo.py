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
