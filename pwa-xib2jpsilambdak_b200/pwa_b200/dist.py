"""Event-sharded likelihood across ranks: every rank evaluates its own event shard and the three
sums (data sw ln fx, MC w fx, MC w fx without interference) are all-reduced once per evaluation
(the reference summed per-device thrust reductions on the host, kernel_calEva.cu:1296-1362)."""
from __future__ import annotations

import math

NLL_SHIFT = 10000000.0


def assemble_nll(data_term: float, sumint: float, sum_noint: float, sum_w_mc: float, sum_w_data: float,
                 nll_shift: float = NLL_SHIFT) -> float:
    """host_store_fx's NLL (kernel_calEva.cu:1341-1361) from the global sums."""
    v = nll_shift + sum_w_data * math.log(sumint / sum_w_mc) - data_term
    if abs(sum_noint / sumint - 1.0) > 0.30000001192092896:  # float 0.3f of the reference
        v += 1000.0
    return v


def allreduce_sums(sums, group=None):
    """In-place all-reduce of a float64 tensor [data_term, sumint, sum_noint, sum_w_mc, sum_w_data]."""
    import torch.distributed as dist
    dist.all_reduce(sums, group=group)
    return sums


def sharded_nll(local: dict, group=None) -> float:
    """local: this rank's partial sums (keys data_term, sumint, sum_noint, sum_w_mc, sum_w_data)."""
    import torch
    t = torch.tensor([local["data_term"], local["sumint"], local["sum_noint"], local["sum_w_mc"],
                      local["sum_w_data"]], dtype=torch.float64)
    allreduce_sums(t, group)
    d, s, sn, wm, wd = t.tolist()
    return assemble_nll(d, s, sn, wm, wd)
