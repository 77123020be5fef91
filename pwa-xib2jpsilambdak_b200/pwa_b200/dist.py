"""Event-sharded likelihood across ranks (one process per GPU, or several contexts in one process).

The reference splits one sample over its devices (kernel_calEva.cu:1237-1243): the global event range
[0, end) (data first, then MC) is cut into DEVICE_NUM contiguous shards, shard i = [Ns[i], Ns[i+1])
with Ns[i] = i * (end / DEVICE_NUM) and the last shard running to `end`; every device evaluates its
shard with the global band arguments, and the per-device sums are added on the host
(kernel_calEva.cu:1296-1362).  Here:

* `shard_bounds` gives the same cut;
* `shard_band_args` turns the global band arguments (Nda_SMR as RooDalitzAmplitude passes it, and
  Nda_SMR_finebinning) into the shard's own, so that a shard evaluated as a sample of its own puts
  every event into the class the whole sample would;
* `ShardedLikelihood` binds one shard of a device sample to a context and evaluates single points
  and batches; the per-shard sums (data sw ln fx, MC w fx, MC w fx without interference; each one
  compensated sum per shard) are combined by an all-reduce of 3 (or P x 3) doubles per evaluation
  over `torch.distributed` (NCCL between GPUs, gloo on CPU), or by `combine` for shards held in
  one process;
* `assemble_nll` forms host_store_fx's NLL from the global sums (kernel_calEva.cu:1341-1361).
"""
from __future__ import annotations

import math

import numpy as np

NLL_SHIFT = 10000000.0
_GUARD = 0.30000001192092896  # the reference's float 0.3f


def assemble_nll(data_term: float, sumint: float, sum_noint: float, sum_w_mc: float, sum_w_data: float,
                 nll_shift: float = NLL_SHIFT) -> float:
    """host_store_fx's NLL (kernel_calEva.cu:1341-1361) from the global sums."""
    v = nll_shift + sum_w_data * math.log(sumint / sum_w_mc) - data_term
    if abs(sum_noint / sumint - 1.0) > _GUARD:
        v += 1000.0
    return v


def shard_bounds(n: int, world: int) -> list:
    """[(begin, end)] of the reference's contiguous split of n events over `world` devices."""
    if world < 1:
        raise ValueError("world must be >= 1")
    step = n // world
    ns = [i * step for i in range(world)] + [n]
    return [(ns[i], ns[i + 1]) for i in range(world)]


def shard_band_args(nda: int, nda_smr: int, nda_fine: int, begin: int, end: int) -> tuple:
    """(shard data events, shard Nda_SMR, shard Nda_SMR_finebinning) of events [begin, end) of a sample
    whose global band arguments are (nda_smr, nda_fine): the 30-offset band is global [0, nda_smr), the
    150-offset band [nda_smr, nda_smr + nda_fine), the rest of the data unsmeared, MC from nda on.
    Shifting Nda_SMR by -begin keeps both band ends in place (a negative value empties band 1)."""
    nd = max(0, min(end, nda) - begin)
    return nd, nda_smr - begin, nda_fine


def combine(results, nll_shift: float, sum_w_mc: float, sum_w_data: float) -> float:
    """Global NLL of shards evaluated in one process (pwa_result-like objects, one per shard)."""
    d = math.fsum(r.data_term for r in results)
    s = math.fsum(r.sumint for r in results)
    sn = math.fsum(r.sum_noint for r in results)
    return assemble_nll(d, s, sn, sum_w_mc, sum_w_data, nll_shift)


def combine_batch(per_shard, nll_shift: float, sum_w_mc: float, sum_w_data: float) -> list:
    """Global NLL per point of batches evaluated shard by shard in one process (per_shard: one list
    of P results per shard)."""
    return [combine([res[p] for res in per_shard], nll_shift, sum_w_mc, sum_w_data)
            for p in range(len(per_shard[0]))]


def allreduce_point_sums(local: np.ndarray, group=None, device=None) -> np.ndarray:
    """All-reduce (sum over ranks) of a [P, 3] float64 array of per-point shard sums (data_term,
    sumint, sum_noint); returns the global [P, 3] array on every rank."""
    import torch
    import torch.distributed as dist
    t = torch.as_tensor(np.ascontiguousarray(local, np.float64), device=device)
    dist.all_reduce(t, group=group)
    return t.cpu().numpy()


def nll_from_point_sums(sums: np.ndarray, sum_w_mc: float, sum_w_data: float,
                        nll_shift: float = NLL_SHIFT) -> list:
    return [assemble_nll(float(d), float(s), float(sn), sum_w_mc, sum_w_data, nll_shift) for d, s, sn in sums]


def sharded_nll(local: dict, group=None) -> float:
    """local: this rank's partial sums (keys data_term, sumint, sum_noint, sum_w_mc, sum_w_data)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([local["data_term"], local["sumint"], local["sum_noint"], local["sum_w_mc"],
                      local["sum_w_data"]], dtype=torch.float64)
    dist.all_reduce(t, group=group)
    d, s, sn, wm, wd = t.tolist()
    return assemble_nll(d, s, sn, wm, wd)


class ShardedLikelihood:
    """One shard of a device sample bound to a context (lib.Context), evaluated with the global
    normalisation weights.  With `group` (a torch.distributed process group, or None for the default
    group when one is initialised) `nll` / `nll_batch` all-reduce the shard sums and return the global
    NLL on every rank; with distributed=False they return this shard's results for `combine`."""

    def __init__(self, ctx, dsample, rank: int, world: int, distributed: bool = True, group=None, device=None):
        from . import lib
        self.ctx, self.rank, self.world = ctx, rank, world
        self.begin, self.end = shard_bounds(dsample.n, world)[rank]
        nda_smr, nda_fine = dsample.reference_band_args()
        self.nda, self.nda_smr, self.nda_fine = shard_band_args(dsample.nda, nda_smr, nda_fine, self.begin, self.end)
        self.sum_w_mc, self.sum_w_data = dsample.sum_w_mc, dsample.sum_w_data
        self.distributed, self.group, self.device = distributed, group, device
        off = 4 * self.begin  # float32 columns: a shard is a column range of every plane (stride n_size)
        lib.check(ctx.L.pwa_ctx_set_device_events(ctx.h, dsample.pp.data_ptr() + off, dsample.pp1.data_ptr() + off,
                                                  dsample.pp2.data_ptr() + off, dsample.sw.data_ptr() + off,
                                                  self.end - self.begin, dsample.n_size, self.nda, self.nda_smr,
                                                  self.nda_fine), "pwa_ctx_set_device_events")
        ctx.sample = self  # the context reads sum_w_mc / sum_w_data / n from here
        ctx.n = self.n = self.end - self.begin
        self._keep = dsample

    def nll(self, block, nll_shift: float = NLL_SHIFT):
        r = self.ctx.eval_nll(block, nll_shift)
        if not self.distributed:
            return r
        g = allreduce_point_sums(np.array([[r.data_term, r.sumint, r.sum_noint]]), self.group, self.device)
        return nll_from_point_sums(g, self.sum_w_mc, self.sum_w_data, nll_shift)[0]

    def nll_batch(self, blocks, nll_shift: float = NLL_SHIFT):
        res, _ = self.ctx.eval_nll_batch(blocks, nll_shift)
        if not self.distributed:
            return res
        local = np.array([[r.data_term, r.sumint, r.sum_noint] for r in res])
        g = allreduce_point_sums(local, self.group, self.device)
        return nll_from_point_sums(g, self.sum_w_mc, self.sum_w_data, nll_shift)
