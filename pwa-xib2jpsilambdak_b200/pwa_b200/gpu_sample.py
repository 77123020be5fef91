"""Benchmark-size samples built on the GPU: MC flat with efficiency weights, data drawn by
hit-or-miss from the model (hit_and_reject.py:40-50 semantics), data sorted into the reference's
m(J/psi p) bands (reOrder.C).  Planes live in torch-owned device memory in the reference layout."""
from __future__ import annotations

import dataclasses

import numpy as np

from . import basis as B
from . import lib


@dataclasses.dataclass
class DeviceSample:
    pp: object  # torch tensors (planes x n_size), float32, cuda
    pp1: object
    pp2: object
    sw: object
    n: int
    n_size: int
    nda: int
    nda_smr1: int
    nda_fine: int
    sum_w_mc: float
    sum_w_data: float
    sum_w2_data: float
    candidates: int = 0

    @property
    def nmc(self):
        return self.n - self.nda

    def reference_band_args(self):
        return self.nda_smr1 - 1, self.nda_fine

    @classmethod
    def from_host(cls, sample, device: int = 0) -> "DeviceSample":
        """Device copy of a host Sample (dataset.Sample, reference layout)."""
        import torch
        dev = torch.device("cuda", device)
        ns = sample.n_size

        def planes(a, rows):
            return torch.as_tensor(np.asarray(a, np.float32).reshape(rows, ns), device=dev)
        return cls(planes(sample.pp, 111), planes(sample.pp1, 96), planes(sample.pp2, 96),
                   torch.as_tensor(np.asarray(sample.sw, np.float32), device=dev), sample.n, ns, sample.nda,
                   sample.nda_smr1, sample.nda_fine, sample.sum_w_mc, sample.sum_w_data, sample.sum_w2_data)

    def to_host(self, data_idx=None, mc_idx=None):
        """Host Sample (dataset.Sample) of a subset: data columns data_idx (in band order) and MC
        columns mc_idx (relative to the MC block)."""
        import torch
        from .dataset import Sample
        di = np.arange(self.nda) if data_idx is None else np.asarray(data_idx)
        mi = np.arange(self.nmc) if mc_idx is None else np.asarray(mc_idx)
        cols = torch.as_tensor(np.concatenate([di, self.nda + mi]), device=self.pp.device, dtype=torch.long)
        n = len(cols)
        ns = B.n_size_of(n)
        out = []
        for t, rows in ((self.pp, 111), (self.pp1, 96), (self.pp2, 96)):
            h = np.zeros((rows, ns), np.float32)
            h[:, :n] = t[:, cols].cpu().numpy()
            out.append(h.reshape(-1))
        sw = np.zeros(ns, np.float32)
        sw[:len(di)] = self.sw[torch.as_tensor(di, device=self.pp.device, dtype=torch.long)].cpu().numpy()
        mz = out[0][ns:ns + len(di)]
        band = B.band_of(mz)
        w = out[0][2 * ns + len(di):2 * ns + n].astype(np.float64)
        swd = sw[:len(di)].astype(np.float64)
        return Sample(out[0], out[1], out[2], sw, n, ns, len(di), int((band == 1).sum()), int((band == 2).sum()),
                      float(w.sum()), float(swd.sum()), float((swd ** 2).sum()))


def _planes(n_size, device):
    import torch
    return (torch.zeros((111, n_size), dtype=torch.float32, device=device),
            torch.zeros((96, n_size), dtype=torch.float32, device=device),
            torch.zeros((96, n_size), dtype=torch.float32, device=device))


def generate(block, n_data: int, n_mc: int, w_range=(0.2, 1.0), seed: int = 1, device: int = 0,
             batch: int = 4_000_000, max_scale: float = 1.05, ordered: bool = True,
             toy_sizes=None) -> DeviceSample:
    """ordered: MC events in the 20-offset smearing windows first, each class sorted by m(J/psi p),
    so every event class is one contiguous, coalesced range (the likelihood does not depend on the
    order; only the summation order changes)."""
    import torch
    L = lib.load()
    dev = torch.device("cuda", device)
    stream = torch.cuda.current_stream(dev).cuda_stream
    n = n_data + n_mc
    ns = B.n_size_of(n)
    pp, pp1, pp2 = _planes(ns, dev)
    # MC directly into its final columns
    lib.check(L.pwa_generate_events(pp.data_ptr(), pp1.data_ptr(), pp2.data_ptr(), ns, n_data, n_mc, seed, 1 << 40,
                                    float(w_range[0]), float(w_range[1]), 0, stream), "pwa_generate_events")
    if ordered and n_mc:
        mzm = pp[1, n_data:n].cpu().numpy()
        win = ((mzm > 4.4) & (mzm < 4.48)) | ((mzm > 4.27) & (mzm < 4.34))
        perm = np.lexsort((mzm, ~win))
        pidx = torch.as_tensor(perm + n_data, device=dev, dtype=torch.long)
        for t in (pp, pp1, pp2):
            t[:, n_data:n] = t[:, pidx]
        del pidx
    # data: hit-or-miss over candidate batches
    ctx = lib.Context(device)
    rng = np.random.default_rng(seed + 17)
    have, cand_total, first = 0, 0, 0
    amp_max = None
    parts = []
    while have < n_data:
        c = batch
        cns = B.n_size_of(c)
        cp, cp1, cp2 = _planes(cns, dev)
        lib.check(L.pwa_generate_events(cp.data_ptr(), cp1.data_ptr(), cp2.data_ptr(), cns, 0, c, seed, first,
                                        1.0, 1.0, 0, stream), "pwa_generate_events")
        first += c
        cand_total += c
        torch.cuda.synchronize(dev)
        csw = torch.zeros(cns, dtype=torch.float32, device=dev)
        ctx.bind_planes(cp, cp1, cp2, csw, c, cns)
        a2 = ctx.amp2(block)
        if amp_max is None:
            amp_max = max_scale * float(a2.max())
        acc = np.nonzero(rng.uniform(0, amp_max, c) < a2)[0][: n_data - have]
        idx = torch.as_tensor(acc, device=dev, dtype=torch.long)
        parts.append((cp[:, idx], cp1[:, idx], cp2[:, idx]))
        have += len(acc)
        del cp, cp1, cp2, csw
    ctx.close()
    dp = torch.cat([p[0] for p in parts], 1)
    dp1 = torch.cat([p[1] for p in parts], 1)
    dp2 = torch.cat([p[2] for p in parts], 1)
    mz = dp[1].cpu().numpy()
    band = B.band_of(mz)
    # bands 1, 2, 3 as the reference requires; inside a band by mass, so neighbouring events share
    # lineshape-table nodes
    if toy_sizes is not None:
        # consecutive accepted events form consecutive toys, each sorted into its own bands
        edges = np.concatenate([[0], np.cumsum(np.asarray(toy_sizes, np.int64))])
        if edges[-1] != n_data:
            raise ValueError("toy sizes must add up to n_data")
        order = np.concatenate([a + (np.lexsort((mz[a:b], band[a:b])) if ordered else B.order_data_by_band(mz[a:b]))
                                for a, b in zip(edges[:-1], edges[1:])]).astype(np.int64)
    else:
        order = np.lexsort((mz, band)) if ordered else B.order_data_by_band(mz)
    o = torch.as_tensor(order, device=dev, dtype=torch.long)
    pp[:, :n_data] = dp[:, o]
    pp[2, :n_data] = -1001.0
    pp1[:, :n_data] = dp1[:, o]
    pp2[:, :n_data] = dp2[:, o]
    del dp, dp1, dp2, parts
    sw = torch.zeros(ns, dtype=torch.float32, device=dev)
    sw[:n_data] = 1.0
    sum_w_mc = float(pp[2, n_data:n].double().sum().item())
    torch.cuda.synchronize(dev)
    return DeviceSample(pp, pp1, pp2, sw, n, ns, n_data, int((band == 1).sum()), int((band == 2).sum()), sum_w_mc,
                        float(n_data), float(n_data), cand_total)
