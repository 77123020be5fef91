"""Toy ensembles: many pseudo-data sets of uneven sizes that share one MC sample.

The reference's toy workflow (gen_toys/: hit-or-miss generation, reOrder.C band sort, one fit per
toy) builds a PDF object per toy, and each object uploads its own copy of the same MC.  Here all toys'
data are uploaded once, toy after toy, each sorted into its own m(J/psi p) bands, followed by the
shared MC; a toy is evaluated (or fitted, with the batched gradient) by selecting its data window on
the context (pwa_ctx_select_data).  The MC normalisation integral is then computed over the shared MC
at each toy's parameter point, exactly as a separate upload would.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import basis as B
from . import dataset as D
from . import kinematics as K


def toy_sizes(n_toys: int = 256, lo: float = 5e3, hi: float = 2e5, seed: int = 42) -> np.ndarray:
    """Toy sizes log-uniform in [lo, hi): floor(exp(U(ln lo, ln hi))), seeded."""
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), n_toys))).astype(np.int64)


@dataclasses.dataclass
class ToyView:
    """One toy of an ensemble, with the attributes the context's evaluation reads from its sample."""
    first: int       # position of the toy's first data event
    nda: int         # the toy's data events
    nda_smr1: int    # its 30-offset band count
    nda_fine: int    # its 150-offset band count
    n: int           # events of the whole upload (per-event outputs have this length)
    sum_w_mc: float
    sum_w_data: float
    sum_w2_data: float

    def reference_band_args(self) -> tuple:
        """Band arguments as RooDalitzAmplitude::IntegralMethod2 passes them (first count minus one)."""
        return self.nda_smr1 - 1, self.nda_fine


@dataclasses.dataclass
class ToyEnsemble:
    sample: D.Sample       # all toys' data, toy after toy, each in band order; then the shared MC
    offsets: np.ndarray    # toy t's data are events [offsets[t], offsets[t + 1])
    band1: np.ndarray      # per toy: 30-offset band count
    band2: np.ndarray      # per toy: 150-offset band count
    sum_w: np.ndarray      # per toy: sum of data weights
    sum_w2: np.ndarray

    @property
    def n_toys(self) -> int:
        return len(self.offsets) - 1

    def view(self, t: int) -> ToyView:
        s = self.sample
        return ToyView(int(self.offsets[t]), int(self.offsets[t + 1] - self.offsets[t]), int(self.band1[t]),
                       int(self.band2[t]), s.n, s.sum_w_mc, float(self.sum_w[t]), float(self.sum_w2[t]))


def build_ensemble(toy_data: list, mc_ang: dict, mc_w: np.ndarray, toy_sw: list | None = None) -> ToyEnsemble:
    """Pack the toys' data (angle dicts, one per toy), each sorted into its bands, then the MC."""
    mks, mzs, bases, sws = [], [], [], []
    offsets, band1, band2, sum_w, sum_w2 = [0], [], [], [], []
    for t, ang in enumerate(toy_data):
        dm, dz, dbas = D.events_from_angles(ang)
        sw = np.ones(len(dm), np.float32) if toy_sw is None else np.asarray(toy_sw[t], np.float32)
        order = B.order_data_by_band(dz)
        band = B.band_of(dz[order])
        mks.append(dm[order])
        mzs.append(dz[order])
        bases.append({k: v[order] for k, v in dbas.items()})
        sws.append(sw[order])
        offsets.append(offsets[-1] + len(dm))
        band1.append(int((band == 1).sum()))
        band2.append(int((band == 2).sum()))
        sum_w.append(float(sw.astype(np.float64).sum()))
        sum_w2.append(float((sw.astype(np.float64) ** 2).sum()))
    mm, mz, mbas = D.events_from_angles(mc_ang)
    nd = offsets[-1]
    mcw = np.asarray(mc_w, np.float32)
    w = np.concatenate([np.full(nd, D.DATA_WEIGHT, np.float32), mcw])
    soa = B.pack_soa(np.concatenate(mks + [mm]), np.concatenate(mzs + [mz]), w, D._concat_basis(bases + [mbas]))
    sw_all = np.zeros(soa["n_size"], np.float32)
    sw_all[:nd] = np.concatenate(sws) if sws else np.zeros(0, np.float32)
    sample = D.Sample(soa["pp"], soa["pp1"], soa["pp2"], sw_all, nd + len(mm), soa["n_size"], nd, int(sum(band1)),
                      int(sum(band2)), float(mcw.astype(np.float64).sum()), float(sum(sum_w)), float(sum(sum_w2)),
                      soa.get("pp3"), soa.get("pp4"))
    return ToyEnsemble(sample, np.array(offsets, np.int64), np.array(band1), np.array(band2), np.array(sum_w),
                       np.array(sum_w2))


def make_ensemble(sizes, n_mc: int, w_range: tuple, seed: int, amp2_of_angles, zcs: bool = False) -> ToyEnsemble:
    """Toys of the given sizes drawn by hit-or-miss from the model (amp2_of_angles: angle dict -> |A|^2
    per event) from one seeded candidate stream, consecutive accepted events forming consecutive
    toys; MC flat with weights uniform in w_range."""
    rng = np.random.default_rng(seed + 7919)
    total = int(np.sum(sizes))
    chunks, have, s = [], 0, seed * 1000 + 1
    amp_max = None
    while have < total:
        cand = K.flat_events(max(4 * (total - have), 2048), s, zcs)
        s += 1
        a2 = amp2_of_angles(cand)
        if amp_max is None:
            amp_max = 1.05 * float(a2.max())
        ok = D.hit_or_miss(a2, rng, amp_max)
        chunks.append({k: v[ok] for k, v in cand.items()})
        have += int(ok.sum())
    data = {k: np.concatenate([c[k] for c in chunks])[:total] for k in chunks[0]}
    edges = np.concatenate([[0], np.cumsum(sizes)])
    toys = [{k: v[edges[t]:edges[t + 1]] for k, v in data.items()} for t in range(len(sizes))]
    mc = K.flat_events(n_mc, seed * 1000 + 999, zcs)
    lo, hi = w_range
    mcw = rng.uniform(lo, hi, n_mc) if hi > lo else np.full(n_mc, lo)
    return build_ensemble(toys, mc, mcw)


def make_ensemble_gpu(block, sizes, n_mc: int, w_range: tuple = (0.2, 1.0), seed: int = 1,
                      device: int = 0) -> ToyEnsemble:
    """The same ensemble drawn on the GPU (flat phase space and hit-or-miss against the model's
    |A|^2 at `block`): toys of the given sizes, each in its own bands, then the shared MC, in
    torch-owned device planes (bind with Context.bind_device(ens.sample))."""
    from . import gpu_sample
    sizes = np.asarray(sizes, np.int64)
    ds = gpu_sample.generate(block, int(sizes.sum()), n_mc, w_range, seed=seed, device=device, toy_sizes=sizes)
    mz = ds.pp[1, :ds.nda].cpu().numpy()
    band = B.band_of(mz)
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    b1 = np.array([int((band[a:b] == 1).sum()) for a, b in zip(offsets[:-1], offsets[1:])])
    b2 = np.array([int((band[a:b] == 2).sum()) for a, b in zip(offsets[:-1], offsets[1:])])
    return ToyEnsemble(ds, offsets, b1, b2, sizes.astype(float), sizes.astype(float))


def select(ctx, ens: ToyEnsemble, t: int) -> ToyView:
    """Make toy t the data the context evaluates (its window of the uploaded ensemble)."""
    v = ens.view(t)
    a, b = v.reference_band_args()
    ctx.select_data(v.first, v.nda, a, b)
    ctx.sample = v
    return v


def select_all(ctx, ens: ToyEnsemble):
    """Back to the selection an upload starts with (all data, the sample's band arguments).  An
    ensemble's bands are per toy, so its likelihood is meaningful one toy at a time."""
    ctx.select_data(0, -1, *ens.sample.reference_band_args())
    ctx.sample = ens.sample


def fit_toys(ctx, ens: ToyEnsemble, model, vals: dict, names: list, toys=None, step: float = 1e-3, **kw) -> list:
    """Fit parameters `names` to each toy in turn (the MC stays resident; every FCN gradient is one
    batched call), starting from vals.  Returns the fit.FitResult of each toy."""
    from . import fit
    out = []
    x0 = np.array([vals[n] for n in names], float)
    for t in (range(ens.n_toys) if toys is None else toys):
        select(ctx, ens, t)
        out.append(fit.migrad(fit.gpu_fcn(ctx, model, vals, names), x0, np.full(len(names), step), **kw))
    select_all(ctx, ens)
    return out
