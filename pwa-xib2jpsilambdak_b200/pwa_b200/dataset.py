"""Synthetic event samples in the reference device layout.

A sample is the data events (hit-or-miss accepted from the model, weight sentinel -1001 in the w
plane, sWeights in the sw plane) followed by the MC events (flat phase space, per-event efficiency
weights), with the data sorted into the reference's m(J/psi p) bands
(gen_toys/rearrange_mJpsip/reOrder.C) and the band counts of RooDalitzAmplitude.cxx:391-396.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import basis as B
from . import kinematics as K

DATA_WEIGHT = -1001.0  # filldlz default weight marks data events (RooDalitzAmplitude.h:235)


@dataclasses.dataclass
class Sample:
    pp: np.ndarray
    pp1: np.ndarray
    pp2: np.ndarray
    sw: np.ndarray
    n: int
    n_size: int
    nda: int
    nda_smr1: int  # events of the 30-offset band (the caller passes nda_smr1 - 1, see below)
    nda_fine: int
    sum_w_mc: float
    sum_w_data: float
    sum_w2_data: float
    pp3: np.ndarray | None = None  # Zcs chain planes (models with NX > 0)
    pp4: np.ndarray | None = None

    @property
    def nmc(self):
        return self.n - self.nda

    def reference_band_args(self) -> tuple:
        """(Nda_SMR, Nda_SMR_finebinning) exactly as RooDalitzAmplitude::IntegralMethod2 passes
        them to host_store_fx (RooDalitzAmplitude.cxx:1943-1946): the first count minus one."""
        return self.nda_smr1 - 1, self.nda_fine

    def shard(self, begin: int, end: int) -> "Sample":
        """Events [begin, end) as a sample of their own (planes copied), with the band arguments that
        keep every event in the class the whole sample gives it (dist.shard_band_args) and the
        whole sample's normalisation weights (sum_w_mc, sum_w_data), as one device of the
        reference's multi-device split evaluates its shard."""
        from .dist import shard_band_args
        n = end - begin
        ns = B.n_size_of(n)

        def cut(a, rows):
            out = np.zeros((rows, ns), np.float32)
            out[:, :n] = np.asarray(a, np.float32).reshape(rows, self.n_size)[:, begin:end]
            return out.reshape(-1)
        nda, smr, fine = shard_band_args(self.nda, *self.reference_band_args(), begin, end)
        sw = np.zeros(ns, np.float32)
        sw[:n] = self.sw[begin:end]
        return Sample(cut(self.pp, 111), cut(self.pp1, 96), cut(self.pp2, 96), sw, n, ns, nda, smr + 1, fine,
                      self.sum_w_mc, self.sum_w_data, self.sum_w2_data,
                      None if self.pp3 is None else cut(self.pp3, 97), None if self.pp4 is None else cut(self.pp4, 96))


def events_from_angles(ang: dict) -> tuple:
    bas = B.fill_basis(ang)
    if "X_cosTheta_Lb" in ang:
        bas.update(B.fill_basis_x(ang))
        bas["mjpsik"] = np.asarray(ang["mjpsik"], np.float32)
    return np.asarray(ang["mLk"], np.float32), np.asarray(ang["mjpsiL"], np.float32), bas


def _concat_basis(parts):
    return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}


def build_sample(data_ang: dict, mc_ang: dict, mc_w: np.ndarray, data_sw: np.ndarray | None = None) -> Sample:
    """Pack data (sorted into bands) followed by MC into the reference planes."""
    dm, dz, dbas = events_from_angles(data_ang)
    mm, mz, mbas = events_from_angles(mc_ang)
    nd, nm = len(dm), len(mm)
    sw_d = np.ones(nd, np.float32) if data_sw is None else np.asarray(data_sw, np.float32)
    order = B.order_data_by_band(dz)
    dm, dz, sw_d = dm[order], dz[order], sw_d[order]
    dbas = {k: v[order] for k, v in dbas.items()}
    band = B.band_of(dz)
    mkp = np.concatenate([dm, mm])
    mzz = np.concatenate([dz, mz])
    w = np.concatenate([np.full(nd, DATA_WEIGHT, np.float32), np.asarray(mc_w, np.float32)])
    soa = B.pack_soa(mkp, mzz, w, _concat_basis([dbas, mbas]))
    sw = np.zeros(soa["n_size"], np.float32)
    sw[:nd] = sw_d
    mcw = np.asarray(mc_w, np.float32)
    return Sample(soa["pp"], soa["pp1"], soa["pp2"], sw, nd + nm, soa["n_size"], nd, int((band == 1).sum()),
                  int((band == 2).sum()), float(mcw.astype(np.float64).sum()), float(sw_d.astype(np.float64).sum()),
                  float((sw_d.astype(np.float64) ** 2).sum()), soa.get("pp3"), soa.get("pp4"))


def hit_or_miss(amp2: np.ndarray, rng, amp2_max: float | None = None) -> np.ndarray:
    """Accept mask of hit-or-miss against a global maximum (hit_and_reject.py:40-50 semantics)."""
    mx = float(amp2.max()) if amp2_max is None else amp2_max
    return rng.uniform(0, mx, amp2.shape[0]) < amp2


def make_sample(n_data: int, n_mc: int, w_range: tuple, seed: int, amp2_of_angles, zcs: bool = False) -> Sample:
    """Data by hit-or-miss from the model (amp2_of_angles: angle dict -> |A|^2 per event), MC flat
    with weights uniform in w_range."""
    rng = np.random.default_rng(seed + 7919)
    chunks, have = [], 0
    s = seed * 1000 + 1
    while have < n_data:
        cand = K.flat_events(max(4 * (n_data - have), 2048), s, zcs)
        s += 1
        a2 = amp2_of_angles(cand)
        ok = hit_or_miss(a2, rng, 1.05 * a2.max())
        chunks.append({k: v[ok] for k, v in cand.items()})
        have += int(ok.sum())
    data = {k: np.concatenate([c[k] for c in chunks])[:n_data] for k in chunks[0]}
    mc = K.flat_events(n_mc, seed * 1000 + 999, zcs)
    lo, hi = w_range
    mcw = rng.uniform(lo, hi, n_mc) if hi > lo else np.full(n_mc, lo)
    return build_sample(data, mc, mcw)
