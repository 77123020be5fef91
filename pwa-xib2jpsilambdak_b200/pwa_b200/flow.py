"""Learned proposal density over the phase space (pwa_flow_* of the C ABI).

The density q(x) lives on unit coordinates x in [0,1]^7 of the Lambda_b -> J/psi(-> mu mu) p K-
phase space (`pwa_events_from_unit` turns x into an event):

* x1, x2: the Dalitz point, m^2(J/psi p) linear in x1 over its range (the narrow Pc bands lie at
  fixed x1) and m^2(Kp) linear in x2 across the Dalitz row at that m^2(J/psi p) (the region's
  boundary lies at x2 = 0 and 1, so no bin of the network straddles it);
* x3, x4, x5: the orientation of the decay in the Lambda_b rest frame (cos of the J/psi polar angle
  to the Lambda_b flight axis, its azimuth, the roll of the decay plane about the J/psi direction);
* x6, x7: the mu+ direction in the J/psi rest frame (cos theta, phi).

Flat phase space has the density `events_from_unit` returns (the Dalitz-row length only).  Each coordinate first passes a fixed monotone pre-map u = F(x) fitted to the target's
weighted marginal (`fit_premap`: a piecewise-linear CDF on 1024 cells with a uniform floor), which
stretches the narrow resonance bands over many of the network's bins.  The network is an
autoregressive 4 x 256 SiLU MLP (MADE masks) giving, per dimension, 64 bin probabilities of u_d
conditional on the earlier dimensions: q(x) = prod_d 64 p_d(bin(u_d) | u_<d) F_d'(x_d), normalised
and sampled exactly.  It is trained by weighted maximum likelihood on flat phase-space events
weighted by |A|^2 (the target density is |A|^2 times flat phase space), with BF16 tcgen05 GEMMs and
FP32 accumulation.

Used (i) for toys: candidates drawn from q, each weighted by |A|^2 flat / q and accepted against the
largest weight (hit-or-miss on the weights), and (ii) for normalisation integrals: the mean of
|A|^2 flat / q over q-samples.  The exact amplitude decides every event, so neither use is biased;
flat phase space stays available (`flat_unit`).  No counterpart in the reference, whose toys are flat
hit-or-miss (gen_toys/create_efficiency/hit_and_reject.py:40-50).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib

D, BINS, IN, H, OUT = 7, 64, 64, 256, 512
PREMAP_NODES = 1025
LAYERS = [(H, IN), (H, H), (H, H), (H, H), (OUT, H)]  # (out, in)


def degree(k: int) -> int:
    """MADE degree of hidden unit k (1 .. D-1); input column c < D is dimension c + 1."""
    return 1 + k % (D - 1)


def masks() -> list:
    """(weight mask, bias mask) per layer, as the library builds them."""
    out = []
    for l, (o, i) in enumerate(LAYERS):
        M = np.zeros((o, i), np.float32)
        mb = np.ones(o, np.float32)
        for r in range(o):
            for c in range(i):
                if l == 0:
                    keep = c < D and degree(r) >= c + 1
                elif l < 4:
                    keep = degree(r) >= degree(c)
                else:
                    keep = r // BINS < D and r // BINS + 1 > degree(c)
                M[r, c] = keep
            if l == 4 and r // BINS >= D:
                mb[r] = 0
        out.append((M, mb))
    return out


def _bind(L):
    if getattr(L, "_flow_bound", False):
        return L
    vp, i64, dp, fp = C.c_void_p, C.c_int64, C.POINTER(C.c_double), C.POINTER(C.c_float)
    L.pwa_flow_create.argtypes = [C.c_int, C.c_int, C.c_uint64, C.POINTER(vp)]
    L.pwa_flow_destroy.argtypes = [vp]
    L.pwa_flow_param_count.restype = i64
    L.pwa_flow_train_step.argtypes = [vp, vp, i64, vp, C.c_int, C.c_float, dp]
    L.pwa_flow_gradients.argtypes = [vp, vp, i64, vp, C.c_int, dp, fp]
    L.pwa_flow_log_density.argtypes = [vp, vp, i64, i64, vp]
    L.pwa_flow_sample.argtypes = [vp, i64, C.c_uint64, vp, i64, vp]
    L.pwa_flow_get_params.argtypes = [vp, fp]
    L.pwa_flow_set_params.argtypes = [vp, fp]
    L.pwa_flow_fit_premap.argtypes = [vp, vp, i64, vp, i64, C.c_double]
    L.pwa_flow_get_premap.argtypes = [vp, dp]
    L.pwa_flow_set_premap.argtypes = [vp, dp]
    L.pwa_events_from_unit.argtypes = [vp, i64, i64, vp, vp, vp, i64, i64, C.c_float, C.c_int, vp, vp]
    L.pwa_unit_flat.argtypes = [i64, C.c_uint64, C.c_uint64, vp, i64, vp]
    L._flow_bound = True
    return L


def _ptr(t):
    return C.c_void_p(t.data_ptr())


class Flow:
    """The proposal network on one device; x arrays are torch float64 [7, n] on that device."""

    def __init__(self, device: int = 0, max_batch: int = 65536, seed: int = 1):
        self.L = _bind(lib.load())
        h = C.c_void_p()
        lib.check(self.L.pwa_flow_create(device, max_batch, seed, C.byref(h)), "pwa_flow_create")
        self.h, self.device, self.max_batch = h, device, max_batch

    def close(self):
        if self.h:
            self.L.pwa_flow_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def train_step(self, x, w, lr: float) -> float:
        loss = C.c_double()
        lib.check(self.L.pwa_flow_train_step(self.h, _ptr(x), x.stride(0), _ptr(w), x.shape[1], lr, C.byref(loss)),
                  "pwa_flow_train_step")
        return loss.value

    def gradients(self, x, w) -> tuple:
        """(loss, [(dW, db) per layer]) of the weighted loss on x (no update)."""
        g = np.zeros(int(self.L.pwa_flow_param_count()), np.float32)
        loss = C.c_double()
        lib.check(self.L.pwa_flow_gradients(self.h, _ptr(x), x.stride(0), _ptr(w), x.shape[1], C.byref(loss),
                                            g.ctypes.data_as(C.POINTER(C.c_float))), "pwa_flow_gradients")
        return loss.value, _split(g)

    def params(self) -> list:
        p = np.zeros(int(self.L.pwa_flow_param_count()), np.float32)
        lib.check(self.L.pwa_flow_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))), "pwa_flow_get_params")
        return _split(p)

    def set_params(self, params: list):
        p = np.concatenate([np.concatenate([W.reshape(-1), b]) for W, b in params]).astype(np.float32)
        lib.check(self.L.pwa_flow_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))), "pwa_flow_set_params")

    def fit_premap(self, x, w, mix: float = 0.1):
        """Fit the coordinates' pre-maps to the weighted marginals of events x [7, n] (weights w [n])."""
        lib.check(self.L.pwa_flow_fit_premap(self.h, _ptr(x), x.stride(0), _ptr(w), x.shape[1], mix),
                  "pwa_flow_fit_premap")

    def premap(self) -> np.ndarray:
        """The pre-maps' nodes [7, PREMAP_NODES] (F_d at x = k / (PREMAP_NODES - 1))."""
        c = np.zeros((D, PREMAP_NODES), np.float64)
        lib.check(self.L.pwa_flow_get_premap(self.h, c.ctypes.data_as(C.POINTER(C.c_double))), "pwa_flow_get_premap")
        return c

    def set_premap(self, cdf: np.ndarray):
        c = np.ascontiguousarray(cdf, np.float64)
        lib.check(self.L.pwa_flow_set_premap(self.h, c.ctypes.data_as(C.POINTER(C.c_double))), "pwa_flow_set_premap")

    def log_density(self, x):
        import torch
        out = torch.empty(x.shape[1], dtype=torch.float32, device=x.device)
        lib.check(self.L.pwa_flow_log_density(self.h, _ptr(x), x.stride(0), x.shape[1], _ptr(out)),
                  "pwa_flow_log_density")
        return out

    def sample(self, n: int, seed: int) -> tuple:
        import torch
        x = torch.empty((D, n), dtype=torch.float64, device=f"cuda:{self.device}")
        lq = torch.empty(n, dtype=torch.float32, device=x.device)
        lib.check(self.L.pwa_flow_sample(self.h, n, seed, _ptr(x), n, _ptr(lq)), "pwa_flow_sample")
        return x, lq

    def train(self, x, w, epochs: int = 4, batch: int = 65536, lr: float = 2e-3, seed: int = 0) -> list:
        """Minibatch Adam over the events (x [7, n], w [n]), cosine-decayed learning rate; returns the
        loss of every step."""
        import torch
        n = x.shape[1] // batch * batch
        steps = epochs * (n // batch)
        g = torch.Generator(device=x.device).manual_seed(seed)
        hist, k = [], 0
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g, device=x.device)
            for b0 in range(0, n, batch):
                idx = perm[b0:b0 + batch]
                rate = lr * 0.5 * (1 + np.cos(np.pi * k / max(steps, 1)))
                hist.append(self.train_step(x[:, idx].contiguous(), w[idx].contiguous(), float(rate)))
                k += 1
        return hist


def _split(flat: np.ndarray) -> list:
    out, o = [], 0
    for (r, c) in LAYERS:
        W = flat[o:o + r * c].reshape(r, c)
        b = flat[o + r * c:o + r * c + r]
        out.append((W, b))
        o += r * c + r
    return out


def flat_unit(n: int, seed: int, device: int = 0, first_id: int = 0):
    """n flat phase-space events in unit coordinates (torch float64 [7, n] on the device)."""
    import torch
    L = _bind(lib.load())
    x = torch.empty((D, n), dtype=torch.float64, device=f"cuda:{device}")
    lib.check(L.pwa_unit_flat(n, seed, first_id, _ptr(x), n, None), "pwa_unit_flat")
    return x


def events_from_unit(x, data: bool = False, weight: float = 1.0):
    """Device planes (pp, pp1, pp2 torch tensors, n_size) of the events at unit coordinates x, and the
    flat phase-space density of x (torch float64 [n])."""
    import torch
    from . import basis as B
    L = _bind(lib.load())
    n = x.shape[1]
    ns = B.n_size_of(n)
    dev = x.device
    pp = torch.zeros((111, ns), dtype=torch.float32, device=dev)
    pp1 = torch.zeros((96, ns), dtype=torch.float32, device=dev)
    pp2 = torch.zeros((96, ns), dtype=torch.float32, device=dev)
    fl = torch.empty(n, dtype=torch.float64, device=dev)
    lib.check(L.pwa_events_from_unit(_ptr(x), x.stride(0), n, _ptr(pp), _ptr(pp1), _ptr(pp2), ns, 0, weight,
                                     int(data), _ptr(fl), None), "pwa_events_from_unit")
    return (pp, pp1, pp2, ns), fl
