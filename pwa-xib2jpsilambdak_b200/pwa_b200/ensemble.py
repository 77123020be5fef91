"""Toy ensembles fitted together on one GPU (pwa_ens_* of the C ABI).

The reference fits a toy study one toy at a time, each with its own PDF object that integrates the
MC anew at every FCN call (src/RooDalitzAmplitude.cxx:1293-1628, gen_toys/).  Here all toys' data and
the one MC sample stay resident (`toys.ToyEnsemble`), and for fits that float the couplings (the
lineshape parameters stay at the ensemble's set-up point):

* every toy's MC normalisation is the Hermitian form c^H M c of its helicity-coupling vector c with the
  FP64 Gram matrix M of the MC, built once;
* one call (one CUDA-graph launch, persistent blocks over (toy, event range) work items) evaluates
  every toy's data term sum sw ln|A|^2 and its gradient in c;
* the couplings c are linear in the fitted LS couplings (checked at set-up), so the FCN gradient in the
  fit parameters follows exactly; a batched variable-metric minimiser (`fit`) steps all toys at once.

The launch shape (warps per block, events per work item) comes from `autotune`, which times the
candidates on the ensemble itself and caches the choice in a JSON file keyed by device and ensemble
shape.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import json
from pathlib import Path

import numpy as np

from . import lib
from .model import BlockBuilder

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_i64p = C.POINTER(C.c_int64)


def _bind(L):
    if getattr(L, "_ens_bound", False):
        return L
    vp = C.c_void_p
    L.pwa_ens_create.argtypes = [vp, _fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                 C.c_int, _i64p, _i64p, _i64p, _i64p, _dp, C.c_double, vp, C.POINTER(vp)]
    L.pwa_ens_destroy.argtypes = [vp]
    L.pwa_ens_slot_count.argtypes = [vp]
    L.pwa_ens_slots.argtypes = [_fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, _dp]
    L.pwa_ens_gram.argtypes = [vp, _dp, _dp]
    L.pwa_ens_set_launch.argtypes = [vp, C.c_int, C.c_int]
    L.pwa_ens_eval.argtypes = [vp, _dp, C.POINTER(C.c_int), C.c_double, _dp, _dp, _i64p]
    L.pwa_ens_last_ms.argtypes = [vp]
    L.pwa_ens_last_ms.restype = C.c_double
    L.pwa_ens_setup_ms.argtypes = [vp, _dp, _dp]
    L._ens_bound = True
    return L


def coupling_names(model) -> list:
    """Fit parameters of an ensemble fit: the LS couplings (Re, Im pairs) in which the helicity couplings
    are linear, i.e. all of them except the common Lambda* scale (a product with every Lambda* coupling),
    each Pc entry's first pair (it scales the entry's others, RooTDalitz's PartWaveCoffZ), and the
    first Lambda* resonance's first pair, which fixes the overall size and phase of the amplitude (the
    likelihood does not depend on them)."""
    out = []
    first_l = True
    for r in model.resonances:
        refs = list(r.couplings)
        if r.chain == "L":
            if first_l:
                refs = refs[2:]
                first_l = False
        else:
            refs = refs[2:]
        for ref in refs:
            if isinstance(ref, str) and ref not in model.derived and ref not in out:
                out.append(ref)
    return out


def _block_args(b):
    pl = np.ascontiguousarray(b.data, np.float32)
    return pl, (pl.ctypes.data_as(_fp), b.para_size, b.vamp_size, b.spline_size, b.NR, b.NZ, b.NX, b.ffr, b.ffb)


@dataclasses.dataclass
class EnsembleFit:
    x: np.ndarray        # [toys, params] fitted values
    fval: np.ndarray     # FCN at the minimum
    errors: np.ndarray   # sqrt(2 up V_ii)
    edm: np.ndarray
    iterations: np.ndarray
    converged: np.ndarray
    calls: int           # ensemble evaluations
    device_ms: float     # summed device time of the evaluations


class Ensemble:
    """A toy ensemble (`toys.ToyEnsemble` bound to `ctx`) with the fit parameters `names` (couplings of
    `model` at `vals`)."""

    def __init__(self, ctx, toy_ens, model, vals: dict, names: list, nll_shift: float = 1e7):
        self.L = _bind(lib.load())
        self.ctx, self.toys, self.model, self.names = ctx, toy_ens, model, list(names)
        self.vals = dict(vals)
        self.nll_shift = nll_shift
        self.builder = BlockBuilder(model, vals)
        b0 = self.builder.block()
        self.x0 = np.array([vals[n] for n in names], float)
        T = toy_ens.n_toys
        first = np.ascontiguousarray(toy_ens.offsets[:-1], np.int64)
        count = np.ascontiguousarray(np.diff(toy_ens.offsets), np.int64)
        band = np.array([toy_ens.view(t).reference_band_args() for t in range(T)], np.int64).reshape(T, 2)
        a, b = np.ascontiguousarray(band[:, 0]), np.ascontiguousarray(band[:, 1])
        self.wdata = np.ascontiguousarray(toy_ens.sum_w, np.float64)
        # slots of the centre and their (linear) dependence on the fit parameters
        self.n_slot = 2 * (6 * b0.NR + 12 * b0.NZ)
        self.s0 = self._slots_host(b0)
        J = np.zeros((self.n_slot, len(names)), complex)
        for j, n in enumerate(names):
            s1 = self._slots_host(self.builder.block({n: self.x0[j] + 1.0}))
            s2 = self._slots_host(self.builder.block({n: self.x0[j] + 2.0}))
            J[:, j] = s1 - self.s0
            curv = np.abs(s2 - 2 * s1 + self.s0)
            scale = np.abs(J[:, j]).max() + 1e-30
            if curv.max() > 1e-5 * scale + 1e-12:
                raise ValueError(f"{n}: the couplings are not linear in this parameter (fix it for the ensemble fit)")
        # jointly linear too (no parameter that scales others)
        d = np.random.default_rng(0).normal(0, 0.3, len(names))
        sj = self._slots_host(self.builder.block(dict(zip(names, self.x0 + d))))
        if np.abs(sj - (self.s0 + J @ d)).max() > 1e-5 * (np.abs(sj).max() + 1e-30):
            raise ValueError("the couplings are not jointly linear in these parameters (one of them scales others)")
        self.J = J
        active = ((np.abs(self.s0) > 0) | (np.abs(J).max(axis=1) > 0)).astype(np.uint8)
        pl, args = _block_args(b0)
        h = C.c_void_p()
        lib.check(self.L.pwa_ens_create(ctx.h, *args, T, first.ctypes.data_as(_i64p), count.ctypes.data_as(_i64p),
                                        a.ctypes.data_as(_i64p), b.ctypes.data_as(_i64p),
                                        self.wdata.ctypes.data_as(_dp), float(toy_ens.sample.sum_w_mc),
                                        active.ctypes.data_as(C.c_void_p), C.byref(h)), "pwa_ens_create")
        self.h = h
        self.n_toys = T
        assert self.L.pwa_ens_slot_count(h) == self.n_slot

    def _slots_host(self, block) -> np.ndarray:
        """Slot vector of a parameter block, decoded as the evaluator decodes it."""
        out = np.zeros(2 * self.n_slot, np.float64)
        pl, args = _block_args(block)
        lib.check(self.L.pwa_ens_slots(*args, out.ctypes.data_as(_dp)), "pwa_ens_slots")
        return out[0::2] + 1j * out[1::2]

    def close(self):
        if getattr(self, "h", None):
            self.L.pwa_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------------ evaluation
    def slots(self, X: np.ndarray) -> np.ndarray:
        """Slot vectors [toys, n_slot] of the parameter vectors X [toys, params]."""
        return self.s0[None, :] + (np.asarray(X, float) - self.x0[None, :]) @ self.J.T

    def exact_slots(self, x: np.ndarray) -> np.ndarray:
        """Slots of the float parameter block at x (as the single-point evaluator sees them)."""
        return self._slots_host(self.builder.block(dict(zip(self.names, map(float, x)))))

    def eval_slots(self, S: np.ndarray, on=None, grad: bool = True):
        """(out [toys, 4] = NLL, data term, sumint, sum_noint; dNLL/dconj(c) [toys, n_slot] or None;
        bad [toys]) at slot vectors S [toys, n_slot]."""
        S = np.ascontiguousarray(np.asarray(S, complex))
        Sr = np.ascontiguousarray(S.view(np.float64))
        on_a = np.ones(self.n_toys, np.int32) if on is None else np.ascontiguousarray(on, np.int32)
        out = np.full((self.n_toys, 4), np.nan)
        g = np.zeros((self.n_toys, 2 * self.n_slot)) if grad else None
        bad = np.zeros(self.n_toys, np.int64)
        lib.check(self.L.pwa_ens_eval(self.h, Sr.ctypes.data_as(_dp), on_a.ctypes.data_as(C.POINTER(C.c_int)),
                                      self.nll_shift, out.ctypes.data_as(_dp),
                                      g.ctypes.data_as(_dp) if grad else None, bad.ctypes.data_as(_i64p)),
                  "pwa_ens_eval")
        gc = g[:, 0::2] + 1j * g[:, 1::2] if grad else None
        return out, gc, bad

    def fcn_grad(self, X: np.ndarray, on=None):
        """FCN = NLL - nll_shift of each toy at its parameter vector (rows of X) and its gradient in
        the fit parameters: dF/dx_j = 2 Re sum_s conj(J_sj) dF/dconj(c_s)."""
        out, gc, _ = self.eval_slots(self.slots(X), on)
        return out[:, 0] - self.nll_shift, 2.0 * np.real(gc @ np.conj(self.J))

    def gram(self):
        M = np.zeros((self.n_slot, self.n_slot), complex)
        Mn = np.zeros_like(M)
        lib.check(self.L.pwa_ens_gram(self.h, M.view(np.float64).ctypes.data_as(_dp),
                                      Mn.view(np.float64).ctypes.data_as(_dp)), "pwa_ens_gram")
        return M, Mn

    def last_ms(self) -> float:
        return float(self.L.pwa_ens_last_ms(self.h))

    def setup_ms(self) -> tuple:
        a, b = C.c_double(), C.c_double()
        lib.check(self.L.pwa_ens_setup_ms(self.h, C.byref(a), C.byref(b)), "pwa_ens_setup_ms")
        return a.value, b.value

    def set_launch(self, warps: int, tile_events: int):
        lib.check(self.L.pwa_ens_set_launch(self.h, int(warps), int(tile_events)), "pwa_ens_set_launch")

    # ------------------------------------------------------------------ fit
    def hessian(self, X: np.ndarray, on=None, rel: float = 1e-4) -> tuple:
        """Hessian of every toy's FCN at X by forward differences of the analytic gradient: one ensemble
        call per parameter, every toy stepped at once.  Returns (H [toys, P, P], calls, device ms)."""
        T, P = X.shape
        _, g0 = self.fcn_grad(X, on)
        H = np.zeros((T, P, P))
        calls, ms = 1, self.last_ms()
        for j in range(P):
            h = rel * max(abs(float(np.abs(X[:, j]).max())), 0.1)
            Xj = X.copy()
            Xj[:, j] += h
            _, gj = self.fcn_grad(Xj, on)
            H[:, :, j] = (gj - g0) / h
            calls += 1
            ms += self.last_ms()
        return 0.5 * (H + np.transpose(H, (0, 2, 1))), calls, ms

    def fit(self, X0=None, tolerance: float = 0.1, up: float = 0.5, max_iter: int = 300, toys=None) -> EnsembleFit:
        """Minimise every toy's FCN together: quasi-Newton (BFGS on the inverse Hessian) per toy, started
        from the finite-difference Hessian of the analytic gradient (eigenvalues floored by modulus, so
        that the first steps are Newton steps wherever the FCN is convex), a backtracking line search
        whose trial points of all toys go into one evaluation, convergence per toy on EDM = g^T V g / 2 <
        0.002 tolerance up (Migrad's criterion); errors sqrt(2 up V_ii).  The toys' inverse Hessians are
        updated together as one batched tensor (on the GPU when the ensemble has one)."""
        import torch
        dev = torch.device("cuda", getattr(self.ctx, "device", 0)) if (getattr(self, "h", None) and
                                                                      torch.cuda.is_available()) else torch.device("cpu")
        T, P = self.n_toys, len(self.names)
        X = np.repeat(self.x0[None, :], T, axis=0) if X0 is None else np.array(X0, float)
        active = np.zeros(T, bool)
        active[list(range(T)) if toys is None else list(toys)] = True
        f, g = self.fcn_grad(X, active)
        calls, dev_ms = 1, self.last_ms()
        H, c, ms = self.hessian(X, active)
        calls += c
        dev_ms += ms
        Ht = torch.as_tensor(H, dtype=torch.float64, device=dev)
        w, U = torch.linalg.eigh(Ht)
        floor = 1e-8 * torch.clamp(w.abs().amax(dim=1, keepdim=True), min=1e-300)
        V = (U / torch.maximum(w.abs(), floor)[:, None, :]) @ U.transpose(1, 2)
        tX = torch.as_tensor(X, dtype=torch.float64, device=dev)
        tf = torch.as_tensor(f, dtype=torch.float64, device=dev)
        tg = torch.as_tensor(g, dtype=torch.float64, device=dev)
        tact = torch.as_tensor(active, device=dev)
        crit = 0.002 * tolerance * up
        edm = 0.5 * torch.einsum("ti,tij,tj->t", tg, V, tg)
        conv = edm < crit
        it = torch.zeros(T, dtype=torch.int64, device=dev)
        alpha = torch.ones(T, dtype=torch.float64, device=dev)
        D = -torch.einsum("tij,tj->ti", V, tg)
        busy = tact & ~conv
        while bool(busy.any()):
            Xt = tX + alpha[:, None] * D
            b_np = busy.cpu().numpy()
            ft_np, gt_np = self.fcn_grad(torch.where(busy[:, None], Xt, tX).cpu().numpy(), b_np)
            calls += 1
            dev_ms += self.last_ms()
            ft = torch.as_tensor(np.nan_to_num(ft_np, nan=np.inf), dtype=torch.float64, device=dev)
            gt = torch.as_tensor(gt_np, dtype=torch.float64, device=dev)
            slope = torch.einsum("ti,ti->t", tg, D)
            ok = busy & torch.isfinite(ft) & (ft <= tf + 1e-4 * alpha * slope)
            fail = busy & ~ok
            # BFGS update of the accepted toys' inverse Hessians (rho = 0 leaves the others as they are)
            sv = torch.where(ok[:, None], Xt - tX, torch.zeros_like(tX))
            yv = torch.where(ok[:, None], gt - tg, torch.zeros_like(tg))
            sy = torch.einsum("ti,ti->t", sv, yv)
            rho = torch.where(ok & (sy > 1e-300), 1.0 / torch.where(sy > 1e-300, sy, torch.ones_like(sy)),
                              torch.zeros_like(sy))
            Vy = torch.einsum("tij,tj->ti", V, yv)
            yVy = torch.einsum("ti,ti->t", yv, Vy)
            V = (V - rho[:, None, None] * (sv[:, :, None] * Vy[:, None, :] + Vy[:, :, None] * sv[:, None, :])
                 + (rho * rho * yVy + rho)[:, None, None] * sv[:, :, None] * sv[:, None, :])
            tX = torch.where(ok[:, None], Xt, tX)
            tf = torch.where(ok, ft, tf)
            tg = torch.where(ok[:, None], gt, tg)
            it = it + ok.to(torch.int64)
            edm_new = 0.5 * torch.einsum("ti,tij,tj->t", tg, V, tg)
            edm = torch.where(ok, edm_new, edm)
            conv = conv | (ok & (edm_new < crit))
            alpha = torch.where(ok, torch.ones_like(alpha), alpha * torch.where(fail, 0.3, 1.0))
            Dn = -torch.einsum("tij,tj->ti", V, tg)
            # not a descent direction: restart that toy's metric from its diagonal
            restart = ok & (torch.einsum("ti,ti->t", tg, Dn) >= 0)
            if bool(restart.any()):
                diag = torch.diag_embed(torch.diagonal(V, dim1=1, dim2=2).abs())
                V = torch.where(restart[:, None, None], diag, V)
                Dn = -torch.einsum("tij,tj->ti", V, tg)
            D = torch.where(ok[:, None], Dn, D)
            stuck = fail & (alpha < 1e-10)  # no descent along the metric: at the precision limit
            conv = conv | (stuck & (edm < 1e3 * crit))
            it = torch.where(stuck, torch.full_like(it, max_iter), it)
            busy = tact & ~conv & (it < max_iter)
        X, f = tX.cpu().numpy(), tf.cpu().numpy()
        edm, it, conv = edm.cpu().numpy(), it.cpu().numpy(), conv.cpu().numpy()
        err = np.sqrt(np.maximum(2 * up * torch.diagonal(V, dim1=1, dim2=2).cpu().numpy(), 0))
        return EnsembleFit(X, f, err, edm, it, conv & active, calls, dev_ms)


# ------------------------------------------------------------------ autotuner
CANDIDATES = [(16, 256), (16, 1024), (16, 4096), (12, 256), (12, 1024), (8, 256), (8, 1024), (4, 1024)]


def _cache_path() -> Path:
    from .autotune import cache_path
    return cache_path("ensemble_tune.json")


def tune_key(ens: Ensemble) -> str:
    import torch
    dev = torch.cuda.get_device_name(getattr(ens.ctx, "device", 0))
    events = int(ens.toys.offsets[-1])
    bucket = int(np.round(np.log2(max(events, 1))))
    return f"{dev}|NR={ens.builder.block().NR}|NZ={ens.builder.block().NZ}|toys={ens.n_toys}|events~2^{bucket}"


def autotune(ens: Ensemble, cache: str | Path | None = None, reps: int = 3, force: bool = False) -> dict:
    """Picks the launch shape of the ensemble kernel: the cached choice for this device and ensemble
    shape, else the fastest candidate (warps per block, events per work item) timed with CUDA events
    over `reps` evaluations at the centre (after one warm-up), written back to the cache."""
    path = Path(cache) if cache else _cache_path()
    key = tune_key(ens)
    table = {}
    if path.exists():
        try:
            table = json.loads(path.read_text())
        except (OSError, ValueError):
            table = {}
    if key in table and not force:
        c = table[key]
        ens.set_launch(c["warps"], c["tile_events"])
        return dict(c, cached=True)
    S = np.repeat(ens.s0[None, :], ens.n_toys, axis=0)
    timings = []
    for w, te in CANDIDATES:
        try:
            ens.set_launch(w, te)
        except lib.PwaError:
            continue  # the shape does not fit this model (shared memory per block)
        ens.eval_slots(S)
        ms = []
        for _ in range(reps):
            ens.eval_slots(S)
            ms.append(ens.last_ms())
        timings.append((float(np.median(ms)), w, te))
    best = min(timings)
    ens.set_launch(best[1], best[2])
    choice = {"warps": best[1], "tile_events": best[2], "ms": best[0],
              "candidates": [{"warps": w, "tile_events": te, "ms": m} for m, w, te in timings]}
    table[key] = choice
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(table, indent=1))
    except OSError:
        pass
    return dict(choice, cached=False)
