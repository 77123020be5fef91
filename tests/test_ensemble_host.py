"""Host side of the toy-ensemble evaluator (no GPU): the slot vector of a parameter block (the helicity
couplings as the device kernels index them), its linear dependence on the ensemble's fit parameters,
and the refusal of models the ensemble evaluator does not take."""
import ctypes as C

import numpy as np
import pytest


def _slots(blk):
    from pwa_b200 import ensemble, lib
    L = ensemble._bind(lib.load())
    n = 2 * (6 * blk.NR + 12 * blk.NZ)
    out = np.zeros(2 * n)
    pl, args = ensemble._block_args(blk)
    rc = L.pwa_ens_slots(*args, out.ctypes.data_as(C.POINTER(C.c_double)))
    return rc, out[0::2] + 1j * out[1::2]


def test_slots_are_the_blocks_helicity_couplings():
    """Each Lambda* resonance's 2 x 6 slots hold the block's helicity-coupling floats (J = 1/2: the
    first four m of each proton helicity), each Pc entry's 2 x 12 slots theirs, in resonance order
    when the Pc entries are Breit-Wigners (group order = resonance order)."""
    from pwa_b200 import configs, model as M
    mdl, vals = configs.small_bw()
    blk = M.build_param_block(mdl, vals)
    rc, s = _slots(blk)
    assert rc == 0
    NR, NZ = blk.NR, blk.NZ
    NS = 6 * NR + 12 * NZ
    vamp = np.asarray(blk.data[blk.para_size:blk.para_size + blk.vamp_size], np.float64)
    pos = 0
    for ir, r in enumerate(mdl.resonances):
        if r.chain == "L":
            for k in range(2):
                for m in range(6):
                    if r.spin2 == 1 and m >= 4:
                        assert s[k * NS + ir * 6 + m] == 0
                        continue
                    assert s[k * NS + ir * 6 + m] == complex(vamp[pos], vamp[pos + 1])
                    pos += 2
        else:
            q = ir - NR
            got = [s[k * NS + 6 * NR + q * 12 + m] for k in range(2) for m in range(12)]
            nz = [g for g in got if g != 0]
            want = [complex(vamp[i], vamp[i + 1]) for i in range(pos, pos + 2 * len(nz), 2)]
            assert nz == [w for w in want if w != 0]
            pos += 2 * len(nz)


def test_fit_parameters_enter_linearly():
    """The coupling parameters of an ensemble fit move the slots linearly: slots(x0 + d) = slots(x0) +
    J d to float rounding, with J from unit steps; the excluded scale parameters do not."""
    from pwa_b200 import configs, ensemble, model as M
    mdl, vals = configs.small_kmatrix()
    names = ensemble.coupling_names(mdl)
    assert "scRe" not in names and len(names) > 10
    b = M.BlockBuilder(mdl, vals)
    x0 = np.array([vals[n] for n in names])
    _, s0 = _slots(b.block())
    J = np.stack([_slots(b.block({n: x0[j] + 1.0}))[1] - s0 for j, n in enumerate(names)], axis=1)
    d = np.random.default_rng(1).normal(0, 0.5, len(names))
    _, sd = _slots(b.block(dict(zip(names, x0 + d))))
    assert np.abs(sd - (s0 + J @ d)).max() < 1e-5 * np.abs(sd).max()
    # the Lambda* scale multiplies every Lambda* coupling: not linear jointly with them
    _, s2 = _slots(b.block({"scRe": vals["scRe"] + 1.0, names[0]: x0[0] + 1.0}))
    _, s1 = _slots(b.block({"scRe": vals["scRe"] + 1.0}))
    assert np.abs((s2 - s1) - J[:, 0]).max() > 1e-3


def test_zcs_models_are_refused():
    from pwa_b200 import configs, model as M
    mdl, vals = configs.small_zcs()
    rc, _ = _slots(M.build_param_block(mdl, vals))
    assert rc == 5  # PWA_E_UNSUPPORTED


def test_batched_minimiser_on_known_functions():
    """The ensemble's batched quasi-Newton minimiser (vectorised BFGS updates, shared line-search calls)
    on a synthetic FCN per toy: a convex quartic-plus-quadratic with a known minimum, a different one
    per toy, and a flat direction (a parameter the FCN does not depend on)."""
    from pwa_b200 import ensemble
    rng = np.random.default_rng(3)
    T, P = 6, 9
    A = rng.normal(size=(T, P, P))
    Q = np.einsum("tij,tkj->tik", A, A) + 0.5 * np.eye(P)
    Q[:, :, -1] = Q[:, -1, :] = 0.0  # the last parameter is flat
    xm = rng.normal(size=(T, P))

    def fcn_grad(X, on=None):
        d = X - xm
        f = 0.5 * np.einsum("ti,tij,tj->t", d, Q, d) + 0.1 * np.sum(d[:, :-1] ** 4, axis=1)
        g = np.einsum("tij,tj->ti", Q, d)
        g[:, :-1] += 0.4 * d[:, :-1] ** 3
        return f, g

    E = ensemble.Ensemble.__new__(ensemble.Ensemble)
    E.n_toys, E.names, E.x0 = T, [f"p{i}" for i in range(P)], np.zeros(P)
    E.fcn_grad = fcn_grad
    E.last_ms = lambda: 0.0
    E.h = None
    fit = E.fit(tolerance=1e-4)
    assert np.all(fit.converged)
    # EDM < 1e-7 leaves |x - x_min| ~ sqrt(2 EDM / lambda_min) ~ 1e-3 at most
    assert np.max(np.abs(fit.x[:, :-1] - xm[:, :-1])) < 1e-3
    assert np.all(fit.x[:, -1] == 0.0)  # the flat direction does not move
