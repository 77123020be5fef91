"""Host model layer: parameter block layout, coupling structure, constraints and the FCN."""
import math

import numpy as np
import pytest

from pwa_b200 import configs, model as M


@pytest.mark.parametrize("name", list(configs.MODELS))
def test_block_layout(name):
    mdl, vals = configs.MODELS[name]()
    b = M.build_param_block(mdl, vals)
    assert b.para_size == 6 * (mdl.NR + mdl.NZ + mdl.NX)
    exp = sum(16 if r.spin2 == 1 else 24 for r in mdl.lstar)
    for r in mdl.pc:
        S = r.spin2 / 2
        exp += 2 * 2 * sum(1 for hpsi in (-1, 0, 1) for _ in range(2) for hp in (-0.5, 0.5) if abs(hpsi - hp) <= S)
    for r in mdl.zcs:
        S = r.spin2 / 2
        exp += 2 * 2 * sum(1 for hpsi in (-1, 0, 1) if abs(hpsi) <= S for hp in (-0.5, 0.5)
                           for hz in (hp - 0.5, hp + 0.5) if abs(hz) <= S)
    assert b.vamp_size == exp
    spl = sum(9 * (M.NUMSP if r.chain == "L" else M.NUMSPZ) for r in mdl.resonances if r.type == M.MODELINDEPENDENT)
    assert b.spline_size == spl
    assert len(b.data) == b.para_size + b.vamp_size + b.spline_size + M.KM_SIZE
    assert b.data.dtype == np.float32


def test_spline_coefficients_not_a_knot():
    """The spline blocks' coefficients: a cubic through the knots with not-a-knot end conditions
    (TSpline3's default), checked against scipy's independent implementation, and the block layout
    (knots, then (y, b, c, d) per knot of Re, then of Im) of RooDalitzAmplitude.cxx:2741-2764."""
    from scipy.interpolate import CubicSpline
    rng = np.random.default_rng(3)
    x = np.sort(rng.uniform(1.43, 2.52, 24))
    y = rng.normal(size=24)
    c = M.spline_coefficients(x, y)
    ref = CubicSpline(x, y, bc_type="not-a-knot")
    assert np.allclose(c[:-1, ::-1].T, ref.c, rtol=1e-9, atol=1e-9)
    t = np.linspace(x[0], x[-1], 777)
    k = np.clip(np.searchsorted(x, t, side="right") - 1, 0, len(x) - 2)
    dt = t - x[k]
    v = c[k, 0] + dt * (c[k, 1] + dt * (c[k, 2] + dt * c[k, 3]))
    assert np.allclose(v, ref(t), rtol=1e-9, atol=1e-9)
    blk = M.spline_block(x, y, 2 * y)
    n = len(x)
    assert len(blk) == 9 * n
    assert np.allclose(np.array(blk[:n]), x.astype(np.float32))
    assert np.allclose(np.array(blk[n:5 * n]).reshape(n, 4), c.astype(np.float32))
    assert np.allclose(np.array(blk[5 * n:]).reshape(n, 4), (2 * c).astype(np.float32))


def test_pc_couplings_do_not_depend_on_proton_helicity():
    mdl, vals = configs.kmatrix()
    b = M.build_param_block(mdl, vals)
    cnt = b.para_size + sum(16 if r.spin2 == 1 else 24 for r in mdl.lstar)
    for r in mdl.pc:
        n = (8 if r.spin2 == 1 else 12) * 2
        c = b.data[cnt:cnt + 2 * n]
        assert np.array_equal(c[:n], c[n:])
        cnt += 2 * n


def test_kmatrix_block_symmetrised():
    mdl, vals = configs.kmatrix()
    b = M.build_param_block(mdl, vals)
    km = b.data[b.kmcount:].reshape(4, 32)
    for ik in range(4):
        f = km[ik, 16:].reshape(4, 4)
        for i in range(1, 4):
            assert f[i, 0] == f[0, i]
    # 1/2- group: two poles (g rows 0..1), four non-resonant scattering values in row 0
    g = km[0, :16].reshape(4, 4)
    assert np.all(g[2:] == 0) and np.all(g[:2] != 0)
    assert vals["fsc_ZM1SC1"] == pytest.approx(float(km[0, 16]))


def test_include_subset_zeroes_other_couplings():
    mdl, vals = configs.small_bw()
    full = M.build_param_block(mdl, vals).data
    part = M.build_param_block(mdl, vals, include=([0], [])).data
    assert np.array_equal(full[:12], part[:12])
    assert np.any(part[12:] != full[12:])


def test_constraint_and_fcn():
    c = M.Constraint("m0", 1.0, 1.2, 0.1, 0.2, 0.5, 2.0)
    assert c.penalty(1.1) == 0.0
    assert c.penalty(0.9) == pytest.approx(0.5)
    assert c.penalty(1.4) == pytest.approx(0.5)
    cons = M.read_constraints("m0 1.0 1.2 0.1 0.2 0.5 2.0\n")
    assert M.fcn(10000010.0, 1e7, 2.0, cons, {"m0": 0.9}) == pytest.approx(20.5)


def test_orbital_l():
    r = configs.lstar_resonance("1520")  # 3/2-
    assert M.orbital_l(r) == 2
    r = configs.lstar_resonance("1600")  # 1/2+
    assert M.orbital_l(r) == 1
    assert M.orbital_l(configs.pc_bw("x", 1, -1)) == 0
    assert M.orbital_l(configs.pc_bw("x", 1, +1)) == 1
    assert M.orbital_l(configs.pc_bw("x", 3, +1)) == 1
