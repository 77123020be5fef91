"""The FP64 oracle's spline, revised K-matrix and triangle-cusp lineshapes pinned against the
reference's own code built for host cores (model `lineshapes`: a Lambda* S-wave spline on the
reference's 24-knot fixture, a Lambda* revised K-matrix of three 1/2- entries, a Pc revised K-matrix
pair, a Pc triangle cusp and a Pc spline wave)."""
import json
from pathlib import Path

import numpy as np
import pytest

from conftest import make_test_sample

BUCKET = (5, 5, 0)
GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def ref(oracle_mod):
    if oracle_mod.ref_lib(*BUCKET, build_if_missing=True) is None:
        pytest.skip("reference host build unavailable")
    return oracle_mod


def _isolated(O, name, include):
    """Unsmeared |A|^2 of one subset of resonances (the others' couplings zeroed) from the oracle and
    from the reference (host_store_fx first: host_store_amp2s uses the spline offsets and barrier radii
    that call configures)."""
    from pwa_b200 import model as M
    mdl, vals, blk, smp = make_test_sample(name, 600, 6000, seed=31)
    b = M.build_param_block(mdl, vals, include=include)
    a_o = O.amp2(smp, b)
    rh = O.RefHost(smp, b)
    rh.store_fx(b)
    return a_o, rh.amp2s(b), smp


def test_full_model_nll_and_events(ref):
    mdl, vals, blk, smp = make_test_sample("lineshapes", 600, 6000, seed=31)
    v, s, fx, _ = ref.nll(smp, blk)
    rh = ref.RefHost(smp, blk)
    rv, rs = rh.store_fx(blk)
    rel = np.abs(rh.fx - fx) / np.abs(fx)
    assert abs(rv - v) < 0.01 and abs(rs / s - 1) < 5e-5
    assert np.median(rel) < 1e-6


@pytest.mark.parametrize("label,include", [("lstar_spline", ([1], [])), ("pc_spline", ([], [4])),
                                           ("lstar_rkm", ([2, 3, 4], [])), ("pc_rkm", ([], [1, 2])),
                                           ("bw", ([0], [0]))])
def test_subsets_agree_to_float32_noise(ref, label, include):
    a_o, a_r, _ = _isolated(ref, "lineshapes", include)
    zero = a_o == 0  # outside a spline's range both give 0
    assert np.all(a_r[zero] == 0)
    rel = np.abs(a_r - a_o)[~zero] / a_o[~zero]
    assert np.median(rel) < 2e-6 and np.max(rel) < 5e-4, (np.median(rel), np.max(rel))


def test_swave_fixture_spline(ref):
    """The reference's own 24-knot S-wave (Fit_Jpsippi/toyr_fine_bin.dat, read from the golden
    fixture) as the Lambda* spline: oracle and reference agree to float noise."""
    from pwa_b200 import configs, dataset as D, model as M
    knots = json.loads((GOLDEN / "swave_knots.json").read_text())
    mdl, vals = configs.lineshapes(swave=[(k[1], k[2]) for k in knots])
    assert [k[0] for k in knots] == list(configs.SWAVE_KNOTS)
    b = M.build_param_block(mdl, vals, include=([1], []))
    smp = D.make_sample(10, 4000, (1.0, 1.0), 5, lambda a: np.ones(len(a["mLk"])))
    a_o = ref.amp2(smp, b)
    rh = ref.RefHost(smp, b)
    rh.store_fx(b)
    rel = np.abs(rh.amp2s(b) - a_o) / a_o
    assert np.max(rel) < 1e-5


def _cusp_np(mz, m_r, g, dt):
    """The triangle cusp (GetCusp_AMP, cu_DPFPropogator.cu:1223-1343) vectorised over masses, with the
    reference's complex square root, logarithm and arctangent (RooTDalitz/cuComplex.h:641-676), in
    float32 (an emulation of the reference's arithmetic) or float64."""
    C = np.complex64 if dt == np.float32 else np.complex128
    f = np.float32

    def csqrt(x):
        r = np.abs(x).astype(dt)
        cosA = (x.real / r).astype(dt)
        out = (np.sqrt((r * (cosA + 1) / 2).astype(dt)) + 1j * np.sqrt((r * (1 - cosA) / 2).astype(dt))).astype(C)
        flip = np.signbit(x.imag) & (np.abs(x.imag / x.real) > dt(0.001))
        out = np.where(flip, np.conj(out), out)
        return np.where((np.abs(x.real) < dt(1e-6)) & (np.abs(x.imag) < dt(1e-6)), C(0), out)

    def catan(x):
        z = ((1 + 1j * x) / (1 - 1j * x)).astype(C)
        r = np.sqrt(z.real * z.real + z.imag * z.imag).astype(dt)
        th = np.arccos((z.real / r).astype(dt)).astype(dt)
        th = np.where(z.imag < 0, -th, th)
        return (C(-0.5) * (1j * (np.log(r).astype(dt) + 1j * th))).astype(C)

    # the reference's float constants and parameters, promoted to dt
    p12, p13, m2, m3 = (dt(np.float32(x)) for x in (5.61951, 0.493677, 3.51067, 0.938272046))
    m_r, g = dt(np.float32(m_r)), dt(np.float32(g))
    m1 = C(complex(m_r, -g / 2))
    p23 = np.asarray(mz, dt)
    dx = dt(f(1.0 / 100))
    out = np.zeros(len(p23), C)
    for i in range(100):
        a = dt(f(i) * f(dx) + f(dx) / f(2))
        b = ((a * (p12 * p12 - p13 * p13 - p23 * p23) + m3 * m3 - m2 * m2) / p23 / p23 + 1 - C(0.001j)).astype(C)
        c = ((a * (m1 * m1 - m3 * m3) + m3 * m3 - a * (1 - a) * p13 * p13) / (p23 * p23)).astype(C)
        sv = csqrt((4 * c - b * b).astype(C))
        out = out + dx * ((1 / sv) * (catan(b / sv) - catan((b + 2 * (a - 1)) / sv)))
    return out * (1 / p23 / p23)


def test_cusp_matches_and_its_deviations_are_float32_branch_flips(ref):
    """The cusp integrates 100 bins, each through the reference's complex square root, whose imaginary
    sign follows the input's only when |Im/Re| > 1e-3: the lineshape jumps wherever one bin crosses that
    threshold, and those masses move with the arithmetic's precision (by up to hundreds of keV in
    float32).  The oracle follows the formula in FP64: it equals a second FP64 restatement; the
    reference agrees with it for the great majority of events; and where it does not, a float32
    emulation of the reference's arithmetic reproduces a large share of the reference's deviations,
    i.e. they are the reference's float32 branch flips, not a difference in the formula."""
    from pwa_b200 import configs, model as M
    mdl, vals = configs.lineshapes()
    blk = M.build_param_block(mdl, vals)
    ms = np.linspace(4.04, 5.12, 301)
    orc = np.array([ref.lineshapes(blk, 1.8, m)[1][3] for m in ms])
    m_r, g = vals["m0_T4337"], vals["width_T4337"]
    bar = np.array([ref.lib().oracle_barrier_lb_pc(0.5, m, m_r, blk.ffb) for m in ms])
    assert np.allclose(orc, _cusp_np(ms, m_r, g, np.float64) * bar, rtol=1e-10, atol=0)
    a_o, a_r, smp = _isolated(ref, "lineshapes", ([], [3]))
    rel = np.abs(a_r - a_o) / a_o
    assert np.mean(rel < 1e-4) > 0.9 and np.median(rel) < 2e-5
    bad = np.nonzero(rel > 1e-3)[0]
    mz = smp.pp[smp.n_size:smp.n_size + smp.n][bad]
    emu = np.abs(_cusp_np(mz, np.float32(m_r), np.float32(g), np.float32)) ** 2 / np.abs(
        _cusp_np(mz.astype(float), m_r, g, np.float64)) ** 2
    ratio = (a_r / a_o)[bad]
    share = np.mean(np.abs(emu - ratio) < 0.02 * np.abs(ratio - 1))
    assert share > 0.3, share


def test_lineshape_diagnostic_matches_reference(ref):
    """host_store_lineshapeLsKM: the revised K-matrix (refactored form) and Breit-Wigner lineshapes of
    every Lambda* entry times the Lambda_b barrier, oracle vs the reference's own function."""
    from pwa_b200 import configs, model as M
    mdl, vals = configs.lineshapes()
    blk = M.build_param_block(mdl, vals)
    m = np.linspace(1.44, 2.5, 64).astype(np.float32)
    km_o, bw_o = ref.lineshapes_lstar_km(blk, m)
    km_r, bw_r = ref.ref_lineshapes_lstar_km(blk, m)
    for o, r in ((km_o, km_r), (bw_o, bw_r)):
        fin = np.isfinite(o)
        assert np.array_equal(fin, np.isfinite(r))  # the non-resonant entry's factor is NaN in both
        assert np.max(np.abs(r[fin] - o[fin]) / np.maximum(np.abs(o[fin]), 1e-12)) < 2e-5
