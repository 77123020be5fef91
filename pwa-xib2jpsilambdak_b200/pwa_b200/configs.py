"""Model configurations of the benchmark workloads, with seeded parameter values.

Resonance masses and widths are PDG-like values; couplings are drawn from a seeded generator.  The
list layouts follow the reference model files (RooTDalitz/JPResL.h:22-36 for Lambda*, RooTDalitz/
ResZKM_alternateCoupling.h:18-46,135-146 for K-matrix Pc entries, RooTDalitz/ResZ.h:7-29 for
Breit-Wigner Pc entries).
"""
from __future__ import annotations

import numpy as np

from .model import (BREITWIGNER, KMATRIX, MODELINDEPENDENT, NONRESONANT, NUMSP, NUMSPZ, REVISEDKMATRIX, TRIANGLE,
                    Model, Resonance)

# name, mass, width, 2J, parity
LSTAR_ALL = [
    ("1405", 1.4051, 0.0505, 1, -1),
    ("1520", 1.5195, 0.0156, 3, -1),
    ("1600", 1.600, 0.150, 1, +1),
    ("1670", 1.670, 0.035, 1, -1),
    ("1690", 1.690, 0.070, 3, -1),
    ("1800", 1.800, 0.200, 1, -1),
    ("1810", 1.810, 0.150, 1, +1),
    ("1820", 1.820, 0.080, 5, +1),
    ("1830", 1.830, 0.090, 5, -1),
    ("1890", 1.890, 0.100, 3, +1),
    ("2100", 2.100, 0.200, 7, -1),
    ("2110", 2.110, 0.200, 5, +1),
    ("2020", 2.020, 0.200, 7, +1),
    ("2050", 2.050, 0.200, 3, -1),
]
LSTAR6 = ["1520", "1600", "1670", "1690", "1800", "1810"]
LSTAR14 = [x[0] for x in LSTAR_ALL]


def _lstar(name: str) -> tuple:
    for x in LSTAR_ALL:
        if x[0] == name:
            return x
    raise KeyError(name)


def lstar_resonance(name: str) -> Resonance:
    _, _, _, s2, par = _lstar(name)
    tags = ["p1p1", "p100", "m100", "m1m1", "p3p1", "m3m1"]
    coup = []
    for t in tags:
        coup += [f"a_{t}_{name}", f"p_{t}_{name}"]
    return Resonance("L", name, s2, par, BREITWIGNER, f"m0_{name}", f"width_{name}", tuple(coup), ("scRe", "scIm"))


def pc_bw(name: str, s2: int, par: int) -> Resonance:
    coup = tuple(f"{ap}_{t}_{name}" for t in ("Bp", "L0", "L1", "L2") for ap in ("a", "p"))
    return Resonance("Z", name, s2, par, BREITWIGNER, f"m0_{name}", f"width_{name}", coup)


def pc_km_pole(name: str, s2: int, par: int, channel: int) -> Resonance:
    coup = tuple(f"{ap}_{t}_{name}" for t in ("Bp", "L0", "L1", "L2") for ap in ("a", "p"))
    g = tuple(f"g{i}_{name}" for i in range(1, 5))
    return Resonance("Z", name, s2, par, KMATRIX, f"m0_{name}", float(channel), coup, g)


def pc_km_nr(name: str, shared: str, s2: int, par: int) -> Resonance:
    # The four non-resonant entries of one J^P group share one set of LS couplings
    # (ResZKM_alternateCoupling.h:166-170).
    coup = tuple(f"{ap}_{t}_{shared}" for t in ("Bp", "L0", "L1", "L2") for ap in ("a", "p"))
    return Resonance("Z", name, s2, par, KMATRIX, -0.5, 0.0, coup, (f"fsc_{name}",))


def zcs_bw(name: str, s2: int, par: int) -> Resonance:
    # RooTDalitz/ResX.h: four Lambda_b -> Zcs p couplings (L0..L3), then the Zcs -> J/psi K one (Bp)
    coup = tuple(f"{ap}_{t}_{name}" for t in ("L0", "L1", "L2", "L3", "Bp") for ap in ("a", "p"))
    return Resonance("X", name, s2, par, BREITWIGNER, f"m0_{name}", f"width_{name}", coup)


def _lstar_couplings(name: str) -> tuple:
    coup = []
    for t in ("p1p1", "p100", "m100", "m1m1", "p3p1", "m3m1"):
        coup += [f"a_{t}_{name}", f"p_{t}_{name}"]
    return tuple(coup)


def lstar_spline(name: str, knot_masses) -> Resonance:
    """Model-independent S-wave (2J = 1, parity -1) of the Lambda* chain: NUMSP spline knots with real
    and imaginary parameters SR_/SI_ at fixed masses (RooTDalitz/ResL.h:1139-1180)."""
    if len(knot_masses) != NUMSP:
        raise ValueError(f"a Lambda* spline wave has {NUMSP} knots")
    knots = tuple((f"SR_{name}_{i:02d}", f"SI_{name}_{i:02d}", float(m)) for i, m in enumerate(knot_masses))
    return Resonance("L", name, 1, -1, MODELINDEPENDENT, f"m0_{name}", f"width_{name}", _lstar_couplings(name),
                     ("scRe", "scIm"), knots)


def lstar_rkm(name: str, s2: int, par: int, mass="", width="") -> Resonance:
    """Lambda* entry of a revised K-matrix (type REVISEDKMATRIX): the entries of one type, spin and
    parity form one coupled set (RooTDalitz/ResL_KM.h)."""
    return Resonance("L", name, s2, par, REVISEDKMATRIX, mass or f"m0_{name}", width or f"width_{name}",
                     _lstar_couplings(name), ("scRe", "scIm"))


def pc_rkm(name: str, s2: int, par: int) -> Resonance:
    """Pc entry of a revised K-matrix (RooTDalitz/ResZKM.h:340-360, the L_Z2BW list)."""
    coup = tuple(f"{ap}_{t}_{name}" for t in ("Bp", "L0", "L1", "L2") for ap in ("a", "p"))
    return Resonance("Z", name, s2, par, REVISEDKMATRIX, f"m0_{name}", f"width_{name}", coup)


def pc_cusp(name: str, s2: int, par: int) -> Resonance:
    """Pc-chain triangle cusp (type TRIANGLE, GetCusp_AMP): mass and width of the particle in the loop."""
    coup = tuple(f"{ap}_{t}_{name}" for t in ("Bp", "L0", "L1", "L2") for ap in ("a", "p"))
    return Resonance("Z", name, s2, par, TRIANGLE, f"m0_{name}", f"width_{name}", coup)


def pc_spline(name: str, s2: int, par: int, knot_masses) -> Resonance:
    """Model-independent wave of the Pc chain: NUMSPZ knots (MakeSplineZ)."""
    if len(knot_masses) != NUMSPZ:
        raise ValueError(f"a Pc spline wave has {NUMSPZ} knots")
    coup = tuple(f"{ap}_{t}_{name}" for t in ("Bp", "L0", "L1", "L2") for ap in ("a", "p"))
    knots = tuple((f"SR_{name}_{i:02d}", f"SI_{name}_{i:02d}", float(m)) for i, m in enumerate(knot_masses))
    return Resonance("Z", name, s2, par, MODELINDEPENDENT, f"m0_{name}", f"width_{name}", coup, (), knots)


def _seed_couplings(model: Model, vals: dict, rng, scale=1.0):
    for r in model.resonances:
        for i in range(0, len(r.couplings), 2):
            a, p = r.couplings[i], r.couplings[i + 1]
            if a not in vals:
                vals[a] = float(rng.normal(0, scale))
                vals[p] = float(rng.normal(0, scale))


def _lstar_vals(names, vals):
    for n in names:
        _, m, w, _, _ = _lstar(n)
        vals[f"m0_{n}"] = m
        vals[f"width_{n}"] = w
    vals["scRe"] = 1.0
    vals["scIm"] = 0.0


def lstar_only(seed: int = 1) -> tuple:
    """Six Lambda* Breit-Wigners, no Pc (the CPU-runnable workload)."""
    m = Model([lstar_resonance(n) for n in LSTAR6], [])
    vals = {}
    _lstar_vals(LSTAR6, vals)
    _seed_couplings(m, vals, np.random.default_rng(seed))
    return m, vals


def full_bw(seed: int = 2) -> tuple:
    """14 Lambda* up to J=7/2 and three narrow Breit-Wigner Pc states."""
    pcs = [pc_bw("Pc4312", 1, -1), pc_bw("Pc4440", 3, -1), pc_bw("Pc4457", 1, -1)]
    m = Model([lstar_resonance(n) for n in LSTAR14], pcs)
    vals = {}
    _lstar_vals(LSTAR14, vals)
    for n, mass, width in (("Pc4312", 4.312, 0.010), ("Pc4440", 4.440, 0.020), ("Pc4457", 4.457, 0.006)):
        vals[f"m0_{n}"] = mass
        vals[f"width_{n}"] = width
    rng = np.random.default_rng(seed)
    _seed_couplings(m, vals, rng)
    for n in ("Pc4312", "Pc4440", "Pc4457"):
        vals[f"a_L0_{n}"] = 1.0
        vals[f"p_L0_{n}"] = 0.0
        vals[f"a_Bp_{n}"] *= 0.3
        vals[f"p_Bp_{n}"] *= 0.3
    return m, vals


def kmatrix(seed: int = 3) -> tuple:
    """Coupled-channel Pc K-matrix (J/psi p, Sigma_c D*, Sigma_c* D*, Sigma_c D) with four poles and
    four non-resonant terms in each of the 1/2- and 3/2- groups, plus six Lambda*."""
    pcs = [
        pc_km_pole("Pc4312", 1, -1, 3),
        pc_km_pole("Pc4457", 1, -1, 1),
        pc_km_pole("Pc4440", 3, -1, 1),
        pc_km_pole("Pc4500", 1, +1, 0),
    ]
    pcs += [pc_km_nr(f"ZM1SC{i}", "ZM1SC1", 1, -1) for i in range(1, 5)]
    pcs += [pc_km_nr(f"ZM3SC{i}", "ZM3SC1", 3, -1) for i in range(1, 5)]
    # K-matrix entries grouped per J^P with poles first (the P-vector output order).
    order = ["Pc4312", "Pc4457", "ZM1SC1", "ZM1SC2", "ZM1SC3", "ZM1SC4", "Pc4440", "ZM3SC1", "ZM3SC2",
             "ZM3SC3", "ZM3SC4", "Pc4500"]
    pcs = sorted(pcs, key=lambda r: order.index(r.name))
    m = Model([lstar_resonance(n) for n in LSTAR6], pcs)
    vals = {}
    _lstar_vals(LSTAR6, vals)
    rng = np.random.default_rng(seed)
    _seed_couplings(m, vals, rng)
    for n, mass in (("Pc4312", 4.312), ("Pc4457", 4.457), ("Pc4440", 4.440), ("Pc4500", 4.50)):
        vals[f"m0_{n}"] = mass
        vals[f"a_L0_{n}"] = 1.0
        vals[f"p_L0_{n}"] = 0.0
        for i in range(1, 5):
            vals[f"g{i}_{n}"] = float(rng.uniform(-0.6, 0.6))
    for grp in ("ZM1SC", "ZM3SC"):
        for i in range(1, 5):
            vals[f"fsc_{grp}{i}"] = float(rng.uniform(-2, 2))
    return m, vals


def small_kmatrix(seed: int = 4) -> tuple:
    """Three Lambda* and a 1/2- K-matrix group with two poles and two non-resonant entries (test size)."""
    pcs = [pc_km_pole("Pc4312", 1, -1, 3), pc_km_pole("Pc4457", 1, -1, 1),
           pc_km_nr("ZM1SC1", "ZM1SC1", 1, -1), pc_km_nr("ZM1SC2", "ZM1SC1", 1, -1)]
    names = ["1520", "1670", "1690"]
    m = Model([lstar_resonance(n) for n in names], pcs)
    vals = {}
    _lstar_vals(names, vals)
    rng = np.random.default_rng(seed)
    _seed_couplings(m, vals, rng)
    for n, mass in (("Pc4312", 4.312), ("Pc4457", 4.457)):
        vals[f"m0_{n}"] = mass
        for i in range(1, 5):
            vals[f"g{i}_{n}"] = float(rng.uniform(-0.6, 0.6))
    for i in (1, 2):
        vals[f"fsc_ZM1SC{i}"] = float(rng.uniform(-2, 2))
    return m, vals


def small_zcs(seed: int = 6) -> tuple:
    """Two Lambda*, a Breit-Wigner Pc and the two Zcs -> J/psi K states of RooTDalitz/ResX.h (1+, 1-)."""
    names = ["1520", "1800"]
    m = Model([lstar_resonance(n) for n in names], [pc_bw("Pc4312", 1, -1)],
              zcs=[zcs_bw("Xplus", 2, +1), zcs_bw("Xminus", 2, -1)])
    vals = {}
    _lstar_vals(names, vals)
    vals["m0_Pc4312"], vals["width_Pc4312"] = 4.312, 0.010
    vals["m0_Xplus"], vals["width_Xplus"] = 4.003, 0.131
    vals["m0_Xminus"], vals["width_Xminus"] = 4.216, 0.091
    _seed_couplings(m, vals, np.random.default_rng(seed))
    return m, vals


def small_bw(seed: int = 5) -> tuple:
    """Two Lambda* and two Breit-Wigner Pc (test size)."""
    names = ["1520", "1800"]
    m = Model([lstar_resonance(n) for n in names], [pc_bw("Pc4312", 1, -1), pc_bw("Pc4440", 3, -1)])
    vals = {}
    _lstar_vals(names, vals)
    for n, mass, width in (("Pc4312", 4.312, 0.010), ("Pc4440", 4.440, 0.020)):
        vals[f"m0_{n}"] = mass
        vals[f"width_{n}"] = width
    _seed_couplings(m, vals, np.random.default_rng(seed))
    return m, vals


# Knot masses of the Lambda* S-wave (24 knots from just above the pK threshold to the upper edge) and
# of the Pc spline wave (11 knots over the m(J/psi p) range the reference's Pc spline covers).
SWAVE_KNOTS = (1.435, 1.44, 1.45, 1.5, 1.525, 1.55, 1.575, 1.6, 1.625, 1.65, 1.675, 1.7, 1.75, 1.8, 1.85, 1.9,
               1.95, 2.0, 2.05, 2.1, 2.2, 2.3, 2.4, 2.5)
PC_SPLINE_KNOTS = (4.04, 4.1, 4.2, 4.25, 4.3, 4.35, 4.4, 4.45, 4.5, 4.55, 4.6)


def lineshapes(seed: int = 8, swave=None) -> tuple:
    """Every lineshape type the reference kernels dispatch on besides Breit-Wigners and the coupled-
    channel K-matrix: a Lambda* S-wave spline, a Lambda* revised K-matrix of three 1/2- entries (one
    below the pK threshold, one non-resonant), a Pc revised K-matrix pair (3/2-), a Pc triangle cusp and
    a Pc spline wave, next to a Breit-Wigner of each chain.  swave: optional NUMSP (Re, Im) knot values
    of the S-wave (default: a smooth seeded shape)."""
    lst = [lstar_resonance("1520"), lstar_spline("S01", SWAVE_KNOTS), lstar_rkm("1405", 1, -1),
           lstar_rkm("1670", 1, -1), lstar_rkm("NRK", 1, -1, mass=-0.5)]
    pcs = [pc_bw("Pc4312", 1, -1), pc_rkm("Z4440", 3, -1), pc_rkm("Z4457", 3, -1), pc_cusp("T4337", 1, +1),
           pc_spline("ZS01", 1, -1, PC_SPLINE_KNOTS)]
    m = Model(lst, pcs)
    vals = {}
    _lstar_vals(["1520", "1405", "1670"], vals)
    vals["m0_S01"], vals["width_S01"] = 0.95, 0.3
    vals["width_NRK"] = 0.3
    rng = np.random.default_rng(seed)
    _seed_couplings(m, vals, rng)
    for i, x in enumerate(SWAVE_KNOTS):
        if swave is not None:
            re, im = swave[i]
        else:
            bw = 1.0 / complex(1.7 ** 2 - x * x, -1.7 * 0.25)
            re, im = 3.0 * bw.real, 3.0 * bw.imag
        vals[f"SR_S01_{i:02d}"], vals[f"SI_S01_{i:02d}"] = float(re), float(im)
    for i, x in enumerate(PC_SPLINE_KNOTS):
        z = 1.0 / complex(4.38 ** 2 - x * x, -4.38 * 0.12)
        vals[f"SR_ZS01_{i:02d}"], vals[f"SI_ZS01_{i:02d}"] = float(0.5 * z.real), float(0.5 * z.imag)
    for n, mass, width in (("Pc4312", 4.312, 0.010), ("Z4440", 4.440, 0.020), ("Z4457", 4.457, 0.006),
                           ("T4337", 1.52, 0.016), ("ZS01", -0.5, 0.0)):
        vals[f"m0_{n}"], vals[f"width_{n}"] = mass, width
    return m, vals


MODELS = {"lstar_only": lstar_only, "full_bw": full_bw, "kmatrix": kmatrix, "small_kmatrix": small_kmatrix,
          "small_bw": small_bw, "small_zcs": small_zcs,
          "lineshapes": lineshapes}

# Workloads: model, data events, MC events, MC weight range.
WORKLOADS = {
    "lstar_only": ("lstar_only", 20_000, 200_000, (1.0, 1.0)),
    "full_bw": ("full_bw", 100_000, 1_000_000, (0.2, 1.0)),
    "kmatrix": ("kmatrix", 500_000, 5_000_000, (0.2, 1.0)),
}
