"""Amplitude model: resonance lists, parameter values and the float parameter block.

The parameter block ("h_paraList") is the hot path's per-call input.  Its layout and contents
restate the reference host code that builds it every FCN call:

* resonance table, 6 floats per resonance [m0, width-or-channel, 2J, L, type, parity]
  (RooDalitzAmplitude::setup_paraList, src/RooDalitzAmplitude.cxx:3068-3139),
* helicity couplings as (Re, Im) float pairs (ConfigureCouplings :2669-2986, PartWaveCoff :5533-5599,
  PartWaveCoffZ :5601-5710),
* spline blocks of the model-independent waves (ConfigureCouplings :2738-2765 for the Lambda* chain,
  the same for the Pc chain with MakeSplineZ :1737-1752): the knot masses, then (y, b, c, d) per
  knot of the real part, then of the imaginary part, from a cubic spline through the knots with
  TSpline3's default (not-a-knot) end conditions,
* K-matrix blocks, per J^P group 16 pole couplings g then the 4x4 scattering matrix f
  (cu_init_data :3141-3210).

Float intermediates of the reference (float sqrt of the kinematic factor, float Clebsch-Gordan
coefficients) are reproduced so the block is bit-identical to the reference's for the same
parameter values.  Parameter files use the reference's text format (see `read_func`).
"""
from __future__ import annotations

import dataclasses
import math
import re
from fractions import Fraction
from functools import lru_cache
from typing import Callable

import numpy as np

BREITWIGNER, MODELINDEPENDENT, TRIANGLE, KMATRIX, REVISEDKMATRIX, NONRESONANT = 1, 3, 7, 240, 360, 361
NUMSP, NUMSPZ = 24, 11  # spline knots of the Lambda* and Pc model-independent waves (Resonances.h:5-6)
NSET, NPMAX, NKMC = 6, 4, 4
KM_BLOCK = (NPMAX + NKMC) * NKMC  # floats per J^P group
KM_SIZE = 4 * KM_BLOCK

HEL1_TWO = (1, 1, -1, -1, 3, -3)
HEL2 = (1, 0, 0, -1, 1, -1)

# Clebsch-Gordan values <L 0; S 1/2 | 1/2 1/2> for 2S = 1..11, 2L = 2S-1, 2S+1, as tabulated by the
# reference (RooDalitzAmplitude.cxx:96-107); the table's last-digit values are kept so couplings are
# bit-identical (tests/test_model.py checks them against the Racah formula).
C2 = ((1.0000000000000000e00, -5.7735026918962584e-01), (-5.7735026918962573e-01, 4.4721359549995765e-01),
      (4.4721359549995754e-01, -3.7796447300922748e-01), (-3.7796447300922759e-01, 3.3333333333333659e-01),
      (3.3333333333332898e-01, -3.0151134457775197e-01), (-3.0151134457772666e-01, 2.7735009811269257e-01))

f32 = np.float32


@lru_cache(maxsize=None)
def clebsch(j1: int, m1: int, j2: int, m2: int, J: int, M: int) -> float:
    """<j1/2 m1/2; j2/2 m2/2 | J/2 M/2> (all arguments doubled), Condon-Shortley phase, by the
    Racah formula in exact rational arithmetic."""
    if m1 + m2 != M or abs(m1) > j1 or abs(m2) > j2 or abs(M) > J:
        return 0.0
    if J < abs(j1 - j2) or J > j1 + j2 or (j1 + j2 + J) % 2 or (j1 + m1) % 2 or (j2 + m2) % 2:
        return 0.0
    f = math.factorial
    a = (j1 + j2 - J) // 2
    b = (j1 - m1) // 2
    c = (j2 + m2) // 2
    d = (J - j2 + m1) // 2
    e = (J - j1 - m2) // 2
    pref = Fraction((J + 1) * f((J + j1 - j2) // 2) * f((J - j1 + j2) // 2) * f(a), f((j1 + j2 + J) // 2 + 1))
    pref *= Fraction(f((J + M) // 2) * f((J - M) // 2) * f((j1 - m1) // 2) * f((j1 + m1) // 2)
                     * f((j2 - m2) // 2) * f((j2 + m2) // 2))
    s = Fraction(0)
    for k in range(0, a + 1):
        if b - k < 0 or c - k < 0 or d + k < 0 or e + k < 0:
            continue
        s += Fraction((-1) ** k, f(k) * f(a - k) * f(b - k) * f(c - k) * f(d + k) * f(e + k))
    if s == 0:
        return 0.0
    return float(math.copysign(math.sqrt(pref * s * s), s))


def _orthogonal_vector(n: int, vectors: list) -> list:
    """Generalised cross product of n-1 vectors of dimension n, accumulated over permutations in the
    order of EvtGen's EvtOrthogVector (src/EvtOrthogVector.cpp:31-127)."""
    orth = [0.0] * n
    holder = [0] * n

    def sign_of_holder() -> int:
        t = list(holder)
        swaps = 0
        for i in range(n - 1):
            for j in range(i + 1, n):
                if t[i] > t[j]:
                    t[i], t[j] = t[j], t[i]
                    swaps += 1
        return -1 if swaps % 2 else 1

    def product() -> float:
        a = 1.0
        for i in range(1, n):
            a *= vectors[i - 1][holder[i]]
        return a

    def rec(dim: int, invect: list):
        if dim == 2:
            holder[0], holder[1] = invect[0], invect[1]
            sign = sign_of_holder()
            orth[holder[0]] += product() * sign
            holder[0], holder[1] = invect[1], invect[0]
            orth[holder[0]] -= product() * sign
            return
        temp = invect + invect
        for i in range(dim):
            holder[dim - 1] = temp[dim - 1 + i]
            rec(dim - 1, temp[i:i + dim - 1])

    rec(n, list(range(n)))
    return orth


@lru_cache(maxsize=None)
def _cg_table(j1: int, j2: int) -> dict:
    """Clebsch-Gordan coefficients for fixed j1, j2 (doubled) built as EvtGen's EvtCGCoefSingle does
    (src/EvtCGCoefSingle.cpp:36-117): highest weight per J by orthogonalisation, then the lowering
    recursion with float square roots.  The float roots leave ~1e-8 relative deviations from the exact
    values; the reference's helicity couplings contain them, so they are reproduced."""
    Jmax, Jmin = j1 + j2, abs(j1 - j2)
    lenmax = min(j1, j2) + 1

    def length(M):
        return min(((j1 + j2) - abs(M)) // 2 + 1, lenmax)

    def mmin(M):
        return max(M - j2, -j1)

    tab = {}

    def cg(J, M, m1):
        return tab[(J, M)][(m1 - mmin(M)) // 2]

    for J in range(Jmax, Jmin - 1, -2):
        for M in range(J, -J - 1, -2):
            tab[(J, M)] = [0.0] * length(M)
        if J == Jmax:
            tab[(J, J)][0] = 1.0
        else:
            n = (Jmax - J) // 2 + 1
            vectors = [[tab[(Jmax - 2 * i, J)][k] for k in range(n)] for i in range(n - 1)]
            orth = _orthogonal_vector(n, vectors)
            sign = -1 if orth[n - 1] < 0 else 1
            tab[(J, J)] = [sign * orth[k] for k in range(n)]
        for M in range(J - 2, -J - 1, -2):
            lo = mmin(M)
            for m1 in range(lo, lo + 2 * length(M), 2):
                m2 = M - m1
                acc = 0.0
                if m1 + 2 <= j1:
                    acc += 0.5 * float(np.sqrt(f32(j1 * (j1 + 2) - (m1 + 2) * m1))) * cg(J, M + 2, m1 + 2)
                if m2 + 2 <= j2:
                    acc += 0.5 * float(np.sqrt(f32(j2 * (j2 + 2) - (m2 + 2) * m2))) * cg(J, M + 2, m1)
                acc /= 0.5 * float(np.sqrt(f32(J * (J + 2) - (M + 2) * M)))
                tab[(J, M)][(m1 - lo) // 2] = acc
    return tab


def cg_evtgen(j1: int, j2: int, J: int, M: int, m1: int, m2: int) -> float:
    """EvtCGCoefSingle(j1, j2).coef(J, M, j1, j2, m1, m2), all arguments doubled."""
    if m1 + m2 != M or abs(M) > J or J > j1 + j2 or J < abs(j1 - j2) or abs(m1) > j1 or abs(m2) > j2:
        raise ValueError((j1, j2, J, M, m1, m2))
    t = _cg_table(j1, j2)
    return t[(J, M)][(m1 - max(M - j2, -j1)) // 2]


# ------------------------------------------------------------------ model description
@dataclasses.dataclass
class Resonance:
    """One entry of a resonance list.  chain: 'L' (Lambda* -> pK), 'Z' (Pc -> J/psi p), 'X' (Zcs -> J/psi K).
    couplings: names of the LS coupling parameters as (Re, Im) pairs (12 for 'L', 8 for 'Z'; for 'X'
    four Lambda_b -> Zcs p couplings, then the Zcs -> J/psi K ones after the first).
    extra: 'L': (scRe, scIm) names; 'Z' K-matrix pole: g1..g4 names; 'Z' K-matrix NR: (fsc,).
    mass / width: parameter names or constants (for a K-matrix pole the width slot holds the
    channel index used for the near-threshold mass shift).
    knots: model-independent (spline) waves only: (Re, Im, mass) references per knot, NUMSP of them
    for 'L', NUMSPZ for 'Z' (RooDalitzAmplitude::MakeSpline / MakeSplineZ read them in this order)."""
    chain: str
    name: str
    spin2: int
    parity: int
    type: int
    mass: str | float
    width: str | float
    couplings: tuple
    extra: tuple = ()
    knots: tuple = ()

    def refs(self) -> list:
        """Every parameter reference this entry reads."""
        return [*self.couplings, *self.extra, self.mass, self.width, *(x for k in self.knots for x in k)]


@dataclasses.dataclass
class Model:
    lstar: list
    pc: list
    ffr: float = 3.0
    ffb: float = 3.0
    derived: dict = dataclasses.field(default_factory=dict)  # name -> callable(values) -> float
    zcs: list = dataclasses.field(default_factory=list)

    @property
    def NR(self):
        return len(self.lstar)

    @property
    def NZ(self):
        return len(self.pc)

    @property
    def NX(self):
        return len(self.zcs)

    @property
    def resonances(self):
        return list(self.lstar) + list(self.pc) + list(self.zcs)

    def value(self, vals: dict, ref) -> float:
        if isinstance(ref, (int, float)):
            return float(ref)
        if ref in self.derived:
            return float(self.derived[ref](vals))
        return float(vals[ref])

    def parameter_names(self) -> list:
        names = []
        for r in self.resonances:
            for ref in r.refs():
                if isinstance(ref, str) and ref not in names and ref not in self.derived:
                    names.append(ref)
        return names


def orbital_l(r: Resonance) -> int:
    """Decay orbital angular momentum stored in the table (setup_paraList :3079-3137)."""
    S = r.spin2 / 2.0
    if r.chain == "X":
        LR = max(abs(int(S - 1)), 0)  # C truncation: int(-1.0) = -1 for a spin-0 Zcs
        if ((-1) ** LR) * r.parity < 0:
            LR += 1
        return LR
    if r.chain == "L":
        LR = int(S - 0.5)
    else:
        LR = max(int(S - 1.5), 0)
    if ((-1) ** (LR + 1)) * r.parity < 0:
        LR += 1
    return LR


def km_group(r: Resonance) -> int:
    return (1 if r.spin2 == 3 else 0) + (2 if r.parity > 0 else 0)


# ------------------------------------------------------------------ LS -> helicity couplings
def _sqrt_f32(x: float) -> np.float32:
    return np.sqrt(f32(x))


def part_wave_lstar(lsc: list, J: int, lam2: int, lam3: int) -> complex:
    """Lambda_b -> Lambda* J/psi helicity coupling from LS couplings (PartWaveCoff, all quantum
    numbers doubled)."""
    c = 0j
    ib = 0
    m1 = lam2 - lam3
    for S in range(abs(J - 2), J + 3, 2):
        for L in (S - 1, S + 1):
            M = lsc[ib]
            if abs(M) ** 2 < 1e-10:
                ib += 1
                continue
            a = _sqrt_f32((L + 1.0) / 2.0)
            ccg = f32(cg_evtgen(J, 2, S, m1, lam2, -lam3))
            pre = float(f32(a * ccg))
            tmp = pre * C2[(S - 1) // 2][(L - S + 1) // 2] * M
            if m1 < 0 and L > S:
                tmp = -tmp
            c += tmp
            ib += 1
    return c


def part_wave_pc(lsc: list, parity: int, J: int, lamZ: int, lamPsi: int, lamp: int) -> complex:
    """Lambda_b -> Pc K and Pc -> J/psi p helicity coupling from LS couplings (PartWaveCoffZ)."""
    HB = 0j
    SB = J
    for LB in (SB - 1, SB + 1):
        tmp = complex(C2[(SB - 1) // 2][(LB - SB + 1) // 2] * math.sqrt((LB + 1.0) / 2.0))
        if LB > SB:
            M = lsc[0]
            if abs(M) ** 2 < 1e-10:
                continue
            tmp = tmp * M
            if lamZ < 0:
                tmp = -tmp
        HB += tmp
    ib = 1
    c = 0j
    m1 = lamPsi - lamp
    for S in (1, 3):
        for L in range(abs(J - S), J + S + 1, 2):
            if ((-1) ** (L // 2 + 1)) * parity < 0:
                continue
            if S < abs(m1):
                ib += 1
                continue
            ccg1 = f32(cg_evtgen(2, 1, S, m1, lamPsi, -lamp))
            M = lsc[ib]
            if abs(M) ** 2 < 1e-10:
                ib += 1
                continue
            a = _sqrt_f32((L + 1.0) / (J + 1.0))
            if J == 1:
                cg = C2[(S - 1) // 2][(L - S + 1) // 2]
                if m1 < 0 and L > S:
                    cg = -cg
                ccg = f32(cg)
            else:
                ccg = f32(cg_evtgen(L, S, J, m1, 0, m1))
            pre = float(f32(f32(a * ccg) * ccg1))
            c += pre * M
            ib += 1
    return c * HB


def part_wave_x(lsc: list, parity: int, J: int, lamZ: int, lamPsi: int, lamp: int) -> complex:
    """Lambda_b -> Zcs p and Zcs -> J/psi K helicity coupling from LS couplings (PartWaveCoffX,
    src/RooDalitzAmplitude.cxx:5724-5830; doubled quantum numbers, double arithmetic, EvtGen
    Clebsch-Gordan coefficients).  As there, the first Zcs -> J/psi K wave has coupling 1 and a
    decay coupling is only moved past when it is zero, so a non-zero one serves every later wave."""
    HZ = 0j
    ib = 4
    SZ = 2
    first = True
    for LZ in range(J - SZ, SZ + J + 1, 2):
        if J == 0 and LZ != SZ:
            continue
        if parity * (-1) ** (LZ // 2) < 0:
            continue
        tmp1 = (LZ + 1.0) / (J + 1.0)
        cg2 = cg_evtgen(LZ, SZ, J, lamPsi, 0, lamPsi)
        if first:
            first = False
            HZ += math.sqrt(tmp1) * cg2
        else:
            M = lsc[ib] if ib < len(lsc) else 0j
            if abs(M) ** 2 < 1e-10:
                ib += 1
                continue
            HZ += M * math.sqrt(tmp1) * cg2
    ib = 0
    c = 0j
    m1 = lamZ - lamp
    for S in (J - 1, J + 1):
        if S < 0:
            continue
        for L in (S - 1, S + 1):
            ccg1 = C2[(S - 1) // 2][(L - S + 1) // 2]
            if m1 < 0 and L > S:
                ccg1 = -ccg1
            M = lsc[ib]
            if abs(M) ** 2 < 1e-10:
                ib += 1
                continue
            ccg = cg_evtgen(J, 1, S, m1, lamZ, -lamp)
            c += math.sqrt((L + 1.0) / 2.0) * ccg * ccg1 * M
            ib += 1
    return c * HZ


def spline_coefficients(x, y) -> np.ndarray:
    """[n, 4] coefficients (y, b, c, d) of the cubic spline through (x_i, y_i), S(x) = y_i + b_i t +
    c_i t^2 + d_i t^3 with t = x - x_i on [x_i, x_i+1], with not-a-knot end conditions (the third
    derivative continuous at the second and the next-to-last knot: the default end conditions of
    TSpline3, which follows de Boor's CUBSPL).  The last knot's row continues the last interval's
    cubic.  Computed in double precision."""
    x = np.asarray(x, float)
    y = np.asarray(y, float)
    n = len(x)
    if n < 4 or np.any(np.diff(x) <= 0):
        raise ValueError("a spline needs at least 4 strictly increasing knots")
    h = np.diff(x)
    A = np.zeros((n, n))
    r = np.zeros(n)
    for i in range(1, n - 1):  # second derivatives M_i: continuity of the first derivative
        A[i, i - 1], A[i, i], A[i, i + 1] = h[i - 1], 2 * (h[i - 1] + h[i]), h[i]
        r[i] = 6 * ((y[i + 1] - y[i]) / h[i] - (y[i] - y[i - 1]) / h[i - 1])
    A[0, 0], A[0, 1], A[0, 2] = h[1], -(h[0] + h[1]), h[0]  # not-a-knot at x_1
    A[n - 1, n - 3], A[n - 1, n - 2], A[n - 1, n - 1] = h[n - 2], -(h[n - 3] + h[n - 2]), h[n - 3]  # at x_n-2
    M = np.linalg.solve(A, r)
    out = np.zeros((n, 4))
    out[:, 0] = y
    out[:-1, 1] = (y[1:] - y[:-1]) / h - h * (2 * M[:-1] + M[1:]) / 6
    out[:, 2] = M / 2
    out[:-1, 3] = (M[1:] - M[:-1]) / (6 * h)
    hl = h[-1]
    out[-1, 1] = out[-2, 1] + 2 * out[-2, 2] * hl + 3 * out[-2, 3] * hl * hl
    out[-1, 3] = out[-2, 3]
    return out


def spline_block(x, re, im) -> list:
    """The float spline block of one model-independent wave: knots, (y, b, c, d) of the real part per
    knot, then of the imaginary part (RooDalitzAmplitude.cxx:2741-2764)."""
    cr, ci = spline_coefficients(x, re), spline_coefficients(x, im)
    return [f32(v) for v in x] + [f32(v) for v in cr.reshape(-1)] + [f32(v) for v in ci.reshape(-1)]


def _pow_m1(e) -> float:
    return 1.0 if int(round(e)) % 2 == 0 else -1.0


@dataclasses.dataclass
class ParamBlock:
    data: np.ndarray  # float32 h_paraList
    para_size: int
    vamp_size: int
    spline_size: int
    NR: int
    NZ: int
    NX: int
    ffr: float
    ffb: float

    @property
    def kmcount(self):
        return self.para_size + self.vamp_size + self.spline_size


def _resonance_parts(model: Model, vals: dict, ir: int, keep: bool = True) -> tuple:
    """The pieces of the parameter block one resonance contributes: its table row (NSET floats), its
    helicity couplings (float Re/Im pairs), its K-matrix inputs (('g', group, g1..g4) for a pole,
    ('f', group, f) for a non-resonant term, or None) and its spline block (empty unless the entry is
    a model-independent wave)."""
    r = model.resonances[ir]
    q = np.zeros(NSET, f32)
    q[0] = f32(model.value(vals, r.mass))
    q[1] = f32(model.value(vals, r.width))
    q[2] = r.spin2
    q[3] = orbital_l(r)
    q[4] = r.type
    q[5] = r.parity
    lsc = [complex(model.value(vals, r.couplings[2 * i]), model.value(vals, r.couplings[2 * i + 1]))
           for i in range(len(r.couplings) // 2)]
    vamp: list = []
    km = None
    if r.chain == "X":
        S = r.spin2 / 2.0
        for k in range(2):
            for hpsi in (-1, 0, 1):
                if abs(hpsi) > S:
                    continue
                for hp in (-0.5, 0.5):
                    for helZ in (hp - 0.5, hp + 0.5):
                        if abs(helZ) > S:
                            continue
                        a = part_wave_x(lsc, r.parity, r.spin2, int(helZ * 2), hpsi * 2, int(hp * 2))
                        vamp += [f32(a.real), f32(a.imag)] if keep else [f32(0), f32(0)]
        if r.type != BREITWIGNER:
            raise NotImplementedError(f"Zcs lineshape type {r.type}")
        return q, vamp, km, []
    if r.chain == "L":
        S = f32(r.spin2) / f32(2)
        sc = complex(model.value(vals, r.extra[0]), model.value(vals, r.extra[1]))
        for k in range(2):
            pp = _pow_m1(int(S - 1.5)) * r.parity if k == 0 else 1.0
            for m in range(6):
                if r.spin2 == 1 and m >= 4:
                    continue
                h2 = HEL2[m]
                a = part_wave_lstar(lsc, r.spin2, HEL1_TWO[m], h2 * 2) * pp
                a = a * _pow_m1(1 - h2)
                a = a * sc
                vamp += [f32(a.real), f32(a.imag)] if keep else [f32(0), f32(0)]
        if r.type not in (BREITWIGNER, NONRESONANT, MODELINDEPENDENT, REVISEDKMATRIX):
            raise NotImplementedError(f"Lambda* lineshape type {r.type}")
    else:
        S = r.spin2 / 2.0
        for k in range(2):
            for hpsi in (-1, 0, 1):
                for ihz in range(2):
                    hz = -0.5 if ihz == 0 else 0.5
                    for ihp in range(2):
                        hp = -0.5 if ihp == 0 else 0.5
                        if abs(hpsi - hp) > S:
                            continue
                        a = part_wave_pc(lsc, r.parity, r.spin2, int(hz * 2), hpsi * 2, int(hp * 2))
                        a = a * _pow_m1(1 - ihp)
                        vamp += [f32(a.real), f32(a.imag)] if keep else [f32(0), f32(0)]
        if r.type == KMATRIX:
            ik = km_group(r)
            if q[0] > 0:
                km = ("g", ik, [f32(model.value(vals, g)) for g in r.extra[:4]])
            else:
                km = ("f", ik, f32(model.value(vals, r.extra[0])))
        elif r.type not in (BREITWIGNER, NONRESONANT, MODELINDEPENDENT, REVISEDKMATRIX, TRIANGLE):
            raise NotImplementedError(f"Pc lineshape type {r.type}")
    spl: list = []
    if r.type == MODELINDEPENDENT:
        nk = NUMSP if r.chain == "L" else NUMSPZ
        if len(r.knots) != nk:
            raise ValueError(f"{r.name}: a model-independent wave of chain {r.chain} has {nk} knots")
        re = [model.value(vals, k[0]) for k in r.knots]
        im = [model.value(vals, k[1]) for k in r.knots]
        xs = [model.value(vals, k[2]) for k in r.knots]
        spl = spline_block(xs, re, im)
    return q, vamp, km, spl


def _assemble_block(model: Model, parts: list) -> ParamBlock:
    table = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, f32)
    vamp = [x for p in parts for x in p[1]]
    spl = [x for p in parts for x in p[3]]  # Lambda* splines, then Pc splines (resonance order)
    galpha = [[] for _ in range(4)]
    fscat = [[] for _ in range(4)]
    for _, _, km, _ in parts:
        if km is None:
            continue
        if km[0] == "g":
            galpha[km[1]] += km[2]
        else:
            fscat[km[1]].append(km[2])
    km = []
    for ik in range(4):
        g = galpha[ik][: NPMAX * NKMC]
        if len(galpha[ik]) > NPMAX * NKMC:
            raise ValueError("more than 4 K-matrix poles in one J^P group")
        f = (fscat[ik] + [f32(0)] * (NKMC * NKMC))[: NKMC * NKMC]
        for i in range(1, NKMC):
            f[NKMC * i] = f[i]
        km += g + [f32(0)] * (NPMAX * NKMC - len(g)) + f
    data = np.concatenate([table.astype(f32), np.array(vamp, f32), np.array(spl, f32),
                           np.array(km, f32)]).astype(f32)
    return ParamBlock(data, len(table), len(vamp), len(spl), model.NR, model.NZ, model.NX, model.ffr, model.ffb)


def build_param_block(model: Model, vals: dict, include: tuple | None = None) -> ParamBlock:
    """The float parameter block for one parameter point (ConfigureCouplings + cu_init_data).
    include: optional (Lambda* indices, Pc indices[, Zcs indices]) whose couplings are kept
    (SetupCoupling); the others are zeroed, as for per-resonance weights."""
    parts = []
    for ir, r in enumerate(model.resonances):
        keep = True
        if include is not None:
            if r.chain == "L":
                keep = ir in include[0]
            elif r.chain == "Z":
                keep = (ir - model.NR) in include[1]
            else:
                keep = (ir - model.NR - model.NZ) in (include[2] if len(include) > 2 else ())
        parts.append(_resonance_parts(model, vals, ir, keep))
    return _assemble_block(model, parts)


class BlockBuilder:
    """Parameter blocks of points that differ from a base point in a few parameters (Minuit's
    gradient and line-search points): only the resonances a changed parameter enters are recomputed,
    and the result is identical to build_param_block of the same values."""

    def __init__(self, model: Model, vals: dict):
        self.model = model
        self.base = dict(vals)
        self.parts = [_resonance_parts(model, vals, i) for i in range(len(model.resonances))]
        self.uses: dict = {}
        everything = list(range(len(model.resonances)))
        for i, r in enumerate(model.resonances):
            refs = [x for x in r.refs() if isinstance(x, str)]
            for x in refs:
                if x in model.derived:  # derived values may read any parameter
                    for n in list(vals):
                        self.uses.setdefault(n, set()).update(everything)
                else:
                    self.uses.setdefault(x, set()).add(i)

    def block(self, changes: dict | None = None) -> ParamBlock:
        changes = changes or {}
        if not changes:
            return _assemble_block(self.model, self.parts)
        vals = dict(self.base)
        vals.update(changes)
        parts = list(self.parts)
        touched = set()
        for n in changes:
            touched |= self.uses.get(n, set())
        for i in touched:
            parts[i] = _resonance_parts(self.model, vals, i)
        return _assemble_block(self.model, parts)


# ------------------------------------------------------------------ parameter files
_FUNC_RE = re.compile(
    r"^\s*(?P<name>[A-Za-z_][\w\.]*)\s*=\s*(?P<val>[-+\w\.]+)(?:\s*\+/-\s*(?P<err>[-+\w\.]+))?"
    r"(?P<const>\s+C)?(?:\s+L\((?P<lo>[-+\w\.]+)\s*-\s*(?P<hi>[-+\w\.]+)\))?\s*$")


def _num(s: str) -> float:
    s = s.strip()
    if s.upper() in ("INF", "+INF"):
        return math.inf
    if s.upper() == "-INF":
        return -math.inf
    return float(s)


@dataclasses.dataclass
class Param:
    name: str
    value: float
    error: float | None = None
    constant: bool = False
    lo: float = -math.inf
    hi: float = math.inf


def read_func(text: str) -> dict:
    """Parse the reference's parameter-file format (RooArgSet::readFromFile, e.g.
    Fit_Jpsippi/func/yujie_test.func):  name = value [+/- error] [C] [L(lo - hi)]."""
    out = {}
    for line in text.splitlines():
        line = line.split("//")[0].rstrip()
        if not line.strip():
            continue
        m = _FUNC_RE.match(line)
        if not m:
            raise ValueError(f"cannot parse parameter line: {line!r}")
        out[m["name"]] = Param(m["name"], _num(m["val"]), _num(m["err"]) if m["err"] else None,
                               bool(m["const"]), _num(m["lo"]) if m["lo"] else -math.inf,
                               _num(m["hi"]) if m["hi"] else math.inf)
    return out


def _fmt(x: float) -> str:
    if math.isinf(x):
        return "+INF" if x > 0 else "-INF"
    return f"{x:.6g}"


def write_func(params: dict) -> str:
    lines = []
    for name in sorted(params):
        p = params[name]
        s = f"{name} = {p.value:.8g}"
        if p.error is not None:
            s += f" +/- {p.error:.5g}"
        if p.constant:
            s += " C"
        s += f" L({_fmt(p.lo)} - {_fmt(p.hi)})"
        lines.append(s)
    return "\n".join(lines) + "\n"


@dataclasses.dataclass
class Constraint:
    """Flat-top two-sided Gaussian penalty (RooFGaussian::evaluate, src/RooFGaussian.cxx:60-75)."""
    name: str
    mean1: float
    mean2: float
    sigma1: float
    sigma2: float
    lo: float
    hi: float

    def penalty(self, x: float) -> float:
        if x < self.mean1:
            return 0.5 * ((x - self.mean1) / self.sigma1) ** 2
        if x > self.mean2:
            return 0.5 * ((x - self.mean2) / self.sigma2) ** 2
        return 0.0


def read_constraints(text: str) -> list:
    """Constraint file: name mean1 mean2 err1 err2 lo hi per line (Fitter::ConstrMW, src/fit.cpp:33-79)."""
    out = []
    for line in text.splitlines():
        f = line.split()
        if len(f) < 7:
            continue
        out.append(Constraint(f[0], *map(float, f[1:7])))
    return out


def fcn(nll: float, nll_shift: float, alpha: float, constraints: list, vals: dict) -> float:
    """Minuit FCN of the reference: (NLL - NLL_SHIFT) * alpha + sum of constraints
    (src/fit.cpp:312-317), alpha = sum w / sum w^2 of the data weights (:201-220)."""
    return (nll - nll_shift) * alpha + sum(c.penalty(vals[c.name]) for c in constraints if c.name in vals)
