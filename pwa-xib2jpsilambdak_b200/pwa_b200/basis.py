"""Per-event angular basis and the reference's SoA device layout.

`fill_basis` restates RooDalitzAmplitude::filldlz (src/RooDalitzAmplitude.cxx:7086-7308) with the
d-functions of :2443-2590 and the phase factors of MEangPart/MEangZPart (:2593-2667), reproducing the
reference's float rounding points: angles are float(acos(cos)), phase sums are accumulated in float,
products are formed in double and stored as float.

`pack_soa` lays the basis out exactly as the reference's device planes
(RooDalitzAmplitude.cxx:548-770): plane stride n_size = (N/32 + 1) * 32, events along the stride.
  pp  (111 planes): 0 mKp, 1 mJ/psi p, 2 weight, 3.. ARe/AIm[i][j][m] interleaved, 51.. DL[s][k][m]
  pp1 (96 planes):  AZRe/AZIm[i][j][m] interleaved
  pp2 (96 planes):  DZ[s][k][m]
  pp3 (97 planes):  0 mJ/psi K, 1.. AXRe/AXIm[i][j][m] interleaved       (Zcs chain, NX > 0 only)
  pp4 (96 planes):  DX[s][k][m]
"""
from __future__ import annotations

import math

import numpy as np

N_PP, N_PP1, N_PP2, N_PP3, N_PP4 = 111, 96, 96, 97, 96
HEL1_TWO = (1, 1, -1, -1, 3, -3)  # 2 x helicity of Lambda* (RooDalitzAmplitude.cxx:110)
HEL2 = (1, 0, 0, -1, 1, -1)  # helicity of J/psi in the Lambda* chain (:111)

_LNFACT = np.array([math.lgamma(n + 1) for n in range(60)])


def n_size_of(n: int) -> int:
    return (n // 32 + 1) * 32


def dfun_half(beta, am, an):
    """d^{1/2}_{am/2, an/2}(beta) (dfunhalf)."""
    if am == an:
        return np.cos(0.5 * beta)
    return -np.sin(0.5 * beta) if am == 1 else np.sin(0.5 * beta)


def dfun_one(beta, am, an):
    """d^1_{am, an}(beta) for an = +-1 (dfunone)."""
    if am == an:
        return (np.cos(beta) + 1.0) / 2.0
    if am == -an and am != 0:
        return (1.0 - np.cos(beta)) / 2.0
    if am == 0:
        return np.sin(beta) * 7.07106781186547461715e-01 * (1 if an == 1 else -1)
    raise ValueError((am, an))


def dfun(beta, j, m, n):
    """Wigner d^j_{m n}(beta) in the log-factorial sum form of Varshalovich 4.3.1(3)
    (the CERNLIB DDJMNB algorithm the reference uses), vectorised over beta."""
    beta = np.asarray(beta, dtype=np.float64)
    jpm, jpn, jmm, jmn, mpn = (int(round(j + m)), int(round(j + n)), int(round(j - m)),
                               int(round(j - n)), int(round(m + n)))
    out = np.zeros_like(beta)
    if min(jpm, jpn, jmm, jmn) < 0:
        return out
    pi, pi2 = 3.141592653589793116, 6.283185307179586232
    at0 = np.abs(beta) < 1e-10
    atpi = np.abs(beta - pi) < 1e-10
    at2pi = np.abs(beta - pi2) < 1e-10
    gen = ~(at0 | atpi | at2pi)
    if jpm == jpn:
        out[at0] = 1.0
    if jpm == jmn:
        out[atpi] = -1.0 if abs(jpm) % 2 == 1 else 1.0
    if jpm == jpn:
        out[at2pi] = -1.0 if abs(mpn) % 2 == 1 else 1.0
    b = 0.5 * beta[gen]
    with np.errstate(divide="ignore"):
        s = np.log(np.sin(b))
        c = np.log(np.abs(np.cos(b)))
    rt = 0.5 * (_LNFACT[jpm] + _LNFACT[jmm] + _LNFACT[jpn] + _LNFACT[jmn])
    k0 = max(0, mpn)
    kq = np.full(b.shape, k0 + jpm)
    kq = kq + np.where(beta[gen] > pi, mpn, 0)
    q = np.where(np.fmod(kq, 2) == 1, -1.0, 1.0)  # C remainder: a negative kq gives q = +1
    cx = 2 * k0 - mpn
    sx = jpm + jpn - 2 * k0
    r = np.zeros_like(b)
    for k in range(k0, min(jpm, jpn) + 1):
        r += q * np.exp(rt - _LNFACT[k] - _LNFACT[jpm - k] - _LNFACT[jpn - k] - _LNFACT[k - mpn] + cx * c + sx * s)
        cx += 2
        sx -= 2
        q = -q
    out[gen] = r
    return out


def fill_basis(ang: dict) -> dict:
    """Angular basis per event.  Returns float32 arrays ARe/AIm (N,2,2,6), DL (N,5,2,6),
    AZRe/AZIm (N,2,2,12), DZ (N,4,2,12)."""
    f32 = np.float32
    acos32 = lambda x: np.arccos(np.asarray(x, np.float64)).astype(f32).astype(np.float64)
    th = acos32(ang["cosTheta_Lb"])
    th1 = acos32(ang["cosTheta_L"])
    th2 = acos32(ang["cosTheta_Jpsi"])
    thB = acos32(ang["Z_cosTheta_Lb"])
    thZ = acos32(ang["Z_cosTheta_Z"])
    thPsi = acos32(ang["Z_cosTheta_Jpsi"])
    thp = acos32(ang["cosTheta_Lambda"])
    phi1 = np.asarray(ang["phiK"]).astype(f32)
    phi2 = np.asarray(ang["phiMu"]).astype(f32)
    phiZ = np.asarray(ang["Z_phiZ"]).astype(f32)
    phiPsi = np.asarray(ang["Z_phiJpsi"]).astype(f32)
    phiMu = np.asarray(ang["Z_phiMu"]).astype(f32)
    alphaMu = np.asarray(ang["alpha_Mu"]).astype(f32)
    n = th.shape[0]
    ARe = np.zeros((n, 2, 2, 6), f32)
    AIm = np.zeros((n, 2, 2, 6), f32)
    for i in range(2):
        dmu = -1 if i == 0 else 1
        for j in range(2):
            hel0 = -0.5 if j == 0 else 0.5
            for m in range(6):
                hel1 = HEL1_TWO[m] / 2.0
                hel2 = HEL2[m]
                part = (f32(hel1) * phi1 + f32(hel2) * phi2).astype(np.float64)
                dh = dfun_half(th, int(hel0 * 2), int((hel1 - hel2) * 2))
                d1 = dfun_one(th2, hel2, dmu)
                ARe[:, i, j, m] = ((np.cos(part) * dh) * d1).astype(f32)
                AIm[:, i, j, m] = ((np.sin(part) * dh) * d1).astype(f32)
    DL = np.zeros((n, 5, 2, 6), f32)
    for s in range(5):
        S = s + 0.5
        for k in range(2):
            hel3 = -0.5 if k == 0 else 0.5
            for m in range(6):
                if s == 0 and m >= 4:
                    continue
                DL[:, s, k, m] = dfun(th1, S, HEL1_TWO[m] / 2.0, hel3).astype(f32)
    AZRe = np.zeros((n, 2, 2, 12), f32)
    AZIm = np.zeros((n, 2, 2, 12), f32)
    for i in range(2):
        dmu = -1 if i == 0 else 1
        for j in range(2):
            hel0 = -0.5 if j == 0 else 0.5
            m = 0
            for hpsi in (-1, 0, 1):
                for helZ in (-0.5, 0.5):
                    part = (((f32(hel0) * phiZ + f32(hpsi) * phiMu) + f32(helZ) * phiPsi)
                            + f32(dmu) * alphaMu).astype(np.float64)
                    d1 = dfun_one(thPsi, hpsi, dmu)
                    dh = dfun_half(thB, int(hel0 * 2), int(helZ * 2))
                    re = ((np.cos(part) * d1) * dh).astype(f32)
                    im = ((np.sin(part) * d1) * dh).astype(f32)
                    for _hp in (-0.5, 0.5):
                        AZRe[:, i, j, m] = re
                        AZIm[:, i, j, m] = im
                        m += 1
    DZ = np.zeros((n, 4, 2, 12), f32)
    for s in range(4):
        S = s + 0.5
        for k in range(2):
            hel3 = -0.5 if k == 0 else 0.5
            m = 0
            for hpsi in (-1, 0, 1):
                for helZ in (-0.5, 0.5):
                    for hp in (-0.5, 0.5):
                        if abs(hpsi - hp) <= S:
                            DZ[:, s, k, m] = (dfun_half(thp, int(hp * 2), int(hel3 * 2))
                                              * dfun(thZ, S, helZ, hpsi - hp)).astype(f32)
                        m += 1
    return {"ARe": ARe, "AIm": AIm, "DL": DL, "AZRe": AZRe, "AZIm": AZIm, "DZ": DZ}


def band_of(mz32) -> np.ndarray:
    """Reference smearing bands of data events by float m(J/psi p): 1 = 30-offset band,
    2 = 150-offset band, 3 = unsmeared (RooDalitzAmplitude.cxx:391-396)."""
    m = np.asarray(mz32, np.float32).astype(np.float64)
    inner = (m > 4.2) & (m < 4.6)
    b1 = inner & ((m < 4.43) | (m > 4.47))
    b2 = inner & ~b1
    return np.where(b1, 1, np.where(b2, 2, 3))


def order_data_by_band(mz) -> np.ndarray:
    """Permutation that sorts data into bands 1, 2, 3 keeping the order inside each band
    (gen_toys/rearrange_mJpsip/reOrder.C)."""
    b = band_of(mz)
    return np.concatenate([np.nonzero(b == 1)[0], np.nonzero(b == 2)[0], np.nonzero(b == 3)[0]])


def fill_basis_x(ang: dict) -> dict:
    """Zcs-chain basis per event (filldlz, RooDalitzAmplitude.cxx:7239-7303, with MEangXPart :2650-2665):
    AXRe/AXIm (N,2,2,12) over all (J/psi, proton, Zcs) helicity combinations, DX (N,4,2,12) for
    Zcs spins 0..3 over the combinations the spin allows (|lambda_psi|, |lambda_Zcs| <= J)."""
    f32 = np.float32
    acos32 = lambda x: np.arccos(np.asarray(x, np.float64)).astype(f32).astype(np.float64)
    thB = acos32(ang["X_cosTheta_Lb"])
    thX = acos32(ang["X_cosTheta_X"])
    thPsi = acos32(ang["X_cosTheta_Jpsi"])
    thp = acos32(ang["X_cosTheta_p"])
    phiX = np.asarray(ang["X_phiX"]).astype(f32)
    phiPsi = np.asarray(ang["X_phiJpsi"]).astype(f32)
    phiMu = np.asarray(ang["X_phiMu"]).astype(f32)
    alphaMu = np.asarray(ang["X_alpha_Mu"]).astype(f32)
    n = thB.shape[0]
    AXRe = np.zeros((n, 2, 2, 12), f32)
    AXIm = np.zeros((n, 2, 2, 12), f32)
    for i in range(2):
        dmu = -1 if i == 0 else 1
        for j in range(2):
            hel0 = -0.5 if j == 0 else 0.5
            m = 0
            for hpsi in (-1, 0, 1):
                for hp in (-0.5, 0.5):
                    for helZ in (hp - 0.5, hp + 0.5):
                        part = (((f32(hel0) * phiX + f32(hpsi) * phiMu) + f32(helZ - hp) * phiPsi)
                                + f32(dmu) * alphaMu).astype(np.float64)
                        d1 = dfun_one(thPsi, hpsi, dmu)
                        dh = dfun_half(thB, int(hel0 * 2), int((helZ - hp) * 2))
                        AXRe[:, i, j, m] = ((np.cos(part) * d1) * dh).astype(f32)
                        AXIm[:, i, j, m] = ((np.sin(part) * d1) * dh).astype(f32)
                        m += 1
    DX = np.zeros((n, 4, 2, 12), f32)
    for s in range(4):
        S = float(s)
        for k in range(2):
            hel3 = -0.5 if k == 0 else 0.5
            m = 0
            for hpsi in (-1, 0, 1):
                if abs(hpsi) > S:
                    continue
                for hp in (-0.5, 0.5):
                    for helZ in (hp - 0.5, hp + 0.5):
                        if abs(helZ) > S:
                            continue
                        DX[:, s, k, m] = (dfun_half(thp, int(hp * 2), int(hel3 * 2))
                                          * dfun(thX, S, helZ, -hpsi)).astype(f32)
                        m += 1
    return {"AXRe": AXRe, "AXIm": AXIm, "DX": DX}


def pack_soa(mkp, mz, w, basis: dict, n_size: int | None = None) -> dict:
    """Pack events into the reference device planes; returns dict pp, pp1, pp2 (float32, flat)."""
    n = len(mkp)
    ns = n_size or n_size_of(n)
    pp = np.zeros((N_PP, ns), np.float32)
    pp1 = np.zeros((N_PP1, ns), np.float32)
    pp2 = np.zeros((N_PP2, ns), np.float32)
    pp[0, :n] = mkp
    pp[1, :n] = mz
    pp[2, :n] = w
    for i in range(2):
        for j in range(2):
            for m in range(6):
                a = 3 + (i * 12 + j * 6 + m) * 2
                pp[a, :n] = basis["ARe"][:, i, j, m]
                pp[a + 1, :n] = basis["AIm"][:, i, j, m]
    for s in range(5):
        for k in range(2):
            for m in range(6):
                pp[51 + s * 12 + k * 6 + m, :n] = basis["DL"][:, s, k, m]
    for i in range(2):
        for j in range(2):
            for m in range(12):
                a = (i * 24 + j * 12 + m) * 2
                pp1[a, :n] = basis["AZRe"][:, i, j, m]
                pp1[a + 1, :n] = basis["AZIm"][:, i, j, m]
    for s in range(4):
        for k in range(2):
            for m in range(12):
                pp2[s * 24 + k * 12 + m, :n] = basis["DZ"][:, s, k, m]
    out = {"pp": pp.reshape(-1), "pp1": pp1.reshape(-1), "pp2": pp2.reshape(-1), "n_size": ns, "n": n}
    if "AXRe" in basis:
        pp3 = np.zeros((N_PP3, ns), np.float32)
        pp4 = np.zeros((N_PP4, ns), np.float32)
        pp3[0, :n] = basis["mjpsik"]
        for i in range(2):
            for j in range(2):
                for m in range(12):
                    a = 1 + (i * 24 + j * 12 + m) * 2
                    pp3[a, :n] = basis["AXRe"][:, i, j, m]
                    pp3[a + 1, :n] = basis["AXIm"][:, i, j, m]
        for s in range(4):
            for k in range(2):
                for m in range(12):
                    pp4[s * 24 + k * 12 + m, :n] = basis["DX"][:, s, k, m]
        out["pp3"] = pp3.reshape(-1)
        out["pp4"] = pp4.reshape(-1)
    return out
