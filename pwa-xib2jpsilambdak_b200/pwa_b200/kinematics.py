"""Synthetic Lambda_b -> J/psi(-> mu+ mu-) p K- events and their helicity angles.

Events are uniform in the Dalitz plane (m^2_Kp, m^2_psip) with an isotropic decay orientation and an
isotropic J/psi -> mu mu decay, i.e. flat three-body phase space.  The angle definitions follow the
reference ntuple maker gen_toys/phsp_toys/tree.C:127-406 (helicityJpsiLam, helicityZK,
helicityTwoFrame); the Lambda_b flight direction (the tree's PBunit) is the z axis of the
Lambda_b rest frame.  Angle names are the ntuple branch names read by the reference
(RooDalitzAmplitude.cxx:305-322).
"""
from __future__ import annotations

import numpy as np

# Masses used by the reference amplitude (cu_DPFPropogator.cu:11-14) and the muon mass of the toy
# generator (gen_toys/phsp_toys/gentoy_formhj.C:11).
M_LB = 5.61951
M_K = 0.493677
M_P = 0.938272046
M_JPSI = 3.096916
M_MU = 0.105658

MKP_MIN, MKP_MAX = M_P + M_K, M_LB - M_JPSI
MZ_MIN, MZ_MAX = M_JPSI + M_P, M_LB - M_K


def _unit(v):
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return v / np.where(n > 0, n, 1.0)


def _dot(a, b):
    return np.einsum("...i,...i->...", a, b)


def _boost(p4, beta):
    """Boost four-vectors p4 (...,4: px,py,pz,E) by velocity beta (...,3)."""
    b2 = _dot(beta, beta)
    gamma = 1.0 / np.sqrt(1.0 - b2)
    bp = _dot(beta, p4[..., :3])
    g2 = np.where(b2 > 0, (gamma - 1.0) / np.where(b2 > 0, b2, 1.0), 0.0)
    vec = p4[..., :3] + (g2 * bp)[..., None] * beta + (gamma * p4[..., 3])[..., None] * beta
    e = gamma * (p4[..., 3] + bp)
    return np.concatenate([vec, e[..., None]], axis=-1)


def _to_rest(p4, parent):
    """Boost p4 into the rest frame of parent (TLorentzVector::Boost(-parent.BoostVector()))."""
    return _boost(p4, -parent[..., :3] / parent[..., 3:4])


def _two_body_p(M, m1, m2):
    return np.sqrt(np.maximum((M * M - (m1 + m2) ** 2) * (M * M - (m1 - m2) ** 2), 0.0)) / (2.0 * M)


def _rotation(rng, n):
    """Uniformly random rotation matrices (n,3,3) via random unit quaternions."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], axis=1)


def generate_phase_space(n: int, seed: int) -> dict:
    """Return n flat phase-space events as four-vectors in the Lambda_b rest frame."""
    rng = np.random.default_rng(seed)
    m12_lo, m12_hi = MKP_MIN ** 2, MKP_MAX ** 2
    m23_lo, m23_hi = MZ_MIN ** 2, MZ_MAX ** 2
    out_s1, out_s2 = [], []
    have = 0
    while have < n:
        k = int((n - have) * 2.2) + 64
        s1 = rng.uniform(m12_lo, m12_hi, k)  # m^2(K p)
        s2 = rng.uniform(m23_lo, m23_hi, k)  # m^2(J/psi p)
        # Dalitz boundary in (s1 = m^2_Kp, s2 = m^2_psip): energies in the (Kp) rest frame.
        m1 = np.sqrt(s1)
        e_p = (s1 - M_K ** 2 + M_P ** 2) / (2 * m1)
        e_psi = (M_LB ** 2 - s1 - M_JPSI ** 2) / (2 * m1)
        pp = np.sqrt(np.maximum(e_p ** 2 - M_P ** 2, 0))
        ppsi = np.sqrt(np.maximum(e_psi ** 2 - M_JPSI ** 2, 0))
        lo = (e_p + e_psi) ** 2 - (pp + ppsi) ** 2
        hi = (e_p + e_psi) ** 2 - (pp - ppsi) ** 2
        ok = (s2 > lo) & (s2 < hi)
        out_s1.append(s1[ok])
        out_s2.append(s2[ok])
        have += int(ok.sum())
    s1 = np.concatenate(out_s1)[:n]
    s2 = np.concatenate(out_s2)[:n]
    s3 = M_LB ** 2 + M_JPSI ** 2 + M_P ** 2 + M_K ** 2 - s1 - s2  # m^2(J/psi K)
    # Energies in the Lambda_b rest frame.
    E_psi = (M_LB ** 2 + M_JPSI ** 2 - s1) / (2 * M_LB)
    E_k = (M_LB ** 2 + M_K ** 2 - s2) / (2 * M_LB)
    E_p = (M_LB ** 2 + M_P ** 2 - s3) / (2 * M_LB)
    q_psi = np.sqrt(np.maximum(E_psi ** 2 - M_JPSI ** 2, 0))
    q_k = np.sqrt(np.maximum(E_k ** 2 - M_K ** 2, 0))
    q_p = np.sqrt(np.maximum(E_p ** 2 - M_P ** 2, 0))
    # Planar configuration: J/psi along +x, p and K in the xy plane balancing the momentum.
    cos_pk = np.clip((q_psi ** 2 - q_p ** 2 - q_k ** 2) / (2 * q_p * q_k), -1, 1)
    # p at angle a from -x, K at angle b; q_p sin a = q_k sin b, q_p cos a + q_k cos b = q_psi.
    cos_a = np.clip((q_psi ** 2 + q_p ** 2 - q_k ** 2) / (2 * q_psi * q_p), -1, 1)
    sin_a = np.sqrt(1 - cos_a ** 2)
    psi3 = np.stack([q_psi, 0 * q_psi, 0 * q_psi], -1)
    p3 = np.stack([-q_p * cos_a, q_p * sin_a, 0 * q_p], -1)
    k3 = -(psi3 + p3)
    del cos_pk
    R = _rotation(rng, n)
    psi3 = np.einsum("nij,nj->ni", R, psi3)
    p3 = np.einsum("nij,nj->ni", R, p3)
    k3 = np.einsum("nij,nj->ni", R, k3)
    psi = np.concatenate([psi3, E_psi[:, None]], -1)
    p = np.concatenate([p3, E_p[:, None]], -1)
    k = np.concatenate([k3, E_k[:, None]], -1)
    # J/psi -> mu+ mu- isotropic in the J/psi rest frame.
    qmu = _two_body_p(M_JPSI, M_MU, M_MU)
    c = rng.uniform(-1, 1, n)
    ph = rng.uniform(-np.pi, np.pi, n)
    sn = np.sqrt(1 - c * c)
    mu3 = qmu * np.stack([sn * np.cos(ph), sn * np.sin(ph), c], -1)
    emu = np.sqrt(qmu ** 2 + M_MU ** 2) * np.ones(n)
    beta_psi = psi[:, :3] / psi[:, 3:4]
    mup = _boost(np.concatenate([mu3, emu[:, None]], -1), beta_psi)
    mum = _boost(np.concatenate([-mu3, emu[:, None]], -1), beta_psi)
    return {"p": p, "k": k, "mup": mup, "mum": mum}


def helicity_angles(ev: dict) -> dict:
    """Helicity angles of both decay chains plus the alignment angles (tree.C conventions)."""
    p, k, mup, mum = ev["p"], ev["k"], ev["mup"], ev["mum"]
    n = p.shape[0]
    psi = mup + mum
    lam = p + k
    zc = psi + p  # Pc candidate (J/psi p)
    zhat = np.broadcast_to(np.array([0.0, 0.0, 1.0]), (n, 3))  # Lambda_b flight direction
    out = {}
    # --- Lambda* chain (helicityJpsiLam)
    L = _unit(lam[:, :3])
    psiU = _unit(psi[:, :3])
    out["cosTheta_Lb"] = _dot(zhat, L)
    p_l = _to_rest(p, lam)
    U = _unit(p_l[:, :3])
    out["cosTheta_L"] = -_dot(psiU, U)
    ab = -_unit(zhat - _dot(zhat, L)[:, None] * L)
    out["phiK"] = np.arctan2(_dot(_unit(np.cross(-psiU, ab)), U), _dot(ab, U))
    ab = -ab
    mum_psi = _to_rest(mum, psi)
    U = _unit(mum_psi[:, :3])
    out["cosTheta_Jpsi"] = _dot(psiU, U)
    out["phiMu"] = np.arctan2(_dot(_unit(np.cross(psiU, ab)), U), _dot(ab, U))
    # --- Pc chain (helicityZK)
    ZU = _unit(zc[:, :3])
    out["Z_cosTheta_Lb"] = _dot(zhat, ZU)
    ab = _unit(lam[:, :3] - _dot(lam[:, :3], zhat)[:, None] * zhat)
    out["Z_phiZ"] = np.arctan2(_dot(_unit(np.cross(zhat, ab)), ZU), _dot(ab, ZU))
    psi_z, k_z, mum_z = _to_rest(psi, zc), _to_rest(k, zc), _to_rest(mum, zc)
    U = _unit(psi_z[:, :3])
    kU = _unit(k_z[:, :3])
    out["Z_cosTheta_Z"] = -_dot(kU, U)
    ab = -_unit(zhat - _dot(zhat, ZU)[:, None] * ZU)
    out["Z_phiJpsi"] = np.arctan2(_dot(_unit(np.cross(-kU, ab)), U), _dot(ab, U))
    psiU_z = U
    mum_zpsi = _to_rest(mum_z, psi_z)
    U = _unit(mum_zpsi[:, :3])
    out["Z_cosTheta_Jpsi"] = _dot(psiU_z, U)
    ab = -_unit(-k_z[:, :3] + _dot(k_z[:, :3], psiU_z)[:, None] * psiU_z)
    out["Z_phiMu"] = np.arctan2(_dot(_unit(np.cross(psiU_z, ab)), U), _dot(ab, U))
    # --- alignment angles (helicityTwoFrame)
    k_p, psi_p = _to_rest(k, p), _to_rest(psi, p)
    out["cosTheta_Lambda"] = _dot(_unit(k_p[:, :3]), _unit(psi_p[:, :3]))  # tree.C cosTheta_p
    mum_ps, p_ps, lam_ps = _to_rest(mum, psi), _to_rest(p, psi), _to_rest(lam, psi)
    z3 = _unit(mum_ps[:, :3])
    x3z = -_unit(-p_ps[:, :3] + _dot(p_ps[:, :3], z3)[:, None] * z3)
    x3l = -_unit(-lam_ps[:, :3] + _dot(lam_ps[:, :3], z3)[:, None] * z3)
    out["alpha_Mu"] = np.arctan2(_dot(_unit(np.cross(z3, x3z)), x3l), _dot(x3z, x3l))

    def mass(v):
        return np.sqrt(np.maximum(v[:, 3] ** 2 - _dot(v[:, :3], v[:, :3]), 0))

    out["mLk"] = mass(lam)
    out["mjpsiL"] = mass(zc)
    out["mjpsik"] = mass(psi + k)
    for key in list(out):
        if key.startswith("cos"):
            out[key] = np.clip(out[key], -1.0, 1.0)
    out["Z_cosTheta_Lb"] = np.clip(out["Z_cosTheta_Lb"], -1, 1)
    out["Z_cosTheta_Z"] = np.clip(out["Z_cosTheta_Z"], -1, 1)
    out["Z_cosTheta_Jpsi"] = np.clip(out["Z_cosTheta_Jpsi"], -1, 1)
    return out


def flat_events(n: int, seed: int, zcs: bool = False) -> dict:
    """n flat phase-space events as the angle dictionary consumed by the basis builder.  zcs: also
    the inputs of the Zcs -> J/psi K chain (zcs_angles)."""
    ang = helicity_angles(generate_phase_space(n, seed))
    if zcs:
        ang.update(zcs_angles(ang, seed))
    return ang


def zcs_angles(ang: dict, seed: int) -> dict:
    """Inputs of the Zcs -> J/psi K chain: m(J/psi K) from the Dalitz relation
    m^2(J/psi K) = M^2(Lb) + m^2(p) + m^2(K) + m^2(J/psi) - m^2(Kp) - m^2(J/psi p), and the eight
    Zcs-chain angles.  The reference reads those angles from its ntuples (X_cosTheta_Lb ...
    X_alpha_Mu, RooDalitzAmplitude.cxx:278-295, 346-353) and its generator does not compute them
    (gen_toys/phsp_toys/tree.C covers the Lambda* and Pc chains only), so they are drawn here,
    seeded, flat in cos(theta) and phi; the amplitude path from them on is the reference's."""
    rng = np.random.default_rng(seed * 7 + 424243)
    n = len(ang["mLk"])
    mkp = np.asarray(ang["mLk"], np.float64)
    mjp = np.asarray(ang["mjpsiL"], np.float64)
    m2 = M_LB ** 2 + M_P ** 2 + M_K ** 2 + M_JPSI ** 2 - mkp ** 2 - mjp ** 2
    out = {"mjpsik": np.sqrt(np.maximum(m2, (M_JPSI + M_K) ** 2))}
    for name in ("X_cosTheta_Lb", "X_cosTheta_X", "X_cosTheta_Jpsi", "X_cosTheta_p"):
        out[name] = rng.uniform(-1.0, 1.0, n)
    for name in ("X_phiX", "X_phiJpsi", "X_phiMu", "X_alpha_Mu"):
        out[name] = rng.uniform(-np.pi, np.pi, n)
    return out
