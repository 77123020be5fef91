"""Synthetic kinematics and the per-event basis: conservation laws, d-function identities, layout."""
import numpy as np

from pwa_b200 import basis as B, dataset as D, kinematics as K


def test_four_momentum_conservation():
    ev = K.generate_phase_space(5000, 1)
    tot = ev["p"] + ev["k"] + ev["mup"] + ev["mum"]
    assert np.allclose(tot[:, :3], 0, atol=1e-9)
    assert np.allclose(tot[:, 3], K.M_LB, atol=1e-9)
    a = K.helicity_angles(ev)
    assert np.all((a["mLk"] > K.MKP_MIN - 1e-9) & (a["mLk"] < K.MKP_MAX + 1e-9))
    assert np.all((a["mjpsiL"] > K.MZ_MIN - 1e-9) & (a["mjpsiL"] < K.MZ_MAX + 1e-9))
    # m^2 sum rule of a three-body decay
    s = a["mLk"] ** 2 + a["mjpsiL"] ** 2 + a["mjpsik"] ** 2
    assert np.allclose(s, K.M_LB ** 2 + K.M_JPSI ** 2 + K.M_P ** 2 + K.M_K ** 2, atol=1e-8)


def test_flat_angles():
    a = K.flat_events(40000, 2)
    for k in ("cosTheta_Lb", "cosTheta_L", "cosTheta_Jpsi", "Z_cosTheta_Z"):
        assert abs(a[k].mean()) < 0.02
    for k in ("phiK", "phiMu", "Z_phiZ", "alpha_Mu"):
        assert abs(a[k].mean()) < 0.05


def test_wigner_d_identities():
    beta = np.linspace(0.05, 3.0, 7)
    for j2 in range(1, 10, 2):
        j = j2 / 2
        ms = [m / 2 for m in range(-j2, j2 + 1, 2)]
        for n in ms:
            tot = sum(B.dfun(beta, j, m, n) ** 2 for m in ms)
            assert np.allclose(tot, 1, atol=1e-12)
            for m in ms:
                assert np.allclose(B.dfun(beta, j, m, n), (-1) ** int(round(m - n)) * B.dfun(beta, j, n, m), atol=1e-12)
    # closed forms
    b = beta
    assert np.allclose(B.dfun(b, 0.5, 0.5, -0.5), -np.sin(b / 2))
    assert np.allclose(B.dfun(b, 1.5, 1.5, 1.5), np.cos(b / 2) ** 3)
    assert np.allclose(B.dfun(b, 1.5, 0.5, 0.5), 0.5 * np.cos(b / 2) * (3 * np.cos(b) - 1))


def test_pack_layout_and_bands():
    a = K.flat_events(3000, 3)
    s = D.build_sample({k: v[:1000] for k, v in a.items()}, {k: v[1000:] for k, v in a.items()}, np.ones(2000))
    pp = s.pp.reshape(111, s.n_size)
    assert s.n_size == (3000 // 32 + 1) * 32
    assert np.all(pp[2, :1000] == -1001.0) and np.all(pp[2, 1000:3000] == 1.0)
    b = B.band_of(pp[1, :1000])
    assert np.all(np.diff(b) >= 0)  # data sorted into bands 1, 2, 3
    assert s.nda_smr1 == int((b == 1).sum()) and s.nda_fine == int((b == 2).sum())
    # Lambda* J=1/2 d-function planes of helicity slots 4, 5 are zero
    assert np.all(pp[51 + 4, :3000] == 0) and np.all(pp[51 + 6 + 5, :3000] == 0)
