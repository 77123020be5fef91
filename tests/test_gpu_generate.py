"""On-device event generator and basis builder vs the host (numpy) restatement."""
import numpy as np
import pytest

from conftest import make_test_sample

pytestmark = pytest.mark.gpu

ANGLE_KEYS = ["mLk", "mjpsiL", "cosTheta_Lb", "cosTheta_L", "cosTheta_Jpsi", "phiK", "phiMu", "Z_cosTheta_Lb",
              "Z_cosTheta_Z", "Z_cosTheta_Jpsi", "Z_phiZ", "Z_phiJpsi", "Z_phiMu", "cosTheta_Lambda", "alpha_Mu"]


def test_angles_from_vectors_match_host():
    import torch
    from pwa_b200 import kinematics as K, lib
    ev = K.generate_phase_space(20000, 3)
    host = K.helicity_angles(ev)
    n = ev["p"].shape[0]
    v = np.concatenate([ev[k].T for k in ("p", "k", "mup", "mum")], 0)  # (16, n)
    dv = torch.as_tensor(np.ascontiguousarray(v), device="cuda")
    da = torch.zeros((15, n), dtype=torch.float64, device="cuda")
    lib.check(lib.load().pwa_angles_from_vectors(dv.data_ptr(), n, da.data_ptr(), None), "angles")
    a = da.cpu().numpy()
    for q, key in enumerate(ANGLE_KEYS):
        d = np.abs(a[q] - host[key])
        if key.startswith(("phi", "Z_phi", "alpha")):
            d = np.minimum(d, 2 * np.pi - d)
        assert d.max() < 1e-9, (key, d.max())


def test_basis_from_angles_matches_host():
    import torch
    from pwa_b200 import basis as B, kinematics as K, lib
    ang = K.flat_events(20000, 4)
    n = len(ang["mLk"])
    ns = B.n_size_of(n)
    hb = B.fill_basis(ang)
    host = B.pack_soa(ang["mLk"].astype(np.float32), ang["mjpsiL"].astype(np.float32), np.full(n, 0.5, np.float32),
                      hb, ns)
    arr = np.stack([ang[k] for k in ANGLE_KEYS] + [np.full(n, 0.5)], 0)
    da = torch.as_tensor(np.ascontiguousarray(arr), device="cuda")
    pp = torch.zeros((111, ns), dtype=torch.float32, device="cuda")
    pp1 = torch.zeros((96, ns), dtype=torch.float32, device="cuda")
    pp2 = torch.zeros((96, ns), dtype=torch.float32, device="cuda")
    lib.check(lib.load().pwa_basis_from_angles(da.data_ptr(), n, pp.data_ptr(), pp1.data_ptr(), pp2.data_ptr(), ns,
                                               None), "basis")
    for name, dev in (("pp", pp), ("pp1", pp1), ("pp2", pp2)):
        g = dev.cpu().numpy().reshape(-1)
        h = host[name]
        # equal up to one float rounding of values below 1 in magnitude (device vs host libm)
        assert np.max(np.abs(g - h)) < 2.5e-7, (name, np.max(np.abs(g - h)))


def test_generated_events_are_flat_phase_space():
    import torch
    from pwa_b200 import basis as B, kinematics as K, lib
    n = 200000
    ns = B.n_size_of(n)
    pp = torch.zeros((111, ns), dtype=torch.float32, device="cuda")
    pp1 = torch.zeros((96, ns), dtype=torch.float32, device="cuda")
    pp2 = torch.zeros((96, ns), dtype=torch.float32, device="cuda")
    lib.check(lib.load().pwa_generate_events(pp.data_ptr(), pp1.data_ptr(), pp2.data_ptr(), ns, 0, n, 7, 0, 0.2, 1.0,
                                             0, None), "generate")
    p = pp.cpu().numpy()
    mkp, mz, w = p[0, :n], p[1, :n], p[2, :n]
    assert mkp.min() >= K.MKP_MIN - 1e-5 and mkp.max() <= K.MKP_MAX + 1e-5
    assert mz.min() >= K.MZ_MIN - 1e-5 and mz.max() <= K.MZ_MAX + 1e-5
    assert 0.2 <= w.min() and w.max() <= 1.0 and abs(w.mean() - 0.6) < 0.01
    # same Dalitz-plane density as the host generator (binned comparison of m^2_Kp and m^2_psip)
    host = K.flat_events(n, 9)
    for a, b in ((mkp, host["mLk"]), (mz, host["mjpsiL"])):
        ha, edges = np.histogram(a ** 2, bins=20)
        hb, _ = np.histogram(b ** 2, bins=edges)
        chi2 = np.sum((ha - hb) ** 2 / np.maximum(ha + hb, 1))
        assert chi2 < 60, chi2
    assert np.all(np.abs(p[3:111, :n]) <= 1.0 + 1e-6) and np.all(np.abs(pp1.cpu().numpy()) <= 1.0 + 1e-6)
    # the same (seed, id) regenerates the same event
    lib.check(lib.load().pwa_generate_events(pp.data_ptr(), pp1.data_ptr(), pp2.data_ptr(), ns, 0, 100, 7, 0, 0.2,
                                             1.0, 0, None), "generate")
    assert np.array_equal(pp.cpu().numpy()[:, :100], p[:, :100])


def test_gpu_sample_bands_and_parity(oracle_mod):
    from pwa_b200 import configs, gpu_sample, lib, model as M
    mdl, vals = configs.small_kmatrix()
    blk = M.build_param_block(mdl, vals)
    ds = gpu_sample.generate(blk, 3000, 30000, seed=3, batch=200000)
    hs = ds.to_host()
    assert (hs.nda_smr1, hs.nda_fine) == (ds.nda_smr1, ds.nda_fine)
    ctx = lib.Context(0)
    ctx.bind_device(ds)
    r = ctx.eval_nll(blk)
    v, s, _, _ = oracle_mod.nll(hs, blk)
    assert abs(r.nll - v) < 1e-6 and abs(r.sumint / s - 1) < 1e-12
    ctx.close()
