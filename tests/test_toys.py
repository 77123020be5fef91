"""Toy ensembles: the seeded size recipe and the packing of toys that share one MC sample (host only)."""
import numpy as np

from pwa_b200 import basis as B, kinematics as K, toys


def test_toy_sizes_recipe():
    s = toys.toy_sizes()
    assert len(s) == 256 and s.dtype == np.int64
    assert s.min() >= 5000 and s.max() < 200000
    assert np.array_equal(s, toys.toy_sizes())  # seeded
    # log-uniform: the median is near the geometric mean of the range
    assert abs(np.log(np.median(s)) - 0.5 * (np.log(5e3) + np.log(2e5))) < 0.3


def test_ensemble_layout_bands_per_toy():
    data = [K.flat_events(n, 100 + t) for t, n in enumerate((40, 75, 9))]
    mc = K.flat_events(120, 7)
    ens = toys.build_ensemble(data, mc, np.full(120, 0.5))
    s = ens.sample
    assert list(ens.offsets) == [0, 40, 115, 124] and s.nda == 124 and s.n == 244
    mz = np.asarray(s.pp[s.n_size:s.n_size + s.n], np.float32)
    w = np.asarray(s.pp[2 * s.n_size:2 * s.n_size + s.n], np.float32)
    assert np.all(w[:124] <= -1000) and np.all(w[124:] == 0.5)
    for t in range(ens.n_toys):
        a, b = ens.offsets[t], ens.offsets[t + 1]
        band = B.band_of(mz[a:b])
        assert np.all(np.diff(band) >= 0)  # each toy sorted into its own bands
        assert ens.band1[t] == (band == 1).sum() and ens.band2[t] == (band == 2).sum()
        v = ens.view(t)
        assert v.first == a and v.nda == b - a and v.sum_w_data == b - a
