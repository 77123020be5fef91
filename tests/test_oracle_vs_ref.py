"""The FP64 oracle pinned against the reference's own likelihood code run on host cores."""
import json
from pathlib import Path

import numpy as np
import pytest

from conftest import make_test_sample

G = json.loads((Path(__file__).resolve().parent / "golden" / "ref_nll.json").read_text())


@pytest.mark.parametrize("row", G, ids=[r["model"] for r in G])
def test_oracle_reproduces_golden(row, oracle_mod):
    mdl, vals, blk, smp = make_test_sample(row["model"], row["n_data"], row["n_mc"], seed=row["seed"])
    import hashlib
    assert hashlib.sha256(np.ascontiguousarray(blk.data).tobytes()).hexdigest()[:16] == row["param_block_sha"]
    v, s, fx, _ = oracle_mod.nll(smp, blk)
    assert abs(v - row["nll_oracle"]) < 1e-7
    assert np.allclose(fx[:8], row["fx_head_oracle"], rtol=1e-12)
    # the reference's FP32 arithmetic agrees with the FP64 restatement to its own rounding noise
    assert abs(row["nll_reference_fp32"] - v) < 0.05
    assert abs(row["sumint_reference_fp32"] / s - 1) < 5e-5


@pytest.mark.parametrize("name", ["small_kmatrix", "small_bw", "small_zcs"])
def test_oracle_vs_reference_live(name, oracle_mod):
    L = oracle_mod.ref_lib(*{"small_kmatrix": (3, 4, 0), "small_bw": (2, 2, 0), "small_zcs": (2, 1, 2)}[name],
                           build_if_missing=True)
    if L is None:
        pytest.skip("reference host build unavailable")
    mdl, vals, blk, smp = make_test_sample(name, 600, 6000, seed=31)
    v, s, fx, _ = oracle_mod.nll(smp, blk)
    ref = oracle_mod.RefHost(smp, blk)
    rv, rs = ref.store_fx(blk)
    rel = np.abs(ref.fx - fx) / np.abs(fx)
    assert np.median(rel) < 1e-5 and np.max(rel) < 2e-3
    assert abs(rv - v) < 0.05
    # swapping the coupling read order breaks agreement by orders of magnitude
    v2, _, _, _ = oracle_mod.nll(smp, blk, swap_coupling_parts=True)
    assert abs(rv - v2) > 100 * abs(rv - v)


def test_oracle_grid_smearing_limits(oracle_mod):
    """The oracle's Gaussian-grid smearing: one offset at zero is the unsmeared |A|^2 (times w for MC),
    and the weights sum to one."""
    from conftest import make_test_sample
    mdl, vals, blk, smp = make_test_sample("small_kmatrix", 300, 3000)
    off, w = oracle_mod.gauss_grid(0.0027, 0.0005, 17)
    assert len(off) == 35 and abs(w.sum() - 1) < 1e-15 and off[17] == 0.0
    fx, fxn = oracle_mod.eval_fx_grid(smp, blk, 0.0027, 0.0005, 0)
    a2 = oracle_mod.amp2(smp, blk)
    wt = np.where(np.arange(smp.n) < smp.nda, 1.0, np.asarray(smp.pp[2 * smp.n_size:2 * smp.n_size + smp.n], np.float64))
    assert np.max(np.abs(fx - a2 * wt) / (a2 * wt)) < 1e-13
