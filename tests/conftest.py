import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "pwa-xib2jpsilambdak_b200"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(ROOT / "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


_samples = {}


def make_test_sample(model_name: str, n_data: int, n_mc: int, seed: int = 11, w_range=(0.2, 1.0)):
    """Seeded sample with data drawn by hit-or-miss from the oracle's unsmeared |A|^2."""
    key = (model_name, n_data, n_mc, seed, w_range)
    if key in _samples:
        return _samples[key]
    from pwa_b200 import configs, dataset as D, model as M
    import oracle as O
    mdl, vals = configs.MODELS[model_name]()
    blk = M.build_param_block(mdl, vals)

    def amp2(ang):
        s = D.build_sample({k: v[:0] for k, v in ang.items()}, ang, np.ones(len(ang["mLk"])))
        fx, _ = O.eval_fx(s, blk, -1, 0)
        return fx

    smp = D.make_sample(n_data, n_mc, w_range, seed, amp2, zcs=mdl.NX > 0)
    _samples[key] = (mdl, vals, blk, smp)
    return _samples[key]


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle as O
    O.build()
    return O
