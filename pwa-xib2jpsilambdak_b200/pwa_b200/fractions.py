"""Fit fractions, interference fractions and per-resonance event weights.

RooDalitzAmplitude::getIFandFF (src/RooDalitzAmplitude.cxx:5250-5435) returns the matrix, in percent
of the total MC integral I = sum_MC w |A|^2, of the integrals of the resonance amplitude products:
diagonal entries are the fit fractions, off-diagonal entries (a, b) half the interference
2 Re sum_MC w sum_h conj(A_a,h) A_b,h, so that all entries add up to 100.  The integrals come from the
normalisation sums of subset parameter blocks (couplings of all other resonances set to zero, as
SetupCoupling does for storeResonanceWeights :985-1292):
  M_aa = I({a}),  M_ab = (I({a, b}) - I({a}) - I({b})) / 2.
"""
from __future__ import annotations

import numpy as np

from .model import Model, build_param_block


def _subset_block(model: Model, vals: dict, members: list):
    lst = [i for i in members if i < model.NR]
    pcs = [i - model.NR for i in members if i >= model.NR]
    return build_param_block(model, vals, include=(lst, pcs))


def interference_matrix(integral, model: Model, vals: dict) -> np.ndarray:
    """(NR + NZ) x (NR + NZ) matrix in percent; integral(block) -> MC integral of a parameter block
    (e.g. lib.Context.mc_integral on the GPU)."""
    n = model.NR + model.NZ
    single = np.array([integral(_subset_block(model, vals, [a])) for a in range(n)])
    total = integral(build_param_block(model, vals))
    M = np.diag(single)
    for a in range(n):
        for b in range(a + 1, n):
            pair = integral(_subset_block(model, vals, [a, b]))
            M[a, b] = M[b, a] = 0.5 * (pair - single[a] - single[b])
    return 100.0 * M / total


def fit_fractions(integral, model: Model, vals: dict) -> dict:
    """{resonance name: fit fraction in percent}."""
    n = model.NR + model.NZ
    total = integral(build_param_block(model, vals))
    names = [r.name for r in model.resonances]
    return {names[a]: 100.0 * integral(_subset_block(model, vals, [a])) / total for a in range(n)}


def resonance_weights(amp2, model: Model, vals: dict, groups: dict) -> dict:
    """Per-event unsmeared |A|^2 of subsets of resonances (storeResonanceWeights): groups maps a label
    to resonance indices; amp2(block) -> per-event values (lib.Context.amp2)."""
    return {label: amp2(_subset_block(model, vals, list(members))) for label, members in groups.items()}
