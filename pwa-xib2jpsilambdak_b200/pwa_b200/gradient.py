"""Parameter points of Minuit's numerical gradient and their batched evaluation.

Minuit (src/fit.cpp:222-288 drives Migrad through RooMinuit) estimates the gradient by evaluating the
FCN at the current point and at points that move one parameter at a time by +-h.  gradient_points
builds those 2N + 1 points; numerical_gradient turns their FCN values into central differences.
"""
from __future__ import annotations

import numpy as np

from .model import BlockBuilder, Model


def default_step(value: float, rel: float = 1e-3, floor: float = 1e-4) -> float:
    return max(abs(value) * rel, floor)


def gradient_points(model: Model, vals: dict, names=None, steps: dict | None = None) -> tuple:
    """([labels], [value dicts]): the centre first, then (name, +1) and (name, -1) for every free
    parameter (default: every parameter the model reads)."""
    names = list(names) if names is not None else model.parameter_names()
    labels = [("centre", 0)]
    points = [dict(vals)]
    for n in names:
        h = (steps or {}).get(n, default_step(vals[n]))
        for sgn in (+1, -1):
            v = dict(vals)
            v[n] = vals[n] + sgn * h
            labels.append((n, sgn))
            points.append(v)
    return labels, points


def gradient_blocks(model: Model, vals: dict, names=None, steps: dict | None = None) -> tuple:
    labels, points = gradient_points(model, vals, names, steps)
    builder = BlockBuilder(model, vals)
    blocks = [builder.block()]
    for (name, _), v in zip(labels[1:], points[1:]):
        blocks.append(builder.block({name: v[name]}))
    return labels, blocks


def numerical_gradient(labels: list, points: list, fvals) -> dict:
    """Central differences {name: dF/dx} from the FCN values of gradient_points' output, divided by
    the difference of the two points' parameter values."""
    f = {lab: x for lab, x in zip(labels, fvals)}
    out = {}
    for (name, sgn), v in zip(labels, points):
        if sgn != +1:
            continue
        vm = points[labels.index((name, -1))]
        out[name] = (f[(name, +1)] - f[(name, -1)]) / (v[name] - vm[name])
    return out
