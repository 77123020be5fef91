"""Launch-shape autotuning with a JSON cache (the project's own; no counterpart in the reference).

`tune_batch` picks, per event class of the batched gradient evaluation, how many waves of resident
blocks its passes launch (pwa_ctx_set_batch_waves): it times the classes' passes with CUDA events over
a few batch calls for each candidate and keeps, per class, the fastest.  `pwa_b200.ensemble.autotune`
does the same for the toy-ensemble kernel.  Choices are cached in a JSON file (`$PWA_B200_TUNE_CACHE`,
default `~/.cache/pwa_b200/tune.json`) under a key of device name and workload shape, so later runs
on the same device and shape take them without timing.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

BATCH_WAVES = (1, 2, 4, 8, 16, 32, 64)


def cache_path(name: str = "tune.json") -> Path:
    base = os.environ.get("PWA_B200_TUNE_CACHE")
    if base:
        return Path(base)
    return Path(os.environ.get("XDG_CACHE_HOME", str(Path.home() / ".cache"))) / "pwa_b200" / name


def load_cache(path: Path) -> dict:
    if path.exists():
        try:
            return json.loads(path.read_text())
        except (OSError, ValueError):
            return {}
    return {}


def store_cache(path: Path, table: dict):
    try:
        path.parent.mkdir(parents=True, exist_ok=True)
        path.write_text(json.dumps(table, indent=1))
    except OSError:
        pass


def device_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def batch_key(ctx, blocks) -> str:
    segs = ctx.segments()
    shape = ",".join(f"{k}:{int(np.round(np.log2(max(n, 1))))}" for k, n, _ in segs)
    b = blocks[0]
    return f"batch|{device_name(getattr(ctx, 'device', 0))}|NR={b.NR}|NZ={b.NZ}|points={len(blocks)}|classes={shape}"


def tune_batch(ctx, blocks, cache=None, candidates=BATCH_WAVES, reps: int = 2, force: bool = False,
               nll_shift: float = 1e7) -> dict:
    """Per event class, the waves whose passes ran fastest over `reps` timed batch calls of `blocks`
    (after one warm-up per candidate); applied to the context and cached.  Returns {kind: waves, ...}
    with the per-candidate times."""
    path = Path(cache) if cache else cache_path()
    table = load_cache(path)
    key = batch_key(ctx, blocks)
    kinds = [k for k, _, _ in ctx.segments()]
    if key in table and not force:
        choice = table[key]
        for k, w in choice["waves"].items():
            ctx.set_batch_waves(int(k), int(w))
        return dict(choice, cached=True)
    timed = {}
    ctx.set_timing(True)
    for w in candidates:
        for k in set(kinds):
            ctx.set_batch_waves(k, w)
        ctx.eval_nll_batch(blocks, nll_shift)
        ms = []
        for _ in range(reps):
            ctx.eval_nll_batch(blocks, nll_shift)
            ms.append(ctx.batch_segment_ms())
        med = np.median(np.array(ms), axis=0)
        for i, k in enumerate(kinds):
            timed.setdefault(k, {})[w] = timed.get(k, {}).get(w, 0.0) + float(med[i])
    best = {str(k): int(min(t, key=t.get)) for k, t in timed.items()}
    for k, w in best.items():
        ctx.set_batch_waves(int(k), w)
    choice = {"waves": best, "ms": {str(k): {str(w): round(v, 3) for w, v in t.items()} for k, t in timed.items()}}
    table[key] = choice
    store_cache(path, table)
    return dict(choice, cached=False)
