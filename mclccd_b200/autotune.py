"""Autotuner for the launch knobs of the batched path (and the single-scene
tree's grid sizes).

``tune_batch`` times every configuration of the batched step on the batch
as it is set: the form (waves or persistent kernel), the compile-time shapes
(threads per block, traversal stack depth) and the run-time knobs (leaf-scan
size; the work-queue chunk of the persistent form, the wave buffer of the
waves form; a knob the form does not use is not varied).  It checks that
every configuration gives the same per-scene results and leaves the fastest
one set.  A configuration whose stack overflows reports an error and is
skipped.  Choices can be cached per GPU and workload signature in a JSON file.
"""
from __future__ import annotations

import itertools
import json
import os

import numpy as np

from .ccd import CCDError

DEFAULT_SPACE = {"form": (0, 1), "block": (128, 256), "stack": (32, 64), "chunk": (1, 4, 16), "leaf": (1, 4),
                 "wave": (1024, 2048, 4096)}
# knobs that only one form reads
_UNUSED = {0: ("chunk",), 1: ("wave",)}


def _signature(batch) -> str:
    import torch
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    return f"{name}|{batch.n_scenes}|{int(np.sum(batch._nv))}|{batch.precision}"


def tune_batch(batch, space: dict | None = None, repeats: int = 3, cache: str | None = None, verbose: bool = False):
    """Returns (best_config, table); table rows are (config, median batch ms or None)."""
    space = space or DEFAULT_SPACE
    sig = _signature(batch)
    if cache and os.path.exists(cache):
        with open(cache) as f:
            known = json.load(f)
        if sig in known:
            batch.set_tuning(**known[sig])
            return known[sig], []
    keys = list(space)
    table, ref, best, best_ms = [], None, None, float("inf")
    seen = set()
    for vals in itertools.product(*(space[k] for k in keys)):
        cfg = dict(zip(keys, vals))
        for k in _UNUSED.get(cfg.get("form"), ()):
            if k in cfg:
                cfg[k] = space[k][0]
        if tuple(cfg.items()) in seen:
            continue
        seen.add(tuple(cfg.items()))
        try:
            batch.set_tuning(**cfg)
            ms = []
            for _ in range(repeats + 1):
                batch.run()
                r = batch.results()
                ms.append(r["batch_ms"])
            t = float(np.median(ms[1:]))   # the first run includes graph capture
        except CCDError as e:
            if verbose:
                print("skip", cfg, e)
            table.append((cfg, None))
            continue
        key = (r["n_hits"].tolist(), r["min_toi"].tolist(), r["n_discrete"].tolist(), r["n_stencils"].tolist())
        if ref is None:
            ref = key
        elif key != ref:
            raise RuntimeError(f"configuration {cfg} changed the results")
        table.append((cfg, t))
        if verbose:
            print(cfg, f"{t:.3f} ms")
        if t < best_ms:
            best, best_ms = cfg, t
    if best is None:
        raise RuntimeError("no configuration ran")
    batch.set_tuning(**best)
    if cache:
        known = {}
        if os.path.exists(cache):
            with open(cache) as f:
                known = json.load(f)
        known[sig] = best
        with open(cache, "w") as f:
            json.dump(known, f, indent=1)
    return best, table
