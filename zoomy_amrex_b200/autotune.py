"""Pick the strip shape of the FP32 stage kernels by measurement.

The FP32 kernels are compiled for a few strip shapes (warps per block NW x
rows per warp CPT; a strip is 30 columns x NW*CPT rows). Which one is fastest
depends on the state width (n_dof_q: more registers per cell favour fewer
rows in flight) and on the box sizes (small boxes waste less of a short
strip). ``tune`` times every shape on a given batch with CUDA events and
records the winner per (n_dof_q, precision, size class) in a JSON cache next
to the library; ``cached_variant`` looks it up.
"""
from __future__ import annotations

import fcntl
import json
import os
import pathlib

import numpy as np

from . import _lib

CACHE = _lib.LIB_PATH.parent / "autotune.json"


def size_class(cells_per_instance: float) -> str:
    """Coarse box-size bucket: the best strip height changes with box size."""
    if cells_per_instance < 128 * 128:
        return "small"
    if cells_per_instance < 1024 * 1024:
        return "medium"
    return "large"


def _key(n_q: int, precision: str, cls: str) -> str:
    return f"n_q={n_q}/{precision}/{cls}"


def _load(path: pathlib.Path = CACHE) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def cached_variant(n_q: int, precision: str, cells_per_instance: float,
                   path: pathlib.Path = CACHE) -> int | None:
    ent = _load(path).get(_key(n_q, precision, size_class(cells_per_instance)))
    return None if ent is None else int(ent["variant"])


def record(n_q: int, precision: str, cells_per_instance: float, variant: int, times_ms: dict,
           shapes: list, path: pathlib.Path = CACHE) -> None:
    entry = dict(variant=int(variant), shape=list(shapes[variant]),
                 ms_per_step={str(k): float(v) for k, v in times_ms.items()})
    # Read-modify-write under an exclusive lock on a sidecar file, so that
    # processes tuning different keys at the same time (one per GPU) each add
    # their key to the latest cache; the new version is written to a
    # per-process temporary file and renamed over the cache atomically, so a
    # reader never sees a partial document.
    tmp = path.with_suffix(f".json.{os.getpid()}.tmp")
    try:
        with open(path.with_suffix(".json.lock"), "a") as lk:
            fcntl.flock(lk, fcntl.LOCK_EX)
            try:
                data = _load(path)
                data[_key(n_q, precision, size_class(cells_per_instance))] = entry
                tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
                tmp.replace(path)
            finally:
                fcntl.flock(lk, fcntl.LOCK_UN)
    except OSError:   # the cache is an optimisation: a read-only install just re-tunes
        tmp.unlink(missing_ok=True)


def time_variant(batch, variant: int, steps: int = 10, warmup: int = 3, repeats: int = 3) -> float:
    """ms per step of ``batch`` with strip shape ``variant`` (device time, best of repeats)."""
    import torch
    batch.set_variant(variant)
    batch.begin()
    batch.evolve(warmup)
    best = float("inf")
    for _ in range(repeats):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        batch.sync()
        e0.record(batch.stream)
        batch.evolve(steps)
        e1.record(batch.stream)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / steps)
    return best


def tune(batch, steps: int = 10, warmup: int = 3, save: bool = True) -> tuple[int, dict]:
    """Time every compiled strip shape on ``batch``; leave it on the fastest.

    The batch's state advances during the measurement: tune on a copy of the
    real inputs (or reload them afterwards).
    """
    from .batch import tile_variants
    shapes = tile_variants()
    times = {v: time_variant(batch, v, steps, warmup) for v in range(len(shapes))}
    best = min(times, key=times.get)
    batch.set_variant(best)
    if save:
        cells = np.mean([c.nx * c.ny for c in batch.cfgs])
        record(4, "fp32", cells, best, times, shapes)
    return best, times
