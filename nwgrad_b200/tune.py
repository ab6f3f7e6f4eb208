"""Autotuner: the fastest kernel geometry per size class of a batch, measured on the device.

A geometry is (lanes per pair, DP rows per lane): one lane per pair (the inter-pair fill), a
quarter, half or whole warp per pair, with 2 to 32 rows per lane.  Every geometry computes
the same cells, so results do not change; speed does, through padding (rows rounded up to
whole stripes), skew (the wavefront's ramp), parallelism and shared memory per group.

Pairs are grouped in size classes: ceil(log2(rows * columns)), the same rule as the library's
planner, so a batch of pairs of 100 to 500 residues spans five classes, each tuned apart.  For each class in a batch
the tuner aligns a sample of the class's own pairs with every candidate geometry, times the
device work (``SeqPairBatch.last_timing``), keeps the fastest and stores the choice in a JSON
cache keyed by device, problem type and class.

Per pair, geometries differ mainly in padding: a pair's rows are rounded up to whole stripes
of lanes x rows DP rows, and each stripe adds the lanes' skew to its columns.  So the tuner
also turns each geometry's measured time into a cost per padded cell and tries the mixed
plan in which every pair of the class takes the geometry with the least cost x padded cells
(``nwg_set_geometry_costs``); the mixed plan is kept when it measures faster than the best
single geometry.  ``apply`` hands the table to the library; ``plain`` selects the plain fill
instead (one fixed geometry, 32 lanes x 4 rows, for every pair).
"""
from __future__ import annotations

import functools
import json
import os

import numpy as np

HARD_GEOS = [(32, 4), (32, 2), (32, 1), (32, 8), (1, 8), (1, 16), (1, 24), (1, 32)]
SOFT_GEOS = [(32, 4), (32, 2), (32, 8), (16, 4), (16, 2), (16, 8), (8, 4), (1, 8), (1, 16), (1, 24), (1, 32)]


def size_class(rows: int, cols: int) -> int:
    """ceil(log2(rows x cols)), in integers (the store's own size_class)."""
    c = max(rows, 1) * max(cols, 1)
    return 0 if c <= 1 else (c - 1).bit_length()


def _cache_path() -> str:
    p = os.environ.get("NWGRAD_B200_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "nwgrad_b200", "tune.json")


def _load_cache() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save_cache(c: dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


@functools.lru_cache(maxsize=None)
def _device_name(dev: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(dev)
    except Exception:   # noqa: BLE001 - the name only keys the cache
        return f"cuda:{dev}"


def _soft(batch) -> bool:
    return batch._grad_mode == "soft"


def _class_of(batch) -> np.ndarray:
    """Every pair's size class: ceil(log2(cells)) in integers, as the store computes it (the
    binary exponent of cells - 1)."""
    m = np.diff(batch._oa).astype(np.int64)
    n = np.diff(batch._ob).astype(np.int64)
    rows = m + 1 if _soft(batch) else m
    cells = np.maximum(rows, 1) * np.maximum(n, 1)
    return np.where(cells <= 1, 0, np.frexp(np.maximum(cells - 1, 1).astype(np.float64))[1]).astype(np.int64)


def _classes(batch, sc=None) -> dict:
    """size class -> indices of the batch's pairs in it."""
    if sc is None:
        sc = _class_of(batch)
    order = np.argsort(sc, kind="stable")
    bounds = np.flatnonzero(np.diff(sc[order])) + 1
    return {int(sc[g[0]]): g for g in np.split(order, bounds) if g.size}   # each in pair order (stable)


def _codes(batch):
    """Concatenated codes of both sides (the batch's own encoding)."""
    if getattr(batch, "_codes", None) is not None:
        return batch._codes
    from .batch import _encode_all
    a, _, _ = _encode_all(batch._alpha, batch._seqs_a, "A")
    b, _, _ = _encode_all(batch._alpha, batch._seqs_b, "B")
    return a, b


def _subset(batch, idx, codes):
    """A batch of the same type over the pairs idx (tracks carried along)."""
    a, b = codes
    oa, ob = batch._oa, batch._ob
    la = (oa[idx + 1] - oa[idx]).astype(np.int64)
    lb = (ob[idx + 1] - ob[idx]).astype(np.int64)
    sa = np.concatenate([a[oa[p]:oa[p + 1]] for p in idx]) if la.sum() else np.zeros(0, np.uint8)
    sb = np.concatenate([b[ob[p]:ob[p + 1]] for p in idx]) if lb.sum() else np.zeros(0, np.uint8)
    noa = np.zeros(len(idx) + 1, np.int64); np.cumsum(la, out=noa[1:])
    nob = np.zeros(len(idx) + 1, np.int64); np.cumsum(lb, out=nob[1:])
    kw = dict(gap_model=batch._gap_model, mode=batch._mode, grad_mode=batch._grad_mode, device=batch._device)
    if batch._flat_t is not None:
        kw["tracks"] = np.concatenate([batch._flat_t[oa[p]:oa[p + 1]] for p in idx])
    if batch._flat_g is not None:
        kw["gap_tracks"] = np.concatenate([batch._flat_g[oa[p] + p:oa[p + 1] + p + 1] for p in idx])
    sub = type(batch).from_codes(sa, noa, sb, nob, batch._params, **kw)
    sub.soft_temperature = batch.soft_temperature
    sub.soft_precision = batch.soft_precision
    return sub, float(np.sum(la.astype(np.float64) * lb.astype(np.float64)))


def _candidates(batch):
    K, N = batch._params.num_sets, batch._alpha.size
    elem = 4 if batch._precision == 32 else 8
    if _soft(batch):
        lane_ok = K * N * N * elem * 32 <= 48 * 1024
        return [g for g in SOFT_GEOS if g[0] > 1 or lane_ok]
    return list(HARD_GEOS)


def _padded(batch, idx, geo) -> float:
    """Cells the geometry computes for the pairs idx: whole stripes, columns plus the skew."""
    G, R = geo
    m = (batch._oa[idx + 1] - batch._oa[idx]).astype(np.float64)
    n = (batch._ob[idx + 1] - batch._ob[idx]).astype(np.float64)
    rows = m + 1 if _soft(batch) else m
    extra = 1 if _soft(batch) else 0
    stripes = np.ceil(np.maximum(rows, 1) / (G * R))
    return float(np.sum(stripes * G * R * (n + extra + G - 1)))


def _set_costs(batch, sc: int, costs) -> None:
    from ._capi import check, ptr, _i32p, _dp
    lanes = np.array([g for g, _, _ in costs], np.int32)
    rows = np.array([r for _, r, _ in costs], np.int32)
    ns = np.array([c for _, _, c in costs], np.float64)
    check(batch._store._L.nwg_set_geometry_costs(batch._store.h, 1 if _soft(batch) else 0, int(sc), len(costs),
                                                ptr(lanes, _i32p), ptr(rows, _i32p), ptr(ns, _dp)))


def describe(entry) -> str:
    """A table entry in words."""
    if isinstance(entry, dict):
        return "per pair by cost: " + ", ".join(f"{g}x{r}" for g, r, _ in entry["costs"])
    return f"{entry[0]} lanes x {entry[1]} rows"


def _key(batch, sc: int) -> str:
    return "|".join(str(x) for x in (_device_name(batch._device), "soft" if _soft(batch) else "hard",
                                     batch._gap_model, batch._mode, batch._precision, batch._alpha.size,
                                     batch._params.num_sets, int(batch._tracked), sc)) + \
        (f"|ends{batch._sg}" if getattr(batch, "_am", 0) == 2 else "")   # semiglobal: its free ends


def tune(batch, sample_pairs: int = 65536, force: bool = False, verbose: bool = False, reps: int = 2,
         mixed: bool = True) -> dict:
    """{size class: (lanes, rows) or {"costs": [(lanes, rows, ns per padded cell), ...]}} for the
    classes of ``batch``, measured (or from the cache).

    The sample should fill the device many times over for every candidate (the narrower
    geometries run several times as many pairs at once): a sample that does not would
    favour them falsely."""
    grad = {"none": 0, "hard": 1, "soft": 2}[batch._grad_mode]
    cache = _load_cache()
    table = {}
    codes = None
    dirty = False
    csc = _class_of(batch)
    present = np.flatnonzero(np.bincount(csc))
    keys = {int(sc): _key(batch, int(sc)) for sc in present}
    if not force and all(k in cache for k in keys.values()):
        groups = {sc: None for sc in keys}           # every class cached: no pair lists needed
    else:
        groups = _classes(batch, csc)
    for sc, idx in sorted(groups.items()):
        key = keys[sc]
        if not force and key in cache:
            ent = cache[key]
            table[sc] = {"costs": [tuple(x) for x in ent["costs"]]} if "costs" in ent else tuple(ent["geo"])
            continue
        if codes is None:
            codes = _codes(batch)
        if idx.size > sample_pairs:   # evenly spread over the class
            idx = idx[np.linspace(0, idx.size - 1, sample_pairs).astype(np.int64)]
        sub, cells = _subset(batch, idx, codes)
        best, best_ms, times = None, float("inf"), {}
        for geo in _candidates(batch):
            sub._tune = geo
            try:
                sub._run(grad)                      # warm: plan, first launch
                ms = min(_timed(sub, grad) for _ in range(reps))
            except (ValueError, RuntimeError):
                continue
            times[f"{geo[0]}x{geo[1]}"] = ms
            if ms < best_ms:
                best, best_ms = geo, ms
        if best is None:
            del sub
            continue
        entry = best
        mixed_ms = None
        if mixed and len(times) > 1:
            # the mixed plan: every pair takes the geometry with the least measured cost x its
            # padded cells; kept when it beats the best single geometry
            sidx = np.arange(len(idx), dtype=np.int64)
            costs = []
            for geo in _candidates(batch):
                k = f"{geo[0]}x{geo[1]}"
                if k in times:
                    costs.append((geo[0], geo[1], times[k] * 1e6 / max(_padded(sub, sidx, geo), 1.0)))
            try:
                sub._tune = (0, 0)
                _set_costs(sub, sc, costs)
                sub._run(grad)
                mixed_ms = min(_timed(sub, grad) for _ in range(reps))
            except (ValueError, RuntimeError):
                mixed_ms = None
            if mixed_ms is not None and mixed_ms < 0.99 * best_ms:
                entry = {"costs": costs}
        del sub
        table[sc] = entry
        use_ms = mixed_ms if isinstance(entry, dict) else best_ms
        cache[key] = {"gcups": cells / (use_ms / 1e3) / 1e9 if use_ms > 0 else None, "ms": times,
                      "mixed_ms": mixed_ms, "sample_pairs": int(idx.size)}
        if isinstance(entry, dict):
            cache[key]["costs"] = [list(x) for x in entry["costs"]]
        else:
            cache[key]["geo"] = list(entry)
        dirty = True
        if verbose:
            print(f"size class 2^{sc}: {idx.size} pairs, best single {best[0]} lanes x {best[1]} rows "
                  f"({best_ms:.3f} ms), mixed {mixed_ms}; " + ", ".join(f"{k} {v:.3f}" for k, v in times.items()))
    if dirty:
        _save_cache(cache)
    return table


def _timed(sub, grad) -> float:
    sub._run(grad)
    return sub.last_timing()[0]


def apply(batch, table: dict) -> None:
    """Use the table's geometries for the batch's later runs."""
    from ._capi import check
    L = batch._store._L
    check(L.nwg_set_geometry(batch._store.h, 0, -1, 0, 0))
    soft = 1 if _soft(batch) else 0
    for sc, entry in table.items():
        if isinstance(entry, dict):
            _set_costs(batch, sc, entry["costs"])
        else:
            lanes, rows = entry
            check(L.nwg_set_geometry(batch._store.h, soft, int(sc), int(lanes), int(rows)))


def plain(batch) -> None:
    """The plain fill: one fixed geometry for every pair."""
    from ._capi import check
    check(batch._store._L.nwg_set_geometry(batch._store.h, 0, -2, 0, 0))
