"""Launch-shape autotuner for the chain kernel.

Candidates are (threads per Gray lane, CTA threads): the lane width and CTA of the CTA-per-stream form, and
for the warp-per-stream form the lane width and the streams per CTA (CTA threads / 32).  The batched
sampler also tunes its length-tier cut points through `tune` (candidates are indices into its list).  `tune` times each candidate on the caller's actual
workload (a callable running one launch with that shape), keeps the fastest, and caches the choice in a
JSON file keyed by the GPU name, the precision and a workload key, so later processes reuse it.  The cache
lives at $PE_TUNE_CACHE (default ~/.cache/photonic_engines_b200/tune.json).
"""
from __future__ import annotations

import json
import os

import torch

# the warp form: (threads per lane, CTA threads = 32 x streams per CTA)
WARP_CANDIDATES = [(1, 256), (2, 256), (1, 128), (2, 128), (1, 64)]
CANDIDATES = {8: [(1, 128), (1, 256), (2, 128), (2, 256)],
              16: [(1, 128), (2, 128), (2, 256), (4, 256)],
              20: [(1, 128), (2, 128), (2, 256), (4, 128), (4, 256)],
              24: [(2, 64), (2, 128), (4, 128), (4, 256)],
              28: [(2, 64), (2, 128), (4, 128), (4, 256)],
              32: [(2, 64), (2, 128), (4, 128), (4, 256)],
              40: [(2, 64), (2, 128), (4, 128)], 48: [(4, 64), (4, 128)], 56: [(4, 64), (4, 128)],
              64: [(4, 64), (4, 128)]}
# the compensated form is compiled for one-thread lanes at 8 columns, two-thread lanes to 20, four beyond
COMP_CANDIDATES = {8: [(1, 128), (2, 128)], 16: [(2, 128)], 20: [(2, 128)], 24: [(4, 128)], 28: [(4, 128)],
                   32: [(4, 128)]}


def _cache_path() -> str:
    return os.environ.get("PE_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "photonic_engines_b200",
                                                        "tune.json"))


def _load() -> dict:
    try:
        with open(_cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(cache: dict) -> None:
    path = _cache_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def tier(n: int) -> int:
    for k in sorted(CANDIDATES):
        if n <= k:
            return k
    raise ValueError(f"at most 64 photons (got {n})")


# bumped whenever the compiled launch shapes change, so that a cached choice the library no longer accepts
# is never replayed
SHAPES_VERSION = 4


def key(device, precision: str, workload: str) -> str:
    return f"v{SHAPES_VERSION}|{torch.cuda.get_device_name(device)}|{precision}|{workload}"


def lookup(device, precision: str, workload: str):
    hit = _load().get(key(device, precision, workload))
    return tuple(hit) if hit else None


def tune(run, device, precision: str, n_tier: int, workload: str, reps: int = 2, force: bool = False,
         candidates=None, keep_first_within: float = 0.0):
    """run(tpl, block) performs one launch on the current stream.  Returns the fastest (tpl, block); with
    keep_first_within = f the first candidate (the default) is kept unless another one is faster by more than
    the fraction f (timing noise must not move a choice)."""
    k = key(device, precision, workload)
    cache = _load()
    if not force and k in cache:
        return tuple(cache[k])
    best, best_ms = None, float("inf")
    if candidates is None:
        candidates = (COMP_CANDIDATES if precision == "compensated" else CANDIDATES)[n_tier]
    first_ms = None
    for tpl, block in candidates:
        run(tpl, block)                                         # warm-up (module load, attribute set-up)
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            run(tpl, block)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        ms = min(times)
        if first_ms is None:
            first_ms = ms
        if ms < best_ms:
            best, best_ms = (tpl, block), ms
    if keep_first_within > 0.0 and best_ms > first_ms * (1.0 - keep_first_within):
        best = tuple(candidates[0])
    cache = _load()
    cache[k] = list(best)
    _store(cache)
    return best
