"""Autotuner of the free-order engine's launch and work-distribution knobs.

For a bucket of instances (one symbol count N, or a mix) it times the batch
launch on a sample for every point of a grid over
  warps per block (block shape),
  steal granularity (items per donation),
  split depth (deepest DFS level whose children may be donated),
  check interval (expansions between idle checks),
and then, with the winning shape, the restart budget base of the root searches
(0 = no restarts); when restarts win, the grid is searched again with that
base and the base swept once more, since restarts shorten the searches that
the donation knobs were tuned for, and last the restart attempt from which a
search races the search of its inverse permutation (0 = no race; the race
needs restarts).  The fastest point by device time is kept,
and the winners per bucket are stored in td16_b200/tuned.json.  `apply(N)`
configures the engine for a bucket.

    python -m td16_b200.autotune [--quick]
"""
from __future__ import annotations

import itertools
import json
import os
import sys
import time

import numpy as np

from . import _lib

TUNED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")
DEFAULT = {"warps": 4, "grain": 4, "split_level": 2, "check_every": 64, "restart": 16,
           "race": 8}  # the library's defaults

GRID = {
    "warps": [4, 8],
    "grain": [1, 2, 4],
    "split_level": [2, 3, 4, 6],
    "check_every": [64, 128, 256, 512, 1024],
}
QUICK = {"warps": [2, 4], "grain": [4, 8], "split_level": [4], "check_every": [32, 128]}


RESTARTS = [0, 16, 24, 32, 48, 64, 128]
RACES = [0, 4, 8, 16]  # restart attempt from which a search races its inverse; 0 = no race


def _configure(p):
    _lib.configure(p["warps"], 1)
    _lib.configure_steal(p["grain"], p["split_level"], p["check_every"])
    _lib.configure_restart(p.get("restart", 0))
    _lib.configure_race(p.get("race", DEFAULT["race"]))


def time_point(slot: int, instances: np.ndarray, params: dict, repeats: int = 2) -> float:
    _configure(params)
    best = float("inf")
    for _ in range(repeats):
        _, st = _lib.search_batch(slot, instances, 0)
        if st.errors:
            return float("inf")
        best = min(best, st.kernel_ms)
    return best


def tune_bucket(slot: int, instances: np.ndarray, grid=None, repeats: int = 2, log=print) -> dict:
    grid = grid or GRID
    keys = list(grid)
    results = []

    def shapes(restart):
        out = []
        for combo in itertools.product(*(grid[k] for k in keys)):
            p = dict(zip(keys, combo), restart=restart)
            ms = time_point(slot, instances, p, repeats)
            out.append((ms, p))
            log(f"  {p} -> {ms:.2f} ms")
        results.extend(out)
        return min(out, key=lambda r: r[0])

    def bases(best_ms, best):
        for base in RESTARTS:
            p = dict(best, restart=base)
            ms = time_point(slot, instances, p, repeats)
            results.append((ms, p))
            log(f"  {p} -> {ms:.2f} ms")
            if ms < best_ms:
                best_ms, best = ms, p
        return best_ms, best

    def races(best_ms, best):
        for attempt in RACES:
            p = dict(best, race=attempt)
            ms = time_point(slot, instances, p, repeats)
            results.append((ms, p))
            log(f"  {p} -> {ms:.2f} ms")
            if ms < best_ms:
                best_ms, best = ms, p
        return best_ms, best

    best_ms, best = bases(*shapes(0))
    if best["restart"]:
        best_ms, best = min([(best_ms, best), shapes(best["restart"])], key=lambda r: r[0])
        best_ms, best = bases(best_ms, best)
        best_ms, best = races(best_ms, best)
    _configure(DEFAULT)
    return {"params": best, "kernel_ms": best_ms, "points": len(results)}


def buckets(quick: bool):
    """Sample workloads per bucket: the batched mix (n 11..13; 65,536 instances,
    the batch it is run as) and S_16 (2^18 instances, so that the launch tail
    weighs about as much as in a full-size batch)."""
    c = 4096 if quick else 16384
    mix = _lib.synth_perms(1, c if quick else 65536, 11, 13, 25, 1, 3)
    s16 = _lib.synth_perms(2, c if quick else 1 << 18, 16, 16, 50, 1, 4)
    return {
        "mix_11_13": _lib.prepare_perms(mix[0], mix[1], (mix[1] // 2 + 1).astype(np.int32)),
        "17": _lib.prepare_perms(s16[0], s16[1], 9),
    }


def load() -> dict:
    if os.path.exists(TUNED):
        with open(TUNED) as f:
            return json.load(f)
    return {}


def apply(bucket: str) -> dict:
    """Configures the engine with the tuned parameters of `bucket` (or the defaults)."""
    p = load().get("buckets", {}).get(bucket, {}).get("params", DEFAULT)
    _configure(p)
    return p


def main(argv):
    quick = "--quick" in argv
    _lib.init_slots(1, [0], 2 << 30)
    out = {"when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()), "grid": QUICK if quick else GRID,
           "buckets": {}}
    try:
        for name, inst in buckets(quick).items():
            print(f"bucket {name}: {len(inst)} instances", flush=True)
            out["buckets"][name] = tune_bucket(0, inst, QUICK if quick else GRID)
            print(f"  best {out['buckets'][name]}", flush=True)
    finally:
        _lib.destroy()
    path = argv[argv.index("--out") + 1] if "--out" in argv else TUNED
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(path)


if __name__ == "__main__":
    main(sys.argv[1:])
