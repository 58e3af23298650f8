"""Generates tests/golden/ref_gpu_fixtures.json from the reference kernel itself.

Runs on a GPU machine with oracle/_ref/libtd16ref.so built by
oracle/build_ref.sh (the reference's unmodified sorting_search.cu and
slot_manager.cu).  Two kinds of cases:

  ordered   performGpuSortingSearch with maxWarps = 1 (one work queue): the
            reference's deterministic witness for each instance
  verdicts  the production launch shape (one queue per resident block): the
            verdict, plus the (order-dependent) witness it returned

Inputs are seeded synthetic instances (the oracle's restatement of the
benchmark generator) converted to reference pairs, some with the caller's
array rotated.

    python tests/golden/make_ref_fixtures.py [out.json]
        the first sets ("ordered", "verdicts")
    python tests/golden/make_ref_fixtures.py screen cases.json
        (CPU) draws the candidates of the later sets and keeps those whose
        search the oracle finishes within an expansion budget, so that every
        kept case is small enough for the tests
    python tests/golden/make_ref_fixtures.py run cases.json [fixtures.json]
        (GPU) runs the reference kernel on the screened cases and adds the
        sets to the fixture file:
          ordered_large      single queue, N = 12..14, bounds 1..6
          at_lower_bound     production shape at the cycle-graph lower bound
                             (N = 14, 15, 17), about a third without a witness
          caller_rates       production shape, minRate = 2 / (maxMoves /
                             (float) target) as UnorientedCycles.java:34,
                             RemainingSuccessorsSolver.java:41 and
                             Oriented9CycleExtensions.java:163-168 compute it,
                             maxMoves 8 and 9, targets 1..17 chosen near the
                             rate's boundary
          caller_rates_ordered  the same rates with a single queue, N = 6..11
          partial            production shape, fullSorting = false
          partial_ordered    single queue, fullSorting = false
"""
from __future__ import annotations

import ctypes as C
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtd16ref.so")


class RefKernel:
    def __init__(self, slots=2, budget=2 << 30):
        self.lib = C.CDLL(REF_LIB)
        self.lib.ref_init.argtypes = [C.c_int, C.c_int, C.c_ulonglong, C.c_char_p, C.c_size_t]
        self.lib.ref_search.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                        C.c_int, C.c_int, C.POINTER(C.c_int16), C.POINTER(C.c_int), C.c_char_p,
                                        C.c_size_t]
        err = C.create_string_buffer(512)
        if self.lib.ref_init(slots, 0, budget, err, 512) != 0:
            raise RuntimeError(err.value.decode())

    def search(self, beta, omega, init, rate, maxd, full, max_warps=-1, slot=0):
        b = (C.c_uint8 * 17)(*beta)
        o = (C.c_uint8 * 17)(*omega)
        out = (C.c_int16 * 27)()
        depth = C.c_int(0)
        err = C.create_string_buffer(512)
        rc = self.lib.ref_search(b, o, len(beta), int(init), float(rate), int(maxd), int(full), slot, max_warps,
                                 out, C.byref(depth), err, 512)
        if rc != 0:
            return "error", err.value.decode(), []
        moves = [[out[3 * d], out[3 * d + 1], out[3 * d + 2]] for d in range(depth.value)]
        return ("found" if moves else "not_found"), "", moves

    def close(self):
        self.lib.ref_destroy()


def _case_inputs(seed, count, n_min, n_max, hard, hmin, hmax, rotate_frac, rng):
    perms, n = O.synth_perms(seed, count, n_min, n_max, hard, hmin, hmax)
    out = []
    for p, k in zip(perms, n):
        beta, omega, init = O.perm_to_pair(p[:k].tolist())
        if rng.random() < rotate_frac:
            r = int(rng.integers(k + 1))
            beta = beta[r:] + beta[:r]
        out.append((beta, omega, init))
    return out


def main(path):
    rng = np.random.default_rng(2024)
    ref = RefKernel()
    ordered, verdicts = [], []
    t0 = time.time()
    # reference smoke input
    st, msg, mv = ref.search([0, 1, 2], [1, 2, 0], 1, 2.0, 1, True)
    ordered.append(dict(beta=[0, 1, 2], omega=[1, 2, 0], init=1, rate=2.0, maxd=1, full=1, status=st, moves=mv))
    # ordered (maxWarps = 1): S_4..S_10, rotated arrays, bounds 1..6, some partial sorting
    for (beta, omega, init) in _case_inputs(31, 700, 4, 10, 20, 1, 3, 0.5, rng):
        maxd = int(rng.integers(1, 7))
        full = int(rng.random() < 0.8)
        rate = float(rng.choice([0.0, 1.0, 1.5, 2.0]))
        init_pass = init if full else max(0, init - int(rng.integers(0, 2)))
        st, msg, mv = ref.search(beta, omega, init_pass, rate, maxd, full, max_warps=1)
        ordered.append(dict(beta=beta, omega=omega, init=init_pass, rate=rate, maxd=maxd, full=full,
                            status=st, moves=mv, error=msg))
    # production shape: batched-mix and S_16 samples
    for (beta, omega, init) in _case_inputs(1, 1200, 11, 13, 25, 1, 3, 0.0, rng):
        maxd = (len(beta) - 1) // 2 + 1
        st, msg, mv = ref.search(beta, omega, init, 0.0, maxd, 1)
        verdicts.append(dict(beta=beta, omega=omega, init=init, rate=0.0, maxd=maxd, full=1, status=st,
                             moves=mv, error=msg))
    for (beta, omega, init) in _case_inputs(2, 300, 16, 16, 50, 1, 4, 0.0, rng):
        st, msg, mv = ref.search(beta, omega, init, 0.0, 9, 1)
        verdicts.append(dict(beta=beta, omega=omega, init=init, rate=0.0, maxd=9, full=1, status=st,
                             moves=mv, error=msg))
    ref.close()
    doc = {
        "_source": "reference kernel sorting_search.cu + slot_manager.cu (unmodified), sm_100a, "
                   "driven by oracle/ref_driver.cu; generated by tests/golden/make_ref_fixtures.py",
        "seconds": round(time.time() - t0, 1),
        "ordered": ordered,
        "verdicts": verdicts,
    }
    with open(path, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    print(f"wrote {path}: {len(ordered)} ordered, {len(verdicts)} verdict cases in {doc['seconds']} s")


# ---- later sets: screened on the CPU, then run on the reference kernel ------

def caller_rate(max_moves: int, target: int) -> float:
    """minRate = 2 / (maxMoves / (float) target) in IEEE single precision."""
    return float(np.float32(2) / (np.float32(max_moves) / np.float32(target)))


CALLER_RATES = sorted({caller_rate(m, t) for m in (8, 9) for t in range(1, 18)})


def _boundary_target(rng, N, init, max_moves):
    """A target whose rate 2t/maxMoves equals gained/depth for some depth the
    search can reach (gained = N - init when fully sorted), else a random one."""
    g = N - init
    cands = [t for t in range(1, 18) for d in range(max(1, (g + 1) // 2), max_moves + 1)
             if 2 * t * d == g * max_moves]
    if cands and rng.random() < 0.8:
        return int(rng.choice(cands))
    return int(rng.integers(1, 18))


def _screen(cases, budget, threads):
    """Keeps the cases the oracle finishes within `budget` expansions."""
    c = len(cases)
    beta = np.zeros((c, 17), np.uint8)
    omega = np.zeros((c, 17), np.uint8)
    for i, k in enumerate(cases):
        beta[i, : len(k["beta"])] = k["beta"]
        omega[i, : len(k["omega"])] = k["omega"]
    get = lambda f, dt: np.array([k[f] for k in cases], dt)  # noqa: E731
    O.set_expansion_budget(budget)
    try:
        st, _, _, _ = O.search_batch(beta, omega, get("N", np.uint8), get("init", np.int32),
                                     get("rate", np.float32), get("maxd", np.int32), get("full", np.uint8), threads)
    finally:
        O.set_expansion_budget(0)
    return [k for k, v in zip(cases, st) if v != O.BUDGET]


def _draw(seed, count, n_min, n_max, hard, hmin, hmax, rotate, rng):
    out = []
    for beta, omega, init in _case_inputs(seed, count, n_min, n_max, hard, hmin, hmax, rotate, rng):
        out.append(dict(beta=beta, omega=omega, N=len(beta), init=init))
    return out


def screen(path, threads=os.cpu_count() or 8):
    rng = np.random.default_rng(4051)
    sets = {}
    # single queue, N = 12..14, small bounds, general rates and rotations
    cases = []
    for k in _draw(41, 900, 11, 13, 40, 1, 3, 0.5, rng):
        lb = (k["N"] - k["init"] + 1) // 2
        k["maxd"] = int(min(6, lb + rng.integers(0, 3))) if rng.random() < 0.7 else int(rng.integers(1, 7))
        k["full"] = int(rng.random() < 0.8)
        k["rate"] = float(rng.choice([0.0, 1.0, 1.5, 2.0] + CALLER_RATES))
        if not k["full"]:
            k["init"] = max(0, k["init"] - int(rng.integers(0, 2)))
        k["max_warps"] = 1
        cases.append(k)
    sets["ordered_large"] = _screen(cases, 20000, threads)[:320]
    # production shape at the lower bound: about a third have no witness
    cases = []
    for seed, n, hard, hmax, count in ((42, 13, 100, 3, 220), (43, 16, 100, 4, 220), (44, 16, 0, 0, 120),
                                       (45, 14, 50, 3, 160)):
        for k in _draw(seed, count, n, n, hard, 1, max(1, hmax), 0.3, rng):
            k["maxd"] = int(min(9, (k["N"] - k["init"] + 1) // 2))
            k.update(full=1, rate=0.0, max_warps=-1)
            cases.append(k)
    sets["at_lower_bound"] = _screen(cases, 200000, threads)
    # the rates the emitter's callers pass, near their boundary
    cases = []
    for k in _draw(46, 600, 8, 16, 50, 1, 4, 0.3, rng):
        mm = int(rng.choice([8, 9]))
        t = _boundary_target(rng, k["N"], k["init"], mm)
        k.update(maxd=mm, full=1, rate=caller_rate(mm, t), target=t, max_warps=-1)
        cases.append(k)
    sets["caller_rates"] = _screen(cases, 200000, threads)[:320]
    cases = []
    for k in _draw(47, 700, 5, 10, 40, 1, 3, 0.3, rng):
        mm = int(rng.choice([8, 9]))
        t = _boundary_target(rng, k["N"], k["init"], mm)
        k.update(maxd=mm, full=1, rate=caller_rate(mm, t), target=t, max_warps=1)
        cases.append(k)
    sets["caller_rates_ordered"] = _screen(cases, 20000, threads)[:240]
    # fullSorting = false
    for name, seed, nlo, nhi, warps, budget, bhi in (("partial", 48, 6, 13, -1, 200000, 7),
                                                     ("partial_ordered", 49, 5, 11, 1, 20000, 6)):
        cases = []
        for k in _draw(seed, 700, nlo, nhi, 40, 1, 3, 0.3, rng):
            k["maxd"] = int(rng.integers(2, bhi))
            k["full"] = 0
            k["rate"] = float(rng.choice([0.5, 1.0, 1.2, 1.5, 2.0] + CALLER_RATES[::3]))
            k["init"] = max(0, k["init"] - int(rng.integers(0, 2)))
            k["max_warps"] = warps
            cases.append(k)
        sets[name] = _screen(cases, budget, threads)[:300]
    with open(path, "w") as f:
        json.dump(sets, f, separators=(",", ":"))
    print(f"wrote {path}: " + ", ".join(f"{k} {len(v)}" for k, v in sets.items()))


def run(cases_path, out_path):
    sets = json.load(open(cases_path))
    doc = json.load(open(out_path)) if os.path.exists(out_path) else {"ordered": [], "verdicts": []}
    ref = RefKernel()
    t0 = time.time()
    for name, cases in sets.items():
        out = []
        for k in cases:
            st, msg, mv = ref.search(k["beta"], k["omega"], k["init"], k["rate"], k["maxd"], k["full"],
                                     max_warps=k["max_warps"])
            rec = {f: k[f] for f in ("beta", "omega", "init", "rate", "maxd", "full")}
            if "target" in k:
                rec["target"] = k["target"]
            rec.update(status=st, moves=mv, error=msg)
            out.append(rec)
        doc[name] = out
        print(f"{name}: {len(out)} cases, " + ", ".join(
            f"{s} {sum(r['status'] == s for r in out)}" for s in ("found", "not_found", "error")), flush=True)
    ref.close()
    doc["_sets"] = "ordered/verdicts: first run; the rest: screened candidates (make_ref_fixtures.py screen)"
    doc["seconds_later_sets"] = round(time.time() - t0, 1)
    with open(out_path, "w") as f:
        json.dump(doc, f, separators=(",", ":"))
    print(f"wrote {out_path} in {doc['seconds_later_sets']} s")


if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    default = os.path.join(here, "ref_gpu_fixtures.json")
    if len(sys.argv) > 1 and sys.argv[1] == "screen":
        screen(sys.argv[2])
    elif len(sys.argv) > 1 and sys.argv[1] == "run":
        run(sys.argv[2], sys.argv[3] if len(sys.argv) > 3 else default)
    else:
        main(sys.argv[1] if len(sys.argv) > 1 else default)
