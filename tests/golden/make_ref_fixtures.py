"""Generates tests/golden/ref_gpu_fixtures.json from the reference kernel itself.

Runs on a GPU machine with oracle/_ref/libtd16ref.so built by
oracle/build_ref.sh (the reference's unmodified sorting_search.cu and
slot_manager.cu).  Two kinds of cases:

  ordered   performGpuSortingSearch with maxWarps = 1 (one work queue): the
            reference's deterministic witness for each instance
  verdicts  the production launch shape (one queue per resident block): the
            verdict, plus the (order-dependent) witness it returned

Inputs are seeded synthetic instances (td16_b200.synth_perms) converted to
reference pairs, some with the caller's array rotated.

    python tests/golden/make_ref_fixtures.py [out.json]
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
import td16_b200 as td  # noqa: E402

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
    perms, n = td.synth_perms(seed, count, n_min, n_max, hard, hmin, hmax)
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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                           "ref_gpu_fixtures.json"))
