"""Same-box speed comparison with the reference kernel (test infrastructure).

Runs the first K instances of the benchmark workload (S_16, seed 2, half
uniform and half near-reverse, bound 9) through
  - the reference's sorting_search.cu + slot_manager.cu compiled unchanged for
    sm_100a (oracle/_ref/libtd16ref.so, built by oracle/build_ref.sh), driven
    the way the emitter drives it: one blocking search per call, one host
    thread per slot, 16 and 7 slots;
  - this engine the same way (td_search, 16 slots);
  - this engine batched (td_search_batch, one launch).
Each per-call arm runs twice: from Python threads (which serialise on the
interpreter lock between calls) and from native threads
(tests/percall_threads.cc, built here with g++), the way Java threads call
the JNI entry.  Prints one JSON line with searches/s for each and checks that
the verdicts agree.  Needs a B200.

    python tests/ref_kernel_speed.py [K] [time limit per arm, s]
"""
from __future__ import annotations

import json
import os
import sys
import threading
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import numpy as np  # noqa: E402

import td16_b200 as td  # noqa: E402
from oracle import oracle as O  # noqa: E402
from make_ref_fixtures import RefKernel  # noqa: E402


def run_threads(k, nthreads, fn, limit):
    idx = [0]
    lock = threading.Lock()
    out = [None] * k
    t0 = time.perf_counter()

    def worker(slot):
        while True:
            with lock:
                i = idx[0]
                idx[0] += 1
            if i >= k or time.perf_counter() - t0 > limit:
                return
            out[i] = fn(slot, i)

    threads = [threading.Thread(target=worker, args=(s,)) for s in range(nthreads)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    return time.perf_counter() - t0, out


def native_threads():
    """Loads tests/percall_threads.cc, compiled on first use."""
    import ctypes as C
    import subprocess
    src = os.path.join(ROOT, "tests", "percall_threads.cc")
    lib = os.path.join(ROOT, "tests", "libpercall_threads.so")
    if not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", lib, src], check=True)
    h = C.CDLL(lib)
    h.percall_run.restype = C.c_double
    h.percall_run.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.c_int, C.c_int, C.c_void_p]
    return h


NAMES = {1: "found", 0: "not_found", -1: "error"}


def run_native(h, kind, fn, arrays, nthreads):
    beta, omega, n, init = arrays
    status = np.zeros(len(n), np.int32)
    dt = h.percall_run(kind, fn, len(n), beta.ctypes.data, omega.ctypes.data, n.ctypes.data, init.ctypes.data, 9,
                       nthreads, status.ctypes.data)
    return dt, [NAMES[int(v)] for v in status]


def main(k=2048, limit=240.0):
    import ctypes as C
    perms, n = td.synth_perms(2, k, 16, 16, 50, 1, 4)
    pairs = [O.perm_to_pair(perms[i, :16].tolist()) for i in range(k)]
    arrays = (np.zeros((k, 17), np.uint8), np.zeros((k, 17), np.uint8), np.full(k, 17, np.int32),
              np.zeros(k, np.int32))
    for i, (b, o, e) in enumerate(pairs):
        arrays[0][i], arrays[1][i], arrays[3][i] = b, o, e
    nat = native_threads()
    res = {"workload": f"first {k} instances of the S_16 benchmark workload, bound 9"}
    verdicts = {}
    for slots in (16, 7):
        ref = RefKernel(slots=slots, budget=1 << 30)
        dt, out = run_threads(k, slots, lambda s, i: ref.search(*pairs[i], 0.0, 9, 1, slot=s)[0], limit)
        done = [o for o in out if o is not None]
        res[f"reference_{slots}_slots"] = {"searches": len(done), "seconds": dt, "per_s": len(done) / dt,
                                           "errors": sum(o == "error" for o in done)}
        verdicts[f"reference_{slots}"] = out
        dt, out = run_native(nat, 1, C.cast(ref.lib.ref_search, C.c_void_p).value, arrays, slots)
        ref.close()
        res[f"reference_{slots}_slots_native_threads"] = {"searches": k, "seconds": dt, "per_s": k / dt,
                                                          "errors": sum(o == "error" for o in out)}
        verdicts[f"reference_{slots}_native"] = out
    td.init_slots(16, [0], 1 << 30)
    try:
        def ours(s, i):
            b, o, e = pairs[i]
            return "found" if td.search(s, bytes(b), bytes(o), e, 0.0, 9) else "not_found"

        # warm-up: a slot allocates its tables and item space on its first search
        run_threads(min(k, 256), 16, ours, limit)
        dt, out = run_threads(k, 16, ours, limit)
        done = [o for o in out if o is not None]
        res["engine_16_slots_per_call"] = {"searches": len(done), "seconds": dt, "per_s": len(done) / dt}
        verdicts["engine_per_call"] = out
        fn = C.cast(td._lib.lib().td_search, C.c_void_p).value
        for slots in (16, 7):
            td.init_slots(slots, [0], 1 << 30)
            run_native(nat, 0, fn, tuple(a[:256] for a in arrays), slots)  # warm-up (slot tables, items)
            dt, out = run_native(nat, 0, fn, arrays, slots)
            res[f"engine_{slots}_slots_native_threads"] = {"searches": k, "seconds": dt, "per_s": k / dt,
                                                           "errors": sum(o == "error" for o in out)}
            verdicts[f"engine_{slots}_native"] = out
        inst = td.prepare_perms(perms, n, 9)
        td.search_batch(0, inst, 0)
        r, st = td.search_batch(0, inst, 0)
        res["engine_batched"] = {"searches": k, "kernel_ms": st.kernel_ms, "per_s": k / (st.kernel_ms / 1e3)}
        verdicts["engine_batched"] = ["found" if s == 1 else "not_found" for s in r["status"]]
    finally:
        td.destroy()
    ref16 = verdicts["reference_16"]
    res["verdicts_agree"] = all(
        a is None or b is None or a == b for name, v in verdicts.items() for a, b in zip(ref16, v))
    print(json.dumps(res), flush=True)
    return 0 if res["verdicts_agree"] else 1


if __name__ == "__main__":
    sys.exit(main(int(sys.argv[1]) if len(sys.argv) > 1 else 2048,
                  float(sys.argv[2]) if len(sys.argv) > 2 else 240.0))
