"""Emitter-shaped end-to-end run.

Synthetic S_16 near-reverse cases (the reverse permutation composed with 1-4
random block transpositions) stream through the slot model the way the
emitter's case families reach GPUSortingSearch: `slots` worker threads, each
owning one slot (stream + `budget` bytes of device scratch), take batches of
cases, search them with the free-order engine plus device replay of every
witness, and hand the witnesses to the certificate sink in the reference's
byte format (CertificateCodec).  Afterwards every stored record is read back
and replayed on the GPU with the checker's rules.

Batching is the one change to the reference's shape: a slot thread searches a
batch of cases per call instead of one case per blocking call.

    python -m td16_b200.emitter_run [--count N] [--slots 16] [--budget-gib 4]
                                    [--batch 65536] [--out certs.bin]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import threading
import time

import numpy as np

from . import _lib


def _pairs(perms, n):
    count = len(n)
    beta = np.zeros((count, 17), np.uint8)
    omega = np.zeros((count, 17), np.uint8)
    _lib.lib().td_pairs_from_perms(count, _lib._ptr(perms), _lib._ptr(n), _lib._ptr(beta), _lib._ptr(omega))
    return beta, omega


def replay_file(path: str, n_symbols: int, chunk: int = 1 << 20) -> dict:
    """Replays every certificate of `path` on the GPU (canonical beta)."""
    import torch
    total, accepted = 0, 0
    t0 = time.perf_counter()
    # a record holds 2 length bytes, the key and a value of at least 2 bytes
    cap = max(1, os.path.getsize(path) // (2 + (5 * n_symbols + 7) // 8 + 2))
    omega = np.zeros((cap, 17), np.uint8)
    abc = np.zeros((cap, 27), np.uint8)
    depth = np.zeros(cap, np.uint8)
    k = _lib.lib().td_cert_read_file(path.encode(), n_symbols, cap, _lib._ptr(omega), _lib._ptr(abc),
                                     _lib._ptr(depth))
    if k < 0:
        raise _lib.TdError(_lib.INVALID_ARG, f"malformed certificate file {path}")
    beta = np.zeros((1, 17), np.uint8)
    beta[0, :n_symbols] = np.arange(n_symbols)
    for lo in range(0, k, chunk):
        hi = min(k, lo + chunk)
        c = hi - lo
        dev = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in
               (np.repeat(beta, c, axis=0), omega[lo:hi], np.full(c, n_symbols, np.uint8),
                np.full(c, 9, np.uint8), depth[lo:hi], abc[lo:hi])]
        ok = torch.zeros(c, dtype=torch.uint8, device="cuda")
        err = C.create_string_buffer(256)
        rc = _lib.lib().td_replay_symbols_device(c, *[C.c_void_p(t.data_ptr()) for t in dev],
                                                 C.c_void_p(ok.data_ptr()), None, err, 256)
        _lib.check(rc, err)
        torch.cuda.synchronize()
        accepted += int(ok.sum().item())
        total += c
    return {"records": total, "accepted": accepted, "replay_s": time.perf_counter() - t0}


def run(count: int, slots: int, budget: int, batch: int, out_path: str, seed: int = 4, device: int = 0) -> dict:
    _lib.init_slots(slots, [device], budget)
    if os.path.exists(out_path):
        os.remove(out_path)
    writer = _lib.CertificateWriter(out_path, 5.0)
    chunks = (count + batch - 1) // batch
    lock = threading.Lock()
    state = {"next": 0, "found": 0, "not_found": 0, "errors": 0, "queued": 0, "expansions": 0}
    failure = []

    def worker(slot: int):
        try:
            while True:
                with lock:
                    k = state["next"]
                    state["next"] += 1
                if k >= chunks:
                    return
                c = min(batch, count - k * batch)
                # chunk k, case j: splitmix64 seeded with (seed ^ k << 32) ^ j
                perms, n = _lib.synth_perms(seed ^ (k << 32), c, 16, 16, 100, 1, 4)
                inst = _lib.prepare_perms(perms, n, 9)
                beta, omega = _pairs(perms, n)
                res, st = _lib.search_batch(slot, inst, _lib.FLAG_VERIFY)
                symbols = (n + 1).astype(np.uint8)  # held: ctypes only keeps its address
                q = _lib.lib().td_cert_writer_enqueue_batch(writer._h, c, _lib._ptr(beta), _lib._ptr(omega),
                                                            _lib._ptr(symbols), _lib._ptr(res))
                if q < 0:
                    raise _lib.TdError(_lib.CUDA_ERROR, "certificate sink rejected a batch")
                with lock:
                    state["found"] += int(st.found)
                    state["not_found"] += int(st.not_found)
                    state["errors"] += int(st.errors)
                    state["queued"] += int(q)
                    state["expansions"] += int(st.expansions)
        except BaseException as e:  # noqa: BLE001 - reported after the join
            failure.append(e)

    t0 = time.perf_counter()
    threads = [threading.Thread(target=worker, args=(s,), daemon=True) for s in range(slots)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    written = writer.close()
    wall = time.perf_counter() - t0
    _lib.destroy()
    if failure:
        raise failure[0]
    rep = replay_file(out_path, 17)
    return {
        "cases": count, "slots": slots, "budget_bytes": budget, "batch": batch,
        "found": state["found"], "not_found": state["not_found"], "errors": state["errors"],
        "certificates": written, "wall_s": wall, "witnesses_per_s": written / wall,
        "expansions": state["expansions"], "replay": rep,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=10_000_000)
    ap.add_argument("--slots", type=int, default=16)
    ap.add_argument("--budget-gib", type=float, default=4.0)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--out", default="certs.bin")
    ap.add_argument("--seed", type=int, default=4)
    a = ap.parse_args()
    print(json.dumps(run(a.count, a.slots, int(a.budget_gib * (1 << 30)), a.batch, a.out, a.seed)))


if __name__ == "__main__":
    main()
