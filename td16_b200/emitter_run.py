"""Emitter-shaped end-to-end run.

Synthetic S_16 near-reverse cases (the reverse permutation composed with 1-4
random block transpositions) stream through the slot model the way the
emitter's case families reach GPUSortingSearch: `slots` worker threads, each
owning one slot (stream + `budget` bytes of device scratch), take batches of
cases, search them with the free-order engine plus device replay of every
witness, and hand the witnesses to the certificate sink in the reference's
byte format (CertificateCodec).  Afterwards every stored record is read back
and replayed on the GPU with the checker's rules.

Four shapes of the host side (--mode):
  batch     a slot thread searches a batch of cases per call (td_search_batch)
  percall   the reference's shape: one blocking td_search per case from
            `slots` native threads, one per slot (GPUSortingSearch.java:134-162)
  consumer  the enumerator's shape: generator threads hand cases one at a
            time to a thread-safe consumer (DirectTwistedBraceletGenerator.
            generateRepresentativesConcurrently), here host.PairBatcher, which
            searches them in batches with td_search_pairs
  native    the same shape in native code: producer threads hand cases one at
            a time to the native pair consumer (td_batcher_*), whose slot
            workers search batches and write the certificates themselves

    python -m td16_b200.emitter_run [--mode batch] [--count N] [--slots 16]
                                    [--budget-gib 4] [--batch 65536] [--out certs.bin]
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


def _chunk(seed: int, k: int, c: int):
    """Chunk k of the case stream: case j uses splitmix64 seeded with
    (seed ^ k << 32) ^ j (near-reverse S_16)."""
    perms, n = _lib.synth_perms(seed ^ (k << 32), c, 16, 16, 100, 1, 4)
    return perms, n


def _records(status, depth, moves):
    """td_result records of per-call outcomes (status 1 found, else not)."""
    res = np.zeros(len(status), _lib.RESULT_DTYPE)
    res["status"] = np.where(status == 1, 1, 0)
    res["depth"] = depth
    m = moves.astype(np.uint16)
    res["moves"] = m[:, :, 0] | (m[:, :, 1] << 5) | (m[:, :, 2] << 10)
    return res


def run_percall(count: int, slots: int, budget: int, out_path: str, seed: int = 4, device: int = 0,
                chunk: int = 1 << 18) -> dict:
    """One blocking td_search per case from `slots` native threads."""
    _lib.init_slots(slots, [device], budget)
    if os.path.exists(out_path):
        os.remove(out_path)
    writer = _lib.CertificateWriter(out_path, 5.0)
    fn = _lib.entry_address("td_search")
    found = not_found = errors = queued = 0
    search_s = 0.0
    t0 = time.perf_counter()
    try:
        for k in range((count + chunk - 1) // chunk):
            c = min(chunk, count - k * chunk)
            perms, n = _chunk(seed, k, c)
            beta, omega = _pairs(perms, n)
            init = (_lib.prepare_perms(perms, n, 9)["packed"] & 31).astype(np.int32)
            r = _lib.slot_threads_run(fn, beta, omega, (n + 1).astype(np.int32), init, 0.0, 9, 1, slots)
            search_s += r["seconds"]
            found += int((r["status"] == 1).sum())
            not_found += int((r["status"] == 0).sum())
            errors += int((r["status"] < 0).sum())
            res = _records(r["status"], r["depth"], r["moves"])
            symbols = (n + 1).astype(np.uint8)
            q = _lib.lib().td_cert_writer_enqueue_batch(writer._h, c, _lib._ptr(beta), _lib._ptr(omega),
                                                        _lib._ptr(symbols), _lib._ptr(res))
            if q < 0:
                raise _lib.TdError(_lib.CUDA_ERROR, "certificate sink rejected a batch")
            queued += int(q)
    finally:
        written = writer.close()
        wall = time.perf_counter() - t0
        _lib.destroy()
    rep = replay_file(out_path, 17)
    return {"mode": "percall", "cases": count, "slots": slots, "found": found, "not_found": not_found,
            "errors": errors, "certificates": written, "wall_s": wall, "search_s": search_s,
            "searches_per_s": count / search_s, "witnesses_per_s": written / wall, "replay": rep}


def run_consumer(count: int, slots: int, budget: int, out_path: str, seed: int = 4, device: int = 0,
                 generators: int = 8, batch: int = 8192) -> dict:
    """Generator threads hand cases one at a time to host.PairBatcher."""
    from .host import PairBatcher
    _lib.init_slots(slots, [device], budget)
    if os.path.exists(out_path):
        os.remove(out_path)
    writer = _lib.CertificateWriter(out_path, 5.0)
    perms, n = _chunk(seed, 0, count)
    beta, omega = _pairs(perms, n)
    init = (_lib.prepare_perms(perms, n, 9)["packed"] & 31).astype(np.int32)
    def batch_sink(b, o, nsym, status, depth, moves):
        # found witnesses of a searched batch go to the certificate writer in one call
        res = _records(np.where(status == _lib.OK, 1, 0), depth, moves)
        q = _lib.lib().td_cert_writer_enqueue_batch(writer._h, len(status), _lib._ptr(b), _lib._ptr(o),
                                                    _lib._ptr(nsym), _lib._ptr(res))
        if q < 0:
            raise _lib.TdError(_lib.CUDA_ERROR, "certificate sink rejected a batch")

    t0 = time.perf_counter()
    batcher = PairBatcher(range(slots), batch_size=batch, max_delay_s=0.005, batch_sink=batch_sink)
    futures = [None] * count

    def generate(g):
        for i in range(g, count, generators):
            futures[i] = batcher.accept(beta[i, :17].tobytes(), omega[i, :17].tobytes(), int(init[i]), 0.0, 9)

    threads = [threading.Thread(target=generate, args=(g,)) for g in range(generators)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    batcher.close()
    results = [f.result() for f in futures]
    written = writer.close()
    wall = time.perf_counter() - t0
    _lib.destroy()
    rep = replay_file(out_path, 17)
    return {"mode": "consumer", "cases": count, "slots": slots, "generators": generators, "batch": batch,
            "batches": batcher.batches, "found": sum(bool(r) for r in results),
            "not_found": sum(not r for r in results), "certificates": written, "wall_s": wall,
            "witnesses_per_s": written / wall, "replay": rep}


def run_native_consumer(count: int, slots: int, budget: int, out_path: str, seed: int = 4, device: int = 0,
                        producers: int = 16, batch: int = 65536) -> dict:
    """Native producer threads hand cases one at a time to the native pair
    consumer (td_batcher_accept); its slot workers search batches and pass
    the witnesses straight to the certificate writer."""
    _lib.init_slots(slots, [device], budget)
    if os.path.exists(out_path):
        os.remove(out_path)
    perms, n = _chunk(seed, 0, count)
    beta, omega = _pairs(perms, n)
    init = (_lib.prepare_perms(perms, n, 9)["packed"] & 31).astype(np.int32)
    writer = _lib.CertificateWriter(out_path, 5.0)
    t0 = time.perf_counter()
    cons = _lib.PairConsumer(0, slots, batch_size=batch, max_delay_s=0.005, cert_writer=writer)
    try:
        produce_s = _lib.producer_threads_run(cons, producers, beta, omega, 17, init, 0.0, 9)
    finally:
        stats = cons.close()
    written = writer.close()
    wall = time.perf_counter() - t0
    _lib.destroy()
    rep = replay_file(out_path, 17)
    return {"mode": "native", "cases": count, "slots": slots, "producers": producers, "batch": batch,
            "batches": stats["batches"], "found": stats["found"], "not_found": stats["not_found"],
            "errors": stats["errors"], "certificates": written, "wall_s": wall, "produce_s": produce_s,
            "search_s_summed": stats["search_s"], "witnesses_per_s": written / wall, "replay": rep}


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
                perms, n = _chunk(seed, k, c)
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
        "mode": "batch", "cases": count, "slots": slots, "budget_bytes": budget, "batch": batch,
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
    ap.add_argument("--mode", default="batch", choices=["batch", "percall", "consumer", "native"])
    a = ap.parse_args()
    budget = int(a.budget_gib * (1 << 30))
    if a.mode == "percall":
        out = run_percall(a.count, a.slots, budget, a.out, a.seed)
    elif a.mode == "consumer":
        out = run_consumer(a.count, a.slots, budget, a.out, a.seed)
    elif a.mode == "native":
        out = run_native_consumer(a.count, a.slots, budget, a.out, a.seed, batch=a.batch)
    else:
        out = run(a.count, a.slots, budget, a.batch, a.out, a.seed)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
