"""Small, seeded workloads that exercise one kernel each, for profiling with
ncu (one kernel per command, `-k regex:<kernel>`) and for quick timings.

    python -m td16_b200.profile_cases <case> [--count N] [--table-bits B]

Every case runs with the benchmark's launch shape (td16_b200/tuned.json).

  steal    td_steal_kernel: the S_16 benchmark instances (seed 2, half
           near-reverse), bound 9, free order (default 2^18 instances)
  ordered  td_persistent_kernel<true>: 4096 x S_10 (seed 0), bound 6, the
           reference's single-queue order (with its split below the root)
  split    td_split_kernel: 4096 x S_13 (seed 5, half near-reverse), bound
           6, the reference's order; most walks outlast the one-warp first
           pass and are split below the root
  plain    td_plain_kernel<false>: the plain one-launch-per-batch form on the
           first 8192 S_16 benchmark instances
  replay   td_replay_symbols_kernel: the certificates of 2^18 S_16 searches,
           read back and replayed with the checker's rules
  validate td_validate_kernel: the pinned-form replay of 2^20 results
  serve    td_serve_kernel<0>: an open-loop Poisson stream of 20,000 requests
           at 100,000 requests/s, n uniform 8..16
  percall  td_serve_kernel<2>: the per-call server under 16 native slot
           threads on the first 4096 S_16 benchmark instances

Each case prints one JSON line with its device time (CUDA events) or rate.
"""
from __future__ import annotations

import argparse
import json
import os
import tempfile
import time

import numpy as np

from . import _lib
from .emitter_run import _pairs, replay_file


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _device_batch(inst, flags, slot=0):
    import torch
    d_in = torch.from_numpy(inst.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(len(inst) * 32, dtype=torch.uint8, device="cuda")
    stream = _lib.lib().td_slot_stream(slot)
    _lib.search_batch_device(slot, len(inst), d_in.data_ptr(), d_out.data_ptr(), flags, 0, stream)  # warm-up
    torch.cuda.synchronize()
    a, b = _events()
    ext = torch.cuda.ExternalStream(stream)
    a.record(ext)
    _lib.search_batch_device(slot, len(inst), d_in.data_ptr(), d_out.data_ptr(), flags, 0, stream)
    b.record(ext)
    torch.cuda.synchronize()
    res = d_out.cpu().numpy().view(_lib.RESULT_DTYPE)
    return a.elapsed_time(b), res, d_in, d_out


def run(case: str, count: int | None, table_bits: int | None = None) -> dict:
    _lib.init_slots(1, [0], 256 << 20)
    from .autotune import apply
    tuned = apply("17")  # the benchmark's launch shape (td16_b200/tuned.json)
    if table_bits is not None:
        _lib.configure_table(table_bits)
    try:
        if case in ("steal", "plain", "validate"):
            k = count or {"steal": 1 << 18, "plain": 8192, "validate": 1 << 20}[case]
            perms, n = _lib.synth_perms(2, k, 16, 16, 50, 1, 4)
            inst = _lib.prepare_perms(perms, n, 9)
            ms, res, d_in, d_out = _device_batch(inst, _lib.FLAG_PLAIN if case == "plain" else 0)
            out = {"case": case, "instances": k, "ms": ms, "found": int((res["status"] == 1).sum()),
                   "expansions": int(res["expansions"].astype(np.int64).sum()), "launch_shape": tuned,
                   "table_bits": 12 if table_bits is None else table_bits}
            if case == "validate":
                import torch
                ok = torch.zeros(k, dtype=torch.uint8, device="cuda")
                a, b = _events()
                a.record()
                _lib.validate_batch_device(k, d_in.data_ptr(), d_out.data_ptr(), ok.data_ptr(),
                                           torch.cuda.current_stream().cuda_stream)
                b.record()
                torch.cuda.synchronize()
                out.update(validate_ms=a.elapsed_time(b), accepted=int(ok.sum().item()))
            return out
        if case in ("ordered", "split"):
            if case == "ordered":
                perms, n = _lib.synth_perms(0, count or 4096, 10, 10, 0, 0, 0)
            else:
                perms, n = _lib.synth_perms(5, count or 4096, 13, 13, 50, 1, 3)
            inst = _lib.prepare_perms(perms, n, 6)
            ms, res, _, _ = _device_batch(inst, _lib.FLAG_ORDERED)
            return {"case": case, "instances": len(inst), "ms": ms, "found": int((res["status"] == 1).sum()),
                    "expansions": int(res["expansions"].astype(np.int64).sum())}
        if case == "replay":
            k = count or (1 << 18)
            perms, n = _lib.synth_perms(2, k, 16, 16, 50, 1, 4)
            inst = _lib.prepare_perms(perms, n, 9)
            res, _ = _lib.search_batch(0, inst, _lib.FLAG_VERIFY)
            beta, omega = _pairs(perms, n)
            path = os.path.join(tempfile.mkdtemp(), "certs.bin")
            w = _lib.CertificateWriter(path, 5.0)
            symbols = (n + 1).astype(np.uint8)
            _lib.lib().td_cert_writer_enqueue_batch(w._h, k, _lib._ptr(beta), _lib._ptr(omega), _lib._ptr(symbols),
                                                    _lib._ptr(res))
            w.close()
            return {"case": case, **replay_file(path, 17)}
        if case == "serve":
            perms, n = _lib.synth_perms(3, count or 20000, 8, 16, 0, 0, 0)
            inst = _lib.prepare_perms(perms, n, (n // 2 + 1).astype(np.int32))
            _, st = _lib.serve_open_loop(0, inst, 100000.0, seed=3)
            return {"case": case, **{k: st[k] for k in ("p50_ms", "p99_ms", "served_per_s", "served")}}
        if case == "percall":
            k = count or 4096
            perms, n = _lib.synth_perms(2, k, 16, 16, 50, 1, 4)
            beta, omega = _pairs(perms, n)
            init = (_lib.prepare_perms(perms, n, 9)["packed"] & 31).astype(np.int32)
            _lib.init_slots(16, [0], 256 << 20)
            fn = _lib.entry_address("td_search")
            r = _lib.slot_threads_run(fn, beta, omega, (n + 1).astype(np.int32), init, 0.0, 9, 1, 16)
            return {"case": case, "searches": k, "per_s": k / r["seconds"], "found": int((r["status"] == 1).sum())}
        raise ValueError(f"unknown case {case}")
    finally:
        _lib.destroy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["steal", "ordered", "split", "plain", "replay", "validate", "serve",
                                         "percall"])
    ap.add_argument("--count", type=int, default=None)
    ap.add_argument("--table-bits", type=int, default=None,
                    help="entries of the explored-state tables (2^bits per warp; 0 = none; default 12)")
    a = ap.parse_args()
    t0 = time.perf_counter()
    out = run(a.case, a.count, a.table_bits)
    out["wall_s"] = time.perf_counter() - t0
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
