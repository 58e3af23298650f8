"""Benchmark of the witness search: verified witnesses/s on S_16, bound 9.

Workload (the full-size decision search): 2^20 seeded permutations of S_16
(nibble-packed), half uniform (Fisher-Yates) and half the reverse permutation
composed with 1-4 random block transpositions; decide whether each sorts
within 9 moves in the reference's move space and emit a witness.  A step is
one pass of the engine over the whole batch followed by the device replay of
every witness; `value` counts replay-verified witnesses per second with the
instances already resident in HBM.  `e2e` is the same metric through the
public host-buffer call (td_search_batch with TD_FLAG_VERIFY): host-to-device
copy of the instances, search, replay and device-to-host copy of the results.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

With --impl reference the CPU restatement of the reference search (the
reference ships no CPU search of its own) is timed on all host cores on a
bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

COUNT = 1 << 20
SEED = 2
MAX_MOVES = 9
METRIC = "verified witnesses/s (S_16, d<=9)"
UNIT = "witnesses/s"
WORKLOAD = "full-size decision search: 2^20 S_16 perms, 50% uniform / 50% reverse o 1-4 transpositions, d<=9"
# Per node expansion at N = 17, the search kernel's warp instructions (all
# pipes) and those of the integer ALU pipe, and its DRAM bytes per launch: one-
# pass ncu captures of td_steal_kernel on one launch of this benchmark's 2^20-
# instance batch with the tuned launch shape and the race from attempt 8,
# summarised with their commands in profiles/td_steal_kernel_s16_2p20_counters.md.
# 36.870 G warp instructions and 19.901 G ALU-pipe instructions over the
# launch's 49.02 M expansions (restarts, races, skipped children, donation and
# scheduling included) in 85.21 M SM cycles: the ALU pipe busy 78.9 % of its 2
# warp instructions per cycle per SM, issue 73.1 % of 4; 0.963 GB read and
# 0.840 GB written.
PLAIN_WARPS = 4  # block shape of the plain one-launch-per-batch leg
INST_PER_EXPANSION = 36.870e9 / 49.02e6
ALU_INST_PER_EXPANSION = 19.901e9 / 49.02e6
ALU_BUSY_MEASURED = 19.901e9 / (85.21e6 * 148 * 2)
ISSUE_MEASURED = 36.870e9 / (85.21e6 * 148 * 4)
DRAM_BYTES_PER_LAUNCH = 0.963e9 + 0.840e9


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_instances(td, rank, count=COUNT, workload="mix"):
    from td16_b200.replicas import rank_seed
    if workload == "replicated":
        # one near-reverse S_16 instance (seed 2, index 0: 895 expansions in
        # free order) copied `count` times: every warp works for the whole
        # launch, so counters describe the search itself, not a tail
        perms, n = td.synth_perms(SEED, 1, 16, 16, 100, 1, 4)
        perms, n = np.repeat(perms, count, axis=0), np.repeat(n, count)
        return td.prepare_perms(perms, n, MAX_MOVES), perms, n
    perms, n = td.synth_perms(rank_seed(SEED, rank), count, 16, 16, 50, 1, 4)
    return td.prepare_perms(perms, n, MAX_MOVES), perms, n


def bench_config(world: int, count: int = COUNT) -> dict:
    """The workload definition both arms report (identical dicts)."""
    return {"workload": WORKLOAD, "count_per_gpu": count, "seed": SEED, "max_moves": MAX_MOVES,
            "l2": "GPU arm: inputs and scratch rewritten, L2 flushed between steps (256 MiB write)",
            "parallelism": f"replicas x{world}"}


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _oracle_pairs(O, first, count):
    """Instances [first, first + count) of the workload as reference pairs,
    generated by the oracle's restatement of the seeded generator (the engine
    library is not loaded)."""
    perms, _ = O.synth_perms(SEED, first + count, 16, 16, 50, 1, 4)
    beta = np.zeros((count, 17), np.uint8)
    omega = np.zeros((count, 17), np.uint8)
    init = np.zeros(count, np.int32)
    for i in range(count):
        b, o, e = O.perm_to_pair(perms[first + i, :16].tolist())
        beta[i], omega[i], init[i] = b, o, e
    return beta, omega, init


def cpu_reference_order(first=0, sample=96):
    """The oracle -- the CPU restatement of the reference search in its
    single-queue order -- on all host cores, on instances [first, first +
    sample) of the workload.  Every witness is replayed by the oracle's
    checker before it counts."""
    from oracle import oracle as O
    beta, omega, init = _oracle_pairs(O, first, sample)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    st, dep, mv, ex = O.search_batch(beta, omega, np.full(sample, 17), init, np.zeros(sample),
                                     np.full(sample, MAX_MOVES), np.ones(sample), cores)
    dt = time.perf_counter() - t0
    verified = 0
    for i in np.nonzero(st == 1)[0]:
        moves = [(int(m) & 31, (int(m) >> 5) & 31, (int(m) >> 10) & 31) for m in mv[i][: dep[i]]]
        abc = O.positions_to_symbols(beta[i].tolist(), moves)
        verified += O.validate(beta[i].tolist(), omega[i].tolist(), abc, MAX_MOVES) is None
    return {"value": verified / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"instances {first}..{first + sample - 1} of the workload (seed {SEED}), {dt:.1f} s on "
                      f"{cores} threads",
            "label": "CPU restatement of the reference algorithm, its single-queue order (the reference has "
                     "no CPU search)",
            "nproc": os.cpu_count(), "cpu_model": cpu_model(), "nodes_per_s": float(ex.sum()) / dt,
            "expansions_per_witness": float(ex.sum()) / max(1, int((st == 1).sum())), "seconds": dt}


def cpu_free_order(sample=16384):
    """The engine's own free-order algorithm (restarts and explored-state
    table; oracle/td_emu.cc, one lane at a time on the host) on all host
    cores: the CPU figure for the same algorithm as the GPU arm."""
    from oracle import oracle as O
    beta, omega, init = _oracle_pairs(O, 0, sample)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    res = O.emu_search_batch(beta, omega, 17, init, 0.0, MAX_MOVES, 1, 0, cores)
    dt = time.perf_counter() - t0
    found = int((res["status"] == 1).sum())
    exp = float(res["expansions"].astype(np.int64).sum())
    return {"searches_per_s": sample / dt, "witnesses_per_s": found / dt, "nodes_per_s": exp / dt,
            "expansions_per_witness": exp / max(1, found), "cores": cores,
            "sample": f"first {sample} instances of the workload, {dt:.1f} s on {cores} threads",
            "label": "the engine's free-order algorithm emulated lane by lane on the host (test "
                     "infrastructure, not tuned CPU code)"}


def cpu_baseline():
    base = cpu_reference_order()
    base["free_order"] = cpu_free_order()
    return base


def run_reference(args):
    """The reference arm: the CPU restatement of the reference search on the
    host cores, each step a bounded consecutive sample of the same workload.
    Loads the oracle only (no engine library)."""
    rank, world, _ = rank_info()
    if rank != 0:
        return
    per_step = 48
    for k in range(args.warmup):
        cpu_reference_order(first=per_step * k, sample=16)
    steps = [cpu_reference_order(first=per_step * k, sample=per_step) for k in range(args.steps)]
    secs = float(np.sum([s["seconds"] for s in steps]))
    verified = float(np.sum([s["value"] * s["seconds"] for s in steps]))
    value = verified / secs
    res = steps[-1]
    cpu = {"value": value, "unit": UNIT, "cores": res["cores"], "kind": "port",
           "sample": f"{args.steps} steps of {per_step} consecutive instances (instances 0.."
                     f"{per_step * args.steps - 1} of the 2^20-instance workload), {secs:.1f} s on "
                     f"{res['cores']} threads",
           "label": res["label"], "nproc": res["nproc"], "cpu_model": res["cpu_model"],
           "nodes_per_s": float(np.mean([s["nodes_per_s"] for s in steps]))}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8/u64 integer",
            "data": "synthetic (seeded)", "config": bench_config(args.gpus),
            "nodes_per_s": cpu["nodes_per_s"], "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serving_legs(td, device):
    """Serving (continuous batching), n uniform 8..16, bound floor(n/2)+1,
    open-loop Poisson arrivals:
      ring     the serving launch fed by one host producer through a mapped
               ring (td_serve_open_loop), one host thread polling all results;
      clients  the per-call server under one client thread per host core
               (at most 16), each polling only its own requests
               (td_percall_open_loop).
    Both are swept up to saturation, then run at 80% of the saturated rate.
    Admission: a request waits for a free client (or worker warp); the 64 GiB
    frame pool of the ring form never binds, since a request's DFS frames live
    in shared memory and its device state is 48 bytes."""
    from td16_b200 import _lib
    perms_s, n_s = td.synth_perms(3, 400000, 8, 16, 0, 0, 0)
    inst_s = td.prepare_perms(perms_s, n_s, (n_s // 2 + 1).astype(np.int32))
    keys = ("p50_ms", "p99_ms", "p999_ms", "served_per_s", "offered_per_s", "served", "admission_wait_ms_mean")
    out = {"workload": "open-loop Poisson, n uniform 8..16, bound floor(n/2)+1",
           "admission": "in-flight requests <= worker warps (ring) or client threads (clients); the 64 GiB frame "
                        "pool never binds (frames live in shared memory)"}
    def sweep(run, rates):
        res, capacity = {}, 0.0
        for rate in rates:
            k = int(min(len(inst_s), max(10000, rate * 0.5)))
            try:
                _, sst = run(inst_s[:k], rate)
            except _lib.TdError as e:
                res[f"{int(rate)}_per_s"] = {"error": str(e)}
                continue
            res[f"{int(rate)}_per_s"] = {key: sst[key] for key in keys}
            capacity = max(capacity, sst["served_per_s"])
        if capacity > 0:
            at80 = 0.8 * capacity
            _, sst = run(inst_s[: int(min(len(inst_s), max(10000, at80 * 0.5)))], at80)
            res["at_80pct_of_saturation"] = {key: sst[key] for key in keys}
        res["saturated_per_s"] = capacity
        return res

    rates = (5000.0, 50000.0, 200000.0, 1000000.0, 2000000.0, 4000000.0)
    out["ring"] = sweep(lambda x, r: _lib.serve_open_loop(device, x, r, seed=3), rates)
    clients = max(1, min(16, os.cpu_count() or 1))
    td.init_slots(1, [device], 64 << 20)
    try:
        out[f"clients_{clients}"] = sweep(lambda x, r: _lib.percall_open_loop(device, x, r, clients=clients, seed=5),
                                          rates[:5])
        # the library's default launch shape (the S_16 bucket's tuned shape,
        # set for the engine leg, is 2.5x slower on this easy mix); the first
        # call on fresh slots also sizes its buffers and tables: untimed; then
        # the median of three
        from td16_b200 import autotune
        out["batched_launch_shape"] = autotune.apply("defaults")
        td.search_batch(0, inst_s[:100000], 0)
        ms = sorted(td.search_batch(0, inst_s[:100000], 0)[1].kernel_ms for _ in range(3))
        out["batched_per_s"] = 100000 / (ms[1] / 1e3)
    finally:
        td.destroy()
    return out


REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libtd16ref.so")


def per_call_legs(td, k=8192, slots=16, budget=1 << 30):
    """One blocking search per call from `slots` native threads, one per slot,
    as the emitter's Java slot workers call searchForSortingSeq: this engine's
    td_search, and the reference kernel itself (sorting_search.cu and
    slot_manager.cu compiled unmodified for sm_100a into oracle/_ref, when that
    build exists) on the same first k instances of the workload."""
    from td16_b200 import _lib
    perms, n = td.synth_perms(SEED, k, 16, 16, 50, 1, 4)
    beta = np.zeros((k, 17), np.uint8)
    omega = np.zeros((k, 17), np.uint8)
    init = np.zeros(k, np.int32)
    pairs_b = np.zeros(17, np.uint8)
    pairs_o = np.zeros(17, np.uint8)
    td_lib = _lib.lib()
    for i in range(k):
        td_lib.td_pairs_from_perms(1, perms[i:].ctypes.data, n[i:].ctypes.data, pairs_b.ctypes.data,
                                   pairs_o.ctypes.data)
        beta[i], omega[i] = pairs_b, pairs_o
    inst = td.prepare_perms(perms, n, MAX_MOVES)
    init[:] = inst["packed"] & 31
    out = {"workload": f"first {k} instances of the benchmark workload, bound {MAX_MOVES}, one blocking "
                       f"search per call from {slots} native threads (one per slot)"}
    td.init_slots(slots, [0], budget)
    try:
        fn = _lib.entry_address("td_search")
        _lib.slot_threads_run(fn, beta[:512], omega[:512], 17, init[:512], 0.0, MAX_MOVES, 1, slots)  # warm-up
        r = _lib.slot_threads_run(fn, beta, omega, 17, init, 0.0, MAX_MOVES, 1, slots)
        lat = np.sort(r["latency_s"]) * 1e3
        out["engine_td_search"] = {"per_s": k / r["seconds"], "seconds": r["seconds"],
                                   "found": int((r["status"] == 1).sum()), "errors": int((r["status"] < 0).sum()),
                                   "p50_ms": float(lat[k // 2]), "p99_ms": float(lat[int(0.99 * (k - 1))])}
        engine_status = r["status"]
    finally:
        td.destroy()
    if not os.path.exists(REF_LIB):
        out["reference_kernel"] = {"unavailable": "oracle/_ref/libtd16ref.so was not built (needs the reference "
                                                  "checkout at build time)"}
        return out
    import ctypes as C
    ref = C.CDLL(REF_LIB)
    ref.ref_init.argtypes = [C.c_int, C.c_int, C.c_ulonglong, C.c_char_p, C.c_size_t]
    err = C.create_string_buffer(512)
    if ref.ref_init(slots, 0, budget, err, 512) != 0:
        out["reference_kernel"] = {"unavailable": err.value.decode()}
        return out
    try:
        fn = C.cast(ref.ref_search, C.c_void_p).value
        _lib.slot_threads_run(fn, beta[:512], omega[:512], 17, init[:512], 0.0, MAX_MOVES, 1, slots, kind=1)
        r = _lib.slot_threads_run(fn, beta, omega, 17, init, 0.0, MAX_MOVES, 1, slots, kind=1)
    finally:
        ref.ref_destroy()
    lat = np.sort(r["latency_s"]) * 1e3
    out["reference_kernel"] = {"per_s": k / r["seconds"], "seconds": r["seconds"],
                               "found": int((r["status"] == 1).sum()), "errors": int((r["status"] < 0).sum()),
                               "p50_ms": float(lat[k // 2]), "p99_ms": float(lat[int(0.99 * (k - 1))]),
                               "source": "sorting_search.cu + slot_manager.cu, unmodified, sm_100a"}
    both = (engine_status >= 0) & (r["status"] >= 0)
    out["verdicts_agree"] = bool((engine_status[both] == r["status"][both]).all())
    out["engine_over_reference"] = out["engine_td_search"]["per_s"] / out["reference_kernel"]["per_s"]
    return out


def run_engine(args):
    import torch
    import td16_b200 as td
    from td16_b200 import _lib

    rank, world, local = rank_info()
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    td.init_slots(1, [local], 256 << 20)
    stream_ptr = _lib.lib().td_slot_stream(0)
    stream = torch.cuda.ExternalStream(stream_ptr, device=dev)

    inst, perms, n = make_instances(td, rank, args.count, args.workload)
    count = len(inst)
    d_in = torch.from_numpy(inst.view(np.uint8).copy()).to(dev)
    d_out = torch.zeros(count * 32, dtype=torch.uint8, device=dev)
    d_ok = torch.zeros(count, dtype=torch.uint8, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # larger than the 126 MB L2

    from td16_b200 import autotune
    # the S_16 bucket's launch shape, restart base and race attempt (a bucket
    # without a race attempt keeps the library's, 8)
    tuned = autotune.apply("17")
    tuned = {**tuned, "race": tuned.get("race", autotune.DEFAULT["race"])}

    def step(flags):
        _lib.search_batch_device(0, count, d_in.data_ptr(), d_out.data_ptr(), flags, 0, stream_ptr)
        _lib.validate_batch_device(count, d_in.data_ptr(), d_out.data_ptr(), d_ok.data_ptr(), stream_ptr)

    # one CUDA graph per step: launch epoch, donation engine, device replay
    graph = _lib.BatchGraph(0, count, d_in.data_ptr(), d_out.data_ptr(), _lib.FLAG_VERIFY)
    for _ in range(args.warmup):
        with torch.cuda.stream(stream):
            flush.zero_()
        graph.launch(stream_ptr)
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    verified, expansions, found, not_found, errors = 0, 0, 0, 0, 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            ev[k][0].record(stream)
            graph.launch(stream_ptr)
            ev[k][1].record(stream)
            torch.cuda.synchronize()
            res = d_out.cpu().numpy().view(_lib.RESULT_DTYPE)
            # a witness that fails the device replay is marked -6, never counted
            verified += int((res["status"] == 1).sum())
            expansions += int(res["expansions"].astype(np.int64).sum())
            found += int((res["status"] == 1).sum())
            not_found += int((res["status"] == 0).sum())
            errors += int((res["status"] < 0).sum())
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_s = sum(step_ms) / 1e3
    if dist:
        from td16_b200 import replicas
        total_s = replicas.max_over_ranks(total_s, dist, dev)
        verified, expansions, found, not_found, errors = [
            int(v) for v in replicas.sum_over_ranks([verified, expansions, found, not_found, errors], dist, dev)]
    value = verified / total_s

    only_engine = args.legs == "engine"
    # end to end through the public host-buffer API: inputs in pinned host
    # memory when the timed region starts; the call copies them in, searches,
    # replays every witness and copies the results back into pinned memory
    host_in = torch.empty(count * inst.dtype.itemsize, dtype=torch.uint8, pin_memory=True).numpy().view(inst.dtype)
    host_in[:] = inst
    host_out = torch.empty(count * _lib.RESULT_DTYPE.itemsize, dtype=torch.uint8,
                           pin_memory=True).numpy().view(_lib.RESULT_DTYPE)
    e2e_s, e2e_verified = 0.0, 0
    if not only_engine:
        td.search_batch(0, host_in, _lib.FLAG_VERIFY, out=host_out)  # untimed: sizes the slot's batch buffer
    e2e_ms = []
    if dist:
        dist.barrier()
    for k in range(0 if only_engine else args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res_h, st = td.search_batch(0, host_in, _lib.FLAG_VERIFY, out=host_out)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
        e2e_verified += int((res_h["status"] == 1).sum())
    e2e_s = sum(e2e_ms) / 1e3
    e2e_steps = max(1, len(e2e_ms))
    if dist:
        # whole job, like `value`: witnesses of every rank over the slowest rank's time
        from td16_b200 import replicas
        e2e_s = replicas.max_over_ranks(e2e_s, dist, dev)
        e2e_verified = int(replicas.sum_over_ranks([e2e_verified], dist, dev)[0])

    # the plain one-launch-per-batch form on the same GPU
    plain_ms, plain_verified = float("nan"), 0
    if not only_engine:
        # in its own faster block shape: 4 warps per block (the library's
        # default; 41.5 k/s against 34.8 k/s with the batch engine's 8-warp
        # blocks)
        _lib.configure(PLAIN_WARPS, 1)
        pe = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        with torch.cuda.stream(stream):
            flush.zero_()
        pe[0].record(stream)
        step(_lib.FLAG_PLAIN)
        pe[1].record(stream)
        torch.cuda.synchronize()
        plain_ms = pe[0].elapsed_time(pe[1])
        plain_verified = int(d_ok.sum().item())
        _lib.configure(tuned["warps"], 1)

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    # roofline: instruction issue of the search kernel against the measured issue peak
    import ctypes as C
    issue_peak, alu_peak = C.c_double(), C.c_double()
    err = C.create_string_buffer(256)
    _lib.lib().td_int_issue_peak.argtypes = [C.c_int, C.c_float, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                             C.c_char_p, C.c_size_t]
    _lib.check(_lib.lib().td_int_issue_peak(local, 200.0, C.byref(issue_peak), C.byref(alu_peak), err, 256), err)
    per_step_exp = expansions / max(1, args.steps) / world
    mean_ms = float(np.mean(step_ms))
    clock = clocks.summary()
    sm_mhz = clock["sm_mhz"] or 1965.0
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    nodes_per_s = per_step_exp / (mean_ms / 1e3)
    triples_per_s = nodes_per_s * 680
    # The bound is the integer ALU pipe (LOP3/shift/compare work of the
    # bit-sliced classification).  achieved: the search's ALU instructions per
    # second (expansions/s x ALU instructions per expansion); peak: LOP3 chains
    # on every SM, measured live.  Issue of all pipes is reported beside it.
    ach = nodes_per_s * ALU_INST_PER_EXPANSION
    roofline = {"bound": "int-alu", "unit": "G warp-inst/s", "achieved": ach / 1e9, "peak": alu_peak.value / 1e9,
                "frac": ach / alu_peak.value,
                "peak_source": "measured live: LOP3 chains on every SM (td_int_issue_peak), of measured",
                "alu_inst_per_expansion": ALU_INST_PER_EXPANSION,
                "issue_achieved": nodes_per_s * INST_PER_EXPANSION / 1e9,
                # issue: 4 warp instructions per clock per SM (one per
                # sub-partition) at the SM clock sampled during the timed steps
                "issue_peak_4_per_clk": 4 * sms * sm_mhz * 1e6 / 1e9,
                "issue_frac": nodes_per_s * INST_PER_EXPANSION / (4 * sms * sm_mhz * 1e6),
                "issue_lop3_imad_measured": issue_peak.value / 1e9,
                "inst_per_expansion": INST_PER_EXPANSION,
                "traffic": DRAM_BYTES_PER_LAUNCH * count / COUNT,
                "traffic_note": "DRAM bytes of one 2^20 launch (ncu, one pass, the benchmark launch itself); the "
                                "algorithmic bytes are 48 per instance (16 in, 32 out): 50 MB; the rest is the "
                                "explored-state tables (4736 warps x 32 KiB = 155 MB > the 126 MB L2)",
                "alu_busy_measured": ALU_BUSY_MEASURED, "issue_measured": ISSUE_MEASURED,
                "nodes_per_s": nodes_per_s, "triples_per_s": triples_per_s}

    graph.close()
    serving = None
    if world == 1 and not only_engine:
        serving = serving_legs(td, local)
    cpu = cpu_baseline() if world == 1 and not only_engine else None
    percall = per_call_legs(td) if world == 1 and not only_engine else None
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/u64 integer", "data": "synthetic (seeded)",
        "config": bench_config(world, count),
        "nodes_per_s": nodes_per_s, "triples_per_s": triples_per_s,
        "found": found, "not_found": not_found, "errors": errors, "verified": verified,
        "plain_one_launch": {"value": plain_verified / (plain_ms / 1e3), "ms": plain_ms, "warps": PLAIN_WARPS},
        "e2e": {"value": e2e_verified / e2e_s if e2e_s else None, "unit": UNIT,
                "h2d_bytes_per_step": count * 16 * world, "d2h_bytes_per_step": count * 32 * world,
                "ms_per_step": e2e_s / e2e_steps * 1e3, "steps": len(e2e_ms),
                "ms_min": min(e2e_ms) if e2e_ms else None, "ms_max": max(e2e_ms) if e2e_ms else None},
        "gpu_launches": args.steps * 4,  # per graph replay: epoch, search, finalize, replay
        "launch_shape": tuned,
        "roofline": roofline,
        "clocks": clock,
        "cpu_baseline": cpu,
        "percall": percall,
        "serving": serving,
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--count", type=int, default=COUNT,
                    help="instances per GPU (default 2^20, the benchmark workload; smaller for profiling)")
    ap.add_argument("--workload", default="mix", choices=["mix", "replicated"],
                    help="'replicated': one hard instance copied, for profiling the search without a tail")
    ap.add_argument("--legs", default="all", choices=["all", "engine"],
                    help="'engine' times only the device-resident batch (no e2e, plain, serving or CPU legs)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
