"""Parity against fixtures produced by the compiled reference kernel
(tests/golden/ref_gpu_fixtures.json, made by tests/golden/make_ref_fixtures.py).

Sets (reference kernel, unmodified sorting_search.cu + slot_manager.cu):
  single queue (maxWarps = 1), witnesses compared move for move:
    ordered               N = 4..11, bounds 1..6, rates {0, 1, 1.5, 2}
    ordered_large         N = 12..14, bounds 1..6
    caller_rates_ordered  N = 6..11, minRate = 2 / (maxMoves / (float) target)
    partial_ordered       fullSorting = false
  production launch (one queue per resident block), verdicts compared:
    verdicts              the n = 11..13 mix and S_16 at bound 9
    at_lower_bound        N = 14, 15, 17 at the cycle-graph lower bound
                          (about a third without a witness)
    caller_rates          N = 9..17, the emitter callers' rates near their
                          boundary, bounds 8 and 9
    partial               fullSorting = false
"""
import ctypes as C
import json
import os

import numpy as np
import pytest

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_gpu_fixtures.json")))
STATUS = {"found": 1, "not_found": 0}
ORDERED_SETS = ["ordered", "ordered_large", "caller_rates_ordered", "partial_ordered"]
VERDICT_SETS = ["verdicts", "at_lower_bound", "caller_rates", "partial"]


def test_fixture_file_is_complete():
    assert len(FIX["ordered"]) > 500 and len(FIX["verdicts"]) > 1000
    sizes = {"ordered_large": 300, "at_lower_bound": 600, "caller_rates": 250, "caller_rates_ordered": 200,
             "partial": 250, "partial_ordered": 250}
    for name, least in sizes.items():
        assert len(FIX[name]) >= least, name
    for name in ORDERED_SETS + VERDICT_SETS:
        assert not [c for c in FIX[name] if c["status"] == "error"], name
    # the later sets hold both verdicts, witnesses at N = 12..14 in the single
    # queue, and searches without a witness at N = 17
    for name in ("ordered_large", "at_lower_bound", "caller_rates", "partial", "partial_ordered"):
        assert {c["status"] for c in FIX[name]} == {"found", "not_found"}, name
    assert {len(c["beta"]) for c in FIX["ordered_large"] if c["status"] == "found"} == {12, 13, 14}
    assert sum(len(c["beta"]) == 17 and c["status"] == "not_found" for c in FIX["at_lower_bound"]) > 50
    rates = {c["rate"] for c in FIX["caller_rates"]}
    assert len(rates) > 10 and all(c["maxd"] in (8, 9) for c in FIX["caller_rates"])


def _f32_accepts(odd, init, depth, rate, N, full):
    """satisfies_rate (sorting_search.cu:336-346) in single precision."""
    if depth <= 0 or (full and odd != N):
        return False
    gained = odd - init
    return gained > 0 and np.float32(gained) / np.float32(depth) >= np.float32(rate)


def _witness_ok(oracle, c, moves):
    """The witness obeys the reference's move filter (no fixed symbol, odd-cycle
    change 0 or +2) and its last node passes the rate test; with full sorting
    the checker's replay also accepts it."""
    beta, omega = list(c["beta"]), list(c["omega"])
    N = len(beta)
    if not moves or len(moves) > c["maxd"]:
        return False
    odd = oracle.count_odd_cycles(omega)
    for (i, j, k) in moves:
        if not (0 <= i < j < k < N):
            return False
        a, b, cc = beta[i], beta[j], beta[k]
        if omega[a] == a or omega[b] == b or omega[cc] == cc:
            return False
        nxt = list(omega)
        nxt[a], nxt[b], nxt[cc] = omega[cc], omega[a], omega[b]
        d = oracle.count_odd_cycles(nxt) - odd
        if d not in (0, 2):
            return False
        odd += d
        omega = nxt
        beta = beta[:i] + beta[j:k] + beta[i:j] + beta[k:]
    if not _f32_accepts(odd, c["init"], len(moves), c["rate"], N, c["full"]):
        return False
    if c["full"]:
        abc = oracle.positions_to_symbols(c["beta"], [tuple(m) for m in moves])
        return oracle.validate(c["beta"], c["omega"], abc, c["maxd"]) is None
    return True


@pytest.mark.parametrize("name", ORDERED_SETS)
def test_oracle_reproduces_reference_single_queue_witnesses(oracle, name):
    for c in FIX[name]:
        rc, moves, _ = oracle.search(c["beta"], c["omega"], c["init"], c["rate"], c["maxd"], bool(c["full"]))
        assert rc == STATUS[c["status"]], c
        assert [list(m) for m in moves] == c["moves"], c


def _arrays(cases):
    c = len(cases)
    beta = np.zeros((c, 17), np.uint8)
    omega = np.zeros((c, 17), np.uint8)
    for i, k in enumerate(cases):
        beta[i, : len(k["beta"])] = k["beta"]
        omega[i, : len(k["omega"])] = k["omega"]
    get = lambda f: np.array([k[f] for k in cases])  # noqa: E731
    return beta, omega, np.array([len(k["beta"]) for k in cases]), get("init"), get("rate"), get("maxd"), get("full")


@pytest.mark.parametrize("name", VERDICT_SETS)
def test_oracle_reproduces_reference_verdicts_and_accepts_its_witnesses(oracle, name):
    cases = FIX[name]
    beta, omega, N, init, rate, maxd, full = _arrays(cases)
    st, _, _, _ = oracle.search_batch(beta, omega, N, init, rate, maxd, full, os.cpu_count() or 8)
    assert [int(v) for v in st] == [STATUS[c["status"]] for c in cases]
    for c in cases:
        if c["moves"]:
            assert _witness_ok(oracle, c, [tuple(m) for m in c["moves"]]), c


@pytest.mark.parametrize("name", ORDERED_SETS)
def test_emulated_engine_reproduces_reference_witnesses(emu, name):
    from tests.test_engine_logic_cpu import Inst, Res, _u8
    for c in FIX[name]:
        x = Inst()
        assert emu.td_emu_prepare_pair(_u8(c["beta"]), _u8(c["omega"]), len(c["beta"]), c["init"],
                                       C.c_float(c["rate"]), c["maxd"], c["full"], C.byref(x)) == 0
        r = Res()
        emu.td_emu_search(C.byref(x), 1, C.byref(r))
        assert r.status == STATUS[c["status"]]
        assert [[m & 31, (m >> 5) & 31, (m >> 10) & 31] for m in r.moves[: r.depth]] == c["moves"]


@pytest.mark.parametrize("name", ["at_lower_bound", "caller_rates", "partial"])
def test_emulated_free_order_reproduces_reference_verdicts(oracle, name):
    cases = FIX[name]
    beta, omega, N, init, rate, maxd, full = _arrays(cases)
    res = oracle.emu_search_batch(beta, omega, N, init, rate, maxd, full, 0, os.cpu_count() or 8)
    assert [int(v) for v in res["status"]] == [STATUS[c["status"]] for c in cases]
    for c, r in zip(cases, res):
        if r["status"] == 1:
            moves = [(int(m) & 31, (int(m) >> 5) & 31, (int(m) >> 10) & 31) for m in r["moves"][: r["depth"]]]
            assert _witness_ok(oracle, c, moves), c


def _batch(td, cases):
    beta, omega, N, init, rate, maxd, full = _arrays(cases)
    return td.prepare_pairs(beta, omega, N, init, rate.astype(np.float32), maxd, full)


@pytest.mark.gpu
def test_engine_reproduces_reference_kernel(td, oracle):
    td.init_slots(1, [0], 64 << 20)
    try:
        for name in ORDERED_SETS:
            inst = _batch(td, FIX[name])
            res, _ = td.search_batch(0, inst, td._lib.FLAG_ORDERED)
            for r, c in zip(res, FIX[name]):
                assert r["status"] == STATUS[c["status"]], (name, c)
                assert [list(m) for m in td.unpack_moves(r)] == c["moves"], (name, c)
        for name in VERDICT_SETS:
            inst = _batch(td, FIX[name])
            want = [STATUS[c["status"]] for c in FIX[name]]
            for flags in (0, td._lib.FLAG_PLAIN, td._lib.FLAG_VERIFY):
                res, _ = td.search_batch(0, inst, flags)
                assert [int(s) for s in res["status"]] == want, (name, flags)
                for r, c in zip(res, FIX[name]):
                    if r["status"] == 1:
                        assert _witness_ok(oracle, c, td.unpack_moves(r)), (name, c)
    finally:
        td.destroy()


@pytest.mark.gpu
def test_per_call_path_reproduces_reference_kernel(td, oracle):
    """The same sets through td_search and td_search_ordered, one blocking
    call per pair from 16 native slot threads."""
    td.init_slots(16, [0], 64 << 20)
    try:
        for name, entry in [(n, "td_search_ordered") for n in ORDERED_SETS] + [(n, "td_search") for n in
                                                                               VERDICT_SETS]:
            cases = FIX[name]
            beta, omega, N, init, rate, maxd, full = _arrays(cases)
            r = td._lib.slot_threads_run(td._lib.entry_address(entry), beta, omega, N, init, rate, maxd, full, 16)
            assert [int(s) for s in r["status"]] == [STATUS[c["status"]] for c in cases], name
            for i, c in enumerate(cases):
                moves = [tuple(int(v) for v in r["moves"][i, d]) for d in range(r["depth"][i])]
                if entry == "td_search_ordered":
                    assert [list(m) for m in moves] == c["moves"], (name, c)
                elif moves:
                    assert _witness_ok(oracle, c, moves), (name, c)
    finally:
        td.destroy()


def test_device_replay_rule_accepts_every_reference_witness_and_rejects_tampering(emu):
    """td_witness_ok, the rule behind TD_FLAG_VERIFY and td_validate_batch_device
    (run here on the host through the emulator): every witness the reference
    kernel returned passes, in full and partial sorting; a witness with a move
    dropped, a move out of range, a depth beyond the bound or a rate it misses
    does not."""
    from tests.test_engine_logic_cpu import Inst, Res, _u8
    checked = rejected = 0
    for name in ORDERED_SETS + VERDICT_SETS:
        for c in FIX[name]:
            if not c["moves"]:
                continue
            x = Inst()
            assert emu.td_emu_prepare_pair(_u8(c["beta"]), _u8(c["omega"]), len(c["beta"]), c["init"],
                                           C.c_float(c["rate"]), c["maxd"], c["full"], C.byref(x)) == 0

            def rec(moves):
                r = Res()
                r.status, r.depth = 1, len(moves)
                for d, (i, j, k) in enumerate(moves):
                    r.moves[d] = (i & 31) | ((j & 31) << 5) | ((k & 31) << 10)
                return r

            moves = [tuple(m) for m in c["moves"]]
            assert emu.td_emu_witness_ok(C.byref(x), C.byref(rec(moves))) == 1, (name, c)
            checked += 1
            bad = [rec(moves[:-1]) if len(moves) > 1 else None,
                   rec(moves[:-1] + [(0, 1, len(c["beta"]))])]
            if len(moves) < 9:
                bad.append(rec(moves + [moves[-1]]))
            for r in bad:
                if r is not None:
                    rejected += emu.td_emu_witness_ok(C.byref(x), C.byref(r)) == 0
            if c["full"] == 0 and c["rate"] > 0:
                x2 = Inst.from_buffer_copy(x)
                x2.min_rate = 100.0  # beyond any gain per move
                assert emu.td_emu_witness_ok(C.byref(x2), C.byref(rec(moves))) == 0
    assert checked > 2000 and rejected > 2 * checked * 0.9
