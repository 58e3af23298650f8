"""Parity against fixtures produced by the compiled reference kernel
(tests/golden/ref_gpu_fixtures.json, made by tests/golden/make_ref_fixtures.py)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

FIX = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_gpu_fixtures.json")))
STATUS = {"found": 1, "not_found": 0}


def test_fixture_file_is_complete():
    assert len(FIX["ordered"]) > 500 and len(FIX["verdicts"]) > 1000
    assert not [c for c in FIX["ordered"] + FIX["verdicts"] if c["status"] == "error"]


def test_oracle_reproduces_reference_single_queue_witnesses(oracle):
    for c in FIX["ordered"]:
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


def test_oracle_reproduces_reference_verdicts_and_replays_its_witnesses(oracle):
    cases = FIX["verdicts"]
    beta, omega, N, init, rate, maxd, full = _arrays(cases)
    st, _, _, _ = oracle.search_batch(beta, omega, N, init, rate, maxd, full, os.cpu_count() or 8)
    assert [int(v) for v in st] == [STATUS[c["status"]] for c in cases]
    for c in cases:
        if c["moves"]:
            abc = oracle.positions_to_symbols(c["beta"], [tuple(m) for m in c["moves"]])
            assert oracle.validate(c["beta"], c["omega"], abc, c["maxd"]) is None


def test_emulated_engine_reproduces_reference_witnesses(emu):
    from tests.test_engine_logic_cpu import Inst, Res, _u8
    for c in FIX["ordered"]:
        x = Inst()
        assert emu.td_emu_prepare_pair(_u8(c["beta"]), _u8(c["omega"]), len(c["beta"]), c["init"],
                                       C.c_float(c["rate"]), c["maxd"], c["full"], C.byref(x)) == 0
        r = Res()
        emu.td_emu_search(C.byref(x), 1, C.byref(r))
        assert r.status == STATUS[c["status"]]
        assert [[m & 31, (m >> 5) & 31, (m >> 10) & 31] for m in r.moves[: r.depth]] == c["moves"]


def _batch(td, cases):
    beta, omega, N, init, rate, maxd, full = _arrays(cases)
    return td.prepare_pairs(beta, omega, N, init, rate.astype(np.float32), maxd, full)


@pytest.mark.gpu
def test_engine_reproduces_reference_kernel(td):
    td.init_slots(1, [0], 64 << 20)
    try:
        inst = _batch(td, FIX["ordered"])
        res, _ = td.search_batch(0, inst, td._lib.FLAG_ORDERED)
        for r, c in zip(res, FIX["ordered"]):
            assert r["status"] == STATUS[c["status"]]
            assert [list(m) for m in td.unpack_moves(r)] == c["moves"]
        inst = _batch(td, FIX["verdicts"])
        for flags in (0, td._lib.FLAG_PLAIN, td._lib.FLAG_VERIFY):
            res, _ = td.search_batch(0, inst, flags)
            assert [int(s) for s in res["status"]] == [STATUS[c["status"]] for c in FIX["verdicts"]]
    finally:
        td.destroy()
