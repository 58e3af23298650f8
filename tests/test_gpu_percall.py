"""Parity of the per-call entry points (td_search, td_search_ordered: the
drop-in for the reference's searchForSortingSeq) with the oracle, called the
way the emitter calls them: one blocking search per call from 16 native slot
threads (GPUSortingSearch.java:134-147), through the C ABI.  Needs a B200."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SLOTS = 16
MiB = 1 << 20


@pytest.fixture(scope="module")
def slots(td):
    td.init_slots(SLOTS, [0], 256 * MiB)
    yield td
    td.destroy()


def _pairs(oracle, perms, n):
    c = len(perms)
    beta = np.zeros((c, 17), np.uint8)
    omega = np.zeros((c, 17), np.uint8)
    init = np.zeros(c, np.int32)
    N = np.zeros(c, np.int32)
    for i, (p, k) in enumerate(zip(perms, n)):
        b, o, e = oracle.perm_to_pair(p[:k].tolist())
        beta[i, : k + 1] = b
        omega[i, : k + 1] = o
        init[i] = e
        N[i] = k + 1
    return beta, omega, init, N


def _oracle(oracle, beta, omega, N, init, maxd, budget=0, rate=0.0, full=1):
    c = len(N)
    oracle.set_expansion_budget(budget)
    try:
        return oracle.search_batch(beta, omega, N, init, np.broadcast_to(np.float32(rate), (c,)),
                                   np.broadcast_to(maxd, (c,)).astype(np.int32),
                                   np.broadcast_to(full, (c,)).astype(np.uint8), 16)
    finally:
        oracle.set_expansion_budget(0)


def _run(td, entry, beta, omega, N, init, maxd, rate=0.0, full=1):
    return td._lib.slot_threads_run(td._lib.entry_address(entry), beta, omega, N, init, rate, maxd, full, SLOTS)


def _replay(oracle, beta, omega, N, r, maxd):
    maxd = np.broadcast_to(maxd, (len(N),))
    for i in np.nonzero(r["status"] == 1)[0]:
        k = int(N[i])
        moves = [tuple(int(v) for v in r["moves"][i, d]) for d in range(r["depth"][i])]
        abc = oracle.positions_to_symbols(beta[i, :k].tolist(), moves)
        err = oracle.validate(beta[i, :k].tolist(), omega[i, :k].tolist(), abc, int(maxd[i]))
        assert err is None, (i, err)


def test_per_call_s16_bound9_from_16_slot_threads(slots, oracle):
    """512 instances of the S_16 benchmark workload (half near-reverse), bound
    9: every search finds a witness that the oracle's checker replays, and the
    oracle agrees on every verdict it reaches within its budget."""
    td = slots
    perms, n = td.synth_perms(2, 512, 16, 16, 50, 1, 4)
    beta, omega, init, N = _pairs(oracle, perms, n)
    r = _run(td, "td_search", beta, omega, N, init, 9)
    assert (r["code"] == 0).all(), np.unique(r["code"])
    _replay(oracle, beta, omega, N, r, 9)
    st, _, _, _ = _oracle(oracle, beta, omega, N, init, 9, budget=200000)
    done = st != oracle.BUDGET
    assert done.sum() > 300
    assert (st[done] == 1).all()


def test_per_call_mix_verdicts_and_ordered_witnesses(slots, oracle):
    """1,024 instances of the n = 11..13 mix at bound floor(n/2)+1 (some
    without a witness): td_search's verdicts equal the oracle's and its
    witnesses replay; td_search_ordered returns the oracle's (the reference's
    single-queue) witness bit for bit."""
    td = slots
    perms, n = td.synth_perms(1, 1024, 11, 13, 25, 1, 3)
    beta, omega, init, N = _pairs(oracle, perms, n)
    maxd = (n // 2 + 1).astype(np.int32)
    st, dep, mv, _ = _oracle(oracle, beta, omega, N, init, maxd)
    free = _run(td, "td_search", beta, omega, N, init, maxd)
    assert (free["status"] >= 0).all()
    assert (free["status"] == st).all()
    _replay(oracle, beta, omega, N, free, maxd)
    ordered = _run(td, "td_search_ordered", beta, omega, N, init, maxd)
    assert (ordered["status"] == st).all()
    for i in range(len(N)):
        assert ordered["depth"][i] == (dep[i] if st[i] == 1 else 0)
        for d in range(ordered["depth"][i]):
            m = int(mv[i, d])
            assert tuple(int(v) for v in ordered["moves"][i, d]) == (m & 31, (m >> 5) & 31, (m >> 10) & 31), i


def test_per_call_server_matches_one_launch_per_call(slots, oracle):
    """The resident server and one launch per call give the same verdicts, on
    hard n = 13 instances at bound 6 (many without a witness)."""
    td = slots
    perms, n = td.synth_perms(5, 384, 13, 13, 100, 1, 3)
    beta, omega, init, N = _pairs(oracle, perms, n)
    served = _run(td, "td_search", beta, omega, N, init, 6)
    try:
        td._lib.configure_percall(0)
        launched = _run(td, "td_search", beta, omega, N, init, 6)
    finally:
        td._lib.configure_percall(1)
    assert (served["status"] >= 0).all() and (served["status"] == launched["status"]).all()
    assert (served["status"] == 0).any() and (served["status"] == 1).any()
    st, _, _, _ = _oracle(oracle, beta, omega, N, init, 6)
    assert (served["status"] == st).all()


def test_server_rotation_and_batches_alongside(slots, oracle):
    """With a rotation age of 20 ms the server is replaced many times while 16
    threads search, and a batch launched meanwhile on another slot shares the
    GPU; every result still equals the oracle's."""
    td = slots
    perms, n = td.synth_perms(9, 1536, 12, 14, 50, 1, 3)
    beta, omega, init, N = _pairs(oracle, perms, n)
    maxd = (n // 2 + 1).astype(np.int32)
    st, _, _, _ = _oracle(oracle, beta, omega, N, init, maxd)
    import threading
    batch = {}

    def run_batch():
        p2, n2 = td.synth_perms(2, 4096, 16, 16, 50, 1, 4)
        res, stats = td.search_batch(0, td.prepare_perms(p2, n2, 9), td._lib.FLAG_VERIFY)
        batch["found"] = int((res["status"] == 1).sum())

    try:
        td._lib.configure_percall(1, 0.02)
        t = threading.Thread(target=run_batch)
        t.start()
        r = td._lib.slot_threads_run(td._lib.entry_address("td_search"), beta, omega, N, init, 0.0, maxd, 1,
                                     SLOTS - 1, first_slot=1)
        t.join()
    finally:
        td._lib.configure_percall(1, 300.0)
    assert (r["status"] == st).all()
    _replay(oracle, beta, omega, N, r, maxd)
    assert batch["found"] == 4096


def test_per_call_edge_cases_through_the_server(slots):
    """The reference's contract on the per-call path: N < 3 gives an empty
    result, the smoke input its one move, invalid input an error."""
    td = slots
    assert td.search(0, b"", b"", 0, 0.0, 1) == []
    assert td.search(3, bytes([0, 1]), bytes([1, 0]), 0, 0.0, 1) == []
    assert td.search(7, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 1) == [(0, 1, 2)]
    assert td.search(7, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 1, ordered=True) == [(0, 1, 2)]
    with pytest.raises(td.TdError):
        td.search(0, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 10)
    with pytest.raises(td.TdError):
        td.search(SLOTS, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 1)


def test_idle_server_exits_and_restarts(slots):
    """The per-call launch exits by itself once idle (5 ms here by default),
    so a device-wide synchronisation afterwards returns at once; searches
    spaced further apart than that each start it again and stay correct."""
    import time
    import torch
    td = slots
    perms, n = td.synth_perms(2, 256, 16, 16, 50, 1, 4)
    beta = np.zeros((256, 17), np.uint8)
    omega = np.zeros((256, 17), np.uint8)
    init = (td.prepare_perms(perms, n, 9)["packed"] & 31).astype(np.int32)
    td._lib.lib().td_pairs_from_perms(256, perms.ctypes.data, n.ctypes.data, beta.ctypes.data, omega.ctypes.data)
    r = _run(td, "td_search", beta, omega, 17, init, 9)
    assert (r["status"] == 1).all()
    time.sleep(0.05)
    t0 = time.perf_counter()
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 0.5
    for i in range(24):  # each of these finds the launch gone and starts a new one
        time.sleep(0.01)
        moves = td.search(i % SLOTS, beta[i].tobytes(), omega[i].tobytes(), int(init[i]), 0.0, 9)
        assert 1 <= len(moves) <= 9
