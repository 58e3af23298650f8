"""The enumerator-shaped case consumer (host.PairBatcher): pairs accepted one
at a time from many generator threads are searched in batches through
td_search_pairs.  The CPU tests drive the batching logic with a stand-in
search; the GPU test compares it with per-call td_search and the oracle."""
import concurrent.futures as cf
import threading
import time

import numpy as np
import pytest


def _fake_search(calls):
    def search(slot, beta, omega, n, init, rate, maxd, full):
        calls.append((slot, len(n)))
        c = len(n)
        status = np.where(init % 2 == 0, 0, 1).astype(np.int32)   # even init: found (OK = 0)
        status[maxd > 9] = 4                                       # the per-call invalid-argument class
        status[maxd == 7] = 2                                      # the overflow class
        depth = np.where(status == 0, 1, 0).astype(np.int32)
        moves = np.zeros((c, 9, 3), np.int16)
        moves[:, 0] = (0, 1, 2)
        return status, depth, moves
    return search


def test_batches_fill_flush_and_complete_every_future(td):
    calls, sunk = [], []
    b = td.PairBatcher([0, 1, 2], batch_size=64, max_delay_s=0.005, search_fn=_fake_search(calls),
                       sink=lambda beta, omega, w: sunk.append(w))
    futs = [None] * 2000

    def gen(t):
        for i in range(t, 2000, 8):
            futs[i] = b.accept(bytes([0, 1, 2]), bytes([1, 2, 0]), i % 4, 0.0, 9)

    threads = [threading.Thread(target=gen, args=(t,)) for t in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    b.close()
    res = [f.result(timeout=5) for f in futs]
    assert all(r == ([(0, 1, 2)] if i % 2 == 0 else []) for i, r in enumerate(res))
    assert len(sunk) == 1000 and b.pairs == 2000
    assert sum(c for _, c in calls) == 2000 and {s for s, _ in calls} <= {0, 1, 2}
    assert max(c for _, c in calls) == 64 and len(calls) >= 2000 // 64


def test_a_lone_pair_is_searched_after_the_delay(td):
    calls = []
    b = td.PairBatcher([0], batch_size=4096, max_delay_s=0.01, search_fn=_fake_search(calls))
    try:
        t0 = time.monotonic()
        assert b.accept(bytes([0, 1, 2]), bytes([1, 2, 0]), 2, 0.0, 9).result(timeout=5) == [(0, 1, 2)]
        assert time.monotonic() - t0 < 1.0 and calls == [(0, 1)]
    finally:
        b.close()


def test_errors_reach_the_callers(td):
    def broken(*a):
        raise RuntimeError("device lost")
    b = td.PairBatcher([0], batch_size=2, max_delay_s=0.01, search_fn=broken)
    f1 = b.accept(bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 0.0, 9)
    f2 = b.accept(bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 0.0, 9)
    b.close()
    for f in (f1, f2):
        with pytest.raises(RuntimeError, match="device lost"):
            f.result(timeout=5)
    calls = []
    b = td.PairBatcher([0], batch_size=3, max_delay_s=0.01, search_fn=_fake_search(calls))
    fs = [b.accept(bytes([0, 1, 2]), bytes([1, 2, 0]), 2, 0.0, m) for m in (9, 7, 10)]
    bad = b.accept(bytes([0, 1, 2]), bytes([1, 2]), 2, 0.0, 9)
    b.close()
    assert fs[0].result() == [(0, 1, 2)]
    with pytest.raises(td.TdError, match="queue overflow"):
        fs[1].result()
    with pytest.raises(td.TdError, match="invalid input"):
        fs[2].result()
    with pytest.raises(td.TdError, match="equal lengths"):
        bad.result()


def test_accept_blocks_while_batches_wait(td):
    gate = threading.Event()
    calls = []

    def slow(*a):
        gate.wait(5)
        return _fake_search(calls)(*a)
    b = td.PairBatcher([0], batch_size=1, max_delay_s=0.01, max_pending=2, search_fn=slow)
    done = []

    def producer():
        for i in range(6):
            b.accept(bytes([0, 1, 2]), bytes([1, 2, 0]), 2, 0.0, 9)
            done.append(i)
    t = threading.Thread(target=producer)
    t.start()
    time.sleep(0.2)
    assert len(done) <= 4   # one batch in the worker, two pending, the producer held back
    gate.set()
    t.join(5)
    b.close()
    assert len(done) == 6


@pytest.mark.gpu
def test_batched_consumer_matches_per_call_search(td, oracle):
    """2,048 pairs from 8 generator threads, half of the n = 11..13 mix at
    bound floor(n/2)+1 and half hard n = 13 pairs at bound 6 (most without a
    witness): the same verdicts as per-call td_search and the oracle; every
    witness replays."""
    p1, n1 = td.synth_perms(1, 1024, 11, 13, 25, 1, 3)
    p2, n2 = td.synth_perms(5, 1024, 13, 13, 100, 1, 3)
    pairs = []
    for (p, k), bound in [((p, k), int(k // 2 + 1)) for p, k in zip(p1, n1)] + [((p, k), 6) for p, k in zip(p2, n2)]:
        beta, omega, init = oracle.perm_to_pair(p[:k].tolist())
        pairs.append((bytes(beta), bytes(omega), init, bound))
    td.init_slots(4, [0], 256 << 20)
    sunk = []
    try:
        b = td.PairBatcher([0, 1, 2, 3], batch_size=256, max_delay_s=0.002,
                           sink=lambda beta, omega, w: sunk.append(1))
        futs = [None] * len(pairs)

        def gen(t):
            for i in range(t, len(pairs), 8):
                futs[i] = b.accept(pairs[i][0], pairs[i][1], pairs[i][2], 0.0, pairs[i][3])
        with cf.ThreadPoolExecutor(8) as ex:
            list(ex.map(gen, range(8)))
        b.close()
        got = [f.result(timeout=60) for f in futs]
        single = [td.search(0, p[0], p[1], p[2], 0.0, p[3]) for p in pairs]
    finally:
        td.destroy()
    c = len(pairs)
    beta = np.zeros((c, 17), np.uint8)
    omega = np.zeros((c, 17), np.uint8)
    for i, p in enumerate(pairs):
        beta[i, : len(p[0])] = list(p[0])
        omega[i, : len(p[1])] = list(p[1])
    st, _, _, _ = oracle.search_batch(beta, omega, [len(p[0]) for p in pairs], [p[2] for p in pairs],
                                      np.zeros(c), [p[3] for p in pairs], np.ones(c), 16)
    assert [int(bool(w)) for w in got] == [int(bool(w)) for w in single] == [int(s) for s in st]
    assert 0 < len(sunk) == sum(bool(w) for w in got) < c
    for p, w in zip(pairs, got):
        if w:
            assert oracle.validate(list(p[0]), list(p[1]), w, p[3]) is None


def test_batch_symbol_conversion_matches_the_c_abi(td):
    """host.positions_to_symbols_batch (the consumer's vectorised conversion)
    gives td_positions_to_symbols's symbol triples for every pair."""
    from td16_b200.host import positions_to_symbols_batch
    rng = np.random.default_rng(1)
    c = 400
    beta = np.zeros((c, 17), np.uint8)
    depth = rng.integers(0, 10, c)
    moves = np.zeros((c, 9, 3), np.int16)
    sizes = []
    for r in range(c):
        N = int(rng.integers(3, 18))
        sizes.append(N)
        beta[r, :N] = rng.permutation(N)
        for d in range(depth[r]):
            moves[r, d] = sorted(rng.choice(N, 3, replace=False))
    out = positions_to_symbols_batch(beta, depth, moves)
    for r in range(c):
        want = td._lib.positions_to_symbols(bytes(beta[r, : sizes[r]]),
                                            [tuple(int(v) for v in moves[r, d]) for d in range(depth[r])])
        assert [tuple(int(v) for v in out[r, d]) for d in range(depth[r])] == want
