"""The native pair consumer (td_batcher_*, td16_b200/csrc/td_batcher.cc): the
enumerator's Consumer<CyclicTargetPair> (DirectTwistedBraceletGenerator.java:
105-156) fed one pair at a time from native producer threads and searched in
batches.  The CPU tests drive its queue, timer, bounded wait, error paths and
certificate sink with a stand-in search of td_search_pairs' signature; the
GPU test compares its verdicts with per-call td_search and the oracle."""
import ctypes as C
import threading
import time

import numpy as np
import pytest

OK, NOT_FOUND, OVERFLOW, CUDA_ERROR, INVALID_ARG = 0, 1, 2, 3, 4


def _fake(calls, gate=None, fail=None):
    """A td_search_pairs stand-in: even init -> found with the one move
    (0, 1, 2); odd -> not found; max_moves 7 -> the overflow class."""
    from td16_b200 import _lib

    def search(slot, count, beta, omega, n, init, rate, maxd, full, flags, status, depth, ijk, err, errlen):
        if gate is not None:
            gate.wait(5)
        calls.append((slot, count, flags))
        if fail is not None:
            C.memmove(err, fail.encode() + b"\0", len(fail) + 1)
            return CUDA_ERROR
        ini = np.ctypeslib.as_array(C.cast(init, C.POINTER(C.c_int32)), (count,))
        mm = np.ctypeslib.as_array(C.cast(maxd, C.POINTER(C.c_int32)), (count,))
        st = np.ctypeslib.as_array(C.cast(status, C.POINTER(C.c_int32)), (count,))
        dp = np.ctypeslib.as_array(C.cast(depth, C.POINTER(C.c_int32)), (count,))
        mv = np.ctypeslib.as_array(C.cast(ijk, C.POINTER(C.c_int16)), (count * 27,)).reshape(count, 9, 3)
        st[:] = np.where(ini % 2 == 0, OK, NOT_FOUND)
        st[mm == 7] = OVERFLOW
        dp[:] = np.where(st == OK, 1, 0)
        mv[:] = 0
        mv[st == OK, 0] = (0, 1, 2)
        return OK
    return _lib.BATCHER_SEARCH(search)


def _pairs(count):
    beta = np.zeros((count, 17), np.uint8)
    omega = np.zeros((count, 17), np.uint8)
    beta[:, :3] = (0, 1, 2)
    omega[:, :3] = (1, 2, 0)
    return beta, omega


def test_producers_batches_and_every_tag_delivered_once(td):
    calls, got = [], []
    lock = threading.Lock()

    def on_batch(tags, status, depth, moves):
        with lock:
            got.append((tags, status, depth, moves))
    cons = td._lib.PairConsumer(0, 3, batch_size=64, max_delay_s=0.005, on_batch=on_batch, search=_fake(calls))
    count = 20000
    beta, omega = _pairs(count)
    init = np.arange(count, dtype=np.int32) % 4
    td._lib.producer_threads_run(cons, 8, beta, omega, 3, init, 0.0, 9)
    stats = cons.close()
    tags = np.concatenate([g[0] for g in got])
    status = np.concatenate([g[1] for g in got])
    depth = np.concatenate([g[2] for g in got])
    moves = np.concatenate([g[3] for g in got])
    assert sorted(tags.tolist()) == list(range(count))
    by_tag = np.empty(count, np.int32)
    by_tag[tags] = status
    assert (by_tag == np.where(init % 2 == 0, OK, NOT_FOUND)).all()
    assert (depth[status == OK] == 1).all() and (moves[status == OK, 0] == (0, 1, 2)).all()
    assert max(c for _, c, _ in calls) == 64 and {s for s, _, _ in calls} <= {0, 1, 2}
    assert sum(c for _, c, _ in calls) == count
    assert stats["pairs"] == count and stats["batches"] == len(calls)
    assert stats["found"] == count // 2 and stats["not_found"] == count // 2 and stats["errors"] == 0


def test_a_lone_pair_is_searched_after_the_delay(td):
    calls, got = [], []
    cons = td._lib.PairConsumer(0, 1, batch_size=4096, max_delay_s=0.01, ordered=True,
                                on_batch=lambda *a: got.append(a), search=_fake(calls))
    try:
        t0 = time.monotonic()
        cons.accept(7, bytes([0, 1, 2]), bytes([1, 2, 0]), 2, 0.0, 9)
        while not got and time.monotonic() - t0 < 2.0:
            time.sleep(0.001)
        assert got and time.monotonic() - t0 < 1.0
        assert got[0][0].tolist() == [7] and got[0][1].tolist() == [OK]
        assert calls == [(0, 1, 1)]  # one pair, slot 0, the ordered flag passed through
    finally:
        cons.close()


def test_statuses_of_a_batch_and_a_failed_batch_call(td):
    calls, got = [], []
    cons = td._lib.PairConsumer(0, 1, batch_size=3, max_delay_s=0.01, on_batch=lambda *a: got.append(a),
                                search=_fake(calls))
    for tag, m in enumerate((9, 7, 9)):
        cons.accept(tag, bytes([0, 1, 2]), bytes([1, 2, 0]), 2 * tag, 0.0, m)
    with pytest.raises(td.TdError):
        cons.accept(9, bytes([0, 1, 2]), bytes([1, 2]), 2, 0.0, 9)  # unequal lengths
    with pytest.raises(td.TdError):
        cons.accept(9, bytes(18), bytes(18), 2, 0.0, 9)             # more than 17 symbols
    stats = cons.close()
    assert got[0][1].tolist() == [OK, OVERFLOW, OK]
    assert stats["found"] == 2 and stats["errors"] == 1

    got = []
    cons = td._lib.PairConsumer(2, 1, batch_size=2, max_delay_s=0.01, on_batch=lambda *a: got.append(a),
                                search=_fake([], fail="device lost"))
    cons.accept(0, bytes([0, 1, 2]), bytes([1, 2, 0]), 2, 0.0, 9)
    cons.accept(1, bytes([0, 1, 2]), bytes([1, 2, 0]), 2, 0.0, 9)
    with pytest.raises(td.TdError, match="device lost"):
        cons.close()
    assert got[0][1].tolist() == [CUDA_ERROR, CUDA_ERROR]
    assert cons.stats["errors"] == 2


def test_accept_blocks_while_batches_wait(td):
    gate = threading.Event()
    cons = td._lib.PairConsumer(0, 1, batch_size=1, max_delay_s=0.01, max_pending=2, search=_fake([], gate=gate))
    done = []

    def producer():
        for i in range(6):
            cons.accept(i, bytes([0, 1, 2]), bytes([1, 2, 0]), 2, 0.0, 9)
            done.append(i)
    t = threading.Thread(target=producer)
    t.start()
    time.sleep(0.2)
    assert len(done) <= 4   # one batch in the worker, two pending, the producer held back
    gate.set()
    t.join(5)
    assert cons.close()["pairs"] == 6 and len(done) == 6


def test_open_rejects_bad_settings(td):
    L = td._lib.lib()
    h = C.c_void_p()
    err = C.create_string_buffer(256)
    null_search, null_done = td._lib.BATCHER_SEARCH(), td._lib.BATCHER_DONE()
    for args in ((0, 0, 64, 0.01, 0, 0), (0, 1, 0, 0.01, 0, 0), (0, 1, 64, 0.0, 0, 0), (-1, 1, 64, 0.01, 0, 0),
                 (0, 1, 64, 0.01, -1, 0), (0, 1, 64, 0.01, 0, 2)):
        assert L.td_batcher_open(*args, null_search, None, null_done, None, C.byref(h), err, 256) == INVALID_ARG
        assert not h.value
    assert L.td_batcher_accept(None, 0, None, None, 0, 0, 0.0, 9, 1) == INVALID_ARG
    assert L.td_batcher_flush(None) == INVALID_ARG
    assert L.td_batcher_close(None, None, err, 256) == INVALID_ARG


def test_found_witnesses_reach_the_certificate_writer(td, tmp_path):
    """The sink path: found pairs become certificate records (the codec's
    bytes) without passing through the caller; the file reads back."""
    path = str(tmp_path / "certs.bin")
    w = td._lib.CertificateWriter(path, 5.0)
    cons = td._lib.PairConsumer(0, 2, batch_size=16, max_delay_s=0.005, cert_writer=w, search=_fake([]))
    count = 100
    beta, omega = _pairs(count)
    td._lib.producer_threads_run(cons, 4, beta, omega, 3, np.arange(count, dtype=np.int32) % 2 * 1, 0.0, 9)
    stats = cons.close()
    assert w.close() == stats["certificates"] == stats["found"] == 50
    om = np.zeros((64, 17), np.uint8)
    abc = np.zeros((64, 27), np.uint8)
    dep = np.zeros(64, np.uint8)
    k = td._lib.lib().td_cert_read_file(path.encode(), 3, 64, om.ctypes.data, abc.ctypes.data, dep.ctypes.data)
    assert k == 50 and (dep[:k] == 1).all()
    assert (om[:k, :3] == (1, 2, 0)).all() and (abc[:k, :3] == (0, 1, 2)).all()


@pytest.mark.gpu
def test_native_consumer_matches_per_call_search(td, oracle):
    """2,048 pairs from 8 native producer threads, half of the n = 11..13 mix
    at bound floor(n/2)+1 and half hard n = 13 pairs at bound 6 (most without
    a witness): the same verdicts as per-call td_search and the oracle; every
    witness replays, and the certificate sink holds one record per witness."""
    import os
    import tempfile
    p1, n1 = td.synth_perms(1, 1024, 11, 13, 25, 1, 3)
    p2, n2 = td.synth_perms(5, 1024, 13, 13, 100, 1, 3)
    rows = [(p, k, int(k // 2 + 1)) for p, k in zip(p1, n1)] + [(p, k, 6) for p, k in zip(p2, n2)]
    c = len(rows)
    beta = np.zeros((c, 17), np.uint8)
    omega = np.zeros((c, 17), np.uint8)
    N = np.zeros(c, np.int32)
    init = np.zeros(c, np.int32)
    bound = np.zeros(c, np.int32)
    for i, (p, k, b) in enumerate(rows):
        be, om, e = oracle.perm_to_pair(p[:k].tolist())
        beta[i, : k + 1], omega[i, : k + 1], N[i], init[i], bound[i] = be, om, k + 1, e, b
    got = {}
    lock = threading.Lock()

    def on_batch(tags, status, depth, moves):
        with lock:
            for t, s, d, m in zip(tags, status, depth, moves):
                got[int(t)] = (int(s), [tuple(int(v) for v in m[q]) for q in range(d)])
    path = os.path.join(tempfile.mkdtemp(), "certs.bin")
    td.init_slots(4, [0], 256 << 20)
    try:
        w = td._lib.CertificateWriter(path, 5.0)
        cons = td._lib.PairConsumer(0, 4, batch_size=256, max_delay_s=0.002, cert_writer=w, on_batch=on_batch)
        td._lib.producer_threads_run(cons, 8, beta, omega, N, init, 0.0, bound)
        stats = cons.close()
        written = w.close()
        single = [td.search(0, bytes(beta[i, : N[i]]), bytes(omega[i, : N[i]]), int(init[i]), 0.0, int(bound[i]))
                  for i in range(c)]
    finally:
        td.destroy()
    st, _, _, _ = oracle.search_batch(beta, omega, N, init, np.zeros(c), bound, np.ones(c), 16)
    assert sorted(got) == list(range(c))
    verdict = [1 if got[i][0] == OK else 0 for i in range(c)]
    assert all(got[i][0] in (OK, NOT_FOUND) for i in range(c))
    assert verdict == [int(bool(s)) for s in single] == [int(s) for s in st]
    assert 0 < stats["found"] == written == sum(verdict) < c
    for i in range(c):
        if verdict[i]:
            abc = oracle.positions_to_symbols(beta[i, : N[i]].tolist(), got[i][1])
            assert oracle.validate(beta[i, : N[i]].tolist(), omega[i, : N[i]].tolist(), abc, int(bound[i])) is None
