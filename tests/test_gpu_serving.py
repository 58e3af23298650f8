"""Serving: requests join a resident launch as they arrive (needs a B200).

Tolerance: in the reference move order every result is bit-identical alone,
in the mix and in the batched form; in free order (where idle warps take
subtrees of running requests) the verdict is identical and every witness
replays with the checker's rules.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(td, count, seed=3, n_max=16):
    perms, n = td.synth_perms(seed, count, 8, n_max, 0, 0, 0)
    return perms, n, td.prepare_perms(perms, n, (n // 2 + 1).astype(np.int32))


def _replays(oracle, td, perms, n, res, maxd):
    for i in np.nonzero(res["status"] == 1)[0]:
        beta, omega, _ = oracle.perm_to_pair(perms[i, : n[i]].tolist())
        abc = oracle.positions_to_symbols(beta, td.unpack_moves(res[i]))
        assert oracle.validate(beta, omega, abc, int(maxd[i])) is None, i


# free order on the full request mix; the reference order (blind, so slow on
# S_16) on n = 8..12
@pytest.mark.parametrize("flags,n_max", [(0, 16), (1, 12)])
def test_results_are_the_same_alone_and_in_the_mix(td, oracle, flags, n_max):
    perms, n, inst = _requests(td, 3000, n_max=n_max)
    maxd = n // 2 + 1
    # alone: one request at a time through a resident launch
    srv = td._lib.Server(0, 64, flags, 60.0)
    alone = []
    try:
        for x in inst[:300]:
            t = srv.submit(x)
            deadline = time.time() + 30
            r = None
            while r is None and time.time() < deadline:
                r = srv.poll(t)
            assert r is not None
            alone.append(r)
    finally:
        srv.close()
    alone = np.array(alone, dtype=td.RESULT_DTYPE)
    # in the mix: open-loop arrivals at 100k/s, many requests on the device at once
    mixed, stats = td._lib.serve_open_loop(0, inst, 100000.0, seed=3, flags=flags)
    # and the batched form
    td.init_slots(1, [0], 64 << 20)
    try:
        batch, _ = td.search_batch(0, inst, flags | td._lib.FLAG_PLAIN)
    finally:
        td.destroy()
    assert (alone["status"] == mixed["status"][:300]).all()
    assert (batch["status"] == mixed["status"]).all()
    if flags & td._lib.FLAG_ORDERED:
        assert (alone["moves"] == mixed["moves"][:300]).all() and (alone["depth"] == mixed["depth"][:300]).all()
        assert (batch["moves"] == mixed["moves"]).all()
    else:
        _replays(oracle, td, perms, n, mixed, maxd)
        _replays(oracle, td, perms[:300], n[:300], alone, maxd[:300])
    assert stats["served"] == 3000 and stats["found"] == int((mixed["status"] == 1).sum())
    assert 0 < stats["p50_ms"] <= stats["p99_ms"] <= stats["p999_ms"] <= stats["max_ms"]


def test_admission_respects_the_pool(td):
    _, _, inst = _requests(td, 1000, seed=4)
    # a pool that holds the frames of about two requests forces arrivals to queue
    res, st = td._lib.serve_open_loop(0, inst, 50000.0, seed=4, pool_bytes=4000)
    assert st["served"] == 1000 and st["admission_wait_ms_mean"] > 0
    assert (res["status"] >= 0).all()


def test_ring_slot_is_reused_only_after_its_result_is_taken(td):
    """A request's ring slot holds its result until the client polls it: with a
    ring of 8, the ninth submission waits for ticket 0 to be taken, even when
    the device finished it long ago."""
    perms, n, inst = _requests(td, 40, seed=5, n_max=12)
    srv = td._lib.Server(0, 8, 0, 60.0)
    try:
        tickets = [srv.submit(x) for x in inst[:8]]
        time.sleep(0.5)  # every one of them is done on the device by now
        with pytest.raises(td.TdError):
            srv.submit(inst[8])
        first = None
        deadline = time.time() + 30
        while first is None and time.time() < deadline:
            first = srv.poll(tickets[0])
        assert first is not None
        tickets.append(srv.submit(inst[8]))
        results = [first]
        for t in tickets[1:]:
            r = None
            deadline = time.time() + 30
            while r is None and time.time() < deadline:
                r = srv.poll(t)
            assert r is not None
            results.append(r)
    finally:
        srv.close()
    td.init_slots(1, [0], 64 << 20)
    try:
        batch, _ = td.search_batch(0, inst[:9], 0)
    finally:
        td.destroy()
    assert [int(r["status"]) for r in results] == [int(s) for s in batch["status"]]


def test_client_side_open_loop_through_the_per_call_server(td, oracle):
    """An open-loop Poisson stream through the per-call server, 8 client
    threads each polling only its own requests (td_percall_open_loop): every
    request is served, verdicts equal the batched form's, witnesses replay,
    and the latency percentiles are ordered."""
    perms, n, inst = _requests(td, 20000, seed=7)
    maxd = n // 2 + 1
    td.init_slots(1, [0], 64 << 20)
    try:
        res, st = td._lib.percall_open_loop(0, inst, 50000.0, clients=8, seed=11)
        batch, _ = td.search_batch(0, inst, 0)
    finally:
        td.destroy()
    assert st["served"] == 20000 and st["max_inflight"] == 8 and st["workers"] > 0
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["p999_ms"] <= st["max_ms"]
    assert (res["status"] == batch["status"]).all()
    _replays(oracle, td, perms, n, res, maxd)
