"""Serving: requests join a resident launch as they arrive (needs a B200)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(td, count, seed=3, n_max=16):
    perms, n = td.synth_perms(seed, count, 8, n_max, 0, 0, 0)
    return td.prepare_perms(perms, n, (n // 2 + 1).astype(np.int32))


# free order on the full request mix; the reference order (blind, so slow on
# S_16) on n = 8..12
@pytest.mark.parametrize("flags,n_max", [(0, 16), (1, 12)])
def test_results_are_the_same_alone_and_in_the_mix(td, flags, n_max):
    inst = _requests(td, 3000, n_max=n_max)
    # alone: each request by itself through a fresh launch, one at a time
    srv = td._lib.Server(0, 64, flags, 60.0)
    alone = []
    try:
        for x in inst[:300]:
            t = srv.submit(x)
            deadline = time.time() + 10
            r = None
            while r is None and time.time() < deadline:
                r = srv.poll(t)
            assert r is not None
            alone.append(r)
    finally:
        srv.close()
    # in the mix: open-loop arrivals at 100k/s, many requests on the device at once
    mixed, stats = td._lib.serve_open_loop(0, inst, 100000.0, seed=3, flags=flags)
    for a, m in zip(alone, mixed[:300]):
        assert a["status"] == m["status"] and a["depth"] == m["depth"]
        assert (a["moves"] == m["moves"]).all()
    # and the batched form gives the same verdicts (and, ordered, the same witnesses)
    td.init_slots(1, [0], 64 << 20)
    try:
        batch, _ = td.search_batch(0, inst, flags | td._lib.FLAG_PLAIN)
    finally:
        td.destroy()
    assert (batch["status"] == mixed["status"]).all()
    assert (batch["moves"] == mixed["moves"]).all()
    assert stats["served"] == 3000 and stats["found"] == int((mixed["status"] == 1).sum())
    assert 0 < stats["p50_ms"] <= stats["p99_ms"] <= stats["p999_ms"] <= stats["max_ms"]


def test_admission_respects_the_pool(td):
    inst = _requests(td, 1000, seed=4)
    # a pool that holds the frames of about two requests forces arrivals to queue
    res, st = td._lib.serve_open_loop(0, inst, 50000.0, seed=4, pool_bytes=4000)
    assert st["served"] == 1000 and st["admission_wait_ms_mean"] > 0
    assert (res["status"] >= 0).all()
