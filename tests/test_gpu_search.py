"""Parity of the CUDA search with the oracle, through the C ABI (needs a B200)."""
import concurrent.futures as cf
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ORDERED, PLAIN = 1, 2
MiB = 1 << 20


def _library_defaults(td):
    """The engine's own defaults (td_engine.cu): donation grain 4, split level
    2, idle check every 64 expansions, 4096-entry tables, restart base 16, the
    race against the inverse from restart attempt 8."""
    td._lib.configure_steal(4, 2, 64)
    td._lib.configure_table(12)
    td._lib.configure_restart(16)
    td._lib.configure_race(8)


@pytest.fixture(scope="module")
def slots(td):
    td.init_slots(2, [0], 64 * MiB)
    yield td
    td.destroy()


def _pairs(oracle, perms, n):
    c = len(perms)
    beta = np.zeros((c, 17), np.uint8)
    omega = np.zeros((c, 17), np.uint8)
    init = np.zeros(c, np.int32)
    N = np.zeros(c, np.uint8)
    for i, (p, k) in enumerate(zip(perms, n)):
        b, o, e = oracle.perm_to_pair(p[:k].tolist())
        beta[i, : k + 1] = b
        omega[i, : k + 1] = o
        init[i] = e
        N[i] = k + 1
    return beta, omega, init, N


def _oracle_batch(oracle, beta, omega, N, init, rate, maxd, full):
    c = len(N)
    return oracle.search_batch(beta, omega, N, init, np.broadcast_to(rate, (c,)).astype(np.float32),
                               np.broadcast_to(maxd, (c,)).astype(np.int32),
                               np.broadcast_to(full, (c,)).astype(np.uint8), os.cpu_count() or 8)


def _keeps_filter(oracle, beta, omega, moves):
    """Every move keeps the reference's move filter: it touches no symbol that
    omega fixes and changes the odd-cycle count by 0 or +2
    (sorting_search.cu:240-332, 375-380)."""
    beta, omega = list(beta), list(omega)
    odd = oracle.count_odd_cycles(omega)
    for (i, j, k) in moves:
        a, b, c = beta[i], beta[j], beta[k]
        if omega[a] == a or omega[b] == b or omega[c] == c:
            return False
        nxt = list(omega)
        nxt[a], nxt[b], nxt[c] = omega[c], omega[a], omega[b]
        d = oracle.count_odd_cycles(nxt) - odd
        if d not in (0, 2):
            return False
        odd += d
        omega = nxt
        beta = beta[:i] + beta[j:k] + beta[i:j] + beta[k:]
    return True


def _replay_all(oracle, beta, omega, N, res, maxd):
    """Every witness replays in the checker and keeps the reference's move
    filter (witnesses found on an inverse's side included)."""
    for i in np.nonzero(res["status"] == 1)[0]:
        k = int(N[i])
        moves = [(int(m) & 31, (int(m) >> 5) & 31, (int(m) >> 10) & 31) for m in res["moves"][i][: res["depth"][i]]]
        abc = oracle.positions_to_symbols(beta[i, :k].tolist(), moves)
        err = oracle.validate(beta[i, :k].tolist(), omega[i, :k].tolist(), abc, int(np.broadcast_to(maxd, (len(N),))[i]))
        assert err is None, (i, err)
        assert _keeps_filter(oracle, beta[i, :k].tolist(), omega[i, :k].tolist(), moves), (i, moves)


def test_smoke_concurrent_three_cycles_through_the_slot_queue(td):
    """GPUSortingSearchSmokeTest: 2 slots, 32 MiB, 32 concurrent N=3 searches."""
    td.GPUSortingSearch.init([0], 2, 32 * MiB, queue_capacity=0)
    try:
        inst = td.GPUSortingSearch.get_instance()
        with cf.ThreadPoolExecutor(32) as ex:
            futs = [ex.submit(inst.search, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 1, True) for _ in range(32)]
            for f in futs:
                assert f.result() == [(0, 1, 2)]
        snap = inst.stats.snapshot(__import__("time").monotonic_ns())
        assert snap.completed == 32 and snap.failed == 0
    finally:
        td.GPUSortingSearch.shutdown()


def test_config1_exact_distance_and_ordered_witnesses(slots, oracle):
    """4096 x S_10 from seed 0: deepening the bound gives the exact restricted
    distance; each witness is the reference single-queue witness."""
    td = slots
    perms, n = td.synth_perms(0, 4096, 10, 10, 0, 0, 0)
    beta, omega, init, N = _pairs(oracle, perms, n)
    dist_gpu = np.full(4096, -1)
    dist_ora = np.full(4096, -1)
    for d in range(1, 7):
        inst = td.prepare_pairs(beta, omega, N, init, 0.0, d, 1)
        res, _ = td.search_batch(0, inst, ORDERED)
        st, dep, mv, ex = _oracle_batch(oracle, beta, omega, N, init, 0.0, d, 1)
        assert (res["status"] == st).all()
        assert (res["depth"] == dep).all()
        assert (res["moves"] == mv).all()
        assert (res["expansions"] == ex + 1).all()
        dist_gpu[(dist_gpu < 0) & (res["status"] == 1)] = d
        dist_ora[(dist_ora < 0) & (st == 1)] = d
    assert (dist_gpu == dist_ora).all() and dist_gpu.max() == 6 and (dist_gpu > 0).all()


def test_ordered_general_pairs_rates_and_partial_sorting(slots, oracle):
    td = slots
    rng = np.random.default_rng(7)
    c = 1500
    perms, n = td.synth_perms(11, c, 4, 11, 20, 1, 3)
    beta, omega, init, N = _pairs(oracle, perms, n)
    for i in range(c):  # rotate the caller's array to exercise betaStart
        k = int(N[i])
        r = int(rng.integers(k))
        beta[i, :k] = np.roll(beta[i, :k], -r)
    maxd = rng.integers(1, 7, c).astype(np.int32)
    rate = rng.choice([0.0, 1.0, 1.5, 2.0], c).astype(np.float32)
    full = (rng.random(c) < 0.7).astype(np.uint8)
    init_pass = np.where(full == 1, init, np.maximum(0, init - rng.integers(0, 2, c))).astype(np.int32)
    inst = td.prepare_pairs(beta, omega, N, init_pass, rate, maxd, full)
    res, _ = td.search_batch(1, inst, ORDERED)
    st, dep, mv, ex = _oracle_batch(oracle, beta, omega, N, init_pass, rate, maxd, full)
    assert (res["status"] == st).all()
    assert (res["depth"] == dep).all() and (res["moves"] == mv).all()
    assert (res["expansions"] == np.where(N >= 3, ex + 1, 0)).all()


def test_split_ordered_search_matches_the_one_warp_walk(slots, oracle):
    """The reference order's split pass (searches that outlast the one-warp
    budget are split into the subtrees of their root's children, searched at
    once and joined in rank order): 8,192 n = 12 instances, half near-reverse,
    at bounds 5 and 6 (both verdicts, over 1,000 walks split at bound 6).
    Status, depth, witness and expansion count equal the oracle's walk and the
    unsplit one-warp launch (a nonzero expansion budget keeps a batch
    unsplit), record for record; also with a record space too small for most
    roots (those walks run whole) and with the split off."""
    td = slots
    perms, n = td.synth_perms(7, 8192, 12, 12, 50, 1, 3)
    beta, omega, init, N = _pairs(oracle, perms, n)
    for d, hard in ((5, 1), (6, 1000)):
        inst = td.prepare_pairs(beta, omega, N, init, 0.0, d, 1)
        res, _ = td.search_batch(0, inst, ORDERED)
        whole, _ = td.search_batch(1, inst, ORDERED, max_expansions=1 << 40)
        st, dep, mv, ex = _oracle_batch(oracle, beta, omega, N, init, 0.0, d, 1)
        assert (ex + 1 > 128).sum() >= hard
        assert (st == 1).any() and (st == 0).any()
        assert (res["status"] == st).all()
        assert (res["depth"] == dep).all() and (res["moves"] == mv).all()
        assert (res["expansions"] == ex + 1).all()
        for key in ("status", "depth", "moves", "expansions"):
            assert (whole[key] == res[key]).all(), key
    # a record space too small for most roots: those walks run whole; and no split
    inst = td.prepare_pairs(beta[:4096], omega[:4096], N[:4096], init[:4096], 0.0, 6, 1)
    ref, _ = td.search_batch(0, inst, ORDERED)
    try:
        for budget, records in ((64, 300), (0, 1)):
            td._lib.configure_split(budget, records)
            got, _ = td.search_batch(0, inst, ORDERED)
            for key in ("status", "depth", "moves", "expansions"):
                assert (got[key] == ref[key]).all(), (budget, key)
    finally:
        td._lib.configure_split()


def test_config2_mix_free_order_verdicts_and_replay(slots, oracle):
    """Sample of the batched uneven mix: n in {11,12,13}, 25% near-reverse,
    bound floor(n/2)+1.  Verdicts equal the oracle's; every witness replays."""
    td = slots
    perms, n = td.synth_perms(1, 4096, 11, 13, 25, 1, 3)
    beta, omega, init, N = _pairs(oracle, perms, n)
    maxd = (n // 2 + 1).astype(np.int32)
    inst = td.prepare_pairs(beta, omega, N, init, 0.0, maxd, 1)
    res, stats = td.search_batch(0, inst, 0)
    st, _, _, _ = _oracle_batch(oracle, beta, omega, N, init, 0.0, maxd, 1)
    assert (res["status"] == st).all()
    assert stats.found + stats.not_found == 4096 and stats.errors == 0
    _replay_all(oracle, beta, omega, N, res, maxd)
    res_p, _ = td.search_batch(0, inst, PLAIN)
    assert (res_p["status"] == res["status"]).all()


def test_config3_s16_witnesses_replay_and_verdict_sample(slots, oracle):
    """S_16, bound 9, half uniform and half near-reverse."""
    td = slots
    perms, n = td.synth_perms(2, 1 << 14, 16, 16, 50, 1, 4)
    inst = td.prepare_perms(perms, n, 9)
    res, stats = td.search_batch(0, inst, 0)
    assert stats.errors == 0
    beta, omega, init, N = _pairs(oracle, perms[:192], n[:192])
    st, _, _, _ = _oracle_batch(oracle, beta, omega, N, init, 0.0, 9, 1)
    assert (res["status"][:192] == st).all()
    sample = np.arange(0, 1 << 14, 7)
    b2, o2, _, N2 = _pairs(oracle, perms[sample], n[sample])
    _replay_all(oracle, b2, o2, N2, res[sample], 9)


def test_device_entry_points_with_validator(slots):
    import torch
    td = slots
    perms, n = td.synth_perms(2, 8192, 16, 16, 50, 1, 4)
    inst = td.prepare_perms(perms, n, 9)
    d_in = torch.from_numpy(inst.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(8192 * 32, dtype=torch.uint8, device="cuda")
    d_ok = torch.zeros(8192, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    td._lib.search_batch_device(0, 8192, d_in.data_ptr(), d_out.data_ptr(), 0, 0, stream)
    td._lib.validate_batch_device(8192, d_in.data_ptr(), d_out.data_ptr(), d_ok.data_ptr(), stream)
    torch.cuda.synchronize()
    res = d_out.cpu().numpy().view(td.RESULT_DTYPE)
    ok = d_ok.cpu().numpy()
    assert ((res["status"] == 1) == (ok == 1)).all()
    host_res, _ = td.search_batch(0, inst, 0)
    assert (host_res["status"] == res["status"]).all()


def test_edge_cases(slots):
    td = slots
    assert td.search(0, b"", b"", 0, 0.0, 1) == []
    assert td.search(0, bytes([0, 1]), bytes([1, 0]), 0, 0.0, 1) == []
    assert td.search(0, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 1, ordered=True) == [(0, 1, 2)]
    # identity omega: every symbol fixed, no move applies
    assert td.search(0, bytes([0, 1, 2, 3]), bytes([0, 1, 2, 3]), 4, 0.0, 3) == []
    for bad in (dict(max_moves=0), dict(max_moves=10)):
        with pytest.raises(td.TdError):
            td.search(0, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, bad["max_moves"])
    with pytest.raises(td.TdError):
        td.search(0, bytes(range(18)), bytes(range(18)), 0, 0.0, 1)
    with pytest.raises(td.TdError):
        td.search(5, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 1)
    with pytest.raises(td.TdError):
        td.search(0, bytes([0, 1, 1]), bytes([1, 2, 0]), 1, 2.0, 1)
    # a work budget that is too small reports the reference's overflow class
    perms, n = td.synth_perms(2, 64, 16, 16, 100, 1, 1)
    inst = td.prepare_perms(perms, n, 9)
    res, _ = td.search_batch(0, inst, ORDERED, max_expansions=2)
    assert (res["status"] == -2).any()


def test_work_donation_keeps_verdicts_and_witnesses(slots, oracle):
    """Hard n=13 instances at bound 7 (several exhaust their tree): with
    donation forced at every expansion, verdicts equal the one-warp-per-
    instance form and the oracle, and every witness replays."""
    td = slots
    perms, n = td.synth_perms(5, 2048, 13, 13, 100, 1, 3)
    inst = td.prepare_perms(perms, n, 7)
    td._lib.configure_steal(4, 6, 1)
    try:
        res, st = td.search_batch(0, inst, 0)
        res2, st2 = td.search_batch(0, inst, 0)
    finally:
        _library_defaults(td)
    assert st.donations > 0 and st.donated_items >= st.donations
    plain, _ = td.search_batch(0, inst, PLAIN)
    assert (res["status"] == plain["status"]).all() and (res2["status"] == plain["status"]).all()
    assert st.errors == 0 and (res["status"] == 0).any()
    beta, omega, init, N = _pairs(oracle, perms[:256], n[:256])
    ost, _, _, _ = _oracle_batch(oracle, beta, omega, N, init, 0.0, 7, 1)
    assert (res["status"][:256] == ost).all()
    b2, o2, _, N2 = _pairs(oracle, perms, n)
    _replay_all(oracle, b2, o2, N2, res, 7)
    # expansions of a shared search are summed over every warp that took part
    assert res["expansions"].sum() > 0


def test_cuda_graph_replays_match_eager_launches(slots):
    import torch
    td = slots
    perms, n = td.synth_perms(6, 4096, 13, 13, 60, 1, 3)
    inst = td.prepare_perms(perms, n, 7)
    eager, _ = td.search_batch(0, inst, 0)
    d_in = torch.from_numpy(inst.view(np.uint8).copy()).cuda()
    d_out = torch.zeros(4096 * 32, dtype=torch.uint8, device="cuda")
    g = td._lib.BatchGraph(0, 4096, d_in.data_ptr(), d_out.data_ptr(), td._lib.FLAG_VERIFY)
    try:
        stream = td._lib.lib().td_slot_stream(0)
        for _ in range(3):
            d_out.zero_()
            torch.cuda.synchronize()
            g.launch(stream)
            torch.cuda.synchronize()
            res = d_out.cpu().numpy().view(td.RESULT_DTYPE)
            assert (res["status"] == eager["status"]).all()  # -6 would mark a witness failing replay
    finally:
        g.close()


def test_explored_state_tables_keep_verdicts(slots, oracle):
    """Free order with and without the per-warp tables of explored states, on
    hard n = 12..13 instances at their bound (several end without a witness):
    identical verdicts, equal to the oracle's on a sample, and every witness
    replays; the tables cut expansions."""
    td = slots
    perms, n = td.synth_perms(8, 4096, 12, 13, 100, 1, 3)
    maxd = (n // 2 + 1).astype(np.int32)
    inst = td.prepare_perms(perms, n, maxd)
    try:
        td._lib.configure_table(0)
        plain, st0 = td.search_batch(0, inst, 0)
        td._lib.configure_table(12)
        tabled, st1 = td.search_batch(0, inst, 0)
        # expansion counts depend on which subtrees are donated, and when; with
        # idle checks too rare to fire, every search stays on one warp and its
        # count is fixed, so the tables' saving is compared there
        td._lib.configure_steal(4, 2, 1 << 24)
        td._lib.configure_table(0)
        solo0, _ = td.search_batch(0, inst, 0)
        td._lib.configure_table(12)
        solo1, _ = td.search_batch(0, inst, 0)
    finally:
        _library_defaults(td)
    assert (plain["status"] == tabled["status"]).all() and st0.errors == st1.errors == 0
    assert (solo0["status"] == plain["status"]).all() and (solo1["status"] == plain["status"]).all()
    e0 = solo0["expansions"].astype(np.int64)
    e1 = solo1["expansions"].astype(np.int64)
    assert e1.sum() < e0.sum()
    beta, omega, init, N = _pairs(oracle, perms[:200], n[:200])
    ost, _, _, _ = _oracle_batch(oracle, beta, omega, N, init, 0.0, maxd[:200], 1)
    assert (tabled["status"][:200] == ost).all()
    b2, o2, _, N2 = _pairs(oracle, perms, n)
    _replay_all(oracle, b2, o2, N2, tabled, maxd)


def test_restarts_keep_verdicts(slots, oracle):
    """Free-order restarts (another child order after 16 x Luby expansions,
    many per search here) against none: identical verdicts on hard S_16 at
    bound 9 and n = 13 at bound 6 (many without a witness, searched to the
    end by the last attempt); every witness replays."""
    td = slots
    p1, n1 = td.synth_perms(3, 2048, 16, 16, 100, 1, 4)
    p2, n2 = td.synth_perms(5, 2048, 13, 13, 100, 1, 3)
    sets = [(p1, n1, 9), (p2, n2, 6)]
    try:
        for perms, n, maxd in sets:
            inst = td.prepare_perms(perms, n, maxd)
            td._lib.configure_restart(0)
            plain, _ = td.search_batch(0, inst, 0)
            td._lib.configure_restart(16)
            restarted, st = td.search_batch(0, inst, 0)
            assert (plain["status"] == restarted["status"]).all() and st.errors == 0
            b, o, _, N = _pairs(oracle, perms, n)
            _replay_all(oracle, b, o, N, restarted, maxd)
        assert (plain["status"] == 0).any()
    finally:
        _library_defaults(td)


def test_batch_stats_match_the_results(slots):
    """td_batch_stats totals (reduced on the device) equal the sums over the
    returned records, in every launch form, with and without per-instance
    budget errors."""
    td = slots
    perms, n = td.synth_perms(11, 3000, 9, 13, 50, 1, 3)
    inst = td.prepare_perms(perms, n, (n // 2 + 1).astype(np.int32))
    for flags, budget in ((0, 0), (ORDERED, 0), (PLAIN, 0), (0, 2), (ORDERED, 2)):
        res, st = td.search_batch(1, inst, flags, max_expansions=budget)
        status = res["status"]
        assert st.found == int((status == 1).sum())
        assert st.not_found == int((status == 0).sum())
        assert st.errors == int(((status != 0) & (status != 1)).sum())
        assert st.expansions == int(res["expansions"].astype(np.uint64).sum())
        if budget:
            assert st.errors > 0
    empty, st = td.search_batch(1, inst[:0], 0)
    assert len(empty) == 0 and st.found == st.not_found == st.errors == st.expansions == 0


def test_inverse_race_keeps_verdicts_and_witnesses(slots, oracle):
    """Free-order batches race a search that reaches a given restart attempt
    against a search of its inverse permutation (td_configure_race).  With and
    without the race: identical verdicts on hard S_16 at bound 9, on hard
    n = 13 at bound 6 and on the n = 11..13 mix one below its bound (the last
    two with many instances that have no witness, which the instance's own
    search decides); the oracle's verdicts on a sample; and every witness,
    many of them found on the inverse's side and converted, replays on the
    device (TD_FLAG_VERIFY) and in the oracle and keeps the reference's move
    filter (a converted witness that leaves it is dropped, and the instance's
    own search decides)."""
    td = slots
    p1, n1 = td.synth_perms(3, 2048, 16, 16, 100, 1, 4)
    p2, n2 = td.synth_perms(5, 2048, 13, 13, 100, 1, 3)
    p3, n3 = td.synth_perms(1, 4096, 11, 13, 25, 1, 3)
    sets = [(p1, n1, np.full(len(n1), 9, np.int32)), (p2, n2, np.full(len(n2), 6, np.int32)),
            (p3, n3, (n3 // 2).astype(np.int32))]
    try:
        for perms, n, maxd in sets:
            inst = td.prepare_perms(perms, n, maxd)
            td._lib.configure_race(0)
            plain, st0 = td.search_batch(0, inst, 0)
            # from the first restart on: the most races, and so the most
            # witnesses found on the inverse's side
            td._lib.configure_race(1)
            raced, st1 = td.search_batch(0, inst, td._lib.FLAG_VERIFY)
            assert st0.races == 0 and st1.races > 0
            assert st0.errors == 0 and st1.errors == 0  # a witness failing the device replay would be -6
            assert (plain["status"] == raced["status"]).all()
            b, o, init, N = _pairs(oracle, perms[:256], n[:256])
            ost, _, _, _ = _oracle_batch(oracle, b, o, N, init, 0.0, maxd[:256], 1)
            assert (raced["status"][:256] == ost).all()
            b, o, _, N = _pairs(oracle, perms, n)
            _replay_all(oracle, b, o, N, raced, maxd)
        assert (plain["status"] == 0).any() and (raced["status"] == 0).sum() == (plain["status"] == 0).sum()
    finally:
        _library_defaults(td)
