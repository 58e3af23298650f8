"""The engine's warp algorithm, emulated one lane at a time on the host,
against the oracle: identical witnesses and expansion counts in ordered mode,
identical verdicts with replayable witnesses in free order (bit-sliced
classification), and the bit-sliced classes equal to the 12-bit class table on
every triple."""
import ctypes as C
import random

import numpy as np
import pytest


class Inst(C.Structure):
    _fields_ = [("perm", C.c_uint64), ("min_rate", C.c_float), ("n_symbols", C.c_uint8),
                ("offset", C.c_uint8), ("max_moves", C.c_uint8), ("packed", C.c_uint8)]


class Res(C.Structure):
    _fields_ = [("status", C.c_int32), ("depth", C.c_int32), ("moves", C.c_uint16 * 9),
                ("reserved", C.c_uint16), ("expansions", C.c_uint32)]


def _u8(v):
    return (C.c_uint8 * 17)(*v)


def _prep(emu, beta, omega, init, rate, maxd, full):
    x = Inst()
    rc = emu.td_emu_prepare_pair(_u8(beta), _u8(omega), len(beta), init, C.c_float(rate), maxd, int(full),
                                 C.byref(x))
    assert rc == 0
    return x


def _run(emu, x, flags):
    r = Res()
    emu.td_emu_search(C.byref(x), flags, C.byref(r))
    return r, [(m & 31, (m >> 5) & 31, (m >> 10) & 31) for m in r.moves[: r.depth]]


def _cases(seed, count):
    rng = random.Random(seed)
    for _ in range(count):
        n = rng.randint(2, 9)
        pi = list(range(n))
        rng.shuffle(pi)
        if rng.random() < 0.25:
            pi = pi[::-1] if rng.random() < 0.5 else list(range(n))[::-1]
        yield rng, n, pi


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_ordered_mode_matches_oracle(oracle, emu, seed):
    for rng, n, pi in _cases(seed, 150):
        beta, omega, init = oracle.perm_to_pair(pi)
        N = n + 1
        r0 = rng.randrange(N)
        beta = beta[r0:] + beta[:r0]  # general pairs: the array may start anywhere
        full = rng.random() < 0.8
        maxd = rng.randint(1, 6)
        rate = rng.choice([0.0, 1.0, 1.5, 2.0])
        init_pass = init if full else max(0, init - rng.randint(0, 1))
        rc, mv, ex = oracle.search(beta, omega, init_pass, rate, maxd, full)
        x = _prep(emu, beta, omega, init_pass, rate, maxd, full)
        r, emv = _run(emu, x, 1)
        assert r.status == rc, (pi, beta, maxd)
        assert emv == mv, (pi, beta, maxd)
        assert r.expansions == (ex + 1 if N >= 3 else 0)


@pytest.mark.parametrize("seed", [3, 4])
def test_free_order_verdicts_and_replay(oracle, emu, seed):
    for rng, n, pi in _cases(seed, 150):
        beta, omega, init = oracle.perm_to_pair(pi)
        maxd = rng.randint(1, 6)
        rc, _, _ = oracle.search(beta, omega, init, 0.0, maxd, True)
        x = _prep(emu, beta, omega, init, 0.0, maxd, True)
        r, emv = _run(emu, x, 0)
        assert r.status == rc
        if rc == 1:
            abc = oracle.positions_to_symbols(beta, emv)
            assert oracle.validate(beta, omega, abc, maxd) is None


def test_bit_sliced_classes_match_class_table(emu):
    """td_row_classes over all k of a pair equals td_class_of_index on the
    pair-table entries of every triple, on random pinned states of S_2..S_16
    with the caller's array starting anywhere."""
    emu.td_emu_row_check.argtypes = [C.c_uint64, C.c_int, C.c_int]
    rng = random.Random(9)
    checked = 0
    for _ in range(3000):
        N = rng.randint(3, 17)
        perm = list(range(N - 1))
        rng.shuffle(perm)
        if rng.random() < 0.2:  # near-identity states have many fixed points
            perm = sorted(perm)
            a, b = sorted(rng.sample(range(N - 1), 2)) if N > 2 else (0, 0)
            perm[a], perm[b] = perm[b], perm[a]
        L = 0
        for m in range(16):
            L |= (perm[m] if m < N - 1 else m) << (4 * m)
        assert emu.td_emu_row_check(L, rng.randrange(N), N) == 0, (perm, N)
        checked += 1
    assert checked == 3000


@pytest.mark.parametrize("seed", [6])
def test_free_order_larger_instances(oracle, emu, seed):
    """Free order on n = 10..13 (several pair slots per lane), bound
    floor(n/2)+1 and one below it."""
    rng = random.Random(seed)
    for _ in range(24):
        n = rng.randint(10, 13)
        pi = list(range(n))
        rng.shuffle(pi)
        if rng.random() < 0.5:
            pi = list(range(n))[::-1]
            a, b = sorted(rng.sample(range(n), 2))
            pi[a], pi[b] = pi[b], pi[a]
        beta, omega, init = oracle.perm_to_pair(pi)
        maxd = n // 2 + 1 - rng.randint(0, 1)
        rc, _, _ = oracle.search(beta, omega, init, 0.0, maxd, True)
        x = _prep(emu, beta, omega, init, 0.0, maxd, True)
        r, emv = _run(emu, x, 0)
        assert r.status == rc, (pi, maxd)
        if rc == 1:
            abc = oracle.positions_to_symbols(beta, emv)
            assert oracle.validate(beta, omega, abc, maxd) is None


def test_pinned_move_matches_block_swap(oracle, emu):
    """td_apply_move on the pinned state equals the block swap of the caller's
    array, including the new array start when i == 0."""
    rng = random.Random(5)
    for _ in range(400):
        n = rng.randint(3, 17)
        N = n
        pi = list(range(n - 1))
        rng.shuffle(pi)
        beta, omega, init = oracle.perm_to_pair(pi)
        r0 = rng.randrange(N)
        beta = beta[r0:] + beta[:r0]
        x = _prep(emu, beta, omega, init, 0.0, 9, True)
        L, off = x.perm, x.offset
        cur = list(beta)
        B = [0] + [((L >> (4 * m)) & 15) + 1 for m in range(N - 1)]
        sigma = {a: B[(p + off) % N] for p, a in enumerate(cur)}  # the instance's fixed relabeling
        assert len(set(sigma.values())) == N
        for _ in range(4):
            i, j, k = sorted(rng.sample(range(N), 3))
            outL, outOff = C.c_uint64(), C.c_int()
            emu.td_emu_apply_move(C.c_uint64(L), off, N, i, j, k, C.byref(outL), C.byref(outOff))
            L, off = outL.value, outOff.value
            cur = cur[:i] + cur[j:k] + cur[i:j] + cur[k:]
            B = [0] + [((L >> (4 * m)) & 15) + 1 for m in range(N - 1)]
            assert [B[(p + off) % N] for p in range(N)] == [sigma[a] for a in cur]


def test_restarts_keep_verdicts_and_witnesses(oracle, emu):
    """Free order with restarts after 16 x Luby expansions (many restarts per
    search, each with another child order) against no restarts: the same
    verdicts on hard S_16 instances at bound 9 and n = 13 instances at bound 6
    (several of the latter have no witness within it, so the last, unbounded
    attempt must search the whole tree), and every witness replays."""
    import td16_b200 as td
    emu.td_emu_set_restart.argtypes = [C.c_uint32]
    cases = []
    for seed, count, lo, hi, maxd in ((3, 24, 16, 16, 9), (5, 48, 13, 13, 6)):
        perms, n = td.synth_perms(seed, count, lo, hi, 100, 1, 3)
        for p, k in zip(perms, n):
            cases.append((p[:k].tolist(), maxd))
    statuses = {}
    try:
        for base in (0, 16):
            emu.td_emu_set_restart(base)
            out = []
            for pi, maxd in cases:
                beta, omega, init = oracle.perm_to_pair(pi)
                x = _prep(emu, beta, omega, init, 0.0, maxd, True)
                r, moves = _run(emu, x, 0)
                if r.status == 1:
                    abc = oracle.positions_to_symbols(beta, moves)
                    assert oracle.validate(beta, omega, abc, maxd) is None
                out.append(r.status)
            statuses[base] = out
    finally:
        emu.td_emu_set_restart(200)
    assert statuses[0] == statuses[16]
    assert 0 in statuses[0] and 1 in statuses[0]


def test_restart_schedule(emu):
    """The restart rule of td_core.cuh: Luby budgets, the first attempt in the
    plain order, and the unbounded attempt after the budgeted ones in the
    plain order too (the best single order for the long searches that get
    that far); the attempts in between use distinct orders."""
    R = emu.td_emu_restarts()
    emu.td_emu_budget.restype = C.c_uint32
    emu.td_emu_order.restype = C.c_uint32
    luby = [1, 1, 2, 1, 1, 2, 4, 1, 1, 2, 1, 1, 2, 4, 8, 1]
    assert [emu.td_emu_budget(16, a) for a in range(16)] == [16 * v for v in luby]
    assert emu.td_emu_budget(16, R) == 0xFFFFFFFF and emu.td_emu_budget(0, 0) == 0xFFFFFFFF
    for level in range(10):
        assert emu.td_emu_order(0, level) == 0
        assert emu.td_emu_order(R, level) == 0
    first_orders = {emu.td_emu_order(a, 0) for a in range(R)}
    assert len(first_orders) == R  # one order per budgeted attempt at the root


@pytest.mark.parametrize("seed", [11, 12])
def test_inverse_instance_gives_the_verdict_and_a_replayable_witness(oracle, emu, seed):
    """The race of a search against the search of its inverse (td_steal_kernel)
    rests on three facts, checked here with full sorting on pairs whose array
    starts anywhere: the inverse instance (td_inverse_pinned, offset 0) has the
    same odd-cycle count; searching it gives the oracle's verdict on the
    original pair; and td_witness_from_inverse turns its witness into one that
    the oracle's replay accepts on the original pair, with the same length."""
    emu.td_emu_pinned_cycles.argtypes = [C.c_uint64, C.c_int, C.c_int]
    rng = random.Random(seed)
    found = 0
    for _ in range(300):
        n = rng.randint(2, 12)
        pi = list(range(n))
        rng.shuffle(pi)
        if rng.random() < 0.3:
            pi = list(range(n))[::-1]
            for _ in range(rng.randint(0, 2)):
                a, b = sorted(rng.sample(range(n), 2)) if n > 1 else (0, 0)
                pi[a], pi[b] = pi[b], pi[a]
        beta, omega, init = oracle.perm_to_pair(pi)
        N = n + 1
        r0 = rng.randrange(N)
        beta = beta[r0:] + beta[:r0]
        maxd = rng.randint(1, 7 if n <= 9 else 6)
        rate = rng.choice([0.0, 0.0, 1.0, 1.5])
        rc, _, _ = oracle.search(beta, omega, init, rate, maxd, True)
        x = _prep(emu, beta, omega, init, rate, maxd, True)
        xi = Inst()
        emu.td_emu_inverse_instance(C.byref(x), C.byref(xi))
        assert xi.offset == 0 and xi.packed == x.packed
        assert emu.td_emu_pinned_cycles(xi.perm, 0, N) == emu.td_emu_pinned_cycles(x.perm, x.offset, N) == init
        ri, _ = _run(emu, xi, 0)
        assert ri.status == rc, (pi, r0, maxd, rate)
        if rc != 1:
            continue
        r = Res()
        assert emu.td_emu_witness_from_inverse(C.byref(x), C.byref(ri), C.byref(r)) == 1
        assert r.depth == ri.depth and emu.td_emu_witness_ok(C.byref(x), C.byref(r)) == 1
        moves = [(m & 31, (m >> 5) & 31, (m >> 10) & 31) for m in r.moves[: r.depth]]
        abc = oracle.positions_to_symbols(beta, moves)
        assert oracle.validate(beta, omega, abc, maxd) is None, (pi, r0, moves)
        found += 1
    assert found > 100


def test_inverse_witness_on_s16(oracle, emu):
    """The same on benchmark-shaped S_16 instances at bound 9 (half
    near-reverse): every inverse-side witness converts and replays."""
    perms, n = oracle.synth_perms(7, 64, 16, 16, 50, 1, 4)
    for p in perms:
        beta, omega, init = oracle.perm_to_pair(p[:16].tolist())
        x = _prep(emu, beta, omega, init, 0.0, 9, True)
        xi = Inst()
        emu.td_emu_inverse_instance(C.byref(x), C.byref(xi))
        ri, _ = _run(emu, xi, 0)
        assert ri.status == 1
        r = Res()
        assert emu.td_emu_witness_from_inverse(C.byref(x), C.byref(ri), C.byref(r)) == 1
        moves = [(m & 31, (m >> 5) & 31, (m >> 10) & 31) for m in r.moves[: r.depth]]
        assert oracle.validate(beta, omega, oracle.positions_to_symbols(beta, moves), 9) is None


def _keeps_move_filter(oracle, beta, omega, moves):
    """The reference's move filter along a witness: no move touches a symbol
    that omega fixes, and each changes the odd-cycle count by 0 or +2
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


def test_converted_witnesses_replay_but_may_leave_the_move_filter(oracle, emu):
    """Why the race checks every converted witness against the move filter on
    the instance's side (td_filtered_witness) before recording it: on
    near-reverse S_16 at bound 9, every witness of the inverse instance,
    converted, replays in the checker, yet some take a -2 move or touch a
    fixed symbol, which the reference's search never does.  The engine's own
    free-order witnesses always keep the filter."""
    perms, n = oracle.synth_perms(2, 600, 16, 16, 100, 1, 4)
    left = 0
    for p in perms:
        beta, omega, init = oracle.perm_to_pair(p[:16].tolist())
        x = _prep(emu, beta, omega, init, 0.0, 9, True)
        r0, own = _run(emu, x, 0)
        assert r0.status == 1 and _keeps_move_filter(oracle, beta, omega, own)
        xi = Inst()
        emu.td_emu_inverse_instance(C.byref(x), C.byref(xi))
        ri, _ = _run(emu, xi, 0)
        r = Res()
        assert emu.td_emu_witness_from_inverse(C.byref(x), C.byref(ri), C.byref(r)) == 1
        moves = [(m & 31, (m >> 5) & 31, (m >> 10) & 31) for m in r.moves[: r.depth]]
        assert oracle.validate(beta, omega, oracle.positions_to_symbols(beta, moves), 9) is None
        left += not _keeps_move_filter(oracle, beta, omega, moves)
    assert 0 < left < len(perms) // 10
