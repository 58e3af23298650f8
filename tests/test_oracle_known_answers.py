"""Pins the CPU oracle to the reference's own known answers (tests/golden/known_answers.json)."""
import itertools
import json
import os

import numpy as np
import pytest

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def test_smoke_three_cycle(oracle):
    g = GOLD["smoke_n3"]
    rc, moves, _ = oracle.search(g["beta"], g["omega"], g["initial_even_cycles"], g["min_rate"],
                                 g["max_moves"], g["full_sorting"])
    assert rc == oracle.FOUND
    assert [list(m) for m in moves] == g["positions"]
    assert [list(m) for m in oracle.positions_to_symbols(g["beta"], moves)] == g["symbols"]


def test_apply_transposition(oracle):
    g = GOLD["apply_transposition"]
    out = oracle.apply_transposition(g["beta"], *g["move"])
    # equal as cycles: rotate to the result's first symbol
    r = g["result_cycle"]
    k = out.index(r[0])
    assert out[k:] + out[:k] == r


def test_compute_product(oracle):
    g = GOLD["compute_product"]
    p = oracle.cycle_oneline(g["p_cycle"], g["n"])
    q = oracle.cycle_oneline(g["q_cycle"], g["n"])
    assert oracle.compose(p, q) == oracle.cycle_oneline(g["result_cycle"], g["n"])
    g2 = GOLD["product_with_inverse"]
    c = oracle.cycle_oneline(g2["cycle"], g2["n"])
    inv = [0] * g2["n"]
    for x, y in enumerate(c):
        inv[y] = x
    assert oracle.compose(c, inv) == list(range(g2["n"]))


def test_codec_round_trip_and_rejections(oracle):
    g = GOLD["codec_n3"]
    key = oracle.codec_key(g["omega"])
    val = oracle.codec_value([tuple(m) for m in g["moves"]])
    assert len(key) == g["key_len"] and len(val) == g["value_len"]
    assert key.hex() == g["key_hex"] and val.hex() == g["value_hex"]
    assert oracle.codec_decode_key(key, 3) == g["omega"]
    assert [list(m) for m in oracle.codec_decode_value(val)] == g["moves"]
    assert oracle.validate(g["beta"], g["omega"], [tuple(m) for m in g["moves"]], 1) is None
    assert oracle.validate(g["beta"], g["omega"], [tuple(m) for m in g["reject_moves"]], 1) is not None
    assert oracle.validate(g["beta"], g["omega"], [tuple(m) for m in g["moves"]], 0) is not None
    with pytest.raises(ValueError):
        oracle.codec_decode_value(bytes(g["reject_value"]))
    # nonzero padding is rejected (CertificateCodec.java:120-129)
    with pytest.raises(ValueError):
        oracle.codec_decode_value(bytes([val[0], val[1] | 1]))


def test_odd_length_witness_replays(oracle):
    g = GOLD["odd_length_witness"]
    omega = oracle.cycle_oneline(g["omega_cycle"], g["n"])
    beta = list(range(g["n"]))
    assert oracle.validate(beta, omega, [tuple(m) for m in g["moves"]], 3) is None
    assert oracle.validate(beta, omega, [tuple(m) for m in g["moves"]], 2) is not None


def _restricted_distances(oracle, perms, n, max_d, threads=8):
    """Exact distance in the reference's move space by deepening the bound."""
    count = len(perms)
    beta = np.zeros((count, 17), np.uint8)
    omega = np.zeros((count, 17), np.uint8)
    init = np.zeros(count, np.int32)
    for i, p in enumerate(perms):
        b, o, e = oracle.perm_to_pair(p)
        beta[i, : n + 1] = b
        omega[i, : n + 1] = o
        init[i] = e
    dist = np.full(count, -1)
    dist[init == n + 1] = 0
    for d in range(1, max_d + 1):
        todo = np.nonzero(dist < 0)[0]
        if len(todo) == 0:
            break
        st, dep, mv, _ = oracle.search_batch(beta[todo], omega[todo], np.full(len(todo), n + 1),
                                             init[todo], np.zeros(len(todo)), np.full(len(todo), d),
                                             np.ones(len(todo)), threads)
        dist[todo[st == 1]] = d
    return dist


@pytest.mark.parametrize("n", [3, 4, 5, 6, 7])
def test_exhaustive_diameter_matches_known_values(oracle, n):
    """Largest restricted distance over all of S_n equals CommonOperations.d(n)."""
    perms = list(itertools.permutations(range(n)))
    dist = _restricted_distances(oracle, perms, n, 9)
    assert (dist >= 0).all()
    assert dist.max() == GOLD["diameters"]["d"][str(n)]


@pytest.mark.parametrize("n", range(3, 13))
def test_reverse_permutation_distance(oracle, n):
    dist = _restricted_distances(oracle, [list(range(n))[::-1]], n, 9, threads=1)
    assert dist[0] == n // 2 + 1
