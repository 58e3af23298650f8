"""Certificate format and replay: the library against the oracle."""
import os
import random

import numpy as np
import pytest


def test_codec_matches_oracle_and_reference_fixture(td, oracle):
    import json
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))["codec_n3"]
    assert td._lib.codec_key(bytes(g["omega"])).hex() == g["key_hex"]
    assert td._lib.codec_value([tuple(g["moves"][0])]).hex() == g["value_hex"]
    rng = random.Random(3)
    for _ in range(300):
        n = rng.randint(1, 17)
        omega = list(range(n))
        rng.shuffle(omega)
        key = td._lib.codec_key(bytes(omega))
        assert key == oracle.codec_key(omega)
        assert td._lib.codec_decode_key(key, n) == omega
        moves = [tuple(rng.randrange(17) for _ in range(3)) for _ in range(rng.randint(1, 9))]
        val = td._lib.codec_value(moves)
        assert val == oracle.codec_value(moves)
        assert td._lib.codec_decode_value(val) == moves
    for bad in (b"\x00", b""):
        with pytest.raises(td.TdError):
            td._lib.codec_decode_value(bad)
    with pytest.raises(td.TdError):
        td._lib.codec_decode_value(bytes([0x00, 0x45]))  # nonzero padding bit


def test_writer_round_trip(td, tmp_path):
    path = str(tmp_path / "certs.bin")
    w = td._lib.CertificateWriter(path, 0.05)
    recs = [([1, 2, 0], [(0, 1, 2)]), ([3, 4, 0, 1, 2], [(0, 3, 4), (0, 1, 2), (1, 2, 4)])]
    for omega, moves in recs:
        w.enqueue(bytes(omega), moves)
    assert w.close() == 2
    back = td._lib.read_certificates(path)
    assert [(td._lib.codec_decode_key(k, len(o)), td._lib.codec_decode_value(v)) for (k, v), (o, _) in
            zip(back, recs)] == [(o, m) for o, m in recs]


@pytest.mark.gpu
def test_device_symbol_replay_matches_oracle(td, oracle):
    import torch
    rng = random.Random(9)
    cases = []
    perms, n = td.synth_perms(21, 600, 5, 12, 30, 1, 3)
    td.init_slots(1, [0], 64 << 20)
    try:
        inst = td.prepare_perms(perms, n, 7)
        res, _ = td.search_batch(0, inst, 0)
    finally:
        td.destroy()
    for i in range(600):
        beta, omega, _ = oracle.perm_to_pair(perms[i, : n[i]].tolist())
        moves = td.unpack_moves(res[i])
        abc = oracle.positions_to_symbols(beta, moves) if moves else [(0, 1, 2)]
        if rng.random() < 0.4:  # corrupt some witnesses
            k = rng.randrange(len(abc))
            a = list(abc[k])
            a[rng.randrange(3)] = rng.randrange(len(beta))
            abc[k] = tuple(a)
        cases.append((beta, omega, abc, 7 if rng.random() < 0.9 else max(0, len(abc) - 1)))
    c = len(cases)
    B = np.zeros((c, 17), np.uint8)
    O = np.zeros((c, 17), np.uint8)
    A = np.zeros((c, 27), np.uint8)
    N = np.zeros(c, np.uint8)
    M = np.zeros(c, np.uint8)
    D = np.zeros(c, np.uint8)
    for i, (b, o, abc, mm) in enumerate(cases):
        B[i, : len(b)] = b
        O[i, : len(o)] = o
        N[i], M[i], D[i] = len(b), mm, len(abc)
        A[i, : 3 * len(abc)] = [v for m in abc for v in m]
    dev = [torch.from_numpy(x).cuda() for x in (B, O, N, M, D, A)]
    ok = torch.zeros(c, dtype=torch.uint8, device="cuda")
    import ctypes as C
    err = C.create_string_buffer(256)
    rc = td._lib.lib().td_replay_symbols_device(c, *[C.c_void_p(t.data_ptr()) for t in dev], C.c_void_p(ok.data_ptr()),
                                               None, err, 256)
    assert rc == 0
    got = ok.cpu().numpy()
    want = [oracle.validate(b, o, abc, mm) is None for b, o, abc, mm in cases]
    assert got.tolist() == [int(w) for w in want]
    assert 0 < sum(want) < c


@pytest.mark.gpu
def test_emitter_shaped_run_replays_every_certificate(td, tmp_path):
    from td16_b200 import emitter_run
    out = str(tmp_path / "certs.bin")
    r = emitter_run.run(count=20000, slots=4, budget=256 << 20, batch=4096, out_path=out, seed=4)
    assert r["errors"] == 0 and r["found"] + r["not_found"] == 20000
    assert r["certificates"] == r["found"] and r["replay"]["records"] == r["found"]
    assert r["replay"]["accepted"] == r["replay"]["records"]
