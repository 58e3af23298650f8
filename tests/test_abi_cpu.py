"""C ABI and host model checks that need no GPU."""
import re
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(td):
    header = open(os.path.join(ROOT, "include", "td16_b200.h")).read()
    declared = set(re.findall(r"^\s*(?:int|void|long long|uint64_t)\s*\*?\s*(td_\w+)\(", header, re.M))
    assert {"td_init_slots", "td_search", "td_search_batch", "td_destroy"} <= declared
    lib = td._lib.lib()
    for name in sorted(declared):
        assert hasattr(lib, name), name


def test_synthetic_generator_is_seeded_and_shaped(td):
    p1, n1 = td.synth_perms(2, 512, 16, 16, 50, 1, 4)
    p2, n2 = td.synth_perms(2, 512, 16, 16, 50, 1, 4)
    assert (p1 == p2).all() and (n1 == n2).all() and (n1 == 16).all()
    for row in p1:
        assert sorted(row.tolist()) == list(range(16))
    p3, n3 = td.synth_perms(1, 4000, 11, 13, 25, 1, 3)
    assert set(np.unique(n3).tolist()) == {11, 12, 13}
    for row, n in zip(p3[:200], n3[:200]):
        assert sorted(row[:n].tolist()) == list(range(n)) and not row[n:].any()
    # index i draws from seed ^ i: a prefix does not depend on the count
    p4, _ = td.synth_perms(2, 7, 16, 16, 50, 1, 4)
    assert (p4 == p1[:7]).all()


def test_prepare_perms_matches_oracle_pairs(td, oracle):
    perms, n = td.synth_perms(0, 64, 10, 10, 0, 0, 0)
    inst = td.prepare_perms(perms, n, 6)
    for row, x in zip(perms, inst):
        beta, omega, init = oracle.perm_to_pair(row[:10].tolist())
        assert x["packed"] & 31 == init and x["packed"] >> 7 == 1
        assert x["n_symbols"] == 11 and x["offset"] == 0 and x["max_moves"] == 6
        # pinned permutation of S_n input pi is pi^-1
        inv = np.argsort(row[:10])
        L = int(x["perm"])
        assert [(L >> (4 * m)) & 15 for m in range(10)] == inv.tolist()


def test_prepare_rejects_invalid_pairs(td):
    beta = np.zeros((1, 17), np.uint8)
    omega = np.zeros((1, 17), np.uint8)
    beta[0, :3] = [0, 1, 1]
    omega[0, :3] = [1, 2, 0]
    with pytest.raises(td.TdError):
        td.prepare_pairs(beta, omega, 3, 1, 0.0, 1, 1)
    beta[0, :3] = [0, 1, 2]
    omega[0, :3] = [0, 1, 2]  # omega . beta = beta is a 3-cycle: valid
    td.prepare_pairs(beta, omega, 3, 3, 0.0, 1, 1)
    omega[0, :3] = [1, 0, 2]  # product is not a 3-cycle
    with pytest.raises(td.TdError):
        td.prepare_pairs(beta, omega, 3, 1, 0.0, 1, 1)
    omega[0, :3] = [1, 2, 0]
    with pytest.raises(td.TdError):
        td.prepare_pairs(beta, omega, 3, 1, 0.0, 10, 1)  # max_moves > 9


def test_positions_to_symbols(td, oracle):
    beta = [3, 0, 4, 1, 2]
    moves = [(0, 2, 4), (1, 2, 3)]
    assert td._lib.positions_to_symbols(bytes(beta), moves) == oracle.positions_to_symbols(beta, moves)


def test_device_layout_round_robin():
    from td16_b200.host import GpuDeviceLayout
    devices = GpuDeviceLayout.parse_devices(" 2, 5 ")
    layout = GpuDeviceLayout(devices, 3)
    assert layout.devices() == [2, 5] and layout.total_slots == 6
    assert [layout.device_for_slot(s) for s in (0, 1, 2, 5)] == [2, 5, 2, 5]
    for bad in (([0, 0], 7), ([-1], 7), ([0], 0)):
        with pytest.raises(ValueError):
            GpuDeviceLayout(*bad)
    for bad in ("0,,1", "gpu0", " "):
        with pytest.raises(ValueError):
            GpuDeviceLayout.parse_devices(bad)
    with pytest.raises(ValueError):
        layout.device_for_slot(6)


def test_search_stats_windows():
    from td16_b200.host import GpuDeviceLayout, GpuSearchStats
    stats = GpuSearchStats(GpuDeviceLayout([0, 1], 2), 0)
    stats.acquired(0, 5, 10)
    stats.acquired(1, 10, 20)
    stats.released(0, 60, False)
    first = stats.snapshot(100)
    assert (first.started, first.completed, first.failed) == (2, 1, 0)
    assert first.queue_wait_nanos == 15 and first.busy_nanos == 130
    assert first.devices[0].completed == 1 and first.devices[0].busy_nanos == 50
    assert first.devices[1].completed == 0 and first.devices[1].busy_nanos == 80
    stats.released(1, 180, True)
    second = stats.snapshot(200)
    assert (second.started, second.completed, second.failed, second.busy_nanos) == (0, 1, 1, 80)
    assert second.devices[0].busy_nanos == 0 and second.devices[1].busy_nanos == 80
    s2 = GpuSearchStats(GpuDeviceLayout([3], 1), 1000)
    s2.acquired(0, 1000, 1100)
    a, b = s2.snapshot(1500), s2.snapshot(1800)
    s2.released(0, 2000, False)
    c = s2.snapshot(2100)
    assert (a.busy_nanos, b.busy_nanos, c.busy_nanos, c.completed, c.started) == (400, 300, 200, 1, 0)
    assert c.latency_p50_ms == pytest.approx((2000 - 1000) / 1e6)


def test_configuration_arguments_are_checked(td):
    """The tuning entry points reject out-of-range values (no GPU needed) and
    leave the configuration unchanged when they do."""
    lib = td._lib.lib()
    INVALID = td._lib.INVALID_ARG
    for bits in (-1, 1, 5, 17, 40):
        assert lib.td_configure_table(bits) == INVALID
    for base in (-1, 1, 15):
        assert lib.td_configure_restart(base) == INVALID
    assert lib.td_configure_restart(0) == td._lib.OK
    assert lib.td_configure_restart(200) == td._lib.OK
    assert lib.td_configure_restart(16) == td._lib.OK  # the default
    for attempt in (-1, 33):
        assert lib.td_configure_race(attempt) == INVALID
    assert lib.td_configure_race(0) == td._lib.OK
    assert lib.td_configure_race(8) == td._lib.OK  # the default
    for args in ((0, 2, 32), (1, -1, 32), (1, 9, 32), (1, 2, 0)):
        assert lib.td_configure_serve(*args) == INVALID
        assert lib.td_configure_steal(*args) == INVALID
    # valid values (the defaults) are accepted
    assert lib.td_configure_table(12) == td._lib.OK
    assert lib.td_configure_table(0) == td._lib.OK
    assert lib.td_configure_table(12) == td._lib.OK
    assert lib.td_configure_serve(1, 2, 32) == td._lib.OK
    with pytest.raises(td.TdError):
        td._lib.configure_table(3)


def test_oracle_generator_matches_the_engine_bit_for_bit(td, oracle):
    """The oracle's restatement of the seeded generator (used where the engine
    library must not be loaded) gives the engine's td_synth_perms output."""
    for args in ((2, 1 << 15, 16, 16, 50, 1, 4), (1, 1 << 14, 11, 13, 25, 1, 3), (0, 4096, 10, 10, 0, 0, 0),
                 (3, 4096, 8, 16, 0, 0, 0), (7, 4096, 1, 16, 37, 0, 5), (9, 512, 16, 16, 100, 4, 4)):
        p_o, n_o = oracle.synth_perms(*args)
        p_t, n_t = td.synth_perms(*args)
        assert (p_o == p_t).all() and (n_o == n_t).all(), args
