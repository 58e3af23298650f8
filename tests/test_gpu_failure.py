"""Failure detection without a GPU fault: every device wait is bounded and
ends with a status the host reads; the context stays usable afterwards."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_expired_deadline_reports_timeout_and_context_survives(td):
    td.init_slots(1, [0], 64 << 20)
    try:
        # unsolvable-heavy batch (n=13, bound 7) that runs for much longer
        # than the deadline set here
        perms, n = td.synth_perms(5, 8192, 13, 13, 100, 1, 3)
        inst = td.prepare_perms(perms, n, 7)
        td._lib.set_time_limit(0.002)
        for flags in (0, td._lib.FLAG_ORDERED):
            try:
                res, st = td.search_batch(0, inst, flags)
                timed_out = (res["status"] == -5).any()
            except td.TdError as e:
                assert e.code == td._lib.TIMEOUT
                timed_out = True
            assert timed_out
    finally:
        td._lib.set_time_limit(float(os.environ.get("TD16_TIME_LIMIT_S", 300)))
    try:
        # the same context still answers correctly
        assert td.search(0, bytes([0, 1, 2]), bytes([1, 2, 0]), 1, 2.0, 1) == [(0, 1, 2)]
        res, st = td.search_batch(0, inst[:256], 0)
        assert st.errors == 0
    finally:
        td.destroy()


def test_budget_exhaustion_is_reported_per_instance(td):
    td.init_slots(1, [0], 64 << 20)
    try:
        perms, n = td.synth_perms(2, 512, 16, 16, 100, 1, 4)
        inst = td.prepare_perms(perms, n, 9)
        for flags in (td._lib.FLAG_ORDERED, 0):  # reference order; free order (per unit of work)
            res, _ = td.search_batch(0, inst, flags, max_expansions=3)
            assert set(np.unique(res["status"]).tolist()) <= {-2, 1}
            assert (res["status"] == -2).any()
        # without a budget the same batch has no errors
        res, _ = td.search_batch(0, inst, 0)
        assert (res["status"] == 1).all()
    finally:
        td.destroy()
