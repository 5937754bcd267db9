"""The bounded device waits give up cleanly.

Every mbarrier wait in the tcgen05 subset-sum hash (ligesis_b200/csrc/hash_tc.cu) is bounded by a
clock budget.  lgs_set_wait_budget shortens that budget to one cycle, far less than a copy or a
tile of MMAs takes, so the waits run out on the GPU: the kernel must stop its roles, drain the
tensor-core work and the copies it issued, free its tensor memory, and the call must report
LGS_ERR_DEVICE_TIMEOUT.  Afterwards the same context, with the default budget again, must give
the oracle's results: nothing is left behind by the failed launch.  Nothing here faults or hangs
the GPU: the wait that gives up is an ordinary bounded spin."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import rng
from ligesis_b200._lib import check, load, ptr64
from tests.helpers import ligesis_inputs

pytestmark = pytest.mark.gpu


def _hash(ctx, A, cw):
    m, cols = cw.shape
    got = np.zeros((32, cols), dtype=np.uint64)
    check(load().lgs_subset_sum_hash(ctx.handle, ptr64(A), m, ptr64(cw), cols, ptr64(got)))
    return got


def test_hash_wait_gives_up_and_the_context_stays_usable(lgs, orc):
    m, cols = 8, 300 * 256  # two tiles per persistent CTA
    A = rng.field_elements(2500, 32 * 64 * m).reshape(32, 64 * m)
    cw = rng.field_elements(2501, m * cols).reshape(m, cols)
    want = orc.hash_columns(A, cw)
    ctx = L.Context(0)
    try:
        for _ in range(2):  # twice: the error word is cleared after it is reported
            ctx.set_wait_budget(1)
            with pytest.raises(L.DeviceTimeout, match="bounded device wait"):
                _hash(ctx, A, cw)
            ctx.set_wait_budget(0)
            assert np.array_equal(_hash(ctx, A, cw), want)
    finally:
        ctx.close()


def test_commit_reports_the_timeout_then_commits(lgs, orc):
    log_m, log_n = 3, 10
    f, A, _, _, _ = ligesis_inputs(log_m, log_n, seed=61)
    ctx = L.Context(0)
    pk, _ = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A), ctx)
    ctx.set_wait_budget(1)
    bad, _ = L.Ligesis.commit(pk, L.MlPoly(f))
    with pytest.raises(L.DeviceTimeout):
        bad.root  # the root (and the device error word) is read on first use
    ctx.set_wait_budget(0)
    commit, _ = L.Ligesis.commit(pk, L.MlPoly(f))
    assert commit.root == orc.Commitment(orc.Key(log_m, log_n, A), f).root
