"""The PolyCommitmentScheme mirror on the CPU: the reference's NoopPcs test (pcs/src/noop.rs:80-108)
and BasefoldPcs's host-side rejections, which decide before any device call."""
from __future__ import annotations

import numpy as np

import ligesis_b200 as L
from ligesis_b200.pcs import BasefoldPcsCommitment, BasefoldPcsProof
from tests.helpers import P


def test_noop_commit_is_empty_and_verify_always_accepts(orc):
    poly = L.MlPoly(np.arange(1, 9, dtype=np.uint64))
    point = [5, 9, 2]
    oracle = L.RandomOracle(3, length=16)
    data, commit = L.NoopPcs.commit(poly)
    assert data is poly and np.array_equal(data.evals, poly.evals)
    assert commit == L.NoopCommit()
    proof = L.NoopPcs.batch_prove([(data, point)], oracle)
    ev = np.stack([poly.evals, np.zeros_like(poly.evals)], axis=1)
    v = orc.mle_eval(ev, np.array([[x, 0] for x in point], dtype=np.uint64))
    bogus = ((v[0] + 1) % P, v[1])
    assert L.NoopPcs.batch_verify([(commit, point, bogus)], proof, oracle)


def test_basefold_pcs_rejects_shape_mismatch_without_device():
    pcs = L.BasefoldPcs()
    oracle = L.RandomOracle(1, length=16)
    com = BasefoldPcsCommitment(bytes(32), 4, True)
    assert not pcs.batch_verify([(com, [1, 2, 3, 4], 0)], None, oracle)
    assert not pcs.batch_verify([(com, [1, 2, 3, 4], 0)], BasefoldPcsProof([]), oracle)
    assert not pcs.batch_verify([(com, [1, 2, 3], 0)], BasefoldPcsProof([b"LGSB" + bytes(60)]),
                                oracle)
    assert not pcs.batch_verify([(com, [1, 2, 3, 4], 0)], BasefoldPcsProof([b"junk"]), oracle)


def test_ligesis_pcs_shapes_and_padding():
    from ligesis_b200.workloads import shape_for_mu

    for n in range(1, 29):
        mu = L.LigesisPcs.padded_vars(n)
        assert mu == max(n, 14)
        log_m, log_n = shape_for_mu(mu)
        assert log_m + log_n == mu and L.shape_ok(log_m, log_n)
    pt = L.LigesisPcs._pad_point([3, 4, 5], 3, 14)
    assert pt.shape == (14, 2) and list(pt[:3, 0]) == [3, 4, 5] and not pt[3:].any()


def test_ligesis_pcs_refuses_extension_values():
    import pytest

    ev = np.zeros((1 << 4, 2), dtype=np.uint64)
    ev[5, 1] = 1
    with pytest.raises(ValueError):
        L.LigesisPcs().commit(L.MlPoly(ev))
