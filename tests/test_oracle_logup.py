"""The oracle's GKR fraction sum and GKR-LogUp lookup against the reference's own tests
(logup/src/frac_sum.rs:262-333, logup/src/lookup.rs:231-270): round trips with the reduced
claims equal to the MLE openings, the cross-multiplied root, and every rejection case."""
from __future__ import annotations

import numpy as np
import pytest

from ligesis_b200 import field as fld
from ligesis_b200 import rng
from tests.helpers import ef_list


def _frac_sum(p, q):
    num, den = (0, 0), (1, 0)
    for pi, qi in zip(p, q):
        num = fld.ef_add(fld.ef_mul(num, qi), fld.ef_mul(pi, den))
        den = fld.ef_mul(den, qi)
    return num, den


def _proof_num_den(proof: bytes, off: int = 0):
    v = np.frombuffer(proof[off + 8: off + 40], dtype=np.uint64)
    return (int(v[0]), int(v[1])), (int(v[2]), int(v[3]))


@pytest.mark.parametrize("k", range(9))
def test_frac_sum_round_trip(orc, k):
    n = 1 << k
    p, q = rng.ext_elements(10 + k, n), rng.ext_elements(20 + k, n)
    fields = rng.ext_elements(30 + k, 64)
    proof, point, pe, qe, cur = orc.frac_sum_prove(p, q, fields)
    assert cur == k * (k + 3) // 2  # lambda, r challenges and beta per layer r
    num, den = _proof_num_den(proof)
    wn, wd = _frac_sum(ef_list(p), ef_list(q))
    assert fld.ef_mul(num, wd) == fld.ef_mul(wn, den)
    got = orc.frac_sum_verify(proof, fields)
    assert got is not None
    vpoint, vpe, vqe, vcur = got
    assert np.array_equal(vpoint, point) and (vpe, vqe) == (pe, qe) and vcur == cur
    assert orc.mle_eval(p, point) == pe and orc.mle_eval(q, point) == qe


def test_frac_sum_ones_numerators(orc):
    q = rng.ext_elements(5, 1 << 7)
    ones = np.zeros((1 << 7, 2), dtype=np.uint64)
    ones[:, 0] = 1
    fields = rng.ext_elements(6, 64)
    assert orc.frac_sum_prove(None, q, fields)[0] == orc.frac_sum_prove(ones, q, fields)[0]


def _tamper(proof: bytes, off: int) -> bytes:
    b = bytearray(proof)
    v = int.from_bytes(b[off:off + 8], "little")
    b[off:off + 8] = ((v + 1) % fld.P).to_bytes(8, "little")
    return bytes(b)


def test_frac_sum_tampered_root_and_round_rejected(orc):
    p, q = rng.ext_elements(1, 64), rng.ext_elements(2, 64)
    fields = rng.ext_elements(3, 64)
    proof = orc.frac_sum_prove(p, q, fields)[0]
    assert orc.frac_sum_verify(_tamper(proof, 8), fields) is None  # num += 1
    # layers[4].round_polys[2][1] += 1: skip layers 0..3 (4 + (4r + 4) * 16 bytes each)
    off = 44 + sum(4 + (4 * r + 4) * 16 for r in range(4))
    off += 4 + (2 * 4 + 1) * 16
    assert orc.frac_sum_verify(_tamper(proof, off), fields) is None
    assert orc.frac_sum_verify(proof[:-1], fields) is None
    assert orc.frac_sum_verify(proof, fields) is not None


def _sample(mu, nu, seed):
    t = rng.ext_elements(seed, 1 << nu)
    idx = rng.ints(seed + 1, 1 << mu) % np.uint64(1 << nu)
    a = t[idx.astype(np.int64)]
    e = np.zeros((1 << nu, 2), dtype=np.uint64)
    np.add.at(e[:, 0], idx.astype(np.int64), 1)
    return a, t, e


@pytest.mark.parametrize("mu,nu", [(0, 0), (4, 2), (8, 4), (10, 6)])
def test_lookup_round_trip(orc, mu, nu):
    a, t, e = _sample(mu, nu, 40 + mu)
    fields = rng.ext_elements(50 + mu, 256)
    proof, zq, zt, cur = orc.lookup_prove(a, t, None, fields)
    assert orc.lookup_prove(a, t, e, fields)[0] == proof  # counted == supplied multiplicities
    got = orc.lookup_verify(proof, fields)
    assert got is not None
    vzq, vzt, va, ve, vt, vcur = got
    assert np.array_equal(vzq, zq) and np.array_equal(vzt, zt) and vcur == cur
    assert orc.mle_eval(a, zq) == va
    assert orc.mle_eval(e, zt) == ve
    assert orc.mle_eval(t, zt) == vt


def test_lookup_non_member_and_wrong_multiplicity_rejected(orc):
    a, t, e = _sample(8, 4, 7)
    fields = rng.ext_elements(8, 256)
    bad_a = a.copy()
    bad_a[3] = rng.ext_elements(9, 1)[0]
    proof = orc.lookup_prove(bad_a, t, None, fields)[0]
    assert orc.lookup_verify(proof, fields) is None
    bad_e = e.copy()
    bad_e[2, 0] += 1
    proof = orc.lookup_prove(a, t, bad_e, fields)[0]
    assert orc.lookup_verify(proof, fields) is None


def test_lookup_openings_via_basefold(orc):
    """lookup.rs:243-268: each returned claim is opened by Basefold over the witness."""
    a, t, e = _sample(10, 6, 11)
    fields = rng.ext_elements(12, 256)
    proof = orc.lookup_prove(a, t, None, fields)[0]
    zq, zt, va, ve, vt, _ = orc.lookup_verify(proof, fields)
    g = rng.SeededRng(13)
    pf, pi = g.ext_elements(64), g.ints(256)
    for poly, point, value in ((a, zq, va), (e, zt, ve), (t, zt, vt)):
        cm = orc.BasefoldCommitment(poly, True, 1, 0)
        bp, _ = orc.basefold_prove(cm, point, pf, pi)
        assert np.frombuffer(bp[24:40], np.uint64).tolist() == list(value)
        assert orc.basefold_verify(cm.root, point, bp, pf, pi)
