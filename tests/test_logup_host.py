"""The library's host verifiers for the GKR fraction sum and the GKR-LogUp lookup
(logup/src/frac_sum.rs:221-258, logup/src/lookup.rs:191-229) on proofs the oracle wrote: the same
reduced claims, the same cursor, and the reference's rejections.  No device work."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import field as fld
from ligesis_b200 import rng


def _oracle(fields):
    o = L.RandomOracle(0, length=4)
    o.fields = np.ascontiguousarray(fields)
    return o


@pytest.mark.parametrize("k", [0, 1, 2, 5, 9])
def test_frac_sum_host_verify_matches_oracle(lgs, orc, k):
    p, q = rng.ext_elements(100 + k, 1 << k), rng.ext_elements(200 + k, 1 << k)
    fields = rng.ext_elements(300 + k, 128)
    proof, point, pe, qe, cur = orc.frac_sum_prove(p, q, fields)
    fp = L.FracSumProof(proof)
    assert fp.num_layers == k and fp.size_bytes() == 16 * (2 + sum(4 * r + 4 for r in range(k)))
    o = _oracle(fields)
    got = L.FracSum.verify(proof, o)
    assert got is not None
    vpoint, vpe, vqe = got
    assert np.array_equal(vpoint, point) and (vpe, vqe) == (pe, qe)
    assert int(o.cursors[0]) == cur


def test_frac_sum_host_verify_rejects(lgs, orc):
    p, q = rng.ext_elements(1, 64), rng.ext_elements(2, 64)
    fields = rng.ext_elements(3, 64)
    proof = orc.frac_sum_prove(p, q, fields)[0]
    b = bytearray(proof)
    v = int.from_bytes(b[8:16], "little")
    b[8:16] = ((v + 1) % fld.P).to_bytes(8, "little")  # num += 1
    assert L.FracSum.verify(bytes(b), _oracle(fields)) is None
    off = 44 + sum(4 + (4 * r + 4) * 16 for r in range(4)) + 4 + (2 * 4 + 1) * 16
    b = bytearray(proof)
    v = int.from_bytes(b[off:off + 8], "little")
    b[off:off + 8] = ((v + 1) % fld.P).to_bytes(8, "little")  # layers[4].round_polys[2][1] += 1
    assert L.FracSum.verify(bytes(b), _oracle(fields)) is None
    assert L.FracSum.verify(proof[:-1], _oracle(fields)) is None
    assert L.FracSum.verify(proof + b"\0", _oracle(fields)) is None
    assert L.FracSum.verify(proof, _oracle(fields[:10])) is None  # oracle exhausted


def _sample(mu, nu, seed):
    t = rng.ext_elements(seed, 1 << nu)
    idx = (rng.ints(seed + 1, 1 << mu) % np.uint64(1 << nu)).astype(np.int64)
    return t[idx], t


@pytest.mark.parametrize("mu,nu", [(0, 0), (4, 2), (8, 4), (10, 6)])
def test_lookup_host_verify_matches_oracle(lgs, orc, mu, nu):
    a, t = _sample(mu, nu, 10 + mu)
    e = L.multiplicity_vector(a, t)
    fields = rng.ext_elements(20 + mu, 256)
    proof, zq, zt, cur = orc.lookup_prove(a, t, None, fields)
    assert orc.lookup_prove(a, t, e, fields)[0] == proof
    lp = L.LookupProof(proof)
    assert lp.query.num_layers == mu and lp.table.num_layers == nu
    o = _oracle(fields)
    claims = L.Lookup.verify(proof, o)
    assert claims is not None and int(o.cursors[0]) == cur
    want = orc.lookup_verify(proof, fields)
    assert [c.poly for c in claims] == [L.Poly.Query, L.Poly.Mult, L.Poly.Table]
    assert np.array_equal(claims[0].point, want[0]) and np.array_equal(claims[1].point, want[1])
    assert [c.value for c in claims] == [want[2], want[3], want[4]]


def test_lookup_host_verify_rejects(lgs, orc):
    a, t = _sample(8, 4, 5)
    fields = rng.ext_elements(6, 256)
    bad = a.copy()
    bad[3] = rng.ext_elements(7, 1)[0]
    assert L.Lookup.verify(orc.lookup_prove(bad, t, None, fields)[0], _oracle(fields)) is None
    e = L.multiplicity_vector(a, t)
    e[2, 0] += 1
    assert L.Lookup.verify(orc.lookup_prove(a, t, e, fields)[0], _oracle(fields)) is None


def test_multiplicity_vector_counts_by_value():
    t = rng.ext_elements(1, 16)
    idx = (rng.ints(2, 300) % np.uint64(16)).astype(np.int64)
    a = t[idx]
    a[7] = rng.ext_elements(3, 1)[0]  # not in the table: counted nowhere
    e = L.multiplicity_vector(a, t)
    want = np.bincount(np.delete(idx, 7), minlength=16)
    assert np.array_equal(e[:, 0], want) and not e[:, 1].any()
