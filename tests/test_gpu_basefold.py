"""Standalone Basefold on the GPU against the CPU oracle (pcs/src/basefold.rs:309-642): roots and
proofs byte for byte, both verifiers accepting, the reference's tamper test, cursor advance."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import rng
from tests.helpers import P

pytestmark = pytest.mark.gpu


def _run(orc, is_ef, n, code_rate, li, seed):
    poly = rng.ext_elements(seed, 1 << n) if is_ef else rng.field_elements(seed, 1 << n)
    pt = rng.ext_elements(seed + 1, n)
    g = rng.SeededRng(seed + 2)
    fields, ints = g.ext_elements(256), g.ints(256)
    mp = L.MlPoly(poly)
    if is_ef:
        state, commit = L.Basefold.commit_ext_on_domain(mp, code_rate, li)
    else:
        state, commit = L.Basefold.commit_base_on_domain(mp, code_rate, li)
    oracle = L.RandomOracle(0, length=8)
    oracle.fields, oracle.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
    proof = L.Basefold.prove(state, pt, oracle)
    cm = orc.BasefoldCommitment(poly, is_ef, code_rate, li)
    want, cur = orc.basefold_prove(cm, pt, fields, ints)
    return dict(poly=poly, pt=pt, fields=fields, ints=ints, state=state, commit=commit,
                oracle=oracle, proof=proof, cm=cm, want=want, cur=cur)


@pytest.mark.parametrize("is_ef,n,code_rate,li", [(False, 12, 2, 6), (True, 12, 2, 6),
                                                  (False, 16, 1, 6), (True, 15, 1, 6),
                                                  (False, 14, 1, 4), (False, 13, 3, 6),
                                                  (False, 20, 1, 6), (False, 22, 1, 6)])
def test_basefold_matches_oracle(lgs, orc, is_ef, n, code_rate, li):
    r = _run(orc, is_ef, n, code_rate, li, seed=100 + n + 10 * code_rate + int(is_ef))
    assert r["commit"].root == r["cm"].root
    assert r["proof"].data == r["want"]
    assert tuple(int(x) for x in r["oracle"].cursors) == r["cur"]
    r["oracle"].restart()
    assert L.Basefold.verify(r["commit"], r["pt"], r["proof"], r["oracle"])
    assert orc.basefold_verify(r["cm"].root, r["pt"], r["proof"].data, r["fields"], r["ints"])


def test_basefold_claimed_eval_and_tamper(lgs, orc):
    r = _run(orc, False, 12, 2, 6, seed=7)
    ev = np.stack([r["poly"], np.zeros_like(r["poly"])], axis=1)
    assert tuple(int(x) for x in orc.mle_eval(ev, r["pt"])) == r["proof"].claimed_eval
    b = bytearray(r["proof"].data)
    c0 = int.from_bytes(b[44:52], "little")
    b[44:52] = ((c0 + 1) % P).to_bytes(8, "little")  # reduction_msgs[0].0 += 1
    r["oracle"].restart()
    assert not L.Basefold.verify(r["commit"], r["pt"], bytes(b), r["oracle"])
    r["oracle"].restart()
    assert not L.Basefold.verify(r["commit"], r["pt"], r["proof"].data[:-8], r["oracle"])
    other = L.BasefoldCommit(bytes(32))
    r["oracle"].restart()
    assert not L.Basefold.verify(other, r["pt"], r["proof"], r["oracle"])


def test_basefold_rejects_bad_arguments(lgs):
    with pytest.raises(L.LgsError):
        L.Basefold.commit_base_on_domain(L.MlPoly(rng.field_elements(1, 1 << 6)), 1, 6)
    state, _ = L.Basefold.commit_base(L.MlPoly(rng.field_elements(1, 1 << 10)), 1)
    oracle = L.RandomOracle(3, length=2)
    with pytest.raises(L.LgsError):
        L.Basefold.prove(state, rng.ext_elements(4, 10), oracle)  # too few oracle fields
    with pytest.raises(L.LgsError):
        L.Basefold.prove(state, rng.ext_elements(4, 9), L.RandomOracle(3, length=512))
