"""BasefoldPcs (the PolyCommitmentScheme trait of pcs/src/noop.rs:23-48 over the GPU Basefold):
a batch of openings on one shared oracle, byte for byte against the oracle's Basefold run task by
task with the cursors carried over, and the verifier's rejections of wrong claims."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import rng
from ligesis_b200.pcs import BasefoldPcsProof
from tests.helpers import P

pytestmark = pytest.mark.gpu


def _polys():
    lifted = rng.field_elements(11, 1 << 12)  # integer witness lifted to EF: base-field leaves
    ext = rng.ext_elements(12, 1 << 13)
    base = rng.field_elements(13, 1 << 15)
    return [
        (L.MlPoly(np.stack([lifted, np.zeros_like(lifted)], axis=1)), lifted, False),
        (L.MlPoly(ext), ext, True),
        (L.MlPoly(base), base, False),
    ]


def _oracle(seed):
    g = rng.SeededRng(seed)
    fields, ints = g.ext_elements(512), g.ints(512)
    o = L.RandomOracle(0, length=8)
    o.fields, o.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
    return o, fields, ints


@pytest.mark.parametrize("code_rate", [1, 2])
def test_basefold_pcs_batch_matches_oracle(lgs, orc, code_rate):
    pcs = L.BasefoldPcs(code_rate=code_rate)
    polys = _polys()
    commits = [pcs.commit(p) for p, _, _ in polys]
    points = [rng.ext_elements(40 + i, p.num_vars) for i, (p, _, _) in enumerate(polys)]
    oracle, fields, ints = _oracle(77)
    proof = pcs.batch_prove([(d, pt) for (d, _), pt in zip(commits, points)], oracle)
    assert len(proof.openings) == 3
    cur = (0, 0)
    for (data, com), (_, raw, is_ef), pt, opening in zip(commits, polys, points, proof.openings):
        assert com.base_field == (not is_ef)
        cm = orc.BasefoldCommitment(raw, is_ef, code_rate, 6)
        assert com.root == cm.root
        want, cur = orc.basefold_prove(cm, pt, fields, ints, cur)
        assert opening == want
    assert tuple(int(x) for x in oracle.cursors) == cur

    evals = []
    for (_, raw, is_ef), pt in zip(polys, points):
        ev = raw if is_ef else np.stack([raw, np.zeros_like(raw)], axis=1)
        evals.append(orc.mle_eval(ev, pt))
    claims = [(com, pt, v) for (_, com), pt, v in zip(commits, points, evals)]
    oracle.restart()
    assert pcs.batch_verify(claims, proof, oracle)
    assert tuple(int(x) for x in oracle.cursors) == cur

    bogus = list(claims)
    v = evals[1]
    bogus[1] = (claims[1][0], claims[1][1], ((v[0] + 1) % P, v[1]))
    oracle.restart()
    assert not pcs.batch_verify(bogus, proof, oracle)

    swapped = [(claims[1][0], claims[0][1], claims[0][2])] + claims[1:]
    oracle.restart()
    assert not pcs.batch_verify(swapped, proof, oracle)

    oracle.restart()
    assert not pcs.batch_verify(claims[:2], proof, oracle)
    oracle.restart()
    assert not pcs.batch_verify(claims, BasefoldPcsProof(proof.openings[::-1]), oracle)

    t = bytearray(proof.openings[2])
    t[-3] ^= 1
    oracle.restart()
    assert not pcs.batch_verify(claims, BasefoldPcsProof(proof.openings[:2] + [bytes(t)]), oracle)


def test_basefold_pcs_small_polys(lgs, orc):
    pcs = L.BasefoldPcs(code_rate=2)
    for n in (1, 2, 3, 7):
        raw = rng.ext_elements(200 + n, 1 << n)
        data, com = pcs.commit(L.MlPoly(raw))
        pt = rng.ext_elements(300 + n, n)
        oracle, fields, ints = _oracle(n)
        proof = pcs.batch_prove([(data, pt)], oracle)
        cm = orc.BasefoldCommitment(raw, True, 2, min(6, n - 1))
        assert com.root == cm.root
        want, _ = orc.basefold_prove(cm, pt, fields, ints)
        assert proof.openings[0] == want
        oracle.restart()
        assert pcs.batch_verify([(com, pt, orc.mle_eval(raw, pt))], proof, oracle)


def test_ligesis_pcs_batch_matches_oracle(lgs, orc):
    """LigesisPcs: lifted integer witnesses of 10, 14 and 16 variables (the first zero-padded to
    14) committed and opened in one batch; every root and proof equals the oracle's LigeSIS run on
    the padded polynomial at the zero-extended point, cursors carried from task to task."""
    pcs = L.LigesisPcs(seed=5)
    raws = [rng.field_elements(60 + n, 1 << n) for n in (10, 14, 16)]
    polys = [L.MlPoly(np.stack([r, np.zeros_like(r)], axis=1)) for r in raws]
    commits = [pcs.commit(p) for p in polys]
    points = [rng.ext_elements(70 + i, p.num_vars) for i, p in enumerate(polys)]
    oracle = L.RandomOracle(9, length=4096)
    fields, ints = oracle.fields.copy(), oracle.ints.copy()
    proof = pcs.batch_prove([(d, pt) for (d, _), pt in zip(commits, points)], oracle)
    cur = (0, 0)
    values = []
    for (d, com), raw, pt, pb in zip(commits, raws, points, proof.proofs):
        mu = com.log_m + com.log_n
        f = np.concatenate([raw, np.zeros((1 << mu) - raw.size, dtype=np.uint64)])
        z = L.LigesisPcs._pad_point(pt, com.num_vars, mu)
        key = orc.Key(com.log_m, com.log_n, d.pk.hash.a)
        cm = orc.Commitment(key, f)
        assert com.root == cm.root
        want, cur = orc.prove(key, cm, z, fields, ints, cur)
        assert pb == want
        v = orc.mle_eval(np.stack([raw, np.zeros_like(raw)], axis=1), pt)
        assert L.LigesisProof(pb).y == v
        values.append(v)
    assert tuple(int(x) for x in oracle.cursors) == cur

    claims = [(com, pt, v) for (_, com), pt, v in zip(commits, points, values)]
    oracle.restart()
    assert pcs.batch_verify(claims, proof, oracle)
    bogus = list(claims)
    bogus[0] = (claims[0][0], claims[0][1], ((values[0][0] + 1) % P, values[0][1]))
    oracle.restart()
    assert not pcs.batch_verify(bogus, proof, oracle)
    oracle.restart()
    assert not pcs.batch_verify(claims[:2], proof, oracle)
    other = [(claims[2][0], claims[1][1], claims[1][2])] + claims[2:]
    oracle.restart()
    assert not pcs.batch_verify([claims[0]] + other, proof, oracle)
