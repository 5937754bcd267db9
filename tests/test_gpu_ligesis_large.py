"""LigeSIS on the GPU at the large reference-valid shapes, against the CPU oracle.

* mu = 24 as 2^7 x 2^17 (the README's row, README.md:175, and the shape bench.py times): the
  oracle runs live (its independent loops split over the host cores) and the commitment root,
  codeword digest H, proof bytes and oracle cursors must equal it byte for byte; both verifiers
  accept.  The same outputs must also match the committed digests in
  tests/golden/ligesis_large.json.
* mu = 26 as 2^7 x 2^19: the oracle needs minutes for it, so the GPU outputs are compared with
  the oracle's digests committed in tests/golden/ligesis_large.json (made by
  tests/golden/make_ligesis_golden.py from the same seeded inputs); the library's verifier
  accepts the proof.

At these shapes the whole path runs together: the four-step RS encode at 2^18 (2^20) columns,
the tcgen05 hash at W = 8192, the 2^18 (2^20)-leaf Merkle tree, the 2^20-entry binary-check
sumcheck over the real B_I and the Basefold batched open."""
from __future__ import annotations

import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import proof as codec
from tests.helpers import ligesis_inputs

pytestmark = pytest.mark.gpu

GOLDEN_FILE = Path(__file__).parent / "golden" / "ligesis_large.json"


def _golden(shape):
    shapes = json.loads(GOLDEN_FILE.read_text())["shapes"]
    return {(s["log_m"], s["log_n"]): s for s in shapes}[shape]


def _gpu(log_m, log_n, f, A, z, fields, ints):
    pk, vk = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A))
    commit, data = L.Ligesis.commit(pk, L.MlPoly(f))
    oracle = L.RandomOracle(0, length=8)
    oracle.fields, oracle.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
    proof = L.Ligesis.prove(pk, data, z, oracle)
    return pk, vk, commit, data, oracle, proof


def _check_golden(shape, vk, commit, data, oracle, proof):
    g = _golden(shape)
    assert vk.com_a.hex() == g["com_a"]
    assert commit.root.hex() == g["root"]
    assert hashlib.sha256(np.ascontiguousarray(data.digest()).tobytes()).hexdigest() == \
        g["digest_sha256"]
    assert len(proof.data) == g["proof_len"]
    assert hashlib.sha256(proof.data).hexdigest() == g["proof_sha256"]
    assert [int(c) for c in oracle.cursors] == g["cursors"]


def test_mu24_commit_and_proof_match_oracle(lgs, orc):
    log_m, log_n = 7, 17
    f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=10 * log_m + log_n)
    pk, vk, commit, data, oracle, proof = _gpu(log_m, log_n, f, A, z, fields, ints)
    orc.set_threads(None)
    try:
        key = orc.Key(log_m, log_n, A)
        cm = orc.Commitment(key, f)
        want, cur = orc.prove(key, cm, z, fields, ints)
        assert vk.com_a == key.com_a
        assert commit.root == cm.root
        assert np.array_equal(data.digest(), cm.digest())
        if proof.data != want:  # name the first differing field before failing
            g, w = codec.decode(proof.data), codec.decode(want)
            for name in ("y", "com_a_vec", "com_i", "y4", "y5", "h_cols", "h_open"):
                assert getattr(g, name) == getattr(w, name), name
            for name in codec.SUMCHECK_NAMES:
                assert g.sumchecks[name] == w.sumchecks[name], name
            assert g.batch == w.batch, "batch"
        assert proof.data == want
        assert tuple(int(c) for c in oracle.cursors) == cur
        _check_golden((log_m, log_n), vk, commit, data, oracle, proof)
        oracle.restart()
        assert L.Ligesis.verify(vk, commit, z, proof, oracle)
        assert orc.verify(key.com_a, log_m, log_n, commit.root, z, proof.data, fields, ints)
    finally:
        orc.set_threads(1)


def test_mu26_commit_and_proof_match_oracle_digests(lgs):
    log_m, log_n = 7, 19
    f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=10 * log_m + log_n)
    pk, vk, commit, data, oracle, proof = _gpu(log_m, log_n, f, A, z, fields, ints)
    _check_golden((log_m, log_n), vk, commit, data, oracle, proof)
    oracle.restart()
    assert L.Ligesis.verify(vk, commit, z, proof, oracle)
