"""LigeSIS on the GPU against the CPU oracle: commitments, intermediates and whole proofs
byte-for-byte, both verifiers accepting, and the reference's tamper tests
(pcs/src/ligesis.rs:808-868) through the library's verifier."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import proof as codec
from ligesis_b200 import rng
from tests.helpers import P, ligesis_inputs

pytestmark = pytest.mark.gpu


def _gpu_run(log_m, log_n, f, A, z, fields, ints):
    pk, vk = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A))
    commit, data = L.Ligesis.commit(pk, L.MlPoly(f))
    oracle = L.RandomOracle(0, length=8)
    oracle.fields, oracle.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
    proof = L.Ligesis.prove(pk, data, z, oracle)
    return pk, vk, commit, data, oracle, proof


@pytest.fixture(scope="module", params=[(3, 10), (5, 13), (6, 14)])
def pair(request, lgs, orc):
    log_m, log_n = request.param
    f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=10 * log_m + log_n)
    pk, vk, commit, data, oracle, proof = _gpu_run(log_m, log_n, f, A, z, fields, ints)
    key = orc.Key(log_m, log_n, A)
    cm = orc.Commitment(key, f)
    oproof, ocur = orc.prove(key, cm, z, fields, ints)
    return dict(log_m=log_m, log_n=log_n, f=f, A=A, z=z, fields=fields, ints=ints, pk=pk, vk=vk,
                commit=commit, data=data, oracle=oracle, proof=proof, key=key, cm=cm,
                oproof=oproof, ocur=ocur)


def test_setup_commitment_matches_oracle(pair):
    assert pair["vk"].com_a == pair["key"].com_a


def test_codeword_and_digest_match_oracle(pair):
    assert np.array_equal(pair["data"].codeword(), pair["cm"].codeword())
    assert np.array_equal(pair["data"].digest(), pair["cm"].digest())


def test_commitment_root_matches_oracle(pair):
    assert pair["commit"].root == pair["cm"].root


def test_proof_bytes_match_oracle(pair):
    got, want = pair["proof"].data, pair["oproof"]
    if got != want:  # name the first differing field before failing
        g, w = codec.decode(got), codec.decode(want)
        for name in ("y", "com_a_vec", "com_i", "y4", "y5", "h_cols", "h_open"):
            assert getattr(g, name) == getattr(w, name), name
        for name in codec.SUMCHECK_NAMES:
            assert g.sumchecks[name] == w.sumchecks[name], name
        assert g.batch == w.batch, "batch"
    assert got == want
    assert tuple(int(c) for c in pair["oracle"].cursors) == pair["ocur"]


def test_both_verifiers_accept(pair, orc):
    o = pair["oracle"]
    o.restart()
    assert L.Ligesis.verify(pair["vk"], pair["commit"], pair["z"], pair["proof"], o)
    assert tuple(int(c) for c in o.cursors) == pair["ocur"]
    assert orc.verify(pair["key"].com_a, pair["log_m"], pair["log_n"], pair["commit"].root,
                      pair["z"], pair["proof"].data, pair["fields"], pair["ints"])


def test_claimed_value_is_the_evaluation(pair, orc):
    lifted = np.stack([pair["f"], np.zeros_like(pair["f"])], axis=1)
    assert pair["proof"].y == orc.mle_eval(lifted, pair["z"])


@pytest.mark.parametrize("what", ["y", "sumcheck", "h_column", "batch_msg", "base_leaf",
                                  "fold_value", "truncate"])
def test_tampered_proof_is_rejected(pair, what):
    pf = codec.decode(pair["proof"].data)
    if what == "y":
        pf.y = ((pf.y[0] + 1) % P, pf.y[1])
    elif what == "sumcheck":
        rp = pf.sumchecks["sc_hash"].round_polys
        rp[0][0] = ((rp[0][0][0] + 1) % P, rp[0][0][1])
    elif what == "h_column":
        pf.h_cols[0][0] = (pf.h_cols[0][0] + 1) % P
    elif what == "batch_msg":
        pf.batch.reduction_msgs[1][0] = ((pf.batch.reduction_msgs[1][0][0] + 1) % P, 0)
    elif what == "base_leaf":
        op = pf.batch.base_bf[1]
        k = max(op.values)
        op.values[k][3] = (op.values[k][3] + 1) % P
    elif what == "fold_value":
        op = pf.batch.fold_openings[0]
        k = min(op.values)
        v = op.values[k][0]
        op.values[k][0] = (v[0], (v[1] + 1) % P)
    bad = codec.encode(pf) if what != "truncate" else pair["proof"].data[:-3]
    o = pair["oracle"]
    o.restart()
    assert not L.Ligesis.verify(pair["vk"], pair["commit"], pair["z"], bad, o)


def test_second_proof_from_advanced_cursors_matches_oracle(pair, orc):
    """A proof made from a used oracle is identical whether made alone or after others."""
    o = pair["oracle"]
    o.cursors[:] = np.array(pair["ocur"], dtype=np.uint64)
    p2 = L.Ligesis.prove(pair["pk"], pair["data"], pair["z"], o)
    o2, cur2 = orc.prove(pair["key"], pair["cm"], pair["z"], pair["fields"], pair["ints"],
                         pair["ocur"])
    assert p2.data == o2
    assert tuple(int(c) for c in o.cursors) == cur2


def test_captured_and_replayed_proofs_match_oracle(lgs, orc):
    """On a fresh context the first prove of a shape runs eagerly, the second is captured into a
    CUDA graph and the rest replay it: every proof, each from its own point and oracle, is the
    oracle's, whichever path made it."""
    log_m, log_n = 4, 11
    f, A, _, _, _ = ligesis_inputs(log_m, log_n, seed=77)
    ctx = L.Context(0)
    pk, _ = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A), ctx)
    commit, data = L.Ligesis.commit(pk, L.MlPoly(f))
    key = orc.Key(log_m, log_n, A)
    cm = orc.Commitment(key, f)
    assert commit.root == cm.root
    for i in range(5):
        z = rng.ext_elements(300 + i, log_m + log_n)
        g = rng.SeededRng(400 + i)
        fields, ints = g.ext_elements(2048), g.ints(2048)
        o = L.RandomOracle(0, length=8)
        o.fields, o.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
        got = L.Ligesis.prove(pk, data, z, o)
        want, cur = orc.prove(key, cm, z, fields, ints)
        assert got.data == want, f"proof {i}"
        assert tuple(int(c) for c in o.cursors) == cur
    # a new commitment (new device buffers) and a new key of the same shape replay the graph too
    f2 = rng.field_elements(78, 1 << (log_m + log_n))
    A2 = rng.field_elements(79, 32 * (64 << log_m)).reshape(32, 64 << log_m)
    for key_a, poly in ((A, f2), (A2, f), (A2, f2)):
        pk2 = pk if key_a is A else L.Ligesis.setup_with_hash(
            log_m, log_n, L.SubsetSumHash(64 << log_m, a=key_a), ctx)[0]
        c2, d2 = L.Ligesis.commit(pk2, L.MlPoly(poly))
        z = rng.ext_elements(310, log_m + log_n)
        o = L.RandomOracle(411, length=2048)
        got = L.Ligesis.prove(pk2, d2, z, o)
        key2 = orc.Key(log_m, log_n, key_a)
        cm2 = orc.Commitment(key2, poly)
        o2 = L.RandomOracle(411, length=2048)
        want, _ = orc.prove(key2, cm2, z, o2.fields, o2.ints)
        assert c2.root == cm2.root and got.data == want


def test_async_commits_overlap_and_match_oracle(lgs, orc):
    # two commits enqueued back to back on one context, a prove of the first while the second is
    # still in flight, roots read afterwards in reverse order: all equal the oracle's
    log_m, log_n = 3, 10
    f1, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=71)
    f2 = rng.field_elements(72, f1.size)
    pk, vk = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A))
    c1, d1 = L.Ligesis.commit(pk, L.MlPoly(f1))
    c2, d2 = L.Ligesis.commit(pk, L.MlPoly(f2))
    oracle = L.RandomOracle(0, length=8)
    oracle.fields, oracle.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
    proof = L.Ligesis.prove(pk, d1, z, oracle)
    key = orc.Key(log_m, log_n, A)
    cm1, cm2 = orc.Commitment(key, f1), orc.Commitment(key, f2)
    assert c2.root == cm2.root
    assert c1.root == cm1.root
    want, _ = orc.prove(key, cm1, z, fields, ints)
    assert proof.data == want
    oracle.restart()
    assert L.Ligesis.verify(vk, c1, z, proof, oracle)


def test_public_api_round_trip(lgs):
    """Ligesis::setup/commit/prove/verify through the reference-shaped API (ligesis.rs:808-822)."""
    g = L.SeededRng(123)
    pk, vk = L.Ligesis.setup(3, 10, g)
    f = L.MlPoly(g.field_elements(1 << 13))
    z = g.ext_elements(13)
    commit, data = L.Ligesis.commit(pk, f)
    oracle = L.RandomOracle(g, length=2048)
    proof = L.Ligesis.prove(pk, data, z, oracle)
    assert proof.y == f.eval(z)
    oracle.restart()
    assert L.Ligesis.verify(vk, commit, z, proof, oracle)
    assert 0 < proof.size_bytes() < len(proof.data)


def test_oracle_exhaustion_is_reported(lgs):
    g = L.SeededRng(5)
    pk, vk = L.Ligesis.setup(3, 10, g)
    commit, data = L.Ligesis.commit(pk, L.MlPoly(g.field_elements(1 << 13)))
    oracle = L.RandomOracle(g, length=100)  # fewer than the 612 ints a proof draws
    with pytest.raises(L.OracleExhausted):
        L.Ligesis.prove(pk, data, g.ext_elements(13), oracle)
    assert oracle.drawn() == (0, 0)


def test_bad_shapes_and_lengths_are_rejected(lgs):
    g = L.SeededRng(6)
    with pytest.raises(L.ShapeError):
        L.Ligesis.setup(10, 10, g)
    pk, vk = L.Ligesis.setup(3, 10, g)
    with pytest.raises(L.LgsError):
        L.Ligesis.commit(pk, L.MlPoly(g.field_elements(1 << 12)))


@pytest.mark.parametrize("log_m,log_n", [(7, 7), (9, 8), (10, 10)])
def test_commit_only_square_shapes_match_oracle(lgs, orc, log_m, log_n):
    """Ligesis::commit at shapes setup's shared-domain window rejects (the square shapes of the
    mu = 20/24/26 commit benchmarks run this way): codeword, digest H and root equal the
    oracle's; the key cannot prove."""
    f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=500 + log_m + log_n)
    with pytest.raises(L.ShapeError):
        L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A))
    pk = L.Ligesis.setup_commit_only(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A))
    commit, data = L.Ligesis.commit(pk, L.MlPoly(f))
    orc.set_threads(None)
    try:
        cm = orc.Commitment(orc.Key(log_m, log_n, A, commit_only=True), f)
    finally:
        orc.set_threads(1)
    assert commit.root == cm.root
    assert np.array_equal(data.codeword(), cm.codeword())
    assert np.array_equal(data.digest(), cm.digest())
    o = L.RandomOracle(0, length=8)
    o.fields, o.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
    with pytest.raises(L.ShapeError):
        L.Ligesis.prove(pk, data, z, o)


def test_tuned_launch_choices_give_the_same_proof(lgs, orc):
    """lgs_tune changes only how kernels are launched: fewer hash CTAs, a smaller sumcheck grid
    and the digest built in row groups under the upload (the host polynomial here takes that
    path) give the oracle's commitment and proof; unknown names are refused."""
    log_m, log_n = 5, 13
    f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=91)
    ctx = L.Context(0)
    pk, _ = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A), ctx)
    key = orc.Key(log_m, log_n, A)
    want, _ = orc.prove(key, orc.Commitment(key, f), z, fields, ints)
    for h, b, g in [(0, 0, 0), (40, 148, 2), (7, 16, 8), (148, 296, 4)]:
        ctx.tune(hash_ctas=h, sumcheck_blocks=b, hash_groups=g)
        assert ctx.tuning() == {"hash_ctas": h, "sumcheck_blocks": b, "hash_groups": g}
        for _ in range(3):  # eager, captured, replayed
            commit, data = L.Ligesis.commit(pk, L.MlPoly(f))
            o = L.RandomOracle(0, length=8)
            o.fields, o.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
            assert L.Ligesis.prove(pk, data, z, o).data == want, (h, b, g)
    with pytest.raises(L.LgsError, match="unknown parameter"):
        ctx.tune(nonsense=1)
    with pytest.raises(L.LgsError):
        ctx.tune(sumcheck_blocks=297)


def test_lent_device_polynomial_gives_the_same_commitment(lgs, orc):
    """commit_device(lend=True) reads the caller's device buffer in place (f_on_device = 2):
    the root and the proof equal the oracle's, as with the copying forms."""
    import torch

    log_m, log_n = 5, 13
    f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=93)
    pk, _ = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A))
    f_dev = torch.from_numpy(f.view(np.int64).copy()).cuda()
    key = orc.Key(log_m, log_n, A)
    cm = orc.Commitment(key, f)
    want, _ = orc.prove(key, cm, z, fields, ints)
    for lend in (False, True):
        commit, data = L.Ligesis.commit_device(pk, f_dev.data_ptr(), f.size, lend=lend)
        o = L.RandomOracle(0, length=8)
        o.fields, o.ints = np.ascontiguousarray(fields), np.ascontiguousarray(ints)
        assert L.Ligesis.prove(pk, data, z, o).data == want, lend
        assert commit.root == cm.root, lend
    assert np.array_equal(f_dev.cpu().numpy().view(np.uint64), f)  # only read


@pytest.mark.parametrize("block,tail,groups", [
    (1, 0, 0), (0, 0, 0), (1 << 30, 0, 0),  # 8, 2 and 1 equal blocks
    (1, 2, 0), (1, 1 << 16, 0),  # a 2-row last block; a tail above a share: equal blocks
    (1, 3, 3), (1, 0, 8), (0, 6, 2), (1, 0, 3),  # hash groups at the block boundaries
])
def test_upload_row_blocks_give_the_same_root(lgs, orc, block, tail, groups):
    """A host polynomial is uploaded and encoded in row blocks of at least upload_block_bytes
    (8, 2 and 1 blocks of a 2 MiB polynomial here), the last one upload_tail_rows long, and
    hashed in hash_groups groups of whole blocks (3 groups over 8 blocks end with blocks 1, 4
    and 7); the commitment must not depend on any of it."""
    log_m, log_n = 5, 13
    f, A, _, _, _ = ligesis_inputs(log_m, log_n, seed=71)
    ctx = L.Context(0)
    ctx.tune(upload_block_bytes=block, upload_tail_rows=tail, hash_groups=groups)
    assert ctx.tuning("upload_tail_rows") == {"upload_tail_rows": tail}
    pk, _ = L.Ligesis.setup_with_hash(log_m, log_n, L.SubsetSumHash(64 << log_m, a=A), ctx)
    commit, _ = L.Ligesis.commit(pk, L.MlPoly(f))
    assert commit.root == orc.Commitment(orc.Key(log_m, log_n, A), f).root
