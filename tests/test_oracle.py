"""The CPU oracle, pinned: field constants by their algebraic properties, BLAKE3 by known
answers from an independent implementation (tests/golden/blake3_kat.json), serialization by the
reference's own test (utils/src/merkle.rs:147-156), and the protocol by the reference's
round-trip and tamper tests (utils/src/sumcheck.rs:156-183, pcs/src/subset_sum.rs:90-124,
utils/src/merkle.rs:127-144, pcs/src/ligesis.rs:808-868).  No GPU needed."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from ligesis_b200 import field as F
from ligesis_b200 import proof as codec
from ligesis_b200 import rng
from tests.helpers import P, ef_list, ligesis_inputs

GOLDEN = Path(__file__).with_name("golden")


# ---- field -----------------------------------------------------------------------------------
def test_base_field_ops_match_big_integers(orc):
    edge = [0, 1, 2, P - 1, P - 2, 1 << 32, (1 << 32) - 1, 1 << 63, (1 << 64) - 1, P, P + 1]
    a = np.array(edge + list(rng.field_elements(7, 500)), dtype=np.uint64)
    b = np.array(edge[::-1] + list(rng.field_elements(8, 500)), dtype=np.uint64)
    s, d, p = orc.bf_ops(a, b)
    for x, y, ss, dd, pp in zip(a.tolist(), b.tolist(), s.tolist(), d.tolist(), p.tolist()):
        assert ss == (x + y) % P
        assert dd == (x - y) % P
        assert pp == (x * y) % P


def test_extension_mul_and_inverse(orc):
    a = rng.ext_elements(9, 200)
    b = rng.ext_elements(10, 200)
    prod, inv = orc.ef_ops(a, b)
    for x, y, pr, iv in zip(ef_list(a), ef_list(b), ef_list(prod), ef_list(inv)):
        assert pr == F.ef_mul(x, y)
        assert F.ef_mul(x, iv) == F.ONE


def test_nonresidue_and_two_adic_generators(orc):
    assert pow(F.W, (P - 1) // 2, P) == P - 1  # 7 is a quadratic non-residue
    for bits in range(0, 33):
        g = orc.two_adic_generator(bits)
        assert pow(g, 1 << bits, P) == 1
        if bits:
            assert pow(g, 1 << (bits - 1), P) == P - 1  # order exactly 2^bits
    assert orc.two_adic_generator(1) == P - 1
    assert orc.two_adic_generator(2) == 1 << 48


# ---- BLAKE3 / Merkle ---------------------------------------------------------------------------
def test_blake3_known_answers(orc):
    kat = json.loads((GOLDEN / "blake3_kat.json").read_text())
    for v in kat["vectors"]:
        data = bytes(j % 251 for j in range(v["len"]))
        assert orc.blake3(data).hex() == v["hash"], v["len"]


def test_serialization_is_canonical_le():
    # utils/src/merkle.rs:147-156: Goldilocks::new(42), Goldilocks::new(u64::MAX)
    vals = [42, (1 << 64) - 1]
    canon = np.array([v % P for v in vals], dtype=np.uint64)
    b = canon.view(np.uint8).tobytes()
    assert len(b) == 16
    assert b[:8] == (42).to_bytes(8, "little")


def test_merkle_commit_and_open(orc):
    # utils/src/merkle.rs:127-144
    leaves = np.array([[2 * x, 2 * x + 1] for x in range(8)], dtype=np.uint64)
    root = orc.merkle_root(leaves)
    proof = orc.merkle_open(leaves, [2, 3])
    assert len(proof) == 2 * 32  # siblings at layers 1 and 2
    assert orc.merkle_verify(root, proof, [2, 3], leaves[[2, 3]], 8)
    bad = leaves[[2, 3]].copy()
    bad[0, 0] += 1
    assert not orc.merkle_verify(root, proof, [2, 3], bad, 8)
    # parent = blake3(left || right), leaf = blake3(serialized fields)
    h = [orc.blake3(l.tobytes()) for l in leaves]
    layer = h
    while len(layer) > 1:
        layer = [orc.blake3(layer[i] + layer[i + 1]) for i in range(0, len(layer), 2)]
    assert layer[0] == root


# ---- DFT / MlPoly ------------------------------------------------------------------------------
def _naive_dft(c, n):
    g = pow(7, 0, P)
    from oracle import orc as o

    g = o.two_adic_generator(n.bit_length() - 1)
    return [sum(int(c[k]) * pow(g, j * k, P) for k in range(len(c))) % P for j in range(n)]


@pytest.mark.parametrize("n_in,size", [(1, 2), (4, 8), (8, 16), (32, 64), (16, 64)])
def test_dft_matches_definition(orc, n_in, size):
    c = rng.field_elements(11, n_in)
    assert orc.dft_bf(c, size).tolist() == _naive_dft(c, size)
    ce = rng.ext_elements(12, n_in)
    out = orc.dft_ef(ce, size)
    assert out[:, 0].tolist() == _naive_dft(ce[:, 0], size)
    assert out[:, 1].tolist() == _naive_dft(ce[:, 1], size)


def _py_eval(evals, point):
    s = ef_list(evals)
    for r in ef_list(point):
        s = [F.ef_add(s[2 * i], F.ef_mul(F.ef_sub(s[2 * i + 1], s[2 * i]), r))
             for i in range(len(s) // 2)]
    return s[0]


def test_mle_eval_fold_new_eq(orc):
    ev = rng.ext_elements(13, 64)
    pt = rng.ext_elements(14, 6)
    assert orc.mle_eval(ev, pt) == _py_eval(ev, pt)
    eq = ef_list(orc.new_eq(pt))
    p = ef_list(pt)
    for idx in [0, 1, 5, 33, 63]:
        want = F.ONE
        for t in range(6):
            want = F.ef_mul(want, p[t] if (idx >> t) & 1 else F.ef_sub(F.ONE, p[t]))
        assert eq[idx] == want  # point[0] is the lowest index bit
    folded = orc.mle_fold(ev, pt[:2])
    assert orc.mle_eval(folded, pt[2:]) == orc.mle_eval(ev, pt)


# ---- sumcheck (utils/src/sumcheck.rs:156-183) ----------------------------------------------------
def _hypercube_sum(polys):
    tot = F.ZERO
    for i in range(polys[0].shape[0]):
        prod = F.ONE
        for p in polys:
            prod = F.ef_mul(prod, (int(p[i, 0]), int(p[i, 1])))
        tot = F.ef_add(tot, prod)
    return tot


def test_product_sumcheck_round_trip(orc):
    polys = [rng.ext_elements(20 + j, 1 << 10) for j in range(3)]
    fields = rng.ext_elements(30, 10)
    rounds, finals, ch = orc.sumcheck_prove(polys, fields)
    claim = _hypercube_sum(polys)
    assert orc.sumcheck_verify(claim, rounds, finals, fields)
    assert not orc.sumcheck_verify(F.ef_add(claim, F.ONE), rounds, finals, fields)
    assert ef_list(ch) == ef_list(fields)


def test_tampered_round_is_rejected(orc):
    polys = [rng.ext_elements(40 + j, 1 << 8) for j in range(3)]
    fields = rng.ext_elements(50, 8)
    rounds, finals, _ = orc.sumcheck_prove(polys, fields)
    claim = _hypercube_sum(polys)
    rounds[2, 3, 0] = (int(rounds[2, 3, 0]) + 1) % P
    assert not orc.sumcheck_verify(claim, rounds, finals, fields)


# ---- subset-sum hash (pcs/src/subset_sum.rs:90-124) ---------------------------------------------
def test_hash_columns_match_naive(orc):
    m, cols = 2, 10  # width 128
    A = rng.field_elements(60, 32 * 64 * m).reshape(32, 64 * m)
    cw = rng.field_elements(61, m * cols).reshape(m, cols)
    H = orc.hash_columns(A, cw)
    for j in range(cols):
        bits = [(int(cw[i // 64, j]) >> (i % 64)) & 1 for i in range(64 * m)]
        for r in range(32):
            assert int(H[r, j]) == sum(int(A[r, i]) for i in range(64 * m) if bits[i]) % P


# ---- LigeSIS (pcs/src/ligesis.rs:808-868) ---------------------------------------------------------
@pytest.fixture(scope="module")
def ligesis_small(orc):
    log_m, log_n = 3, 10
    f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=100)
    key = orc.Key(log_m, log_n, A)
    cm = orc.Commitment(key, f)
    proof, cur = orc.prove(key, cm, z, fields, ints)
    return dict(log_m=log_m, log_n=log_n, f=f, A=A, z=z, fields=fields, ints=ints, key=key, cm=cm,
                proof=proof, cur=cur)


def test_ligesis_round_trip(orc, ligesis_small):
    s = ligesis_small
    pf = codec.decode(s["proof"])
    lifted = np.stack([s["f"], np.zeros_like(s["f"])], axis=1)
    assert pf.y == orc.mle_eval(lifted, s["z"])
    assert orc.verify(s["key"].com_a, s["log_m"], s["log_n"], s["cm"].root, s["z"], s["proof"],
                      s["fields"], s["ints"])
    assert codec.encode(pf) == s["proof"]


def _tamper(proof: bytes, edit) -> bytes:
    pf = codec.decode(proof)
    edit(pf)
    return codec.encode(pf)


@pytest.mark.parametrize("what", ["y", "sumcheck", "h_column", "batch_msg", "base_leaf"])
def test_ligesis_tampering_is_rejected(orc, ligesis_small, what):
    s = ligesis_small

    def edit(pf):
        if what == "y":
            pf.y = ((pf.y[0] + 1) % P, pf.y[1])
        elif what == "sumcheck":
            rp = pf.sumchecks["sc_hash"].round_polys
            rp[0][0] = ((rp[0][0][0] + 1) % P, rp[0][0][1])
        elif what == "h_column":
            pf.h_cols[0][0] = (pf.h_cols[0][0] + 1) % P
        elif what == "batch_msg":
            m = pf.batch.reduction_msgs[0]
            m[0] = ((m[0][0] + 1) % P, m[0][1])
        else:
            op = pf.batch.base_bf[0]
            k = min(op.values)
            op.values[k][0] = (op.values[k][0] + 1) % P

    bad = _tamper(s["proof"], edit)
    assert bad != s["proof"]
    assert not orc.verify(s["key"].com_a, s["log_m"], s["log_n"], s["cm"].root, s["z"], bad,
                          s["fields"], s["ints"])


def test_ligesis_rejects_truncated_and_wrong_point(orc, ligesis_small):
    s = ligesis_small
    args = (s["key"].com_a, s["log_m"], s["log_n"], s["cm"].root)
    assert not orc.verify(*args, s["z"], s["proof"][:-1], s["fields"], s["ints"])
    z2 = s["z"].copy()
    z2[0, 0] = (int(z2[0, 0]) + 1) % P
    assert not orc.verify(*args, z2, s["proof"], s["fields"], s["ints"])


def test_setup_rejects_shapes_outside_window(orc):
    assert orc.lib().orc_shape_ok(7, 17) == 1
    assert orc.lib().orc_shape_ok(10, 10) == 0  # counts [21, 23, 10]
    assert orc.lib().orc_shape_ok(3, 10) == 1


# ---- standalone Basefold (pcs/src/basefold.rs:1055-1146, restated on the oracle) ----
def _basefold_case(orc, is_ef, n=12, code_rate=2, li=6, seed=90):
    poly = rng.ext_elements(seed, 1 << n) if is_ef else rng.field_elements(seed, 1 << n)
    cm = orc.BasefoldCommitment(poly, is_ef, code_rate, li)
    pt = rng.ext_elements(seed + 1, n)
    g = rng.SeededRng(seed + 2)
    fields, ints = g.ext_elements(512), g.ints(512)
    pf, cur = orc.basefold_prove(cm, pt, fields, ints)
    return poly, cm, pt, fields, ints, pf, cur


@pytest.mark.parametrize("is_ef", [False, True])
def test_basefold_round_trip(orc, is_ef):
    # commit_prove_verify_round_trip / commit_ext_round_trip: claimed_eval is the MLE value and
    # verify accepts from the restarted oracle
    poly, cm, pt, fields, ints, pf, cur = _basefold_case(orc, is_ef)
    ev = poly if is_ef else np.stack([poly, np.zeros_like(poly)], axis=1)
    want = orc.mle_eval(ev, pt)
    got = np.frombuffer(pf[24:40], dtype=np.uint64)
    assert [int(x) for x in got] == [int(x) for x in want]
    assert cur == (12 - 6, 50)  # n - log_interleave fields, ceil(100 / code_rate) ints
    assert orc.basefold_verify(cm.root, pt, pf, fields, ints)


def test_basefold_tampered_message_is_rejected(orc):
    # tampered_proof_is_rejected: reduction_msgs[0].0 += 1
    _, cm, pt, fields, ints, pf, _ = _basefold_case(orc, False)
    b = bytearray(pf)
    c0 = int.from_bytes(b[44:52], "little")
    b[44:52] = ((c0 + 1) % P).to_bytes(8, "little")
    assert not orc.basefold_verify(cm.root, pt, bytes(b), fields, ints)
    assert not orc.basefold_verify(cm.root, pt, pf[:-1], fields, ints)
    wrong_pt = np.array(pt, dtype=np.uint64).copy()
    wrong_pt[0, 0] ^= np.uint64(1)
    assert not orc.basefold_verify(cm.root, wrong_pt, pf, fields, ints)


def test_commit_only_key_commits_like_setup_key(orc):
    """The oracle's commit-only key gives the same commitment as setup's key where both exist."""
    from tests.helpers import ligesis_inputs

    f, A, _, _, _ = ligesis_inputs(3, 10, seed=44)
    full = orc.Commitment(orc.Key(3, 10, A), f)
    only = orc.Commitment(orc.Key(3, 10, A, commit_only=True), f)
    assert full.root == only.root
    assert np.array_equal(full.digest(), only.digest())
