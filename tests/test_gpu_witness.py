"""proofsys' rescaled linear-layer witness on the GPU against the oracle (proofsys/src/tensor.rs,
model.rs:360-361): q, rem, y and encode_i64(y) equal element for element at GPT-2's layer shapes
and ragged ones, both operand layouts, host and device arrays, and the overflow error."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import proofsys as ps
from tests.helpers import tiny_gpt

pytestmark = pytest.mark.gpu


def _rand(seed, shape, bits):
    g = np.random.default_rng(seed)
    return g.integers(-(1 << bits), 1 << bits, size=shape, dtype=np.int64)


@pytest.mark.parametrize("rows,inner,cols,wt", [(31, 768, 3072, False), (31, 3072, 768, False),
                                                (31, 768, 2304, False), (5, 70, 33, False),
                                                (31, 768, 4099, True), (1, 1, 1, True),
                                                (67, 129, 65, True)])
def test_linear_witness_matches_oracle(lgs, orc, rows, inner, cols, wt):
    x = _rand(rows + inner, (rows, inner), 20)
    w = _rand(cols + 1, (cols, inner) if wt else (inner, cols), 15)
    b = _rand(cols + 2, cols, 30)
    got = ps.linear_witness(x, w, b, 1 << 12, wt)
    want = orc.linear_witness(x, w, b, 1 << 12, wt)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)
    assert np.array_equal(got[3], ps.encode_i64(got[2]))


def test_linear_witness_device_and_odd_divisor(lgs, orc):
    torch = pytest.importorskip("torch")
    x, w = _rand(1, (31, 768), 20), _rand(2, (768, 3072), 15)
    want = orc.linear_witness(x, w, None, 4097)
    got = ps.linear_witness(torch.from_numpy(x).cuda(), torch.from_numpy(w).cuda(), None, 4097)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_.cpu().numpy().view(w_.dtype), w_)


def test_linear_witness_overflow_is_an_error(lgs):
    big = np.full((2, 4), 1 << 40, dtype=np.int64)
    with pytest.raises(L.ShapeError):
        ps.linear_witness(big, big.T.copy(), None, 1)
    with pytest.raises(L.ShapeError):
        ps.linear_witness(big[:, :1], big[:1, :], None, 0)


@pytest.mark.parametrize("rows,d", [(31, 768), (1, 1), (3, 257), (64, 3072)])
def test_layer_norm_witness_matches_oracle(lgs, orc, rows, d):
    x = _rand(rows * 7 + d, (rows, d), 20)
    gain = _rand(d + 3, d, 13)
    bias = _rand(d + 4, d, 13)
    got = ps.layer_norm_witness(x, gain, bias)
    want = orc.layer_norm_witness(x, gain, bias)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)


def test_layer_norm_witness_constant_row(lgs, orc):
    x = np.full((2, 16), -12345, dtype=np.int64)  # zero variance: std = round_sqrt(1) = 1
    got = ps.layer_norm_witness(x, np.ones(16, np.int64), np.zeros(16, np.int64))
    assert got[3].tolist() == [1, 1] and not got[4].any()
    for g_, w_ in zip(got, orc.layer_norm_witness(x, np.ones(16, np.int64), np.zeros(16, np.int64))):
        assert np.array_equal(g_, w_)


@pytest.mark.parametrize("cfg_over", [{}, {"n_seq": 5, "d_model": 64, "mlp_hidden": 128,
                                           "n_head": 4}])
def test_block_witness_matches_oracle(lgs, orc, cfg_over):
    """One GPT-2 block's whole witness (36 arrays: ln1, attention with per-head scores, softmax
    and weighted values, ln2, MLP with the GELU lookup) equals the oracle's element for element."""
    cfg = {**ps.GPT2_31, "n_head": 12, **cfg_over}
    x, w, el, gl = ps.synthetic_block(11, cfg)
    got = ps.block_witness(x, w, el, gl, cfg)
    want = orc.block_witness(x, w, el, gl, cfg)
    assert set(got) == set(want) == set(ps.BLOCK_FIELDS)
    for k in ps.BLOCK_FIELDS:
        assert np.array_equal(got[k], want[k]), k


def test_softmax_and_gather_reject_out_of_table(lgs):
    s = np.zeros((1, 3, 3), dtype=np.int64)
    s[0, 2, 0] = -1000  # index -1000 + offset 10 < 0
    with pytest.raises(L.ShapeError):
        ps.softmax_witness(s, np.ones(11, np.int64), 10, 4)
    with pytest.raises(L.ShapeError):
        ps.lut_gather(np.array([5, 6], np.int64), np.ones(11, np.int64), 5)  # 6 + 5 = 11
    xm, ex, se, pr = ps.softmax_witness(np.zeros((1, 3, 3), np.int64), np.ones(11, np.int64), 10, 4)
    assert se.tolist() == [[1, 2, 3]] and pr[0].tolist() == [[4, 0, 0], [2, 2, 0], [1, 1, 1]]


def test_forward_witness_matches_oracle(lgs, orc):
    """A three-block forward with the final layer norm and a 4099-token vocabulary head (the
    block shape of GPT-2 small, fewer blocks and tokens to keep the oracle quick)."""
    cfg = {**ps.GPT2_31, "n_head": 12}
    x0, _, el, gl = ps.synthetic_block(20, cfg)
    blocks = [ps.synthetic_block(21 + i, cfg)[1] for i in range(3)]
    g = np.random.default_rng(30)
    ln_g = g.integers(cfg["scale"] // 48, cfg["scale"] // 24, size=768, dtype=np.int64)
    ln_b = g.integers(-1024, 1024, size=768, dtype=np.int64)
    wte = g.integers(-64, 64, size=(4099, 768), dtype=np.int64)
    got = ps.forward_witness(x0, blocks, ln_g, ln_b, wte, el, gl, cfg)
    want = orc.forward_witness(x0, blocks, ln_g, ln_b, wte, el, gl, cfg)
    for gb, wb in zip(got["blocks"], want["blocks"]):
        for k in ps.BLOCK_FIELDS:
            assert np.array_equal(gb[k], wb[k]), k
    for a, b in zip(got["lnf"], want["lnf"]):
        assert np.array_equal(a, b)
    assert np.array_equal(got["q_log"], want["q_log"])
    assert np.array_equal(got["rem_log"], want["rem_log"])


def test_canonical_commitment_of_the_reference_tiny_model(lgs, orc):
    """The reference's tiny model through the GPU forward witness equals the oracle's; its
    canonical merged polynomials equal an independent restatement of build_online; the
    reference's check (canonical.rs:363-385): q_ln's instance 1 (ln2 of layer 0) at row 1,
    column 0 reads ln2's quotient there; and every merged polynomial commits and opens with the
    Basefold backend of the PolyCommitmentScheme."""
    cfg, x0, w, lg, lb, wte, el, gl = tiny_gpt()
    fw = ps.forward_witness(x0, [w], lg, lb, wte, el, gl, cfg)
    ofw = orc.forward_witness(x0, [w], lg, lb, wte, el, gl, cfg)
    for k in ps.BLOCK_FIELDS:
        assert np.array_equal(fw["blocks"][0][k], ofw["blocks"][0][k]), k
    assert np.array_equal(fw["q_log"], ofw["q_log"])
    canon = ps.canonical_online(fw)
    want = orc.canonical_online(ofw)
    assert list(canon) == list(ps.CANONICAL_TYPES)
    for k in ps.CANONICAL_TYPES:
        assert canon[k].tolist() == want[k], k
    # q_ln: 3 instances -> 2 instance vars, rows 2 -> 1 var, cols 2 -> 1 var
    point = np.array([[0, 0], [1, 0], [1, 0], [0, 0]], dtype=np.uint64)  # col 0, row 1, inst 1
    ev = np.stack([canon["q_ln"], np.zeros_like(canon["q_ln"])], axis=1)
    want_v = int(ps.encode_i64(fw["blocks"][0]["ln2.quotient"][1, 0]))
    assert orc.mle_eval(ev, point) == (want_v, 0)
    pcs = L.BasefoldPcs(code_rate=1)
    from ligesis_b200 import rng

    oracle = L.RandomOracle(4, length=4096)
    tasks, claims = [], []
    for i, k in enumerate(ps.CANONICAL_TYPES):
        poly = L.MlPoly(canon[k])
        data, com = pcs.commit(poly)
        pt = rng.ext_elements(500 + i, poly.num_vars)
        tasks.append((data, pt))
        claims.append((com, pt, orc.mle_eval(np.stack([canon[k], np.zeros_like(canon[k])], 1), pt)))
    proof = pcs.batch_prove(tasks, oracle)
    oracle.restart()
    assert pcs.batch_verify(claims, proof, oracle)


@pytest.mark.parametrize("xb,wb,inner", [(20, 15, 3072), (40, 8, 64), (28, 28, 64), (40, 15, 64),
                                         (40, 21, 1), (31, 30, 2)])
def test_linear_witness_arithmetic_paths(lgs, orc, xb, wb, inner):
    """Operand sizes that select each exact path: fused multiply-adds of doubles (GPT-2's
    sizes), 64-bit products with 64-bit sums (40 + 8 and 40 + 15 bits), 32-bit products
    (28 + 28 bits), and 128-bit sums (wide operands whose results still fit an i64)."""
    ctx = L.Context(0)
    ctx.tune(witness_path=1)  # the CUDA-core kernel (the tensor cores would take 20 x 15 bits)
    x = _rand(xb + inner, (7, inner), xb)
    w = _rand(wb + inner, (inner, 9), wb)
    got = ps.linear_witness(x, w, None, 3, False, ctx)
    want = orc.linear_witness(x, w, None, 3)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)


@pytest.mark.parametrize("wt", [False, True])
def test_linear_witness_mixed_widths_across_k(lgs, orc, wt):
    """Each K stage of 32 picks its own exact arithmetic from the operands it stages: here the
    first stage needs 128-bit sums (38-bit x, 20-bit w), the second 64-bit products (36-bit x,
    18-bit w), the third 32-bit products (26-bit operands) and the rest doubles (12-bit
    operands), in one product and with K split over CTAs."""
    rows, inner, cols = 7, 4096, 9
    x = _rand(5, (rows, inner), 12)
    x[:, :32] = _rand(6, (rows, 32), 38)
    x[:, 32:64] = _rand(7, (rows, 32), 36)
    x[:, 64:96] = _rand(11, (rows, 32), 26)
    w = _rand(8, (inner, cols), 12)
    w[:32] = _rand(9, (32, cols), 20)
    w[32:64] = _rand(10, (32, cols), 18)
    w[64:96] = _rand(12, (32, cols), 26)
    if wt:
        w = np.ascontiguousarray(w.T)
    got = ps.linear_witness(x, w, None, 1 << 12, wt)
    want = orc.linear_witness(x, w, None, 1 << 12, wt)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)


@pytest.mark.parametrize("sign", [1, -1])
def test_linear_witness_double_path_at_its_bound(lgs, orc, sign):
    """Stages whose sums come closest to 2^53 still take the double path (40-bit by 8-bit
    operands, 32 products per stage: 32 (2^40 - 1) 255 < 2^53) and stay exact."""
    x = np.full((3, 96), sign * ((1 << 40) - 1), dtype=np.int64)
    w = np.full((96, 5), 255, dtype=np.int64)
    x[1, ::7] = -x[1, ::7]
    got = ps.linear_witness(x, w, None, 1 << 12)
    want = orc.linear_witness(x, w, None, 1 << 12)
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)
