"""The oracle's proofsys linear-layer witness (proofsys/src/tensor.rs:51-133, :194-216;
witness.rs:102-108) against Python integers: i128-exact products, floor division with a
non-negative remainder for negative values, the bias row, encode_i64, and the overflow check."""
from __future__ import annotations

import numpy as np
import pytest

from ligesis_b200 import field as fld


def _py(x, w, bias, d, wt):
    rows, inner = x.shape
    cols = w.shape[0] if wt else w.shape[1]
    q = np.zeros((rows, cols), dtype=object)
    r = np.zeros_like(q)
    y = np.zeros_like(q)
    for i in range(rows):
        for j in range(cols):
            acc = sum(int(x[i, k]) * int(w[j, k] if wt else w[k, j]) for k in range(inner))
            qq = acc // d  # Python floors
            q[i, j], r[i, j] = qq, acc - qq * d
            y[i, j] = qq + (0 if bias is None else int(bias[j]))
    return q, r, y


@pytest.mark.parametrize("wt", [False, True])
def test_linear_witness_matches_python(orc, wt):
    g = np.random.default_rng(3)
    x = g.integers(-(1 << 20), 1 << 20, size=(7, 33), dtype=np.int64)
    w = g.integers(-(1 << 15), 1 << 15, size=(5, 33) if wt else (33, 5), dtype=np.int64)
    b = g.integers(-(1 << 30), 1 << 30, size=5, dtype=np.int64)
    q, r, y, yf = orc.linear_witness(x, w, b, 4096, wt)
    wq, wr, wy = _py(x, w, b, 4096, wt)
    assert (q == wq.astype(np.int64)).all() and (r == wr.astype(np.int64)).all()
    assert (y == wy.astype(np.int64)).all()
    assert (r >= 0).all() and (r < 4096).all() and (q < 0).any()
    assert all(int(yf.flat[i]) == int(y.flat[i]) % fld.P for i in range(y.size))


def test_linear_witness_edges(orc):
    x = np.array([[-1, 0], [1 << 62, 1]], dtype=np.int64)
    w = np.array([[1], [1]], dtype=np.int64)
    q, r, y, yf = orc.linear_witness(x, w, None, 3)
    assert q.ravel().tolist() == [-1, (1 << 62) // 3] and r.ravel().tolist() == [2, ((1 << 62) + 1) % 3]
    assert int(yf[0, 0]) == fld.P - 1
    big = np.array([[1 << 40]], dtype=np.int64)
    with pytest.raises(Exception):
        orc.linear_witness(big, big, None, 1)  # 2^80 does not fit an i64


def test_encode_i64_mirror():
    from ligesis_b200.proofsys import encode_i64

    xs = np.array([0, 1, -1, 5, -5, (1 << 63) - 1, -(1 << 63), fld.P - 1 - (1 << 63)], dtype=object)
    a = np.array([int(v) for v in xs], dtype=np.int64)
    want = [int(v) % fld.P for v in a.tolist()]
    assert encode_i64(a).tolist() == want


def test_layer_norm_witness_matches_python(orc):
    import math

    g = np.random.default_rng(5)
    x = g.integers(-(1 << 20), 1 << 20, size=(4, 48), dtype=np.int64)
    gain = g.integers(-(1 << 13), 1 << 13, size=48, dtype=np.int64)
    bias = g.integers(-(1 << 13), 1 << 13, size=48, dtype=np.int64)
    sx, sx2, vs, st, dv, qu, out = orc.layer_norm_witness(x, gain, bias)
    d = 48
    for r in range(4):
        row = [int(v) for v in x[r]]
        s1, s2 = sum(row), sum(v * v for v in row)
        v = s2 * d - s1 * s1
        root = math.sqrt(float(v + 1))
        rs = math.floor(root + 0.5)  # half away from zero for a non-negative value
        assert (int(sx[r]), int(sx2[r]), int(vs[r]), int(st[r])) == (s1, s2, v, rs)
        for c in range(d):
            a = int(gain[c]) * (d * row[c] - s1)
            assert int(dv[r, c]) == a and int(qu[r, c]) == a // rs
            assert int(out[r, c]) == a // rs + int(bias[c])


def test_block_witness_structure(orc):
    """The oracle's GPT-2 block (proofsys/src/model.rs:213-443) on a small config: causal softmax
    (zeros above the diagonal, row maxima over the causal part, probabilities summing to at most
    scale), residuals, and the GELU lookup."""
    from ligesis_b200 import proofsys as ps

    cfg = dict(ps.GPT2_31, n_seq=5, d_model=64, mlp_hidden=128, n_head=4)
    x, w, el, gl = ps.synthetic_block(9, cfg)
    o = orc.block_witness(x, w, el, gl, cfg)
    n, sc, off = 5, cfg["scale"], cfg["max_v"] * cfg["scale"]
    ex, pr, sco = o["attn.exp"], o["attn.q_prob"], o["attn.scores"]
    for h in range(4):
        for i in range(n):
            assert o["attn.x_max"][h, i] == sco[h, i, :i + 1].max()
            assert not ex[h, i, i + 1:].any() and not pr[h, i, i + 1:].any()
            assert 0 < pr[h, i, :i + 1].sum() <= sc
            assert ex[h, i, :i + 1].tolist() == [int(el[v - sco[h, i, :i + 1].max() + off])
                                                 for v in sco[h, i, :i + 1]]
    assert np.array_equal(o["attn.x_out"], x + o["attn.q_apr"] + w["attn_proj_b"])
    assert np.array_equal(o["mlp.act"], gl[o["mlp.fc"] + off])
    assert np.array_equal(o["mlp.x_out"], o["attn.x_out"] + o["mlp.q_fpr"] + w["fproj_b"])


def test_canonical_layout_of_the_reference_tiny_model(orc):
    """The library's canonical layout (numpy) against the independent restatement of build_online
    (proofsys/src/canonical.rs:249-331) on the oracle's witness of the reference's tiny model."""
    from ligesis_b200 import proofsys as ps
    from tests.helpers import tiny_gpt

    cfg, x0, w, lg, lb, wte, el, gl = tiny_gpt()
    fw = orc.forward_witness(x0, [w], lg, lb, wte, el, gl, cfg)
    got, want = ps.canonical_online(fw), orc.canonical_online(fw)
    assert list(got) == list(ps.CANONICAL_TYPES) == list(want)
    for k in ps.CANONICAL_TYPES:
        assert got[k].tolist() == want[k], k
    assert len(got["q_ln"]) == 16 and got["std"].tolist()[-2:] == [1, 1]
