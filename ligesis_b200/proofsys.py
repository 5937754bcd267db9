"""proofsys' integer witness on the GPU, over liblgs.so (include/lgs.h):

* `linear_witness(x, w, bias, divisor)`: the rescaled linear layer of the integer GPT-2
  (proofsys/src/model.rs:360-374 with the Matrix kernels of proofsys/src/tensor.rs) ->
  (q, rem, y, y_field): q, rem = x.matmul(w).floor_div_const_with_rem(divisor),
  y = q.add_row_vector(bias), y_field = encode_i64(y) as canonical Goldilocks.  With
  w_transposed, x.matmul_transposed_rhs(w) (the vocabulary head, model.rs:225-228).  int64 numpy
  arrays, or CUDA int64 tensors (then the outputs are CUDA tensors too).
* `layer_norm_witness(x, gain, bias)`: layer_norm (model.rs:241-279) -> (sum_x, sum_x2, var_sum,
  std, dividend, quotient, output).
* `softmax_witness`, `lut_gather`: the attention's causal softmax with its exp table and the
  MLP's GELU table (model.rs:409-443, :362-373).
* `block_witness`, `forward_witness`: one block's and the whole forward's witness
  (model.rs:208-237), every step on the GPU.
* `canonical_online`: the merged polynomials of the witness types in the canonical commitment
  layout (proofsys/src/canonical.rs:249-331), ready for a PolyCommitmentScheme backend
  (ligesis_b200.pcs).
* `encode_i64` (proofsys/src/witness.rs:102-108).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import field as fld
from ._lib import Context, check, i64p, load, ptr64

GPT2_31 = {"n_seq": 31, "d_model": 768, "mlp_hidden": 3072, "vocab": 50257, "scale": 1 << 12,
           "max_v": 200}  # Config::gpt2_31 (proofsys/src/witness.rs:19-31)


def encode_i64(x) -> np.ndarray:
    """encode_i64 (proofsys/src/witness.rs:102-108): x >= 0 -> x mod p, else -(|x| mod p)."""
    a = np.asarray(x, dtype=np.int64)
    flat = np.atleast_1d(a)
    u = flat.view(np.uint64)
    neg = flat < 0
    p = np.uint64(fld.P)
    mag = np.where(neg, (~u) + np.uint64(1), u) % p  # |x|, two's complement (exact at -2^63)
    return np.where(neg & (mag != 0), p - mag, mag).reshape(a.shape)


def _ptr(t):
    return C.cast(C.c_void_p(t.data_ptr()), i64p)


def linear_witness(x, w, bias, divisor: int, w_transposed: bool = False,
                   ctx: Context | None = None):
    ctx = ctx or Context.default()
    if hasattr(x, "is_cuda") and x.is_cuda:
        import torch

        rows, inner = x.shape
        cols = w.shape[0] if w_transposed else w.shape[1]
        if (w.shape[1] if w_transposed else w.shape[0]) != inner:
            raise ValueError("linear witness: inner dimensions differ")
        dev = x.device
        xc, wc = x.contiguous(), w.contiguous()
        bc = None if bias is None else bias.contiguous()
        q = torch.empty((rows, cols), dtype=torch.int64, device=dev)
        rem, y, yf = torch.empty_like(q), torch.empty_like(q), torch.empty_like(q)
        # the context's stream waits for the operands' producer (torch's current stream), in
        # stream order; the call returns once its own stream has finished
        torch.cuda.ExternalStream(ctx.stream_ptr, device=dev).wait_stream(
            torch.cuda.current_stream(dev))
        check(load().lgs_linear_witness(ctx.handle, _ptr(xc), rows, inner, _ptr(wc), cols,
                                        int(w_transposed), None if bc is None else _ptr(bc),
                                        int(divisor), 1, _ptr(q), _ptr(rem), _ptr(y),
                                        C.cast(C.c_void_p(yf.data_ptr()), C.POINTER(C.c_uint64))))
        return q, rem, y, yf
    xa = np.ascontiguousarray(x, dtype=np.int64)
    wa = np.ascontiguousarray(w, dtype=np.int64)
    rows, inner = xa.shape
    cols = wa.shape[0] if w_transposed else wa.shape[1]
    if (wa.shape[1] if w_transposed else wa.shape[0]) != inner:
        raise ValueError("linear witness: inner dimensions differ")
    ba = None if bias is None else np.ascontiguousarray(bias, dtype=np.int64)
    if ba is not None and ba.shape != (cols,):
        raise ValueError("linear witness: bias must hold one value per column")
    q = np.empty((rows, cols), np.int64)
    rem, y = np.empty_like(q), np.empty_like(q)
    yf = np.empty((rows, cols), np.uint64)
    p = lambda a: a.ctypes.data_as(i64p)
    check(load().lgs_linear_witness(ctx.handle, p(xa), rows, inner, p(wa), cols,
                                    int(w_transposed), None if ba is None else p(ba),
                                    int(divisor), 0, p(q), p(rem), p(y), ptr64(yf)))
    return q, rem, y, yf


def layer_norm_witness(x, gain, bias, ctx: Context | None = None):
    """layer_norm (proofsys/src/model.rs:241-279) on the GPU: (sum_x, sum_x2, var_sum, std,
    dividend, quotient, output), the first four per row, the rest per entry.  Host int64 arrays."""
    ctx = ctx or Context.default()
    xa = np.ascontiguousarray(x, dtype=np.int64)
    rows, d = xa.shape
    ga = np.ascontiguousarray(gain, dtype=np.int64)
    ba = np.ascontiguousarray(bias, dtype=np.int64)
    if ga.shape != (d,) or ba.shape != (d,):
        raise ValueError("layer norm witness: gain and bias hold one value per column")
    per_row = [np.empty(rows, np.int64) for _ in range(4)]
    per_ent = [np.empty((rows, d), np.int64) for _ in range(3)]
    p = lambda a: a.ctypes.data_as(i64p)
    check(load().lgs_layer_norm_witness(ctx.handle, p(xa), rows, d, p(ga), p(ba), 0,
                                        *[p(a) for a in per_row + per_ent]))
    return tuple(per_row + per_ent)


def _call_small(fn, *args):
    check(fn(*args))


def softmax_witness(scores, exp_lut, offset: int, scale: int, ctx: Context | None = None):
    """The causal softmax of the integer GPT-2 (model.rs:409-443) over heads x n x n scores:
    (x_max (heads, n), exp (heads, n, n), sum_exp (heads, n), prob (heads, n, n))."""
    ctx = ctx or Context.default()
    s = np.ascontiguousarray(scores, dtype=np.int64)
    if s.ndim == 2:
        s = s[None]
    heads, n, n2 = s.shape
    if n != n2:
        raise ValueError("softmax witness: square score matrices")
    lut = np.ascontiguousarray(exp_lut, dtype=np.int64)
    xm, se = np.empty((heads, n), np.int64), np.empty((heads, n), np.int64)
    ex, pr = np.empty((heads, n, n), np.int64), np.empty((heads, n, n), np.int64)
    p = lambda a: a.ctypes.data_as(i64p)
    check(load().lgs_softmax_witness(ctx.handle, p(s), heads, n, p(lut), lut.size, int(offset),
                                     int(scale), 0, p(xm), p(ex), p(se), p(pr)))
    return xm, ex, se, pr


def lut_gather(v, lut, offset: int, ctx: Context | None = None):
    """lut[v + offset] elementwise (the GELU activation, model.rs:362-373)."""
    ctx = ctx or Context.default()
    va = np.ascontiguousarray(v, dtype=np.int64)
    la = np.ascontiguousarray(lut, dtype=np.int64)
    out = np.empty_like(va)
    p = lambda a: a.ctypes.data_as(i64p)
    check(load().lgs_lut_gather(ctx.handle, p(va), va.size, p(la), la.size, int(offset), 0,
                                p(out)))
    return out


# The fields of one block's witness (BlockWitness of proofsys/src/witness.rs: ln1, attention, ln2,
# mlp), in the order block_witness returns them.
LN_FIELDS = ("sum_x", "sum_x2", "var_sum", "std", "dividend", "quotient", "output")
ATTN_FIELDS = ("q_qkv", "qkv", "scores", "x_max", "exp", "sum_exp", "q_prob", "q_ao_heads",
               "q_ao", "q_apr", "x_out", "rem_qkv", "rem_sc", "rem_ao_heads", "rem_apr")
MLP_FIELDS = ("q_fc", "fc", "act", "q_fpr", "x_out", "rem_fc", "rem_fpr")
BLOCK_FIELDS = (tuple("ln1." + f for f in LN_FIELDS) + tuple("attn." + f for f in ATTN_FIELDS)
                + tuple("ln2." + f for f in LN_FIELDS) + tuple("mlp." + f for f in MLP_FIELDS))
WEIGHT_NAMES = ("ln_1_g", "ln_1_b", "attn_w", "attn_b", "attn_proj_w", "attn_proj_b", "ln_2_g",
                "ln_2_b", "fc_w", "fc_b", "fproj_w", "fproj_b")


def block_witness(x, w: dict, exp_lut, gelu_lut, cfg: dict = GPT2_31,
                  ctx: Context | None = None) -> dict:
    """One block of the integer GPT-2 forward (model.rs:213-221): ln1, attention (qkv, per-head
    scores, softmax, weighted values, projection, residual), ln2 and the MLP (fc, GELU lookup,
    projection, residual), every step on the GPU.  `w` holds WEIGHT_NAMES (matrices row-major:
    attn_w d x 3d, attn_proj_w d x d, fc_w d x hidden, fproj_w hidden x d).  Returns the witness
    keyed by BLOCK_FIELDS."""
    n, d = cfg["n_seq"], cfg["d_model"]
    H = cfg.get("n_head", 12)
    dh = d // H
    sc = cfg["scale"]
    sqrt_d_scale = sc * int(round(dh ** 0.5))  # Config::sqrt_d_scale (witness.rs:33-35)
    offset = cfg["max_v"] * sc
    x = np.ascontiguousarray(x, dtype=np.int64)
    out = {}
    ln1 = layer_norm_witness(x, w["ln_1_g"], w["ln_1_b"], ctx)
    out.update({"ln1." + f: v for f, v in zip(LN_FIELDS, ln1)})
    q_qkv, rem_qkv, qkv, _ = linear_witness(ln1[6], w["attn_w"], w["attn_b"], sc, False, ctx)
    qh = qkv[:, :d].reshape(n, H, dh).transpose(1, 0, 2)
    kh = qkv[:, d:2 * d].reshape(n, H, dh).transpose(1, 0, 2)
    vh = qkv[:, 2 * d:].reshape(n, H, dh).transpose(1, 0, 2)
    scores = np.empty((H, n, n), np.int64)
    rem_sc = np.empty_like(scores)
    for h in range(H):
        scores[h], rem_sc[h], _, _ = linear_witness(qh[h], kh[h], None, sqrt_d_scale, True, ctx)
    xm, ex, se, prob = softmax_witness(scores, exp_lut, offset, sc, ctx)
    aoh = np.empty((H, n, dh), np.int64)
    rao = np.empty_like(aoh)
    for h in range(H):
        aoh[h], rao[h], _, _ = linear_witness(prob[h], vh[h], None, sc, False, ctx)
    merged = np.ascontiguousarray(aoh.transpose(1, 0, 2).reshape(n, d))
    q_apr, rem_apr, proj, _ = linear_witness(merged, w["attn_proj_w"], w["attn_proj_b"], sc,
                                             False, ctx)
    attn_out = x + proj
    vals = (q_qkv, qkv, scores, xm, ex, se, prob, aoh, merged, q_apr, attn_out, rem_qkv, rem_sc,
            rao, rem_apr)
    out.update({"attn." + f: v for f, v in zip(ATTN_FIELDS, vals)})
    ln2 = layer_norm_witness(attn_out, w["ln_2_g"], w["ln_2_b"], ctx)
    out.update({"ln2." + f: v for f, v in zip(LN_FIELDS, ln2)})
    q_fc, rem_fc, fc, _ = linear_witness(ln2[6], w["fc_w"], w["fc_b"], sc, False, ctx)
    act = lut_gather(fc, gelu_lut, offset, ctx)
    q_fpr, rem_fpr, fpr, _ = linear_witness(act, w["fproj_w"], w["fproj_b"], sc, False, ctx)
    vals = (q_fc, fc, act, q_fpr, attn_out + fpr, rem_fc, rem_fpr)
    out.update({"mlp." + f: v for f, v in zip(MLP_FIELDS, vals)})
    return out


def synthetic_block(seed: int, cfg: dict = GPT2_31):
    """Seeded weights, lookup tables and input for one block, sized so that every lookup index
    stays inside its table (no exported model here): x ~ +-2^18, gains ~ scale / 32, matrix entries
    ~ +-2^6, biases ~ +-2^10; exp table positive and decreasing toward small indices, GELU table
    increasing."""
    g = np.random.default_rng(seed)
    n, d, hid, sc = cfg["n_seq"], cfg["d_model"], cfg["mlp_hidden"], cfg["scale"]
    r = lambda shape, b: g.integers(-(1 << b), 1 << b, size=shape, dtype=np.int64)
    w = {"ln_1_g": g.integers(sc // 48, sc // 24, size=d, dtype=np.int64), "ln_1_b": r(d, 10),
         "attn_w": r((d, 3 * d), 6), "attn_b": r(3 * d, 10), "attn_proj_w": r((d, d), 6),
         "attn_proj_b": r(d, 10), "ln_2_g": g.integers(sc // 48, sc // 24, size=d, dtype=np.int64),
         "ln_2_b": r(d, 10), "fc_w": r((d, hid), 6), "fc_b": r(hid, 10), "fproj_w": r((hid, d), 6),
         "fproj_b": r(d, 10)}
    off = cfg["max_v"] * sc
    idx = np.arange(off + 1, dtype=np.float64)
    exp_lut = np.maximum(1, np.round(sc * np.exp((idx - off) / sc))).astype(np.int64)
    gidx = np.arange(2 * off + 1, dtype=np.float64) - off
    gelu_lut = np.round(np.maximum(gidx, 0) + gidx / 64).astype(np.int64)
    return r((n, d), 18), w, exp_lut, gelu_lut


def forward_witness(x0, blocks, ln_f_g, ln_f_b, wte, exp_lut, gelu_lut, cfg: dict = GPT2_31,
                    ctx: Context | None = None) -> dict:
    """The integer GPT-2 forward's witness (proofsys/src/model.rs:208-237) on the GPU: every
    block's witness (`block_witness`, each block's input the previous mlp.x_out), the final
    layer norm, and the vocabulary head q_log, rem_log = floor_div(lnf.output wteᵀ, scale).
    Returns {"blocks": [block dicts], "lnf": 7 layer-norm arrays, "q_log", "rem_log"}."""
    x = np.ascontiguousarray(x0, dtype=np.int64)
    out = {"blocks": []}
    for w in blocks:
        b = block_witness(x, w, exp_lut, gelu_lut, cfg, ctx)
        out["blocks"].append(b)
        x = b["mlp.x_out"]
    out["lnf"] = layer_norm_witness(x, ln_f_g, ln_f_b, ctx)
    q, rem, _, _ = linear_witness(out["lnf"][6], wte, None, cfg["scale"], True, ctx)
    out["q_log"], out["rem_log"] = q, rem
    return out


# ---- the canonical online commitment layout (proofsys/src/canonical.rs:75-331) ----------------
def _np2(x: int) -> int:
    return 1 << max(0, (int(x) - 1).bit_length())


def _stack_matrices(mats, pad: int = 0) -> np.ndarray:
    """commit_matrices (canonical.rs:135-158) with stack_instances (commit.rs:32-41): each matrix
    padded to row_pow x col_pow (column on the low variables), instances on the high variables,
    values encode_i64'd."""
    m0 = np.asarray(mats[0])
    rows, cols = (m0.shape[0], 1) if m0.ndim == 1 else m0.shape
    rp, cp = _np2(rows), _np2(cols)
    k = _np2(len(mats))
    out = np.full((k, rp, cp), encode_i64(np.int64(pad)), dtype=np.uint64)
    if pad == 0:
        out[:] = 0
    for i, m in enumerate(mats):
        a = np.asarray(m, dtype=np.int64)
        a = a.reshape(-1, 1) if a.ndim == 1 else a
        out[i, :a.shape[0], :a.shape[1]] = encode_i64(a)
    return out.reshape(-1)


def _stack_vectors_padded(vecs, pad: int) -> np.ndarray:
    """commit_vectors_padded (canonical.rs:164-181): padding rows and instances hold pad."""
    rp, k = _np2(len(vecs[0])), _np2(len(vecs))
    out = np.full((k, rp), int(encode_i64(np.int64(pad))), dtype=np.uint64)
    for i, v in enumerate(vecs):
        out[i, :len(v)] = encode_i64(np.asarray(v, dtype=np.int64))
    return out.reshape(-1)


CANONICAL_TYPES = ("q_ln", "a_ln", "std", "var", "q_sc", "exp", "q_prob", "x_max", "sum_exp",
                   "q_qkv", "q_ao", "q_apr", "q_fc", "act", "q_fpr", "x_out", "q_log")


def canonical_online(fw: dict) -> dict:
    """build_online (canonical.rs:249-331): the merged polynomial of every witness type of a
    `forward_witness`, as Goldilocks values (uint64) of 2^(instance + row + column variables)
    entries, keyed by CANONICAL_TYPES.  Layer norms in the order [ln1_0, ln2_0, ..., lnf], heads
    12 l + h, x_out [attn_0, mlp_0, ...]; `std` and `sum_exp` pad with 1, everything else with 0."""
    blocks = fw["blocks"]
    lns = []
    for b in blocks:
        lns.append([b["ln1." + f] for f in LN_FIELDS])
        lns.append([b["ln2." + f] for f in LN_FIELDS])
    lns.append(list(fw["lnf"]))
    heads = lambda key: [b[key][h] for b in blocks for h in range(b[key].shape[0])]
    per_layer = lambda key: [b[key] for b in blocks]
    x_out = []
    for b in blocks:
        x_out += [b["attn.x_out"], b["mlp.x_out"]]
    return {
        "q_ln": _stack_matrices([ln[5] for ln in lns]),
        "a_ln": _stack_matrices([ln[4] for ln in lns]),
        "std": _stack_vectors_padded([ln[3] for ln in lns], 1),
        "var": _stack_vectors_padded([ln[2] for ln in lns], 0),
        "q_sc": _stack_matrices(heads("attn.scores")),
        "exp": _stack_matrices(heads("attn.exp")),
        "q_prob": _stack_matrices(heads("attn.q_prob")),
        "x_max": _stack_matrices(heads("attn.x_max")),
        "sum_exp": _stack_vectors_padded(heads("attn.sum_exp"), 1),
        "q_qkv": _stack_matrices(per_layer("attn.q_qkv")),
        "q_ao": _stack_matrices(per_layer("attn.q_ao")),
        "q_apr": _stack_matrices(per_layer("attn.q_apr")),
        "q_fc": _stack_matrices(per_layer("mlp.q_fc")),
        "act": _stack_matrices(per_layer("mlp.act")),
        "q_fpr": _stack_matrices(per_layer("mlp.q_fpr")),
        "x_out": _stack_matrices(x_out),
        "q_log": _stack_matrices([fw["q_log"]]),
    }
