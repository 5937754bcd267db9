"""proofsys' integer witness on the GPU, over liblgs.so (include/lgs.h):

* `linear_witness(x, w, bias, divisor)`: the rescaled linear layer of the integer GPT-2
  (proofsys/src/model.rs:360-374 with the Matrix kernels of proofsys/src/tensor.rs) ->
  (q, rem, y, y_field): q, rem = x.matmul(w).floor_div_const_with_rem(divisor),
  y = q.add_row_vector(bias), y_field = encode_i64(y) as canonical Goldilocks.  With
  w_transposed, x.matmul_transposed_rhs(w) (the vocabulary head, model.rs:225-228).  int64 numpy
  arrays, or CUDA int64 tensors (then the outputs are CUDA tensors too).
* `layer_norm_witness(x, gain, bias)`: layer_norm (model.rs:241-279) -> (sum_x, sum_x2, var_sum,
  std, dividend, quotient, output).
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
    mag = np.where(a >= 0, a.astype(np.uint64),
                   (-(a + 1)).astype(np.uint64) + np.uint64(1)) % np.uint64(fld.P)
    neg = (a < 0) & (mag != 0)
    return np.where(neg, np.uint64(fld.P) - mag, mag)


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
        q = torch.empty((rows, cols), dtype=torch.int64, device=dev)
        rem, y, yf = torch.empty_like(q), torch.empty_like(q), torch.empty_like(q)
        torch.cuda.synchronize(dev)
        check(load().lgs_linear_witness(ctx.handle, _ptr(x.contiguous()), rows, inner,
                                        _ptr(w.contiguous()), cols, int(w_transposed),
                                        None if bias is None else _ptr(bias.contiguous()),
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
