"""ORACLE (test infrastructure only): ctypes access to the CPU restatement in oracle/*.hpp,
built into oracle/_build/liborc.so by oracle/Makefile.  Imported only by tests/, the smoke
check and bench.py's CPU-baseline leg, always as the checker or the timed CPU baseline."""
from __future__ import annotations

import ctypes as C
import struct
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liborc.so"
_lib = None
_lock = threading.Lock()

u64p = C.POINTER(C.c_uint64)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p


def build() -> Path:
    srcs = list(HERE.glob("*.hpp")) + list(HERE.glob("*.cpp")) + [HERE / "Makefile"]
    if LIB.exists() and LIB.stat().st_mtime >= max(s.stat().st_mtime for s in srcs):
        return LIB
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            l = C.CDLL(str(LIB))
            sig = {
                "orc_last_error": (C.c_char_p, []),
                "orc_free_buf": (None, [vp]),
                "orc_set_threads": (None, [C.c_uint]),
                "orc_get_threads": (C.c_uint, []),
                "orc_two_adic_generator": (C.c_int, [C.c_uint, u64p]),
                "orc_bf_ops": (C.c_int, [u64p, u64p, C.c_size_t, u64p, u64p, u64p]),
                "orc_ef_ops": (C.c_int, [u64p, u64p, C.c_size_t, u64p, u64p]),
                "orc_blake3": (C.c_int, [u8p, C.c_size_t, u8p]),
                "orc_dft_bf": (C.c_int, [u64p, C.c_size_t]),
                "orc_dft_ef": (C.c_int, [u64p, C.c_size_t]),
                "orc_mle_eval": (C.c_int, [u64p, C.c_size_t, u64p, u64p]),
                "orc_mle_fold": (C.c_int, [u64p, C.c_size_t, u64p, C.c_size_t]),
                "orc_new_eq": (C.c_int, [u64p, C.c_size_t, u64p]),
                "orc_hash_columns": (C.c_int, [u64p, C.c_size_t, u64p, C.c_size_t, C.c_size_t, u64p]),
                "orc_sumcheck_prove": (C.c_int, [u64p, C.c_size_t, C.c_size_t, u64p, C.c_size_t,
                                                 u64p, u64p, u64p]),
                "orc_sumcheck_verify": (C.c_int, [u64p, u64p, C.c_size_t, C.c_size_t, u64p, u64p,
                                                  C.c_size_t]),
                "orc_merkle_root": (C.c_int, [u8p, C.c_size_t, C.c_size_t, u8p]),
                "orc_merkle_open": (C.c_int, [u8p, C.c_size_t, C.c_size_t, u64p, C.c_size_t,
                                              C.POINTER(u8p), C.POINTER(C.c_size_t)]),
                "orc_merkle_verify": (C.c_int, [u8p, u8p, C.c_size_t, u64p, C.c_size_t, u8p,
                                                C.c_size_t, C.c_size_t]),
                "orc_shape_ok": (C.c_int, [C.c_uint, C.c_uint]),
                "orc_setup": (vp, [C.c_uint, C.c_uint, u64p, u8p]),
                "orc_setup_commit_only": (vp, [C.c_uint, C.c_uint, u64p]),
                "orc_key_free": (None, [vp]),
                "orc_commit": (vp, [vp, u64p, C.c_size_t, u8p]),
                "orc_commit_free": (None, [vp]),
                "orc_commit_codeword": (C.c_int, [vp, u64p]),
                "orc_commit_digest": (C.c_int, [vp, u64p]),
                "orc_prove": (C.c_int, [vp, vp, u64p, C.c_size_t, u64p, C.c_size_t, u64p,
                                        C.c_size_t, u64p, C.POINTER(u8p), C.POINTER(C.c_size_t)]),
                "orc_verify": (C.c_int, [u8p, C.c_uint, C.c_uint, u8p, u64p, C.c_size_t, u8p,
                                         C.c_size_t, u64p, C.c_size_t, u64p, C.c_size_t, u64p]),
                "orc_basefold_commit": (vp, [u64p, C.c_size_t, C.c_int, C.c_uint, C.c_uint, u8p]),
                "orc_basefold_free": (None, [vp]),
                "orc_basefold_prove": (C.c_int, [vp, u64p, C.c_size_t, u64p, C.c_size_t, u64p,
                                                 C.c_size_t, u64p, C.POINTER(u8p),
                                                 C.POINTER(C.c_size_t)]),
                "orc_basefold_verify": (C.c_int, [u8p, u64p, C.c_size_t, u8p, C.c_size_t, u64p,
                                                  C.c_size_t, u64p, C.c_size_t, u64p]),
                "orc_frac_sum_prove": (C.c_int, [u64p, u64p, C.c_size_t, u64p, C.c_size_t, u64p,
                                                 C.POINTER(u8p), C.POINTER(C.c_size_t), u64p,
                                                 u64p]),
                "orc_frac_sum_verify": (C.c_int, [u8p, C.c_size_t, u64p, C.c_size_t, u64p, u64p,
                                                  C.c_size_t, u64p]),
                "orc_lookup_prove": (C.c_int, [u64p, C.c_size_t, u64p, C.c_size_t, u64p, u64p,
                                               C.c_size_t, u64p, C.POINTER(u8p),
                                               C.POINTER(C.c_size_t), u64p, u64p]),
                "orc_linear_witness": (C.c_int, [i64p, C.c_size_t, C.c_size_t, i64p, C.c_size_t,
                                                 C.c_int, i64p, C.c_int64, i64p, i64p, i64p,
                                                 u64p]),
                "orc_layer_norm_witness": (C.c_int, [i64p, C.c_size_t, C.c_size_t, i64p, i64p,
                                                     i64p, i64p, i64p, i64p, i64p, i64p, i64p]),
                "orc_block_witness": (C.c_int, [i64p, u64p, i64p, C.POINTER(i64p), i64p,
                                                C.c_size_t, i64p, C.c_size_t, C.POINTER(i64p)]),
                "orc_lookup_verify": (C.c_int, [u8p, C.c_size_t, u64p, C.c_size_t, u64p, u64p,
                                                C.c_size_t, u64p, C.c_size_t, u64p]),
            }
            for name, (res, args) in sig.items():
                fn = getattr(l, name)
                fn.restype = res
                fn.argtypes = args
            _lib = l
    return _lib


def set_threads(n: int | None = None) -> int:
    """Threads for the oracle's independent bulk loops; None = every core this process may use.
    The outputs do not depend on the count (exact residues mod p)."""
    import os

    if n is None:
        n = len(os.sched_getaffinity(0))
    lib().orc_set_threads(int(n))
    return int(lib().orc_get_threads())


def _p64(a):
    return a.ctypes.data_as(u64p)


def _p8(a):
    return a.ctypes.data_as(u8p)


def _u64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


def _ok(rc):
    if rc < 0:
        raise RuntimeError("oracle: " + (lib().orc_last_error() or b"").decode())
    return rc


def two_adic_generator(bits: int) -> int:
    out = np.zeros(1, np.uint64)
    _ok(lib().orc_two_adic_generator(bits, _p64(out)))
    return int(out[0])


def bf_ops(a, b):
    a, b = _u64(a), _u64(b)
    s, d, p = (np.zeros_like(a) for _ in range(3))
    _ok(lib().orc_bf_ops(_p64(a), _p64(b), a.size, _p64(s), _p64(d), _p64(p)))
    return s, d, p


def ef_ops(a, b):
    a, b = _u64(a).reshape(-1, 2), _u64(b).reshape(-1, 2)
    prod, inv = np.zeros_like(a), np.zeros_like(a)
    _ok(lib().orc_ef_ops(_p64(a), _p64(b), a.shape[0], _p64(prod), _p64(inv)))
    return prod, inv


def blake3(data: bytes) -> bytes:
    buf = np.frombuffer(bytes(data) or b"\0", dtype=np.uint8).copy()
    out = np.zeros(32, np.uint8)
    _ok(lib().orc_blake3(_p8(buf), len(data), _p8(out)))
    return out.tobytes()


def dft_bf(coeffs, size: int) -> np.ndarray:
    a = np.zeros(size, np.uint64)
    c = _u64(coeffs)
    a[: c.size] = c
    _ok(lib().orc_dft_bf(_p64(a), size))
    return a


def dft_ef(coeffs, size: int) -> np.ndarray:
    a = np.zeros((size, 2), np.uint64)
    c = _u64(coeffs).reshape(-1, 2)
    a[: c.shape[0]] = c
    _ok(lib().orc_dft_ef(_p64(a), size))
    return a


def mle_eval(evals, point):
    e = _u64(evals).reshape(-1, 2).copy()
    p = _u64(point).reshape(-1, 2).copy()
    out = np.zeros(2, np.uint64)
    _ok(lib().orc_mle_eval(_p64(e), p.shape[0], _p64(p), _p64(out)))
    return (int(out[0]), int(out[1]))


def mle_fold(evals, point):
    e = _u64(evals).reshape(-1, 2).copy()
    p = _u64(point).reshape(-1, 2).copy()
    k = e.shape[0].bit_length() - 1
    _ok(lib().orc_mle_fold(_p64(e), k, _p64(p), p.shape[0]))
    return e[: e.shape[0] >> p.shape[0]]


def new_eq(point):
    p = _u64(point).reshape(-1, 2).copy()
    out = np.zeros((1 << p.shape[0], 2), np.uint64)
    _ok(lib().orc_new_eq(_p64(p), p.shape[0], _p64(out)))
    return out


def hash_columns(A, cw):
    A, cw = _u64(A), _u64(cw)
    m, two_n = cw.shape
    W = A.shape[1]
    H = np.zeros((32, two_n), np.uint64)
    _ok(lib().orc_hash_columns(_p64(A), W, _p64(cw), m, two_n, _p64(H)))
    return H


def sumcheck_prove(polys, fields):
    ps = [_u64(p).reshape(-1, 2) for p in polys]
    d, k = len(ps), ps[0].shape[0].bit_length() - 1
    flat = np.ascontiguousarray(np.concatenate(ps))
    f = _u64(fields).reshape(-1, 2).copy()
    rounds = np.zeros((k, d + 1, 2), np.uint64)
    finals = np.zeros((d, 2), np.uint64)
    ch = np.zeros((k, 2), np.uint64)
    _ok(lib().orc_sumcheck_prove(_p64(flat), d, k, _p64(f), f.shape[0], _p64(rounds),
                                 _p64(finals), _p64(ch)))
    return rounds, finals, ch


def sumcheck_verify(claim, rounds, finals, fields) -> bool:
    c = _u64(claim).reshape(2).copy()
    r = np.ascontiguousarray(_u64(rounds))
    f = np.ascontiguousarray(_u64(finals))
    fl = _u64(fields).reshape(-1, 2).copy()
    k, w = r.shape[0], r.shape[1]
    return bool(_ok(lib().orc_sumcheck_verify(_p64(c), _p64(r), k, w - 1, _p64(f), _p64(fl),
                                              fl.shape[0])))


def merkle_root(leaves: np.ndarray) -> bytes:
    lv = np.ascontiguousarray(leaves).view(np.uint8).reshape(leaves.shape[0], -1)
    out = np.zeros(32, np.uint8)
    _ok(lib().orc_merkle_root(_p8(lv), lv.shape[0], lv.shape[1], _p8(out)))
    return out.tobytes()


def merkle_open(leaves: np.ndarray, idx) -> bytes:
    lv = np.ascontiguousarray(leaves).view(np.uint8).reshape(leaves.shape[0], -1)
    ix = _u64(idx)
    p = u8p()
    n = C.c_size_t()
    _ok(lib().orc_merkle_open(_p8(lv), lv.shape[0], lv.shape[1], _p64(ix), ix.size, C.byref(p),
                              C.byref(n)))
    b = C.string_at(p, n.value)
    lib().orc_free_buf(p)
    return b


def merkle_verify(root: bytes, proof: bytes, idx, leaves: np.ndarray, total: int) -> bool:
    lv = np.ascontiguousarray(leaves).view(np.uint8).reshape(len(idx), -1)
    r = np.frombuffer(root, np.uint8).copy()
    pb = np.frombuffer(proof or b"\0", np.uint8).copy()
    ix = _u64(idx)
    return bool(_ok(lib().orc_merkle_verify(_p8(r), _p8(pb), len(proof), _p64(ix), ix.size, _p8(lv),
                                            lv.shape[1], total)))


class Key:
    """setup (commit_only=False) or a key for commit alone, at any shape (commit_only=True)."""

    def __init__(self, log_m: int, log_n: int, A, commit_only: bool = False):
        self.A = _u64(A)
        self.log_m, self.log_n = log_m, log_n
        com = np.zeros(32, np.uint8)
        if commit_only:
            h = lib().orc_setup_commit_only(log_m, log_n, _p64(self.A))
        else:
            h = lib().orc_setup(log_m, log_n, _p64(self.A), _p8(com))
        if not h:
            raise RuntimeError("oracle setup: " + lib().orc_last_error().decode())
        self.h, self.com_a = h, (None if commit_only else com.tobytes())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_key_free(self.h)
            self.h = None


class Commitment:
    def __init__(self, key: Key, f):
        f = _u64(f)
        root = np.zeros(32, np.uint8)
        h = lib().orc_commit(key.h, _p64(f), f.size, _p8(root))
        if not h:
            raise RuntimeError("oracle commit: " + lib().orc_last_error().decode())
        self.h, self.root, self.key = h, root.tobytes(), key

    def codeword(self):
        m, two_n = 1 << self.key.log_m, 2 << self.key.log_n
        out = np.zeros((m, two_n), np.uint64)
        _ok(lib().orc_commit_codeword(self.h, _p64(out)))
        return out

    def digest(self):
        out = np.zeros((32, 2 << self.key.log_n), np.uint64)
        _ok(lib().orc_commit_digest(self.h, _p64(out)))
        return out

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_commit_free(self.h)
            self.h = None


def prove(key: Key, cm: Commitment, z, fields, ints, cursors=(0, 0)):
    z = _u64(z).reshape(-1, 2).copy()
    f = _u64(fields).reshape(-1, 2).copy()
    i = _u64(ints).copy()
    cur = np.array(cursors, dtype=np.uint64)
    p = u8p()
    n = C.c_size_t()
    _ok(lib().orc_prove(key.h, cm.h, _p64(z), z.shape[0], _p64(f), f.shape[0], _p64(i), i.size,
                        _p64(cur), C.byref(p), C.byref(n)))
    b = C.string_at(p, n.value)
    lib().orc_free_buf(p)
    return b, (int(cur[0]), int(cur[1]))


def verify(com_a: bytes, log_m: int, log_n: int, root: bytes, z, proof: bytes, fields, ints,
           cursors=(0, 0)) -> bool:
    z = _u64(z).reshape(-1, 2).copy()
    f = _u64(fields).reshape(-1, 2).copy()
    i = _u64(ints).copy()
    cur = np.array(cursors, dtype=np.uint64)
    ca = np.frombuffer(com_a, np.uint8).copy()
    rt = np.frombuffer(root, np.uint8).copy()
    pb = np.frombuffer(proof or b"\0", np.uint8).copy()
    rc = lib().orc_verify(_p8(ca), log_m, log_n, _p8(rt), _p64(z), z.shape[0], _p8(pb), len(proof),
                          _p64(f), f.shape[0], _p64(i), i.size, _p64(cur))
    return bool(_ok(rc))


# ---- standalone Basefold (pcs/src/basefold.rs:309-642) ----
class BasefoldCommitment:
    """Basefold::commit_{base,ext}_on_domain of `poly` (2^n BF, or 2^n x 2 EF)."""

    def __init__(self, poly, is_ef: bool, code_rate: int, log_interleave: int = 6):
        p = _u64(poly).reshape(-1)
        n = p.size // 2 if is_ef else p.size
        root = np.zeros(32, np.uint8)
        h = lib().orc_basefold_commit(_p64(p), n, int(is_ef), code_rate, log_interleave, _p8(root))
        if not h:
            raise RuntimeError("oracle basefold commit: " + lib().orc_last_error().decode())
        self.h, self.root, self.is_ef = h, root.tobytes(), is_ef

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_basefold_free(self.h)
            self.h = None


def basefold_prove(cm: BasefoldCommitment, point, fields, ints, cursors=(0, 0)):
    pt = _u64(point).reshape(-1, 2).copy()
    f = _u64(fields).reshape(-1, 2).copy()
    i = _u64(ints).copy()
    cur = np.array(cursors, dtype=np.uint64)
    p = u8p()
    n = C.c_size_t()
    _ok(lib().orc_basefold_prove(cm.h, _p64(pt), pt.shape[0], _p64(f), f.shape[0], _p64(i), i.size,
                                 _p64(cur), C.byref(p), C.byref(n)))
    b = C.string_at(p, n.value)
    lib().orc_free_buf(p)
    return b, (int(cur[0]), int(cur[1]))


def basefold_verify(root: bytes, point, proof: bytes, fields, ints, cursors=(0, 0)) -> bool:
    pt = _u64(point).reshape(-1, 2).copy()
    f = _u64(fields).reshape(-1, 2).copy()
    i = _u64(ints).copy()
    cur = np.array(cursors, dtype=np.uint64)
    rt = np.frombuffer(root, np.uint8).copy()
    pb = np.frombuffer(proof or b"\0", np.uint8).copy()
    rc = lib().orc_basefold_verify(_p8(rt), _p64(pt), pt.shape[0], _p8(pb), len(proof), _p64(f),
                                   f.shape[0], _p64(i), i.size, _p64(cur))
    return bool(_ok(rc))


# ---- GKR fraction sum / GKR-LogUp lookup (logup/src/frac_sum.rs, logup/src/lookup.rs) ---------
i64p = C.POINTER(C.c_int64)


def linear_witness(x, w, bias, divisor: int, w_transposed: bool = False):
    """proofsys' rescaled linear layer: (q, rem, y, encode_i64(y)) of x.matmul(w) (or
    x.matmul_transposed_rhs(w)), floor-divided by divisor, plus the bias row."""
    xa = np.ascontiguousarray(x, dtype=np.int64)
    wa = np.ascontiguousarray(w, dtype=np.int64)
    rows, inner = xa.shape
    cols = wa.shape[0] if w_transposed else wa.shape[1]
    ba = None if bias is None else np.ascontiguousarray(bias, dtype=np.int64)
    q = np.zeros((rows, cols), np.int64)
    rem = np.zeros_like(q)
    y = np.zeros_like(q)
    yf = np.zeros((rows, cols), np.uint64)
    p64 = lambda a: a.ctypes.data_as(i64p)
    _ok(lib().orc_linear_witness(p64(xa), rows, inner, p64(wa), cols, int(w_transposed),
                                 None if ba is None else p64(ba), int(divisor), p64(q), p64(rem),
                                 p64(y), _p64(yf)))
    return q, rem, y, yf


def layer_norm_witness(x, gain, bias):
    """proofsys' layer_norm: (sum_x, sum_x2, var_sum, std, dividend, quotient, output)."""
    xa = np.ascontiguousarray(x, dtype=np.int64)
    rows, d = xa.shape
    ga = np.ascontiguousarray(gain, dtype=np.int64)
    ba = np.ascontiguousarray(bias, dtype=np.int64)
    per_row = [np.zeros(rows, np.int64) for _ in range(4)]
    per_ent = [np.zeros((rows, d), np.int64) for _ in range(3)]
    p64 = lambda a: a.ctypes.data_as(i64p)
    _ok(lib().orc_layer_norm_witness(p64(xa), rows, d, p64(ga), p64(ba),
                                     *[p64(a) for a in per_row + per_ent]))
    return tuple(per_row + per_ent)


def block_witness(x, w: dict, exp_lut, gelu_lut, cfg: dict) -> dict:
    """One GPT-2 block's witness (proofsys/src/model.rs:213-443) on the CPU, keyed like
    ligesis_b200.proofsys.block_witness."""
    from ligesis_b200 import proofsys as ps

    n, d, hid = cfg["n_seq"], cfg["d_model"], cfg["mlp_hidden"]
    H = cfg.get("n_head", 12)
    dh = d // H
    sc = cfg["scale"]
    dims = np.array([n, d, H, dh, hid], dtype=np.uint64)
    consts = np.array([sc, sc * int(round(dh ** 0.5)), cfg["max_v"] * sc], dtype=np.int64)
    ws = [np.ascontiguousarray(w[k], dtype=np.int64).ravel() for k in ps.WEIGHT_NAMES]
    shapes = {"ln": [(n,)] * 4 + [(n, d)] * 3,
              "attn": [(n, 3 * d), (n, 3 * d), (H, n, n), (H, n), (H, n, n), (H, n), (H, n, n),
                       (H, n, dh), (n, d), (n, d), (n, d), (n, 3 * d), (H, n, n), (H, n, dh),
                       (n, d)],
              "mlp": [(n, hid), (n, hid), (n, hid), (n, d), (n, d), (n, hid), (n, d)]}
    outs = ([np.zeros(s, np.int64) for s in shapes["ln"]] +
            [np.zeros(s, np.int64) for s in shapes["attn"]] +
            [np.zeros(s, np.int64) for s in shapes["ln"]] +
            [np.zeros(s, np.int64) for s in shapes["mlp"]])
    xa = np.ascontiguousarray(x, dtype=np.int64)
    el = np.ascontiguousarray(exp_lut, dtype=np.int64)
    gl = np.ascontiguousarray(gelu_lut, dtype=np.int64)
    p64 = lambda a: a.ctypes.data_as(i64p)
    wptr = (i64p * 12)(*[p64(a) for a in ws])
    optr = (i64p * len(outs))(*[p64(a) for a in outs])
    _ok(lib().orc_block_witness(p64(xa), _p64(dims), p64(consts), wptr, p64(el), el.size,
                                p64(gl), gl.size, optr))
    return dict(zip(ps.BLOCK_FIELDS, outs))


def forward_witness(x0, blocks, ln_f_g, ln_f_b, wte, exp_lut, gelu_lut, cfg: dict) -> dict:
    """The integer GPT-2 forward's witness (proofsys/src/model.rs:208-237) from the oracle's
    blocks, layer norm and linear layer, keyed like ligesis_b200.proofsys.forward_witness."""
    x = np.ascontiguousarray(x0, dtype=np.int64)
    out = {"blocks": []}
    for w in blocks:
        b = block_witness(x, w, exp_lut, gelu_lut, cfg)
        out["blocks"].append(b)
        x = b["mlp.x_out"]
    out["lnf"] = layer_norm_witness(x, ln_f_g, ln_f_b)
    q, rem, _, _ = linear_witness(out["lnf"][6], wte, None, cfg["scale"], True)
    out["q_log"], out["rem_log"] = q, rem
    return out


def canonical_online(fw: dict) -> dict:
    """build_online (proofsys/src/canonical.rs:249-331) restated with plain Python integers:
    {type: list of Goldilocks values}, for checking the library's layout."""
    P_ = 0xFFFFFFFF00000001
    enc = lambda v: int(v) % P_
    np2 = lambda x: 1 if x <= 1 else 1 << (int(x) - 1).bit_length()

    def mats(ms, pad=0):
        rows = len(ms[0])
        a0 = np.asarray(ms[0])
        cols = 1 if a0.ndim == 1 else a0.shape[1]
        rp, cp, k = np2(rows), np2(cols), np2(len(ms))
        out = [enc(pad)] * (k * rp * cp) if pad else [0] * (k * rp * cp)
        for i, m in enumerate(ms):
            a = np.asarray(m)
            for r in range(a.shape[0]):
                for c in range(1 if a.ndim == 1 else a.shape[1]):
                    out[(i * rp + r) * cp + c] = enc(a[r] if a.ndim == 1 else a[r, c])
        return out

    def vecs(vs, pad):
        rp, k = np2(len(vs[0])), np2(len(vs))
        out = [enc(pad)] * (k * rp)
        for i, v in enumerate(vs):
            for r, x in enumerate(v):
                out[i * rp + r] = enc(x)
        return out

    bl = fw["blocks"]
    lns = []
    for b in bl:
        for which in ("ln1.", "ln2."):
            lns.append({f: b[which + f] for f in ("var_sum", "std", "dividend", "quotient")})
    lf = fw["lnf"]
    lns.append({"var_sum": lf[2], "std": lf[3], "dividend": lf[4], "quotient": lf[5]})
    heads = lambda key: [b[key][h] for b in bl for h in range(len(b[key]))]
    xo = []
    for b in bl:
        xo += [b["attn.x_out"], b["mlp.x_out"]]
    return {"q_ln": mats([l["quotient"] for l in lns]), "a_ln": mats([l["dividend"] for l in lns]),
            "std": vecs([l["std"] for l in lns], 1), "var": vecs([l["var_sum"] for l in lns], 0),
            "q_sc": mats(heads("attn.scores")), "exp": mats(heads("attn.exp")),
            "q_prob": mats(heads("attn.q_prob")), "x_max": mats(heads("attn.x_max")),
            "sum_exp": vecs(heads("attn.sum_exp"), 1),
            "q_qkv": mats([b["attn.q_qkv"] for b in bl]), "q_ao": mats([b["attn.q_ao"] for b in bl]),
            "q_apr": mats([b["attn.q_apr"] for b in bl]), "q_fc": mats([b["mlp.q_fc"] for b in bl]),
            "act": mats([b["mlp.act"] for b in bl]), "q_fpr": mats([b["mlp.q_fpr"] for b in bl]),
            "x_out": mats(xo), "q_log": mats([fw["q_log"]])}


def _ef2(a):
    return _u64(a).reshape(-1, 2).copy()


def _take(p, n):
    b = C.string_at(p, n.value)
    lib().orc_free_buf(p)
    return b


def frac_sum_prove(p, q, fields, cursor: int = 0):
    """frac_sum::prove over EF arrays p, q (p None: all ones).  Returns (proof bytes, point,
    p_in(point), q_in(point), fields cursor after)."""
    qq = _ef2(q)
    n = qq.shape[0]
    pp = None if p is None else _ef2(p)
    f = _ef2(fields)
    cur = np.array([cursor, 0], dtype=np.uint64)
    k = n.bit_length() - 1
    point = np.zeros((max(k, 1), 2), np.uint64)
    pq = np.zeros(4, np.uint64)
    b, ln = u8p(), C.c_size_t()
    _ok(lib().orc_frac_sum_prove(None if pp is None else _p64(pp), _p64(qq), n, _p64(f),
                                 f.shape[0], _p64(cur), C.byref(b), C.byref(ln), _p64(point),
                                 _p64(pq)))
    return (_take(b, ln), point[:k], (int(pq[0]), int(pq[1])), (int(pq[2]), int(pq[3])),
            int(cur[0]))


def frac_sum_verify(proof: bytes, fields, cursor: int = 0):
    """frac_sum::verify: None on reject, else (point, p_in, q_in, fields cursor after)."""
    f = _ef2(fields)
    cur = np.array([cursor, 0], dtype=np.uint64)
    point = np.zeros((64, 2), np.uint64)
    pq = np.zeros(4, np.uint64)
    pb = np.frombuffer(proof or b"\0", np.uint8).copy()
    rc = _ok(lib().orc_frac_sum_verify(_p8(pb), len(proof), _p64(f), f.shape[0], _p64(cur),
                                       _p64(point), 64, _p64(pq)))
    if rc != 1:
        return None
    k = struct.unpack_from("<I", proof, 40)[0]
    return point[:k], (int(pq[0]), int(pq[1])), (int(pq[2]), int(pq[3])), int(cur[0])


def lookup_prove(a, t, e, fields, cursor: int = 0):
    """lookup::prove_with_opening_points (e None: multiplicities counted as lookup::prove does).
    Returns (proof bytes, zq, zt, fields cursor after)."""
    aa, tt = _ef2(a), _ef2(t)
    ee = None if e is None else _ef2(e)
    f = _ef2(fields)
    cur = np.array([cursor, 0], dtype=np.uint64)
    mu, nu = aa.shape[0].bit_length() - 1, tt.shape[0].bit_length() - 1
    zq = np.zeros((max(mu, 1), 2), np.uint64)
    zt = np.zeros((max(nu, 1), 2), np.uint64)
    b, ln = u8p(), C.c_size_t()
    _ok(lib().orc_lookup_prove(_p64(aa), aa.shape[0], _p64(tt), tt.shape[0],
                               None if ee is None else _p64(ee), _p64(f), f.shape[0], _p64(cur),
                               C.byref(b), C.byref(ln), _p64(zq), _p64(zt)))
    return _take(b, ln), zq[:mu], zt[:nu], int(cur[0])


def lookup_verify(proof: bytes, fields, cursor: int = 0):
    """lookup::verify: None on reject, else (zq, zt, a(zq), e(zt), t(zt), fields cursor after)."""
    f = _ef2(fields)
    cur = np.array([cursor, 0], dtype=np.uint64)
    zq = np.zeros((64, 2), np.uint64)
    zt = np.zeros((64, 2), np.uint64)
    vals = np.zeros(6, np.uint64)
    pb = np.frombuffer(proof or b"\0", np.uint8).copy()
    rc = _ok(lib().orc_lookup_verify(_p8(pb), len(proof), _p64(f), f.shape[0], _p64(cur),
                                     _p64(zq), 64, _p64(zt), 64, _p64(vals)))
    if rc != 1:
        return None
    kq = struct.unpack_from("<I", proof, 48)[0]
    kt = _frac_sum_layers(proof, 8 + _frac_sum_len(proof, 8))
    v = [(int(vals[2 * i]), int(vals[2 * i + 1])) for i in range(3)]
    return zq[:kq], zt[:kt], v[0], v[1], v[2], int(cur[0])


def _frac_sum_layers(proof: bytes, off: int) -> int:
    return struct.unpack_from("<I", proof, off + 40)[0]


def _frac_sum_len(proof: bytes, off: int) -> int:
    """Byte length of the FracSumProof encoded at off."""
    nl = _frac_sum_layers(proof, off)
    pos = off + 44
    for _ in range(nl):
        r = struct.unpack_from("<I", proof, pos)[0]
        pos += 4 + (4 * r + 4) * 16
    return pos - off
