"""GKR fraction sum and GKR-LogUp lookup on the GPU: the host mirror of logup/src/frac_sum.rs
(`prove`, `verify`, `FracSumProof`) and logup/src/lookup.rs (`prove`, `prove_with_mults`,
`prove_with_query_point`, `prove_with_opening_points`, `verify`, `multiplicity_vector`,
`OpeningClaim`) over liblgs.so (lgs_frac_sum_* / lgs_lookup_* in include/lgs.h).  Proofs are the
"LGSF" / "LGSL" byte encodings documented there.  EF arrays are (n, 2) uint64, canonical.
"""
from __future__ import annotations

import ctypes as C
import enum
import struct
from dataclasses import dataclass

import numpy as np

from ._lib import Context, check, load, ptr64, ptr8, u64, u8p
from .ligesis import RandomOracle, _ef_array


def _ef(v) -> tuple[int, int]:
    return (int(v[0]), int(v[1]))


class FracSumProof:
    """An encoded FracSumProof: the root fraction and one layer proof per reduction."""

    def __init__(self, data: bytes):
        if data[:4] != b"LGSF":
            raise ValueError("not a fraction-sum proof")
        self.data = bytes(data)

    @property
    def num(self) -> tuple[int, int]:
        return struct.unpack_from("<QQ", self.data, 8)

    @property
    def den(self) -> tuple[int, int]:
        return struct.unpack_from("<QQ", self.data, 24)

    @property
    def num_layers(self) -> int:
        return struct.unpack_from("<I", self.data, 40)[0]

    def layers(self):
        """[(round_polys: (r, 4, 2) uint64, leaves: (4, 2) uint64)] for r = 0 .. k-1."""
        out, pos = [], 44
        for _ in range(self.num_layers):
            r = struct.unpack_from("<I", self.data, pos)[0]
            pos += 4
            polys = np.frombuffer(self.data, np.uint64, 8 * r, pos).reshape(r, 4, 2)
            pos += 64 * r
            leaves = np.frombuffer(self.data, np.uint64, 8, pos).reshape(4, 2)
            pos += 64
            out.append((polys, leaves))
        return out

    def size_bytes(self) -> int:
        """The reference's accounting (frac_sum.rs:42-52): 2 + sum (4 r + 4) field elements."""
        return 16 * (2 + sum(4 * p.shape[0] + 4 for p, _ in self.layers()))

    def __len__(self) -> int:
        return len(self.data)


def _fs_len(data: bytes, off: int) -> int:
    nl = struct.unpack_from("<I", data, off + 40)[0]
    pos = off + 44
    for _ in range(nl):
        r = struct.unpack_from("<I", data, pos)[0]
        pos += 4 + 64 * r + 64
    return pos - off


class LookupProof:
    """An encoded LookupProof: the query-side and the table-side fraction-sum proofs."""

    def __init__(self, data: bytes):
        if data[:4] != b"LGSL":
            raise ValueError("not a lookup proof")
        self.data = bytes(data)

    @property
    def query(self) -> FracSumProof:
        return FracSumProof(self.data[8:8 + _fs_len(self.data, 8)])

    @property
    def table(self) -> FracSumProof:
        n = _fs_len(self.data, 8)
        return FracSumProof(self.data[8 + n:])

    def size_bytes(self) -> int:
        return self.query.size_bytes() + self.table.size_bytes()

    def __len__(self) -> int:
        return len(self.data)


class Poly(enum.Enum):
    """Which committed polynomial an OpeningClaim refers to (lookup.rs:20-28)."""
    Query = 0
    Table = 1
    Mult = 2


@dataclass
class OpeningClaim:
    poly: Poly
    point: np.ndarray  # (k, 2) uint64, low-bit-first
    value: tuple[int, int]


def _input(x, ctx: Context):
    """(pointer, length, on_device, keepalive) for an EF array on the host or a CUDA tensor."""
    if hasattr(x, "is_cuda") and x.is_cuda:
        if x.device.index != ctx.device:
            raise ValueError("tensor on another device than the context")
        if not x.is_contiguous() or x.element_size() != 8 or x.numel() % 2:
            raise ValueError("device EF input: a contiguous 64-bit tensor of (n, 2) values")
        return C.cast(C.c_void_p(x.data_ptr()), C.POINTER(C.c_uint64)), x.numel() // 2, 1, x
    a = _ef_array(x)
    return ptr64(a), a.shape[0], 0, a


class FracSum:
    @staticmethod
    def prove(p, q, oracle: RandomOracle, ctx: Context | None = None):
        """frac_sum::prove: (FracSumProof, point (k, 2), p_in(point), q_in(point)).  p None: every
        numerator is one (the query side of a lookup).  p and q are EF arrays on the host or
        CUDA tensors on the context's device."""
        ctx = ctx or Context.default()
        qp, n, on_dev, keep_q = _input(q, ctx)
        if p is None:
            pp, keep_p = None, None
        else:
            pp, n_p, on_dev_p, keep_p = _input(p, ctx)
            if n_p != n or on_dev_p != on_dev:
                raise ValueError("p and q: one length, one memory")
        k = max(n.bit_length() - 1, 0)
        point = np.zeros((max(k, 1), 2), dtype=np.uint64)
        claim = np.zeros(4, dtype=np.uint64)
        cur = C.c_uint64(int(oracle.cursors[0]))
        b, ln = u8p(), C.c_size_t()
        check(load().lgs_frac_sum_prove(ctx.handle, pp, qp, n, on_dev, ptr64(oracle.fields),
                                        oracle.fields.shape[0], C.byref(cur), C.byref(b),
                                        C.byref(ln), ptr64(point), ptr64(claim)))
        oracle.cursors[0] = cur.value
        del keep_p, keep_q
        return (FracSumProof(C.string_at(b, ln.value)), point[:k], _ef(claim[:2]),
                _ef(claim[2:]))

    @staticmethod
    def verify(proof: FracSumProof | bytes, oracle: RandomOracle):
        """frac_sum::verify: None, or (point, p_in(point), q_in(point)) to discharge."""
        data = proof.data if isinstance(proof, FracSumProof) else bytes(proof)
        buf = np.frombuffer(data or b"\0", dtype=np.uint8).copy()
        point = np.zeros((64, 2), dtype=np.uint64)
        claim = np.zeros(4, dtype=np.uint64)
        cur = C.c_uint64(int(oracle.cursors[0]))
        acc = C.c_int()
        check(load().lgs_frac_sum_verify(ptr8(buf), len(data), ptr64(oracle.fields),
                                         oracle.fields.shape[0], C.byref(cur), ptr64(point), 64,
                                         ptr64(claim), C.byref(acc)))
        oracle.cursors[0] = cur.value
        if not acc.value:
            return None
        k = FracSumProof(data).num_layers
        return point[:k].copy(), _ef(claim[:2]), _ef(claim[2:])


def multiplicity_vector(a, t) -> np.ndarray:
    """lookup::multiplicity_vector (lookup.rs:66-81): how often each table entry occurs among the
    queries, by value (the table's entries distinct; a query outside the table counts nowhere)."""
    aa, tt = _ef_array(a), _ef_array(t)
    dt = np.dtype([("c0", "<u8"), ("c1", "<u8")])
    ta = np.ascontiguousarray(tt).view(dt).reshape(-1)
    qa = np.ascontiguousarray(aa).view(dt).reshape(-1)
    order = np.argsort(ta, kind="stable")
    ts = ta[order]
    pos = np.searchsorted(ts, qa)
    pos_c = np.minimum(pos, len(ts) - 1)
    hit = ts[pos_c] == qa
    counts = np.bincount(order[pos_c[hit]], minlength=len(ta)).astype(np.uint64)
    e = np.zeros((len(ta), 2), dtype=np.uint64)
    e[:, 0] = counts
    return e


class Lookup:
    @staticmethod
    def prove(a, t, oracle: RandomOracle, ctx: Context | None = None) -> LookupProof:
        """lookup::prove: multiplicities counted on the host, then prove_with_mults."""
        return Lookup.prove_with_mults(a, t, multiplicity_vector(a, t), oracle, ctx)

    @staticmethod
    def prove_with_mults(a, t, e, oracle: RandomOracle, ctx: Context | None = None) -> LookupProof:
        return Lookup.prove_with_opening_points(a, t, e, oracle, ctx)[0]

    @staticmethod
    def prove_with_query_point(a, t, e, oracle: RandomOracle, ctx: Context | None = None):
        proof, zq, _ = Lookup.prove_with_opening_points(a, t, e, oracle, ctx)
        return proof, zq

    @staticmethod
    def prove_with_opening_points(a, t, e, oracle: RandomOracle, ctx: Context | None = None):
        """(LookupProof, zq, zt).  a, t, e are EF arrays on the host, or CUDA tensors."""
        ctx = ctx or Context.default()
        ap, m, on_a, ka = _input(a, ctx)
        tp, n, on_t, kt = _input(t, ctx)
        ep, n_e, on_e, ke = _input(e, ctx)
        if n_e != n or not (on_a == on_t == on_e):
            raise ValueError("lookup: |e| == |t| and all inputs in one memory")
        mu, nu = max(m.bit_length() - 1, 0), max(n.bit_length() - 1, 0)
        zq = np.zeros((max(mu, 1), 2), dtype=np.uint64)
        zt = np.zeros((max(nu, 1), 2), dtype=np.uint64)
        cur = C.c_uint64(int(oracle.cursors[0]))
        b, ln = u8p(), C.c_size_t()
        check(load().lgs_lookup_prove(ctx.handle, ap, m, tp, ep, n, on_a, ptr64(oracle.fields),
                                      oracle.fields.shape[0], C.byref(cur), C.byref(b),
                                      C.byref(ln), ptr64(zq), ptr64(zt)))
        oracle.cursors[0] = cur.value
        del ka, kt, ke
        return LookupProof(C.string_at(b, ln.value)), zq[:mu], zt[:nu]

    @staticmethod
    def verify(proof: LookupProof | bytes, oracle: RandomOracle):
        """lookup::verify: None, or the three OpeningClaims [a(zq), e(zt), t(zt)]."""
        data = proof.data if isinstance(proof, LookupProof) else bytes(proof)
        buf = np.frombuffer(data or b"\0", dtype=np.uint8).copy()
        zq = np.zeros((64, 2), dtype=np.uint64)
        zt = np.zeros((64, 2), dtype=np.uint64)
        vals = np.zeros(6, dtype=np.uint64)
        cur = C.c_uint64(int(oracle.cursors[0]))
        acc = C.c_int()
        check(load().lgs_lookup_verify(ptr8(buf), len(data), ptr64(oracle.fields),
                                       oracle.fields.shape[0], C.byref(cur), ptr64(zq), 64,
                                       ptr64(zt), 64, ptr64(vals), C.byref(acc)))
        oracle.cursors[0] = cur.value
        if not acc.value:
            return None
        lp = LookupProof(data)
        kq, kt = lp.query.num_layers, lp.table.num_layers
        return [OpeningClaim(Poly.Query, zq[:kq].copy(), _ef(vals[0:2])),
                OpeningClaim(Poly.Mult, zt[:kt].copy(), _ef(vals[2:4])),
                OpeningClaim(Poly.Table, zt[:kt].copy(), _ef(vals[4:6]))]
