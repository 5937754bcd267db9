"""Python view of the encoded LigesisProof (layout documented in csrc/proof.hpp; field order of
pcs/src/ligesis.rs:99-119 and BatchProof of pcs/src/basefold.rs:151-162).  Used to inspect a
proof, to compute the reference's `size_bytes`, and by tamper tests to edit and re-encode."""
from __future__ import annotations

import struct
from dataclasses import dataclass, field


@dataclass
class SumcheckProof:
    round_polys: list[list[tuple[int, int]]]
    final_evals: list[tuple[int, int]]

    def size_bytes(self) -> int:  # utils/src/sumcheck.rs:16-20
        return 16 * (sum(len(r) for r in self.round_polys) + len(self.final_evals))


@dataclass
class Opening:
    proof_bytes: bytes
    values: dict[int, list]  # key -> list of BF ints or EF tuples


@dataclass
class BatchProof:
    code_rate: int
    log_len: int
    reduction_msgs: list[list[tuple[int, int]]]
    fold_roots: list[bytes]
    final_codeword: list[tuple[int, int]]
    fold_openings: list[Opening]
    base_bf: list[Opening]
    base_ef: list[Opening]

    def size_bytes(self) -> int:  # pcs/src/basefold.rs:168-193
        s = 16 * sum(len(c) for c in self.reduction_msgs) + 32 * len(self.fold_roots)
        s += 16 * len(self.final_codeword)
        for op in self.fold_openings:
            s += len(op.proof_bytes) + 16 * sum(len(v) for v in op.values.values())
        for op in self.base_bf:
            s += len(op.proof_bytes) + 8 * sum(len(v) for v in op.values.values())
        for op in self.base_ef:
            s += len(op.proof_bytes) + 16 * sum(len(v) for v in op.values.values())
        return s


SUMCHECK_NAMES = ("sc_binary", "sc_hash", "sc_recon", "sc_table", "sc_rslink", "sc_bi_batch",
                  "sc_a_batch")


@dataclass
class ProofFields:
    y: tuple[int, int]
    com_a_vec: bytes
    com_i: bytes
    y4: tuple[int, int]
    y5: tuple[int, int]
    h_cols: list[list[int]]
    h_open: bytes
    sumchecks: dict[str, SumcheckProof] = field(default_factory=dict)
    batch: BatchProof | None = None

    def size_bytes(self) -> int:  # pcs/src/ligesis.rs:124-138
        s = 16 * 3 + 64 + len(self.h_open) + 8 * sum(len(c) for c in self.h_cols)
        s += sum(p.size_bytes() for p in self.sumchecks.values())
        return s + self.batch.size_bytes()


class _R:
    def __init__(self, b: bytes):
        self.b, self.p = b, 0

    def take(self, n: int) -> bytes:
        if self.p + n > len(self.b):
            raise ValueError("truncated proof")
        v = self.b[self.p:self.p + n]
        self.p += n
        return v

    def u32(self) -> int:
        return struct.unpack("<I", self.take(4))[0]

    def u64(self) -> int:
        return struct.unpack("<Q", self.take(8))[0]

    def ef(self):
        return (self.u64(), self.u64())

    def opening(self, ext: bool) -> Opening:
        pb = self.take(self.u32())
        vals = {}
        for _ in range(self.u32()):
            key = self.u64()
            n = self.u32()
            vals[key] = [self.ef() if ext else self.u64() for _ in range(n)]
        return Opening(pb, vals)


def decode(b: bytes) -> ProofFields:
    r = _R(bytes(b))
    if r.take(4) != b"LGSP" or r.u32() != 1:
        raise ValueError("not an encoded LigesisProof")
    y = r.ef()
    com_a_vec, com_i = r.take(32), r.take(32)
    y4, y5 = r.ef(), r.ef()
    ncols, nrows = r.u32(), r.u32()
    h_cols = [[r.u64() for _ in range(nrows)] for _ in range(ncols)]
    h_open = r.take(r.u32())
    pf = ProofFields(y, com_a_vec, com_i, y4, y5, h_cols, h_open)
    for name in SUMCHECK_NAMES:
        rounds, width = r.u32(), r.u32()
        rp = [[r.ef() for _ in range(width)] for _ in range(rounds)]
        fe = [r.ef() for _ in range(r.u32())]
        pf.sumchecks[name] = SumcheckProof(rp, fe)
    code_rate, log_len = r.u32(), r.u32()
    msgs = [[r.ef() for _ in range(r.u32())] for _ in range(r.u32())]
    roots = [r.take(32) for _ in range(r.u32())]
    final = [r.ef() for _ in range(r.u32())]
    folds = [r.opening(True) for _ in range(r.u32())]
    bbf = [r.opening(False) for _ in range(r.u32())]
    bef = [r.opening(True) for _ in range(r.u32())]
    if r.p != len(r.b):
        raise ValueError("trailing bytes in proof")
    pf.batch = BatchProof(code_rate, log_len, msgs, roots, final, folds, bbf, bef)
    return pf


def encode(pf: ProofFields) -> bytes:
    out = [b"LGSP", struct.pack("<I", 1)]
    u32 = lambda v: out.append(struct.pack("<I", v))  # noqa: E731
    u64 = lambda v: out.append(struct.pack("<Q", v))  # noqa: E731

    def ef(e):
        u64(e[0])
        u64(e[1])

    def opening(op: Opening, ext: bool):
        u32(len(op.proof_bytes))
        out.append(op.proof_bytes)
        u32(len(op.values))
        for k in sorted(op.values):
            u64(k)
            u32(len(op.values[k]))
            for v in op.values[k]:
                ef(v) if ext else u64(v)

    ef(pf.y)
    out += [pf.com_a_vec, pf.com_i]
    ef(pf.y4)
    ef(pf.y5)
    u32(len(pf.h_cols))
    u32(len(pf.h_cols[0]) if pf.h_cols else 32)
    for c in pf.h_cols:
        for v in c:
            u64(v)
    u32(len(pf.h_open))
    out.append(pf.h_open)
    for name in SUMCHECK_NAMES:
        sc = pf.sumchecks[name]
        u32(len(sc.round_polys))
        u32(len(sc.round_polys[0]) if sc.round_polys else 0)
        for rp in sc.round_polys:
            for e in rp:
                ef(e)
        u32(len(sc.final_evals))
        for e in sc.final_evals:
            ef(e)
    b = pf.batch
    u32(b.code_rate)
    u32(b.log_len)
    u32(len(b.reduction_msgs))
    for ch in b.reduction_msgs:
        u32(len(ch))
        for e in ch:
            ef(e)
    u32(len(b.fold_roots))
    out += list(b.fold_roots)
    u32(len(b.final_codeword))
    for e in b.final_codeword:
        ef(e)
    u32(len(b.fold_openings))
    for op in b.fold_openings:
        opening(op, True)
    u32(len(b.base_bf))
    for op in b.base_bf:
        opening(op, False)
    u32(len(b.base_ef))
    for op in b.base_ef:
        opening(op, True)
    return b"".join(out)
