"""The reference's API for the LigeSIS path, backed by liblgs.so on the GPU:

* `MlPoly`            — utils/src/poly.rs:4-61
* `RandomOracle`      — utils/src/oracle.rs:10-64
* `SubsetSumHash`     — pcs/src/subset_sum.rs:23-79
* `Ligesis`           — pcs/src/ligesis.rs:205-757 (`setup`, `commit`, `prove`, `verify`)

Field elements: BF values are Python ints / numpy uint64 in [0, p); EF values are (c0, c1)
pairs or (k, 2) uint64 arrays.  Points are low-bit-first as in the reference.
"""
from __future__ import annotations

import ctypes as C
import sys
from dataclasses import dataclass

import numpy as np

from . import field as fld
from . import proof as proof_codec
from ._lib import Context, check, load, ptr64, ptr8, u64, u64p, u8p, vp
from .rng import SeededRng

ETA = 64                # pcs/src/ligesis.rs:53
CODE_RATE = 1           # pcs/src/ligesis.rs:56
NUM_COLS_OPENED = 128   # pcs/src/ligesis.rs:59
C_ROWS = 32             # pcs/src/subset_sum.rs:19
LOG_INTERLEAVE = 6      # pcs/src/basefold.rs:16
RANDOM_ORACLE_LEN = 4_000_000  # utils/src/oracle.rs:8


def _ef_array(x) -> np.ndarray:
    a = np.asarray(x, dtype=object if isinstance(x, list) else None)
    if a.dtype == object:
        a = np.array([fld.ef(v) for v in x], dtype=np.uint64)
    a = u64(a)
    if a.ndim == 1:  # BF values -> lift
        a = np.stack([a, np.zeros_like(a)], axis=1)
    return np.ascontiguousarray(a.reshape(-1, 2))


class MlPoly:
    """Multilinear polynomial as its 2^k hypercube evaluations (BF: shape (2^k,), EF: (2^k, 2))."""

    def __init__(self, evals):
        a = u64(evals)
        if a.ndim not in (1, 2) or (a.ndim == 2 and a.shape[1] != 2):
            raise ValueError("MlPoly takes a BF vector or an (n, 2) EF array")
        n = a.shape[0]
        if n == 0 or n & (n - 1):
            raise ValueError("MlPoly needs a power-of-two number of evaluations")
        self.evals = a

    @property
    def is_ext(self) -> bool:
        return self.evals.ndim == 2

    @property
    def num_vars(self) -> int:
        return int(self.evals.shape[0]).bit_length() - 1

    def __len__(self) -> int:
        return int(self.evals.shape[0])

    def eval(self, point, ctx: Context | None = None) -> tuple[int, int]:
        """MlPoly::eval (utils/src/poly.rs:7-18) on the GPU."""
        pt = _ef_array(point)
        if pt.shape[0] != self.num_vars:
            raise ValueError("point length must equal the number of variables")
        ev = _ef_array(self.evals)
        ctx = ctx or Context.default()
        out = np.zeros(2, dtype=np.uint64)
        check(load().lgs_mle_eval(ctx.handle, ptr64(ev), self.num_vars, ptr64(pt), ptr64(out)))
        return (int(out[0]), int(out[1]))

    @staticmethod
    def new_eq(point, ctx: Context | None = None) -> "MlPoly":
        """MlPoly::new_eq (utils/src/poly.rs:44-53): point[0] on the lowest index bit."""
        pt = _ef_array(point)
        k = pt.shape[0]
        if k == 0:
            return MlPoly(np.array([[1, 0]], dtype=np.uint64))
        ctx = ctx or Context.default()
        out = np.zeros(((1 << k), 2), dtype=np.uint64)
        check(load().lgs_new_eq(ctx.handle, ptr64(pt), k, ptr64(out)))
        return MlPoly(out)

    @staticmethod
    def eval_eq(p1, p2) -> tuple[int, int]:
        """MlPoly::eval_eq (utils/src/poly.rs:55-61), O(k) scalar work."""
        return fld.eval_eq(list(map(fld.ef, _ef_array(p1))), list(map(fld.ef, _ef_array(p2))))

    def split(self, n: int) -> list["MlPoly"]:
        """MlPoly::split (utils/src/poly.rs:20-31): chunk j holds evals j, j + len/n, ..."""
        if n <= 0 or n & (n - 1):
            raise ValueError("split size must be a power of two")
        chunks = len(self) // n
        a = self.evals.reshape((n, chunks) + self.evals.shape[1:])
        return [MlPoly(np.ascontiguousarray(a[:, j])) for j in range(chunks)]


class RandomOracle:
    """Pre-drawn Fiat-Shamir stand-in (utils/src/oracle.rs:10-64): `fields` EF and `ints` u64
    arrays read by two cursors.  The reference pre-draws RANDOM_ORACLE_LEN of each; `length`
    sets a smaller pool (one LigeSIS proof needs a few hundred fields and 612 ints)."""

    def __init__(self, rng: SeededRng | int, length: int = 1 << 16):
        rng = rng if isinstance(rng, SeededRng) else SeededRng(int(rng))
        self.fields = np.ascontiguousarray(rng.ext_elements(length))
        self.ints = np.ascontiguousarray(rng.ints(length))
        self.cursors = np.zeros(2, dtype=np.uint64)

    def next_field(self) -> tuple[int, int]:
        i = int(self.cursors[0])
        if i >= len(self.fields):
            raise IndexError("oracle exhausted (fields)")
        self.cursors[0] += 1
        return (int(self.fields[i, 0]), int(self.fields[i, 1]))

    def next_n_fields(self, n: int) -> list[tuple[int, int]]:
        return [self.next_field() for _ in range(n)]

    def next_int(self) -> int:
        i = int(self.cursors[1])
        if i >= len(self.ints):
            raise IndexError("oracle exhausted (ints)")
        self.cursors[1] += 1
        return int(self.ints[i])

    def next_n_ints(self, n: int) -> list[int]:
        return [self.next_int() for _ in range(n)]

    def drawn(self) -> tuple[int, int]:
        return (int(self.cursors[0]), int(self.cursors[1]))

    def restart(self) -> None:
        self.cursors[:] = 0


class SubsetSumHash:
    """H = A * B over Goldilocks (pcs/src/subset_sum.rs:23-79); A is C_ROWS x width."""

    def __init__(self, width: int, rng: SeededRng | None = None, a: np.ndarray | None = None):
        if a is None:
            a = (rng or SeededRng(0)).field_elements(C_ROWS * width).reshape(C_ROWS, width)
        self.a = np.ascontiguousarray(u64(a).reshape(C_ROWS, width))
        self.width = width

    def a_mle_flat(self) -> np.ndarray:
        """subset_sum.rs:73-79: flat[r * width + i] = A[r][i]."""
        return self.a.reshape(-1).copy()

    def hash_columns(self, cols, ctx: Context | None = None) -> np.ndarray:
        """subset_sum.rs:58-67 on the GPU.  cols: (ncols, width) booleans; returns (C, ncols)."""
        b = np.asarray(cols, dtype=bool)
        ncols, width = b.shape
        if width != self.width:
            raise ValueError("column length must equal the hash width")
        m = -(-width // ETA)
        pad_w = m * ETA
        pad_c = -(-ncols // 128) * 128
        bits = np.zeros((pad_c, pad_w), dtype=bool)
        bits[:ncols, :width] = b
        # word[i][j] = sum_b bit[j][64 i + b] << b
        packed = np.packbits(bits.reshape(pad_c, m, ETA), axis=2, bitorder="little")
        cw = np.ascontiguousarray(packed.view("<u8").reshape(pad_c, m).T)
        a = np.zeros((C_ROWS, pad_w), dtype=np.uint64)
        a[:, :width] = self.a
        h = np.zeros((C_ROWS, pad_c), dtype=np.uint64)
        ctx = ctx or Context.default()
        check(load().lgs_subset_sum_hash(ctx.handle, ptr64(a), m, ptr64(cw), pad_c, ptr64(h)))
        return h[:, :ncols]

    def hash_column(self, x, ctx: Context | None = None) -> np.ndarray:
        return self.hash_columns(np.asarray(x, dtype=bool)[None, :], ctx)[:, 0]


@dataclass
class VerifyingKey:
    com_a: bytes
    log_m: int
    log_n: int
    width: int


class ProvingKey:
    def __init__(self, handle, hash_: SubsetSumHash, com_a: bytes, log_m: int, log_n: int,
                 ctx: Context):
        self.handle, self.hash, self.com_a = handle, hash_, com_a
        self.log_m, self.log_n, self.ctx = log_m, log_n, ctx

    def __del__(self):
        try:
            if self.handle and not sys.is_finalizing():
                load().lgs_pk_free(self.handle)
            self.handle = None
        except Exception:
            pass


class LigesisCommit:
    """The commitment (pcs/src/ligesis.rs:85-86): the 32-byte Merkle root of H's columns.  A
    commitment returned by `Ligesis.commit` is resolved on first use of `root`, which waits for
    the commit's device work; until then the device runs the commit while the host goes on."""

    def __init__(self, root: bytes | None = None, *, data: "CommitData | None" = None):
        if root is None and data is None:
            raise ValueError("a commitment needs its root or its pending commit data")
        self._root, self._data = root, data

    @property
    def root(self) -> bytes:
        if self._root is None:
            r = np.zeros(32, dtype=np.uint8)
            check(load().lgs_commit_root(self._data.pk.ctx.handle, self._data.handle, ptr8(r)))
            self._root, self._data = r.tobytes(), None
        return self._root

    def __eq__(self, other):
        return isinstance(other, LigesisCommit) and self.root == other.root

    def __hash__(self):
        return hash(self.root)

    def __repr__(self):
        return f"LigesisCommit({self.root.hex()})"


class CommitData:
    """Device-resident prover data retained between commit and prove (the reference keeps f,
    the bit columns, H and its Merkle tree, pcs/src/ligesis.rs:88-97)."""

    def __init__(self, handle, pk: ProvingKey):
        self.handle, self.pk = handle, pk

    def codeword(self) -> np.ndarray:
        m, two_n = 1 << self.pk.log_m, 2 << self.pk.log_n
        out = np.zeros(m * two_n, dtype=np.uint64)
        check(load().lgs_commit_read(self.pk.ctx.handle, self.handle, 0, ptr64(out), out.size))
        return out.reshape(m, two_n)

    def digest(self) -> np.ndarray:
        two_n = 2 << self.pk.log_n
        out = np.zeros(C_ROWS * two_n, dtype=np.uint64)
        check(load().lgs_commit_read(self.pk.ctx.handle, self.handle, 1, ptr64(out), out.size))
        return out.reshape(C_ROWS, two_n)

    def __del__(self):
        try:
            if self.handle and not sys.is_finalizing():
                load().lgs_commit_data_free(self.handle)
            self.handle = None
        except Exception:
            pass


class LigesisProof:
    """An encoded proof (bytes) with a lazily decoded view of its fields."""

    def __init__(self, data: bytes):
        self.data = bytes(data)
        self._fields = None

    @property
    def fields(self) -> proof_codec.ProofFields:
        if self._fields is None:
            self._fields = proof_codec.decode(self.data)
        return self._fields

    @property
    def y(self) -> tuple[int, int]:
        return self.fields.y

    def size_bytes(self) -> int:
        """The reference's accounting (pcs/src/ligesis.rs:124-138)."""
        return self.fields.size_bytes()

    def __bytes__(self) -> bytes:
        return self.data

    def __len__(self) -> int:
        return len(self.data)


def shape_ok(log_m: int, log_n: int) -> bool:
    """setup's shared-domain precondition (pcs/src/ligesis.rs:246-251)."""
    v = (5 + 6 + log_m, 6 + log_m + 7, log_n)
    return max(v) - min(v) <= LOG_INTERLEAVE


def oracle_need(log_m: int, log_n: int) -> tuple[int, int]:
    f, i = C.c_size_t(), C.c_size_t()
    check(load().lgs_oracle_need(log_m, log_n, C.byref(f), C.byref(i)))
    return f.value, i.value


class Ligesis:
    """Ligesis<Goldilocks, BinomialExtensionField<Goldilocks, 2>> (pcs/src/ligesis.rs:205-757)."""

    @staticmethod
    def setup(log_m: int, log_n: int, rng: SeededRng, ctx: Context | None = None):
        """Ligesis::setup: sample A (SubsetSumHash::new) from `rng`, commit the flat A."""
        return Ligesis.setup_with_hash(log_m, log_n, SubsetSumHash(ETA << log_m, rng), ctx)

    @staticmethod
    def setup_with_hash(log_m: int, log_n: int, hash_: SubsetSumHash,
                        ctx: Context | None = None):
        """setup with a caller-provided subset-sum matrix (width must be 64 * 2^log_m)."""
        ctx = ctx or Context.default()
        width = ETA << log_m
        if hash_.width != width:
            raise ValueError("the hash width must be 64 * 2^log_m")
        h = vp()
        com = np.zeros(32, dtype=np.uint8)
        check(load().lgs_setup(ctx.handle, log_m, log_n, ptr64(hash_.a), C.byref(h), ptr8(com)))
        pk = ProvingKey(h, hash_, com.tobytes(), log_m, log_n, ctx)
        vk = VerifyingKey(com.tobytes(), log_m, log_n, width)
        return pk, vk

    @staticmethod
    def setup_commit_only(log_m: int, log_n: int, hash_: SubsetSumHash,
                          ctx: Context | None = None) -> ProvingKey:
        """A key for `commit` alone, at any shape the commit takes (log_m <= 13, log_n >= 7):
        setup's shared-domain assertion (pcs/src/ligesis.rs:246-251) binds only the prove, so
        square shapes such as 2^12 x 2^12 are committed through this key.  It cannot prove."""
        ctx = ctx or Context.default()
        if hash_.width != ETA << log_m:
            raise ValueError("the hash width must be 64 * 2^log_m")
        h = vp()
        check(load().lgs_setup_commit_only(ctx.handle, log_m, log_n, ptr64(hash_.a), C.byref(h)))
        return ProvingKey(h, hash_, b"", log_m, log_n, ctx)

    @staticmethod
    def commit(pk: ProvingKey, f: MlPoly) -> tuple[LigesisCommit, CommitData]:
        """Enqueues the commit (lgs_commit_async) and returns at once: the root is read when
        first used, and a prove on the same context runs after the commit on the device."""
        if f.is_ext:
            raise ValueError("LigeSIS commits base-field polynomials")
        ev = f.evals
        h = vp()
        check(load().lgs_commit_async(pk.ctx.handle, pk.handle, ptr64(ev), ev.size, 0,
                                      C.byref(h)))
        data = CommitData(h, pk)
        return LigesisCommit(data=data), data

    @staticmethod
    def commit_device(pk: ProvingKey, f_dev_ptr: int, length: int, lend: bool = False):
        """commit with f already in device memory (e.g. a torch uint64/int64 CUDA tensor); f must
        stay unchanged until the commitment's root has been read or a prove has returned.  With
        lend=True f is not copied: the commitment reads the caller's buffer for as long as it
        lives (as the reference's commit owns its MlPoly), so the buffer must stay allocated and
        unchanged until the CommitData is released."""
        h = vp()
        check(load().lgs_commit_async(pk.ctx.handle, pk.handle, vp(f_dev_ptr), length,
                                      2 if lend else 1, C.byref(h)))
        data = CommitData(h, pk)
        return LigesisCommit(data=data), data

    @staticmethod
    def prove(pk: ProvingKey, data: CommitData, z, oracle: RandomOracle) -> LigesisProof:
        zz = _ef_array(z)
        p = u8p()
        n = C.c_size_t()
        cur = oracle.cursors
        check(load().lgs_prove(pk.ctx.handle, pk.handle, data.handle, ptr64(zz), zz.shape[0],
                               ptr64(oracle.fields), oracle.fields.shape[0], ptr64(oracle.ints),
                               oracle.ints.shape[0], ptr64(cur), C.byref(p), C.byref(n)))
        return LigesisProof(C.string_at(p, n.value))

    @staticmethod
    def verify(vk: VerifyingKey, commit: LigesisCommit, z, proof: LigesisProof | bytes,
               oracle: RandomOracle) -> bool:
        zz = _ef_array(z)
        data = bytes(proof)
        buf = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, np.uint8)
        ca = np.frombuffer(vk.com_a, dtype=np.uint8).copy()
        rt = np.frombuffer(commit.root, dtype=np.uint8).copy()
        acc = C.c_int(0)
        check(load().lgs_verify(vk.log_m, vk.log_n, ptr8(ca), ptr8(rt), ptr64(zz), zz.shape[0],
                                ptr8(buf), len(data), ptr64(oracle.fields),
                                oracle.fields.shape[0], ptr64(oracle.ints), oracle.ints.shape[0],
                                ptr64(oracle.cursors), C.byref(acc)))
        return bool(acc.value)


def sumcheck_prove(polys, challenges, ctx: Context | None = None):
    """utils::sumcheck::prove (utils/src/sumcheck.rs:37-84) on the GPU.  polys: list of d EF
    arrays (2^k, 2); challenges: the k oracle fields it draws.  Returns (round_polys (k, d+1, 2),
    final_evals (d, 2))."""
    ps = [_ef_array(p) for p in polys]
    d, length = len(ps), ps[0].shape[0]
    k = length.bit_length() - 1
    flat = np.ascontiguousarray(np.concatenate(ps, axis=0))
    ch = _ef_array(challenges)
    rounds = np.zeros((k, d + 1, 2), dtype=np.uint64)
    finals = np.zeros((d, 2), dtype=np.uint64)
    ctx = ctx or Context.default()
    check(load().lgs_sumcheck_prove(ctx.handle, ptr64(flat), d, k, ptr64(ch), ptr64(rounds),
                                    ptr64(finals)))
    return rounds, finals


def dft(coeffs, log_size: int, ctx: Context | None = None) -> np.ndarray:
    """Radix2Dit::dft of each row of `coeffs` (zero-padded to 2^log_size)."""
    a = u64(coeffs)
    if a.ndim == 1:
        a = a[None, :]
    a = np.ascontiguousarray(a)
    out = np.zeros((a.shape[0], 1 << log_size), dtype=np.uint64)
    ctx = ctx or Context.default()
    check(load().lgs_dft(ctx.handle, ptr64(a), a.shape[1], a.shape[0], log_size, ptr64(out)))
    return out


def merkle_root(leaves, ctx: Context | None = None) -> bytes:
    """MerkleTreeProver::new(...).commit() over leaves given as (n, words) u64."""
    a = u64(leaves)
    root = np.zeros(32, dtype=np.uint8)
    ctx = ctx or Context.default()
    check(load().lgs_merkle_root(ctx.handle, ptr64(a), a.shape[0], a.shape[1], ptr8(root)))
    return root.tobytes()
