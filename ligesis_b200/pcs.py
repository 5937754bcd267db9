"""The `PolyCommitmentScheme` trait of the reference (pcs/src/noop.rs:23-48) and three backends.

`NoopPcs` mirrors the reference's measurement fake (pcs/src/noop.rs:53-78): an empty commitment,
no proof, and a `batch_verify` that accepts anything.  It is not sound; it exists so that callers
written against the trait run unchanged.

`LigesisPcs` is a sound backend: the adapter that puts LigeSIS (pcs/src/ligesis.rs:239-575)
behind the trait.  LigeSIS commits base-field polynomials, so `commit` projects the F_{p^2} values
onto F_p, which is exact for integer witnesses and refused for any value with c1 != 0.  A
polynomial of mu variables is committed as a 2^log_m x 2^log_n matrix of the reference-valid
shape (log_m = min(7, (mu - 7) / 2)); one of fewer than 14 variables is zero-padded to 14 at the
high variables and opened at its point with zeros appended, at which the padded polynomial takes
the same value.  Each proof's `y` is the opened value.

`BasefoldPcs` is the other sound backend, over F_{p^2} (the field proofsys instantiates the trait over,
proofsys/src/commit.rs:24) built on the GPU Basefold of this package.  `commit` commits the
polynomial with Basefold.  When every value lies in the base field (proofsys witnesses are
integers lifted with encode_i64, proofsys/src/witness.rs:102-108), it uses base-field leaves,
which halves the committed and opened data; otherwise it uses extension-field leaves.
`batch_prove` opens each task in order on the shared oracle, and `batch_verify` checks each
opening and that its claimed value is the one the caller states.  Points are low-bit-first, as
for `MlPoly.eval`.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from ._lib import Context
from .basefold import Basefold, BasefoldCommit, BasefoldProof, BasefoldProverState
from .ligesis import (Ligesis, LigesisCommit, LigesisProof, MlPoly, RandomOracle, SeededRng,
                      _ef_array, shape_ok)
from .workloads import shape_for_mu


# ---- the reference's no-op backend ----------------------------------------------------------
@dataclass(frozen=True)
class NoopCommit:
    """An empty commitment: nothing is sent to the verifier."""


class NoopPcs:
    """PolyCommitmentScheme with no binding at all (pcs/src/noop.rs:53-78); not sound."""

    @staticmethod
    def commit(poly: MlPoly):
        return poly, NoopCommit()

    @staticmethod
    def batch_prove(tasks, oracle: RandomOracle):
        return None

    @staticmethod
    def batch_verify(claims, proof, oracle: RandomOracle) -> bool:
        return True


# ---- Basefold on the GPU ----------------------------------------------------------------------
@dataclass
class BasefoldPcsCommitment:
    root: bytes
    num_vars: int
    base_field: bool


@dataclass
class BasefoldPcsData:
    state: BasefoldProverState
    commitment: BasefoldPcsCommitment


@dataclass
class BasefoldPcsProof:
    """One encoded Basefold opening per task, in task order."""
    openings: list[bytes] = field(default_factory=list)

    def size_bytes(self) -> int:
        return sum(len(o) for o in self.openings)


class BasefoldPcs:
    """PolyCommitmentScheme over F_{p^2} backed by Basefold on the GPU (see the module doc)."""

    def __init__(self, code_rate: int = 1, log_interleave: int = 6, ctx: Context | None = None):
        self.code_rate, self.log_interleave = code_rate, log_interleave
        self.ctx = ctx

    def _li(self, num_vars: int) -> int:
        return min(self.log_interleave, num_vars - 1)

    def commit(self, poly: MlPoly):
        if poly.num_vars < 1:
            raise ValueError("BasefoldPcs commits polynomials of at least one variable")
        li = self._li(poly.num_vars)
        if poly.is_ext and not np.any(poly.evals[:, 1]):
            base = MlPoly(np.ascontiguousarray(poly.evals[:, 0]))
            state, com = Basefold.commit_base_on_domain(base, self.code_rate, li, self.ctx)
            is_base = True
        elif poly.is_ext:
            state, com = Basefold.commit_ext_on_domain(poly, self.code_rate, li, self.ctx)
            is_base = False
        else:
            state, com = Basefold.commit_base_on_domain(poly, self.code_rate, li, self.ctx)
            is_base = True
        c = BasefoldPcsCommitment(com.root, poly.num_vars, is_base)
        return BasefoldPcsData(state, c), c

    def batch_prove(self, tasks, oracle: RandomOracle) -> BasefoldPcsProof:
        proof = BasefoldPcsProof()
        for data, point in tasks:
            proof.openings.append(Basefold.prove(data.state, point, oracle).data)
        return proof

    def batch_verify(self, claims, proof: BasefoldPcsProof, oracle: RandomOracle) -> bool:
        if proof is None or len(proof.openings) != len(claims):
            return False
        for (com, point, value), opening in zip(claims, proof.openings):
            pt = _ef_array(point)
            if pt.shape[0] != com.num_vars:
                return False
            try:
                bp = BasefoldProof(opening)
            except ValueError:
                return False
            if len(opening) < 40 or bp.num_vars != com.num_vars \
                    or bp.leaf_ef == com.base_field:
                return False
            want = tuple(int(x) for x in _ef_array([value])[0])
            if bp.claimed_eval != want:
                return False
            if not Basefold.verify(BasefoldCommit(com.root), pt, bp, oracle):
                return False
        return True


# ---- LigeSIS behind the trait ----------------------------------------------------------------
LIGESIS_MIN_VARS = 14  # 2^3 x 2^11, the smallest shape the padded commits use
LIGESIS_MAX_VARS = 28  # 2^7 x 2^21, the largest shape setup takes


@dataclass
class LigesisPcsCommitment:
    root: bytes
    num_vars: int  # of the committed polynomial, before padding
    log_m: int
    log_n: int


@dataclass
class LigesisPcsData:
    data: object  # CommitData, device-resident
    commitment: LigesisPcsCommitment
    pk: object


@dataclass
class LigesisPcsProof:
    """One encoded LigeSIS proof per task, in task order."""
    proofs: list[bytes] = field(default_factory=list)

    def size_bytes(self) -> int:
        return sum(LigesisProof(p).size_bytes() for p in self.proofs)


class LigesisPcs:
    """PolyCommitmentScheme over F_{p^2} backed by LigeSIS on the GPU (see the module doc).
    Keys are made once per matrix shape from `seed` (setup samples the subset-sum matrix) and
    shared by prover and verifier."""

    def __init__(self, seed: int = 0, ctx: Context | None = None):
        self.seed, self.ctx = seed, ctx
        self._keys: dict[tuple[int, int], tuple] = {}

    def keys(self, log_m: int, log_n: int):
        k = (log_m, log_n)
        if k not in self._keys:
            rng = SeededRng((self.seed << 16) ^ (log_m << 8) ^ log_n)
            self._keys[k] = Ligesis.setup(log_m, log_n, rng, self.ctx)
        return self._keys[k]

    @staticmethod
    def padded_vars(num_vars: int) -> int:
        if num_vars > LIGESIS_MAX_VARS:
            raise ValueError(f"LigesisPcs commits at most {LIGESIS_MAX_VARS} variables")
        return max(num_vars, LIGESIS_MIN_VARS)

    @staticmethod
    def _pad_point(point, num_vars: int, mu: int) -> np.ndarray:
        pt = _ef_array(point)
        if pt.shape[0] != num_vars:
            raise ValueError("the point must have num_vars coordinates")
        if mu > num_vars:
            pt = np.concatenate([pt, np.zeros((mu - num_vars, 2), dtype=np.uint64)])
        return np.ascontiguousarray(pt)

    def commit(self, poly: MlPoly):
        if poly.is_ext:
            if np.any(poly.evals[:, 1]):
                raise ValueError("LigesisPcs commits integer (base-field) values only: "
                                 "a value has a nonzero c1")
            f = poly.evals[:, 0]
        else:
            f = poly.evals
        n = poly.num_vars
        mu = self.padded_vars(n)
        log_m, log_n = shape_for_mu(mu)
        assert shape_ok(log_m, log_n)
        if mu > n:
            f = np.concatenate([f, np.zeros((1 << mu) - f.size, dtype=np.uint64)])
        pk, _ = self.keys(log_m, log_n)
        com, data = Ligesis.commit(pk, MlPoly(np.ascontiguousarray(f)))
        c = LigesisPcsCommitment(com.root, n, log_m, log_n)
        return LigesisPcsData(data, c, pk), c

    def batch_prove(self, tasks, oracle: RandomOracle) -> LigesisPcsProof:
        proof = LigesisPcsProof()
        for d, point in tasks:
            c = d.commitment
            z = self._pad_point(point, c.num_vars, c.log_m + c.log_n)
            proof.proofs.append(Ligesis.prove(d.pk, d.data, z, oracle).data)
        return proof

    def batch_verify(self, claims, proof: LigesisPcsProof, oracle: RandomOracle) -> bool:
        if proof is None or len(proof.proofs) != len(claims):
            return False
        for (com, point, value), pb in zip(claims, proof.proofs):
            if self.padded_vars(com.num_vars) != com.log_m + com.log_n \
                    or shape_for_mu(com.log_m + com.log_n) != (com.log_m, com.log_n):
                return False
            try:
                z = self._pad_point(point, com.num_vars, com.log_m + com.log_n)
                y = LigesisProof(pb).y
            except ValueError:
                return False
            if y != tuple(int(x) for x in _ef_array([value])[0]):
                return False
            _, vk = self.keys(com.log_m, com.log_n)
            if not Ligesis.verify(vk, LigesisCommit(com.root), z, pb, oracle):
                return False
        return True
