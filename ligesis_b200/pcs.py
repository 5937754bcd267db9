"""The `PolyCommitmentScheme` trait of the reference (pcs/src/noop.rs:23-48) and two backends.

`NoopPcs` mirrors the reference's measurement fake (pcs/src/noop.rs:53-78): an empty commitment,
no proof, and a `batch_verify` that accepts anything.  It is not sound; it exists so that callers
written against the trait run unchanged.

`BasefoldPcs` is a sound backend over F_{p^2} (the field proofsys instantiates the trait over,
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
from .ligesis import MlPoly, RandomOracle, _ef_array


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
