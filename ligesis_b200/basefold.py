"""Standalone Basefold PCS on the GPU: the host mirror of pcs/src/basefold.rs's
`Basefold::{commit_base, commit_ext, commit_base_on_domain, commit_ext_on_domain, prove, verify}`
over liblgs.so (lgs_basefold_* in include/lgs.h).  Proofs are the "LGSB" byte encoding of
`BasefoldProof` (pcs/src/basefold.rs:84-103) that ligesis_b200/csrc/proof.hpp documents.
"""
from __future__ import annotations

import ctypes as C
import struct
import sys

import numpy as np

from ._lib import Context, check, load, ptr64, ptr8, u64p, u8p, vp
from .ligesis import MlPoly, RandomOracle, _ef_array

LOG_INTERLEAVE = 6  # pcs/src/basefold.rs:15-16


class BasefoldCommit:
    """The commitment: the Merkle root over the interleaved codeword columns."""

    def __init__(self, root: bytes):
        self.root = root

    def __eq__(self, other):
        return isinstance(other, BasefoldCommit) and self.root == other.root

    def __repr__(self):
        return f"BasefoldCommit({self.root.hex()})"


class BasefoldProverState:
    """BasefoldProverState (pcs/src/basefold.rs:46-58), resident on the device."""

    def __init__(self, handle, ctx: Context, num_vars: int, code_rate: int, log_interleave: int,
                 is_ext: bool):
        self.handle, self.ctx = handle, ctx
        self.num_vars, self.code_rate = num_vars, code_rate
        self.log_interleave, self.is_ext = log_interleave, is_ext

    def __del__(self):
        try:
            if self.handle and not sys.is_finalizing():
                load().lgs_basefold_free(self.handle)
            self.handle = None
        except Exception:
            pass


class BasefoldProof:
    """An encoded BasefoldProof."""

    def __init__(self, data: bytes):
        if data[:4] != b"LGSB":
            raise ValueError("not a Basefold proof")
        self.data = data

    @property
    def claimed_eval(self) -> tuple[int, int]:
        return struct.unpack_from("<QQ", self.data, 24)

    @property
    def num_vars(self) -> int:
        return struct.unpack_from("<I", self.data, 8)[0]

    @property
    def leaf_ef(self) -> bool:
        return struct.unpack_from("<I", self.data, 20)[0] != 0

    def __len__(self) -> int:
        return len(self.data)


class Basefold:
    @staticmethod
    def commit_base_on_domain(poly: MlPoly, code_rate: int, log_interleave: int,
                              ctx: Context | None = None):
        return Basefold._commit(poly, code_rate, log_interleave, False, ctx)

    @staticmethod
    def commit_ext_on_domain(poly: MlPoly, code_rate: int, log_interleave: int,
                             ctx: Context | None = None):
        return Basefold._commit(poly, code_rate, log_interleave, True, ctx)

    @staticmethod
    def commit_base(poly: MlPoly, code_rate: int, ctx: Context | None = None):
        return Basefold._commit(poly, code_rate, LOG_INTERLEAVE, False, ctx)

    @staticmethod
    def commit_ext(poly: MlPoly, code_rate: int, ctx: Context | None = None):
        return Basefold._commit(poly, code_rate, LOG_INTERLEAVE, True, ctx)

    @staticmethod
    def _commit(poly: MlPoly, code_rate: int, log_interleave: int, is_ext: bool,
                ctx: Context | None):
        if poly.is_ext != is_ext:
            raise ValueError("commit_base takes a BF polynomial, commit_ext an EF one")
        ctx = ctx or Context.default()
        ev = np.ascontiguousarray(poly.evals)
        root = np.zeros(32, dtype=np.uint8)
        h = vp()
        check(load().lgs_basefold_commit(ctx.handle, ptr64(ev), len(poly), int(is_ext),
                                         code_rate, log_interleave, ptr8(root), C.byref(h)))
        state = BasefoldProverState(h, ctx, poly.num_vars, code_rate, log_interleave, is_ext)
        return state, BasefoldCommit(root.tobytes())

    @staticmethod
    def prove(state: BasefoldProverState, point, oracle: RandomOracle) -> BasefoldProof:
        pt = _ef_array(point)
        p = u8p()
        n = C.c_size_t()
        check(load().lgs_basefold_prove(state.ctx.handle, state.handle, ptr64(pt), pt.shape[0],
                                        ptr64(oracle.fields), oracle.fields.shape[0],
                                        ptr64(oracle.ints), oracle.ints.shape[0],
                                        ptr64(oracle.cursors), C.byref(p), C.byref(n)))
        return BasefoldProof(C.string_at(p, n.value))

    @staticmethod
    def verify(commit: BasefoldCommit, point, proof: BasefoldProof | bytes,
               oracle: RandomOracle) -> bool:
        pt = _ef_array(point)
        data = proof.data if isinstance(proof, BasefoldProof) else bytes(proof)
        buf = np.frombuffer(data or b"\0", dtype=np.uint8).copy()
        rt = np.frombuffer(commit.root, dtype=np.uint8).copy()
        acc = C.c_int()
        check(load().lgs_basefold_verify(ptr8(rt), ptr64(pt), pt.shape[0], ptr8(buf), len(data),
                                         ptr64(oracle.fields), oracle.fields.shape[0],
                                         ptr64(oracle.ints), oracle.ints.shape[0],
                                         ptr64(oracle.cursors), C.byref(acc)))
        return bool(acc.value)
