"""Batched and served proving: many LigeSIS commit + prove jobs of uneven sizes in flight on one
GPU at once (lgs_engine_* in include/lgs.h).  The reference proves one polynomial at a time on a
single thread; `ProverEngine` keeps `lanes` independent contexts busy, admits queued jobs as lanes
and device memory free up (FIFO against an HBM budget), and returns, per job, the same root and
proof bytes as `Ligesis.commit` + `Ligesis.prove` would.
"""
from __future__ import annotations

import ctypes as C
import sys
from dataclasses import dataclass

import numpy as np

from ._lib import check, load, u64, vp
from .ligesis import LigesisCommit, LigesisProof, ProvingKey, RandomOracle, _ef_array


class _Job(C.Structure):
    _fields_ = [("pk", vp), ("f", C.POINTER(C.c_uint64)), ("len", C.c_size_t),
                ("z", C.POINTER(C.c_uint64)), ("zlen", C.c_size_t),
                ("fields", C.POINTER(C.c_uint64)), ("nfields", C.c_size_t),
                ("ints", C.POINTER(C.c_uint64)), ("nints", C.c_size_t),
                ("cursors", C.c_uint64 * 2)]


class _Result(C.Structure):
    _fields_ = [("status", C.c_int), ("root", C.c_uint8 * 32), ("proof", C.POINTER(C.c_uint8)),
                ("proof_len", C.c_size_t), ("cursors", C.c_uint64 * 2), ("submit_ms", C.c_double),
                ("start_ms", C.c_double), ("done_ms", C.c_double)]


_SIGS = {
    "lgs_engine_create": (C.c_int, [C.c_int, C.c_uint, C.c_size_t, C.POINTER(vp)]),
    "lgs_engine_destroy": (None, [vp]),
    "lgs_engine_submit": (C.c_int, [vp, C.POINTER(_Job), C.POINTER(C.c_uint64)]),
    "lgs_engine_wait": (C.c_int, [vp, C.c_uint64, C.c_double, C.POINTER(_Result)]),
    "lgs_engine_free_proof": (None, [C.POINTER(C.c_uint8)]),
    "lgs_engine_pending": (C.c_int, [vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "lgs_engine_prepare": (C.c_int, [vp, C.POINTER(vp), C.c_size_t]),
    "lgs_engine_tune": (C.c_int, [vp, C.c_char_p, C.c_uint64]),
}


def _lib():
    lib = load()
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        if fn.argtypes != args:
            fn.restype, fn.argtypes = res, args
    return lib


@dataclass
class JobResult:
    commit: LigesisCommit
    proof: LigesisProof
    cursors: tuple[int, int]
    submit_ms: float
    start_ms: float
    done_ms: float

    @property
    def latency_ms(self) -> float:
        return self.done_ms - self.submit_ms


class ProverEngine:
    """`lanes` contexts on `device`; hbm_budget in bytes (0: 90% of free device memory)."""

    def __init__(self, device: int = 0, lanes: int = 4, hbm_budget: int = 0, tuned: bool = True):
        lib = _lib()
        h = vp()
        check(lib.lgs_engine_create(int(device), int(lanes), int(hbm_budget), C.byref(h)))
        self.handle, self._lib = h, lib
        self._keep: dict[int, tuple] = {}
        self.tuning = None
        if tuned:  # the lanes' launch choices from the autotuner's cache, if it has them
            from . import autotune

            self.tuning = autotune.lookup_engine(lanes, device)
            if self.tuning:
                self.tune(**self.tuning)

    def submit(self, pk: ProvingKey, f, z, oracle: RandomOracle) -> int:
        """Queue one commit + prove of f (2^mu BF) at z, starting at the oracle's cursors.
        The oracle's cursors are advanced as the proof will advance them."""
        fa = u64(f).reshape(-1)
        za = _ef_array(z)
        job = _Job()
        job.pk = pk.handle
        job.f = fa.ctypes.data_as(C.POINTER(C.c_uint64))
        job.len = fa.size
        job.z = za.ctypes.data_as(C.POINTER(C.c_uint64))
        job.zlen = za.shape[0]
        job.fields = oracle.fields.ctypes.data_as(C.POINTER(C.c_uint64))
        job.nfields = oracle.fields.shape[0]
        job.ints = oracle.ints.ctypes.data_as(C.POINTER(C.c_uint64))
        job.nints = oracle.ints.shape[0]
        job.cursors[0], job.cursors[1] = int(oracle.cursors[0]), int(oracle.cursors[1])
        t = C.c_uint64()
        check(self._lib.lgs_engine_submit(self.handle, C.byref(job), C.byref(t)))
        self._keep[t.value] = (fa, za, oracle, pk)  # buffers must outlive the job
        return t.value

    def wait(self, ticket: int, timeout_ms: float = -1.0) -> JobResult:
        r = _Result()
        check(self._lib.lgs_engine_wait(self.handle, ticket, timeout_ms, C.byref(r)))
        keep = self._keep.pop(ticket)
        try:
            check(r.status)
            proof = LigesisProof(C.string_at(r.proof, r.proof_len))
        finally:
            self._lib.lgs_engine_free_proof(r.proof)
        oracle = keep[2]
        oracle.cursors[:] = np.array([r.cursors[0], r.cursors[1]], dtype=np.uint64)
        return JobResult(LigesisCommit(bytes(r.root)), proof, (r.cursors[0], r.cursors[1]),
                         r.submit_ms, r.start_ms, r.done_ms)

    def run(self, jobs) -> list[JobResult]:
        """Batch: submit every (pk, f, z, oracle) job, then collect them in order."""
        tickets = [self.submit(*j) for j in jobs]
        return [self.wait(t) for t in tickets]

    def prepare(self, pks) -> None:
        """Warm every lane for these proving keys' shapes (sizes scratch buffers and captures
        each shape's prove as a CUDA graph).  Call before submitting jobs."""
        pks = list(pks)
        arr = (vp * max(1, len(pks)))(*[pk.handle for pk in pks])
        check(self._lib.lgs_engine_prepare(self.handle, arr, len(pks)))

    def tune(self, **params: int) -> None:
        """lgs_tune on every lane (hash_ctas, sumcheck_blocks, hash_groups; 0 = default).
        Call with no job queued or running; prepare again after a sumcheck_blocks change."""
        for name, value in params.items():
            check(self._lib.lgs_engine_tune(self.handle, name.encode(), int(value)))

    def pending(self) -> tuple[int, int]:
        q, b = C.c_size_t(), C.c_size_t()
        check(self._lib.lgs_engine_pending(self.handle, C.byref(q), C.byref(b)))
        return q.value, b.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.lgs_engine_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            if not sys.is_finalizing():
                self.close()
        except Exception:
            pass
