"""ctypes binding of liblgs.so (include/lgs.h).  The library is the only compute path: if it is
missing or cannot be loaded, every call raises; there is no CPU fallback."""
from __future__ import annotations

import ctypes as C
import sys
import threading
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "liblgs.so"

STATUS = {
    0: "ok",
    1: "bad shape",
    2: "out of memory",
    3: "oracle exhausted",
    4: "device timeout",
    5: "bad argument",
    6: "cuda error",
    7: "internal error",
    8: "buffer too small",
}


class LgsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class ShapeError(LgsError):
    pass


class OracleExhausted(LgsError):
    pass


class DeviceTimeout(LgsError):
    """A bounded device wait gave up (LGS_ERR_DEVICE_TIMEOUT); the context stays usable."""


_lib = None
_lock = threading.Lock()

u64p = C.POINTER(C.c_uint64)
u8p = C.POINTER(C.c_uint8)
i64p = C.POINTER(C.c_int64)
vp = C.c_void_p

_SIGS = {
    "lgs_last_error": (C.c_char_p, []),
    "lgs_version": (C.c_char_p, []),
    "lgs_ctx_create": (C.c_int, [C.c_int, C.c_uint, C.POINTER(vp)]),
    "lgs_ctx_destroy": (None, [vp]),
    "lgs_ctx_stream": (C.c_int, [vp, C.POINTER(vp)]),
    "lgs_setup": (C.c_int, [vp, C.c_uint, C.c_uint, u64p, C.POINTER(vp), u8p]),
    "lgs_setup_commit_only": (C.c_int, [vp, C.c_uint, C.c_uint, u64p, C.POINTER(vp)]),
    "lgs_pk_free": (None, [vp]),
    "lgs_commit": (C.c_int, [vp, vp, u64p, C.c_size_t, u8p, C.POINTER(vp)]),
    "lgs_commit_device": (C.c_int, [vp, vp, vp, C.c_size_t, u8p, C.POINTER(vp)]),
    "lgs_commit_data_free": (None, [vp]),
    "lgs_commit_async": (C.c_int, [vp, vp, vp, C.c_size_t, C.c_int, C.POINTER(vp)]),
    "lgs_commit_root": (C.c_int, [vp, vp, u8p]),
    "lgs_commit_read": (C.c_int, [vp, vp, C.c_int, u64p, C.c_size_t]),
    "lgs_oracle_need": (C.c_int, [C.c_uint, C.c_uint, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "lgs_prove": (C.c_int, [vp, vp, vp, u64p, C.c_size_t, u64p, C.c_size_t, u64p, C.c_size_t,
                            u64p, C.POINTER(u8p), C.POINTER(C.c_size_t)]),
    "lgs_verify": (C.c_int, [C.c_uint, C.c_uint, u8p, u8p, u64p, C.c_size_t, u8p, C.c_size_t,
                             u64p, C.c_size_t, u64p, C.c_size_t, u64p, C.POINTER(C.c_int)]),
    "lgs_profile": (C.c_int, [vp, C.c_int]),
    "lgs_profile_get": (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]),
    "lgs_launch_count": (C.c_uint64, []),
    "lgs_set_wait_budget": (C.c_int, [vp, C.c_uint64]),
    "lgs_tune": (C.c_int, [vp, C.c_char_p, C.c_uint64]),
    "lgs_tune_get": (C.c_int, [vp, C.c_char_p, C.POINTER(C.c_uint64)]),
    "lgs_profile_names": (C.c_int, [vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "lgs_sumcheck_prove_dev": (C.c_int, [vp, vp, C.c_uint, C.c_uint, vp, vp, vp]),
    "lgs_new_eq_dev": (C.c_int, [vp, vp, C.c_uint, vp]),
    "lgs_mle_fold_dev": (C.c_int, [vp, vp, C.c_uint, vp, C.c_uint, vp]),
    "lgs_mle_eval_dev": (C.c_int, [vp, vp, C.c_uint, vp, vp]),
    "lgs_basefold_commit": (C.c_int, [vp, u64p, C.c_size_t, C.c_int, C.c_uint, C.c_uint, u8p,
                                      C.POINTER(vp)]),
    "lgs_basefold_free": (None, [vp]),
    "lgs_basefold_prove": (C.c_int, [vp, vp, u64p, C.c_size_t, u64p, C.c_size_t, u64p,
                                     C.c_size_t, u64p, C.POINTER(u8p), C.POINTER(C.c_size_t)]),
    "lgs_basefold_verify": (C.c_int, [u8p, u64p, C.c_size_t, u8p, C.c_size_t, u64p, C.c_size_t,
                                      u64p, C.c_size_t, u64p, C.POINTER(C.c_int)]),
    "lgs_frac_sum_prove": (C.c_int, [vp, u64p, u64p, C.c_size_t, C.c_int, u64p, C.c_size_t,
                                     C.POINTER(C.c_uint64), C.POINTER(u8p), C.POINTER(C.c_size_t),
                                     u64p, u64p]),
    "lgs_frac_sum_verify": (C.c_int, [u8p, C.c_size_t, u64p, C.c_size_t, C.POINTER(C.c_uint64),
                                      u64p, C.c_size_t, u64p, C.POINTER(C.c_int)]),
    "lgs_lookup_prove": (C.c_int, [vp, u64p, C.c_size_t, u64p, u64p, C.c_size_t, C.c_int, u64p,
                                   C.c_size_t, C.POINTER(C.c_uint64), C.POINTER(u8p),
                                   C.POINTER(C.c_size_t), u64p, u64p]),
    "lgs_lookup_verify": (C.c_int, [u8p, C.c_size_t, u64p, C.c_size_t, C.POINTER(C.c_uint64),
                                    u64p, C.c_size_t, u64p, C.c_size_t, u64p, C.POINTER(C.c_int)]),
    "lgs_linear_witness": (C.c_int, [vp, i64p, C.c_size_t, C.c_size_t, i64p, C.c_size_t, C.c_int,
                                     i64p, C.c_int64, C.c_int, i64p, i64p, i64p, u64p]),
    "lgs_layer_norm_witness": (C.c_int, [vp, i64p, C.c_size_t, C.c_size_t, i64p, i64p, C.c_int,
                                         i64p, i64p, i64p, i64p, i64p, i64p, i64p]),
    "lgs_softmax_witness": (C.c_int, [vp, i64p, C.c_uint, C.c_uint, i64p, C.c_size_t, C.c_int64,
                                      C.c_int64, C.c_int, i64p, i64p, i64p, i64p]),
    "lgs_lut_gather": (C.c_int, [vp, i64p, C.c_size_t, i64p, C.c_size_t, C.c_int64, C.c_int,
                                 i64p]),
    "lgs_tensor_peak_i8": (C.c_int, [vp, C.c_uint, C.POINTER(C.c_double)]),
    "lgs_rs_alu_rates": (C.c_int, [vp, C.c_uint, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "lgs_dft": (C.c_int, [vp, u64p, C.c_size_t, C.c_size_t, C.c_uint, u64p]),
    "lgs_subset_sum_hash": (C.c_int, [vp, u64p, C.c_size_t, u64p, C.c_size_t, u64p]),
    "lgs_merkle_root": (C.c_int, [vp, u64p, C.c_size_t, C.c_uint, u8p]),
    "lgs_sumcheck_prove": (C.c_int, [vp, u64p, C.c_uint, C.c_uint, u64p, u64p, u64p]),
    "lgs_mle_eval": (C.c_int, [vp, u64p, C.c_uint, u64p, u64p]),
    "lgs_new_eq": (C.c_int, [vp, u64p, C.c_uint, u64p]),
    "lgs_sumcheck_prove_noalloc": (C.c_int, [vp, C.c_uint, C.c_uint, vp, vp, vp, vp]),
}


def load(path: Path | None = None):
    """Load liblgs.so (building it first if the CUDA toolkit is here and it is absent)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            from . import build as _build

            _build.build()
        lib = C.CDLL(str(p))
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int) -> None:
    if status == 0:
        return
    msg = (load().lgs_last_error() or b"").decode(errors="replace")
    if status == 1:
        raise ShapeError(status, msg)
    if status == 3:
        raise OracleExhausted(status, msg)
    if status == 4:
        raise DeviceTimeout(status, msg)
    raise LgsError(status, msg)


def ptr64(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"], "expected a contiguous uint64 array"
    return a.ctypes.data_as(u64p)


def ptr8(a: np.ndarray):
    assert a.dtype == np.uint8 and a.flags["C_CONTIGUOUS"], "expected a contiguous uint8 array"
    return a.ctypes.data_as(u8p)


def u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


class Context:
    """One device, one CUDA stream (lgs_ctx).  Not shared between host threads."""

    _default: dict[int, "Context"] = {}

    def __init__(self, device: int = 0):
        lib = load()
        h = vp()
        check(lib.lgs_ctx_create(int(device), 0, C.byref(h)))
        self.handle = h
        self.device = device
        self._lib = lib

    @classmethod
    def default(cls, device: int = 0) -> "Context":
        ctx = cls._default.get(device)
        if ctx is None:
            ctx = cls._default[device] = cls(device)
        return ctx

    @property
    def stream_ptr(self) -> int:
        s = vp()
        check(self._lib.lgs_ctx_stream(self.handle, C.byref(s)))
        return int(s.value or 0)

    def tune(self, **params: int) -> None:
        """Launch choices of this context's kernels (lgs_tune): hash_ctas, sumcheck_blocks,
        hash_groups, witness_path, witness_ctas, upload_block_bytes, upload_tail_rows."""
        for name, value in params.items():
            check(self._lib.lgs_tune(self.handle, name.encode(), int(value)))

    def tuning(self, *names: str) -> dict:
        out = {}
        for name in names or ("hash_ctas", "sumcheck_blocks", "hash_groups"):
            v = C.c_uint64()
            check(self._lib.lgs_tune_get(self.handle, name.encode(), C.byref(v)))
            out[name] = int(v.value)
        return out

    def set_wait_budget(self, cycles: int) -> None:
        """Clock-cycle budget of the bounded device waits of this context's kernels (0 = the
        default of about 2 s); a short budget makes them give up (DeviceTimeout)."""
        check(self._lib.lgs_set_wait_budget(self.handle, int(cycles)))

    def close(self):
        if getattr(self, "handle", None):
            self._lib.lgs_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            if not sys.is_finalizing():  # at exit the driver tears the context down itself
                self.close()
        except Exception:
            pass
