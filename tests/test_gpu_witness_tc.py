"""The rescaled linear layer's contraction on the int8 tensor cores (witness_tc.cu) against the
oracle (proofsys/src/tensor.rs:76-133, model.rs:360-374, :225-228): Q, REM, Y and encode_i64(Y)
equal element for element, whichever path ran, and the tensor path is the one that runs for
operands within its limb encodings (activations in [-2^23, 2^23), weights in [-2^15, 2^15))."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import proofsys as ps

pytestmark = pytest.mark.gpu


def _rand(seed, shape, lo, hi):
    return np.random.default_rng(seed).integers(lo, hi, size=shape, dtype=np.int64)


def _paths(ctx, fn):
    """Runs fn with the context's profile on; returns (tensor-core launches, CUDA-core launches)."""
    lib = L.load()
    L._lib.check(lib.lgs_profile(ctx.handle, 1))
    try:
        fn()
        counts = []
        for name in (b"linear_witness_tc", b"linear_witness_cores"):
            tot, cnt = C.c_double(), C.c_uint64()
            L._lib.check(lib.lgs_profile_get(ctx.handle, name, C.byref(tot), C.byref(cnt)))
            counts.append(cnt.value)
        return tuple(counts)
    finally:
        L._lib.check(lib.lgs_profile(ctx.handle, 0))


def _check(got, want):
    for g_, w_ in zip(got, want):
        assert np.array_equal(g_, w_)
    assert np.array_equal(got[3], ps.encode_i64(got[2]))


@pytest.mark.parametrize("rows,inner,cols,wt", [
    (31, 768, 4099, True),    # the vocabulary head's layout, ragged columns
    (31, 768, 3072, False),   # MLP fc
    (31, 3072, 768, False),   # MLP projection (K split over CTAs)
    (5, 70, 33, False),       # ragged K inside one chunk
    (67, 129, 65, True),      # two row tiles, K one past a chunk
    (1, 1, 1, True),
    (3, 20000, 40, True),     # more K than one CTA may sum: split by the int32 bound
    (64, 300, 130, False),
])
def test_tensor_path_matches_oracle(lgs, orc, rows, inner, cols, wt):
    ctx = L.Context(0)
    x = _rand(rows + inner, (rows, inner), -(1 << 21), 1 << 21)
    w = _rand(cols + 1, (cols, inner) if wt else (inner, cols), -(1 << 15), 1 << 15)
    b = _rand(cols + 2, cols, -(1 << 30), 1 << 30)
    out = {}
    tc, cores = _paths(ctx, lambda: out.setdefault("r", ps.linear_witness(x, w, b, 1 << 12, wt,
                                                                          ctx)))
    assert (tc, cores) == (1, 0)
    _check(out["r"], orc.linear_witness(x, w, b, 1 << 12, wt))


@pytest.mark.parametrize("rows,inner,cols,wt", [
    (63, 512, 300, True),     # N = 64: two accumulator sets fill all 512 TMEM columns
    (63, 512, 300, False),
    (7, 256, 10, False),      # fewer columns than one 16-column box
    (5, 2, 200, True),        # K of two values: one chunk, mostly past the matrix
    (31, 20000, 300, False),  # K split by the int32 bound, weights as inner x cols
    (40, 1000, 2, True),      # two output columns
])
def test_persistent_kernel_edges(lgs, orc, rows, inner, cols, wt):
    """Shapes at the edges of the persistent kernel's boxes, tiles and TMEM."""
    ctx = L.Context(0)
    x = _rand(rows + 11, (rows, inner), -(1 << 23), 1 << 23)
    w = _rand(cols + 12, (cols, inner) if wt else (inner, cols), -(1 << 15), 1 << 15)
    b = _rand(cols + 13, cols, -(1 << 35), 1 << 35)
    out = {}
    tc, cores = _paths(ctx, lambda: out.setdefault("r", ps.linear_witness(x, w, b, 1 << 12, wt,
                                                                          ctx)))
    assert (tc, cores) == (1, 0)
    _check(out["r"], orc.linear_witness(x, w, b, 1 << 12, wt))


@pytest.mark.parametrize("rows,inner,cols,wt,ctas", [
    (31, 768, 1300, True, 8),     # one wave of whole tiles, three tiles split in two after it
    (70, 300, 700, False, 5),     # two row tiles, ragged K and columns, the tail split in two
    (64, 2000, 1000, True, 3),    # one tail tile split in three
    (3, 20000, 700, True, 4),     # every tile split by the int32 bound
])
def test_tensor_path_whole_waves_and_split_tail(lgs, orc, rows, inner, cols, wt, ctas):
    """The work plan with fewer resident CTAs than tiles (witness_ctas caps what it assumes):
    whole tiles in full waves, the remaining tiles split over K into one more wave."""
    ctx = L.Context(0)
    ctx.tune(witness_ctas=ctas)
    x = _rand(rows + 7, (rows, inner), -(1 << 22), 1 << 22)
    w = _rand(cols + 8, (cols, inner) if wt else (inner, cols), -(1 << 15), 1 << 15)
    b = _rand(cols + 9, cols, -(1 << 40), 1 << 40)
    out = {}
    tc, cores = _paths(ctx, lambda: out.setdefault("r", ps.linear_witness(x, w, b, 3 << 11, wt,
                                                                          ctx)))
    assert (tc, cores) == (1, 0)
    _check(out["r"], orc.linear_witness(x, w, b, 3 << 11, wt))


@pytest.mark.parametrize("wt", [False, True])
def test_tensor_path_at_the_encoding_bounds(lgs, orc, wt):
    """Every activation and weight at an end of its range, in sign patterns, with an odd
    divisor: the offset corrections and the int32 limb sums stay exact."""
    ctx = L.Context(0)
    rows, inner, cols = 9, 1000, 150
    g = np.random.default_rng(3)
    x = np.where(g.integers(0, 2, (rows, inner)) == 1, (1 << 23) - 1, -(1 << 23)).astype(np.int64)
    w = np.where(g.integers(0, 2, (inner, cols)) == 1, (1 << 15) - 1, -(1 << 15)).astype(np.int64)
    x[0] = (1 << 23) - 1
    w[:, 0] = (1 << 15) - 1
    x[1] = -(1 << 23)
    w[:, 1] = -(1 << 15)
    if wt:
        w = np.ascontiguousarray(w.T)
    out = {}
    tc, cores = _paths(ctx, lambda: out.setdefault("r", ps.linear_witness(x, w, None, 4097, wt,
                                                                          ctx)))
    assert (tc, cores) == (1, 0)
    _check(out["r"], orc.linear_witness(x, w, None, 4097, wt))


@pytest.mark.parametrize("wt", [False, True])
@pytest.mark.parametrize("which", ["x", "w"])
def test_operand_outside_the_limbs_takes_the_cuda_cores(lgs, orc, which, wt):
    ctx = L.Context(0)
    x = _rand(1, (31, 768), -(1 << 20), 1 << 20)
    w = _rand(2, (768, 300), -(1 << 15), 1 << 15)
    if which == "x":
        x[17, 500] = 1 << 23
    else:
        w[700, 299] = -(1 << 15) - 1
    if wt:
        w = np.ascontiguousarray(w.T)
    out = {}
    tc, cores = _paths(ctx, lambda: out.setdefault("r", ps.linear_witness(x, w, None, 1 << 12,
                                                                          wt, ctx)))
    assert (tc, cores) == (1, 1)
    _check(out["r"], orc.linear_witness(x, w, None, 1 << 12, wt))


def test_device_arrays_both_paths_agree(lgs, orc):
    torch = pytest.importorskip("torch")
    x = _rand(4, (31, 768), -(1 << 20), 1 << 20)
    w = _rand(5, (2000, 768), -(1 << 15), 1 << 15)
    b = _rand(6, 2000, -(1 << 20), 1 << 20)
    want = orc.linear_witness(x, w, b, 1 << 12, True)
    for path in (0, 1):
        ctx = L.Context(0)
        ctx.tune(witness_path=path)
        got = ps.linear_witness(torch.from_numpy(x).cuda(), torch.from_numpy(w).cuda(),
                                torch.from_numpy(b).cuda(), 1 << 12, True, ctx)
        for g_, w_ in zip(got, want):
            assert np.array_equal(g_.cpu().numpy().view(w_.dtype), w_)


def test_results_beyond_i64_still_an_error_on_the_tensor_path(lgs):
    """Q + bias overflowing i64 is reported (the reference panics), also from the tensor path."""
    ctx = L.Context(0)
    x = np.full((2, 4), 1 << 20, dtype=np.int64)
    w = np.full((4, 3), 1 << 14, dtype=np.int64)
    b = np.full(3, (1 << 63) - 1, dtype=np.int64)
    with pytest.raises(L.ShapeError):
        ps.linear_witness(x, w, b, 1, False, ctx)
