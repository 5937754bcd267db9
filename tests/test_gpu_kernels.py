"""Device operations against the CPU oracle, bit-exact (integer field arithmetic): DFT, subset-sum
hash, Merkle roots, eq tables, MLE evaluation and the product sumcheck."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import rng
from tests.helpers import P

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_size,n_in,batch", [(1, 1, 3), (4, 8, 2), (10, 512, 4), (12, 4096, 2),
                                                 (13, 4096, 3), (15, 16384, 2), (18, 131072, 2),
                                                 (20, 1 << 19, 1), (14, 5, 2), (17, 1 << 17, 1),
                                                 (14, 8192, 3), (14, 16384, 2), (16, 1 << 15, 5),
                                                 (16, 1 << 16, 1), (18, 1 << 18, 1)])
def test_dft_matches_oracle(lgs, orc, log_size, n_in, batch):
    c = rng.field_elements(1000 + log_size, batch * n_in).reshape(batch, n_in)
    got = L.dft(c, log_size)
    for b in range(batch):
        assert np.array_equal(got[b], orc.dft_bf(c[b], 1 << log_size)), b


def test_dft_reduces_noncanonical_input(lgs, orc):
    c = np.array([P, P + 5, (1 << 64) - 1, 3], dtype=np.uint64)
    got = L.dft(c, 3)[0]
    want = orc.dft_bf(np.array([0, 5, (1 << 64) - 1 - P, 3], dtype=np.uint64), 8)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("log_size", [14, 18])
def test_dft_large_reduces_noncanonical_input(lgs, orc, log_size):
    # the four-step row transform (2^14 .. 2^18) canonicalises what it reads, like the small one
    n_in = 1 << (log_size - 1)
    c = rng.field_elements(555, 2 * n_in).reshape(2, n_in)
    c[0, ::7] = np.uint64(P)
    c[1, 3::11] = np.uint64((1 << 64) - 1)
    got = L.dft(c, log_size)
    canon = np.where(c >= np.uint64(P), c - np.uint64(P), c)
    for b in range(2):
        assert np.array_equal(got[b], orc.dft_bf(canon[b], 1 << log_size)), b


@pytest.mark.parametrize("m,cols", [(1, 128), (2, 256), (8, 2048), (16, 384), (128, 1024)])
def test_subset_sum_hash_matches_oracle(lgs, orc, m, cols):
    A = rng.field_elements(2000 + m, 32 * 64 * m).reshape(32, 64 * m)
    cw = rng.field_elements(3000 + m, m * cols).reshape(m, cols)
    h = L.SubsetSumHash(64 * m, a=A)
    got = np.zeros((32, cols), dtype=np.uint64)
    from ligesis_b200._lib import Context, check, load, ptr64

    check(load().lgs_subset_sum_hash(Context.default().handle, ptr64(A), m, ptr64(cw), cols,
                                     ptr64(got)))
    assert np.array_equal(got, orc.hash_columns(A, cw))
    assert h.width == 64 * m


@pytest.mark.parametrize("m,cols", [(8, 297 * 256 + 77), (3, 600 * 256)])
def test_subset_sum_hash_many_tiles_per_cta(lgs, orc, m, cols):
    # more 256-column tiles than SMs: every persistent CTA walks several tiles, and the pipeline
    # stages wrap across tile boundaries (m = 3 and 8 give 2 and 4 stages per tile)
    A = rng.field_elements(2100 + m, 32 * 64 * m).reshape(32, 64 * m)
    cw = rng.field_elements(3100 + m, m * cols).reshape(m, cols)
    from ligesis_b200._lib import Context, check, load, ptr64

    got = np.zeros((32, cols), dtype=np.uint64)
    check(load().lgs_subset_sum_hash(Context.default().handle, ptr64(A), m, ptr64(cw), cols,
                                     ptr64(got)))
    assert np.array_equal(got, orc.hash_columns(A, cw))


@pytest.mark.parametrize("m,cols,hash_ctas", [(1000, 512, 0), (999, 300, 0), (2048, 256, 0),
                                               (4096, 1024, 0), (512, 1024, 37)])
def test_subset_sum_hash_split_over_k(lgs, orc, m, cols, hash_ctas):
    """Few column tiles and many rows (the square commit shapes): the K rows are split over CTAs
    into digest slices that a second kernel sums and hashes; also with a CTA cap and an odd row
    count (which keeps a single slice)."""
    A = rng.field_elements(2200 + m, 32 * 64 * m).reshape(32, 64 * m)
    cw = rng.field_elements(3200 + m, m * cols).reshape(m, cols)
    from ligesis_b200._lib import Context, check, load, ptr64

    ctx = Context(0)
    ctx.tune(hash_ctas=hash_ctas)
    got = np.zeros((32, cols), dtype=np.uint64)
    check(load().lgs_subset_sum_hash(ctx.handle, ptr64(A), m, ptr64(cw), cols, ptr64(got)))
    assert np.array_equal(got, orc.hash_columns(A, cw))


def test_subset_sum_hash_extremes(lgs, orc):
    # every bit set and every limb 0xff-heavy: the largest int32 limb sums the kernel sees
    m, cols = 128, 256
    A = np.full((32, 64 * m), P - 1, dtype=np.uint64)
    cw = np.full((m, cols), P - 1, dtype=np.uint64)
    cw[:, ::2] = 0
    from ligesis_b200._lib import Context, check, load, ptr64

    got = np.zeros((32, cols), dtype=np.uint64)
    check(load().lgs_subset_sum_hash(Context.default().handle, ptr64(A), m, ptr64(cw), cols,
                                     ptr64(got)))
    assert np.array_equal(got, orc.hash_columns(A, cw))


def test_subset_sum_hash_api_on_bool_columns(lgs, orc):
    # SubsetSumHash::hash_columns on explicit bit columns (pcs/src/subset_sum.rs:110-124)
    width = 64
    A = rng.field_elements(77, 32 * width).reshape(32, width)
    bits = (rng.ints(78, 10 * width) & np.uint64(1)).astype(bool).reshape(10, width)
    h = L.SubsetSumHash(width, a=A)
    got = h.hash_columns(bits)
    for j in range(10):
        for r in range(32):
            assert int(got[r, j]) == sum(int(A[r, i]) for i in range(width) if bits[j, i]) % P


@pytest.mark.parametrize("nleaves,words", [(2, 1), (8, 2), (64, 16), (1024, 32), (4096, 64),
                                           (1 << 15, 2), (256, 128), (1 << 18, 4)])
def test_merkle_root_matches_oracle(lgs, orc, nleaves, words):
    leaves = rng.field_elements(4000 + words, nleaves * words).reshape(nleaves, words)
    assert L.merkle_root(leaves) == orc.merkle_root(leaves)


@pytest.mark.parametrize("k", [1, 3, 10, 20])
def test_new_eq_and_mle_eval_match_oracle(lgs, orc, k):
    pt = rng.ext_elements(5000 + k, k)
    eq = L.MlPoly.new_eq(pt).evals
    assert np.array_equal(eq, orc.new_eq(pt))
    ev = rng.ext_elements(5100 + k, 1 << k)
    assert L.MlPoly(ev).eval(pt) == orc.mle_eval(ev, pt)
    bf = rng.field_elements(5200 + k, 1 << k)
    lifted = np.stack([bf, np.zeros_like(bf)], axis=1)
    assert L.MlPoly(bf).eval(pt) == orc.mle_eval(lifted, pt)


@pytest.mark.parametrize("d,k", [(1, 4), (2, 1), (2, 12), (2, 13), (3, 12), (3, 14), (2, 18),
                                 (3, 20)])
def test_sumcheck_matches_oracle(lgs, orc, d, k):
    polys = [rng.ext_elements(6000 + 10 * d + j, 1 << k) for j in range(d)]
    ch = rng.ext_elements(7000 + k, k)
    rounds, finals = L.sumcheck_prove(polys, ch)
    r_o, f_o, _ = orc.sumcheck_prove(polys, ch)
    assert np.array_equal(rounds, r_o)
    assert np.array_equal(finals, f_o)


def test_rs_alu_rates_measure_the_encodings_arithmetic(lgs):
    """lgs_rs_alu_rates (the RS encoding's arithmetic floor) runs and gives plausible rates: a
    radix-8 DFT holds 12 butterflies, so it runs slower than a single multiplication."""
    import ctypes as C

    ctx = L.Context(0)
    r8, mul = C.c_double(), C.c_double()
    L._lib.check(L.load().lgs_rs_alu_rates(ctx.handle, 256, C.byref(r8), C.byref(mul)))
    assert 1e9 < r8.value < mul.value < 1e14
