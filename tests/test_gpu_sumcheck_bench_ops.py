"""The sumcheck microbenchmark's operations on device-resident inputs, against the oracle.

The reference's sumcheck bench proves a product of 3 multilinears (pcs/benches/sumcheck.rs:64-68);
bench.py's sumcheck mode times it over F_{p^2} at mu = 20, 22, 24, the eq-product variant
[eq_z, f, g] (the shape of the binary check, pcs/src/ligesis.rs:424-428) and an MlPoly
fold/new_eq/eval sweep (utils/src/poly.rs:7-53), all through the device-pointer entry points
lgs_sumcheck_prove_dev, lgs_new_eq_dev, lgs_mle_fold_dev and lgs_mle_eval_dev.  Here each of
them is compared with the C++ oracle on the same seeded inputs, round polynomials and final
evaluations bit for bit, at the benchmark's sizes."""
from __future__ import annotations

import numpy as np
import pytest

from ligesis_b200 import rng
from ligesis_b200._lib import Context, check, load

pytestmark = pytest.mark.gpu


def _dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).reshape(-1)).cuda()


def _host(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


def _sync(ctx):
    import torch

    torch.cuda.synchronize()


@pytest.fixture(scope="module")
def orc_threads(orc):
    orc.set_threads(None)
    yield orc
    orc.set_threads(1)


@pytest.mark.parametrize("k", [20, 22, 24])
def test_three_factor_sumcheck_matches_oracle(lgs, orc_threads, k):
    import torch

    orc, d = orc_threads, 3
    polys = [rng.ext_elements(7000 + 10 * k + j, 1 << k) for j in range(d)]
    ch = rng.ext_elements(7100 + k, k)
    want_rounds, want_finals, _ = orc.sumcheck_prove(polys, ch)
    ctx = Context.default()
    d_polys = _dev(np.concatenate(polys))
    del polys
    d_ch = _dev(ch)
    d_rounds = torch.zeros(k * (d + 1) * 2, dtype=torch.int64, device="cuda")
    d_finals = torch.zeros(d * 2, dtype=torch.int64, device="cuda")
    check(load().lgs_sumcheck_prove_dev(ctx.handle, d_polys.data_ptr(), d, k, d_ch.data_ptr(),
                                        d_rounds.data_ptr(), d_finals.data_ptr()))
    _sync(ctx)
    assert np.array_equal(_host(d_rounds).reshape(k, d + 1, 2), want_rounds)
    assert np.array_equal(_host(d_finals).reshape(d, 2), want_finals)


def test_eq_product_sumcheck_matches_oracle(lgs, orc_threads):
    """[eq_z, f, g] with eq_z built on the device by lgs_new_eq_dev."""
    import torch

    orc, k, d = orc_threads, 22, 3
    z = rng.ext_elements(7201, k)
    f = rng.ext_elements(7202, 1 << k)
    g = rng.ext_elements(7203, 1 << k)
    ch = rng.ext_elements(7204, k)
    eq = orc.new_eq(z)
    want_rounds, want_finals, _ = orc.sumcheck_prove([eq, f, g], ch)
    ctx = Context.default()
    d_polys = torch.empty(3 * (2 << k), dtype=torch.int64, device="cuda")
    d_z = _dev(z)
    check(load().lgs_new_eq_dev(ctx.handle, d_z.data_ptr(), k, d_polys.data_ptr()))
    d_polys[(2 << k):(4 << k)] = _dev(f)
    d_polys[(4 << k):] = _dev(g)
    _sync(ctx)
    assert np.array_equal(_host(d_polys[:(2 << k)]).reshape(-1, 2), eq)
    d_ch = _dev(ch)
    d_rounds = torch.zeros(k * 4 * 2, dtype=torch.int64, device="cuda")
    d_finals = torch.zeros(3 * 2, dtype=torch.int64, device="cuda")
    check(load().lgs_sumcheck_prove_dev(ctx.handle, d_polys.data_ptr(), 3, k, d_ch.data_ptr(),
                                        d_rounds.data_ptr(), d_finals.data_ptr()))
    _sync(ctx)
    assert np.array_equal(_host(d_rounds).reshape(k, 4, 2), want_rounds)
    assert np.array_equal(_host(d_finals).reshape(3, 2), want_finals)


@pytest.mark.parametrize("k", [20, 24])
def test_new_eq_fold_and_eval_match_oracle(lgs, orc_threads, k):
    import torch

    orc = orc_threads
    ctx = Context.default()
    pt = rng.ext_elements(7300 + k, k)
    evals = rng.ext_elements(7400 + k, 1 << k)
    d_pt, d_ev = _dev(pt), _dev(evals)
    d_eq = torch.empty(2 << k, dtype=torch.int64, device="cuda")
    check(load().lgs_new_eq_dev(ctx.handle, d_pt.data_ptr(), k, d_eq.data_ptr()))
    d_val = torch.zeros(2, dtype=torch.int64, device="cuda")
    check(load().lgs_mle_eval_dev(ctx.handle, d_ev.data_ptr(), k, d_pt.data_ptr(),
                                  d_val.data_ptr()))
    _sync(ctx)
    assert np.array_equal(_host(d_eq).reshape(-1, 2), orc.new_eq(pt))
    assert tuple(int(v) for v in _host(d_val)) == tuple(int(v) for v in orc.mle_eval(evals, pt))
    for np_ in (1, 3, 8):
        d_out = torch.empty(2 << (k - np_), dtype=torch.int64, device="cuda")
        check(load().lgs_mle_fold_dev(ctx.handle, d_ev.data_ptr(), k, d_pt.data_ptr(), np_,
                                      d_out.data_ptr()))
        _sync(ctx)
        assert np.array_equal(_host(d_out).reshape(-1, 2), orc.mle_fold(evals, pt[:np_])), np_
