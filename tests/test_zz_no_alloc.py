"""The allocation-free sumcheck entry point (lgs_sumcheck_prove_noalloc).

It exists for callers that cannot allocate device memory themselves or through the library: a
process whose HBM belongs to another allocator, or a serving loop that must not pay for
cudaMalloc's device-wide synchronisation.  They pass device buffers for inputs and outputs and
the library works in a fixed device array.  This test drives it through the C ABI with device
buffers and requires the same round polynomials and final evaluations, bit for bit, as the CPU
oracle's sumcheck prover (an independent restatement of utils/src/sumcheck.rs:37-84) and as the
allocating entry point lgs_sumcheck_prove, on two calls in a row (different shapes and inputs,
so the second call also shows that the shared array carries nothing over)."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import rng
from ligesis_b200._lib import LgsError, check, load

pytestmark = pytest.mark.gpu


def _dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64).reshape(-1).copy()).cuda()


def _host(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64)


def test_noalloc_sumcheck_matches_oracle(orc):
    import torch

    lib = load()
    for call, (d, k) in enumerate([(3, 14), (2, 16)]):
        polys = [rng.ext_elements(900 + 10 * call + j, 1 << k) for j in range(d)]
        ch = rng.ext_elements(950 + call, k)
        want_rounds, want_finals, used = orc.sumcheck_prove(polys, ch)
        assert np.array_equal(used, ch), call
        alloc_rounds, alloc_finals = L.sumcheck_prove(polys, ch)
        assert np.array_equal(alloc_rounds, want_rounds), call
        assert np.array_equal(alloc_finals, want_finals), call

        d_polys = _dev(np.concatenate(polys))
        d_ch = _dev(ch)
        d_rounds = torch.zeros(k * (d + 1) * 2, dtype=torch.int64, device="cuda")
        d_finals = torch.zeros(d * 2, dtype=torch.int64, device="cuda")
        stream = torch.cuda.current_stream()
        check(lib.lgs_sumcheck_prove_noalloc(d_polys.data_ptr(), d, k, d_ch.data_ptr(),
                                             d_rounds.data_ptr(), d_finals.data_ptr(),
                                             stream.cuda_stream))
        stream.synchronize()
        assert np.array_equal(_host(d_rounds).reshape(k, d + 1, 2), want_rounds), call
        assert np.array_equal(_host(d_finals).reshape(d, 2), want_finals), call
        # the inputs are only read
        assert np.array_equal(_host(d_polys).reshape(-1, 2), np.concatenate(polys)), call


def test_noalloc_sumcheck_rejects_sizes_beyond_its_scratch():
    import torch

    lib = load()
    k = 17
    d_buf = torch.zeros(4, dtype=torch.int64, device="cuda")
    p = d_buf.data_ptr()
    with pytest.raises(LgsError, match="1 <= k <= 16"):
        check(lib.lgs_sumcheck_prove_noalloc(p, 2, k, p, p, p, None))
    with pytest.raises(LgsError, match="1 <= d <= 3"):
        check(lib.lgs_sumcheck_prove_noalloc(p, 4, 8, p, p, p, None))
