"""GKR fraction sum and GKR-LogUp lookup on the GPU against the CPU oracle
(logup/src/frac_sum.rs, logup/src/lookup.rs): proofs byte for byte, reduced claims, cursors,
the host verifier accepting, and the reference's rejections on GPU-made proofs.  Sizes cross the
kernels' boundaries: one pass folds 10 rounds, one build launch 10 levels."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import field as fld
from ligesis_b200 import rng

pytestmark = pytest.mark.gpu


def _oracle(fields):
    o = L.RandomOracle(0, length=4)
    o.fields = np.ascontiguousarray(fields)
    return o


@pytest.mark.parametrize("k", [0, 1, 2, 3, 9, 10, 11, 12, 21, 22])
def test_frac_sum_matches_oracle(lgs, orc, k):
    p, q = rng.ext_elements(500 + k, 1 << k), rng.ext_elements(600 + k, 1 << k)
    fields = rng.ext_elements(700 + k, 512)
    o = _oracle(fields)
    o.cursors[0] = 3  # start mid-oracle
    proof, point, pe, qe = L.FracSum.prove(p, q, o)
    want, wpoint, wpe, wqe, wcur = orc.frac_sum_prove(p, q, fields, 3)
    assert proof.data == want
    assert np.array_equal(point, wpoint) and (pe, qe) == (wpe, wqe)
    assert int(o.cursors[0]) == wcur
    o.cursors[0] = 3
    got = L.FracSum.verify(proof, o)
    assert got is not None and np.array_equal(got[0], point) and got[1:] == (pe, qe)


@pytest.mark.parametrize("k", [1, 11, 22])
def test_frac_sum_unit_numerators(lgs, orc, k):
    q = rng.ext_elements(800 + k, 1 << k)
    fields = rng.ext_elements(900 + k, 512)
    proof, point, pe, qe = L.FracSum.prove(None, q, _oracle(fields))
    want, wpoint, wpe, wqe, _ = orc.frac_sum_prove(None, q, fields)
    assert proof.data == want and (pe, qe) == (wpe, wqe) and pe == (1, 0)


def _sample(mu, nu, seed):
    t = rng.ext_elements(seed, 1 << nu)
    idx = (rng.ints(seed + 1, 1 << mu) % np.uint64(1 << nu)).astype(np.int64)
    return t[idx], t


@pytest.mark.parametrize("mu,nu", [(0, 0), (4, 2), (8, 4), (10, 6), (14, 3), (20, 12), (22, 16)])
def test_lookup_matches_oracle(lgs, orc, mu, nu):
    a, t = _sample(mu, nu, 40 + mu + nu)
    e = L.multiplicity_vector(a, t)
    fields = rng.ext_elements(60 + mu, 1024)
    o = _oracle(fields)
    proof, zq, zt = L.Lookup.prove_with_opening_points(a, t, e, o)
    want, wzq, wzt, wcur = orc.lookup_prove(a, t, e, fields)
    assert proof.data == want
    assert np.array_equal(zq, wzq) and np.array_equal(zt, wzt) and int(o.cursors[0]) == wcur
    o.restart()
    claims = L.Lookup.verify(proof, o)
    assert claims is not None
    if mu <= 14:
        assert claims[0].value == orc.mle_eval(a, zq)
        assert claims[1].value == orc.mle_eval(e, zt)
        assert claims[2].value == orc.mle_eval(t, zt)


def test_lookup_rejections_on_gpu_proofs(lgs):
    a, t = _sample(12, 5, 3)
    fields = rng.ext_elements(4, 512)
    o = _oracle(fields)
    good = L.Lookup.prove(a, t, o)
    o.restart()
    assert L.Lookup.verify(good, o) is not None
    bad = a.copy()
    bad[3] = rng.ext_elements(5, 1)[0]
    o.restart()
    assert L.Lookup.verify(L.Lookup.prove(bad, t, o), _oracle(fields)) is None
    e = L.multiplicity_vector(a, t)
    e[2, 0] += 1
    o.restart()
    assert L.Lookup.verify(L.Lookup.prove_with_mults(a, t, e, o), _oracle(fields)) is None
    b = bytearray(good.data)
    v = int.from_bytes(b[16:24], "little")  # query num, c0 (after "LGSL" and "LGSF" headers)
    b[16:24] = ((v + 1) % fld.P).to_bytes(8, "little")
    assert L.Lookup.verify(bytes(b), _oracle(fields)) is None


def test_device_inputs_same_bytes(lgs):
    torch = pytest.importorskip("torch")
    a, t = _sample(16, 8, 9)
    e = L.multiplicity_vector(a, t)
    fields = rng.ext_elements(10, 512)
    host = L.Lookup.prove_with_mults(a, t, e, _oracle(fields))
    dev = [torch.from_numpy(x.view(np.int64)).cuda() for x in (a, t, e)]
    torch.cuda.synchronize()
    got = L.Lookup.prove_with_mults(*dev, _oracle(fields))
    assert got.data == host.data
    q = rng.ext_elements(11, 1 << 13)
    hp = L.FracSum.prove(None, q, _oracle(fields))[0]
    qd = torch.from_numpy(q.view(np.int64)).cuda()
    torch.cuda.synchronize()
    assert L.FracSum.prove(None, qd, _oracle(fields))[0].data == hp.data


def test_frac_sum_zero_coordinates(lgs, orc):
    """Challenges equal to zero or one (a lambda, a beta, fold challenges): layers whose point has
    a zero coordinate sum S(1) instead of taking it from the claim chain, and eq(z, c) factors can
    vanish; the bytes still equal the oracle's."""
    k = 14
    p, q = rng.ext_elements(31, 1 << k), rng.ext_elements(32, 1 << k)
    fields = rng.ext_elements(33, 512).copy()
    # offset o = r (r + 3) / 2 of layer r: lambda at o, ch[r][t] at o + 1 + t, beta at o + 1 + r
    for r, t in ((5, 1), (12, 3), (12, 12), (12, 13), (13, 0)):
        fields[r * (r + 3) // 2 + t] = 0
    fields[9 * 12 // 2 + 2] = (1, 0)
    proof, point, pe, qe = L.FracSum.prove(p, q, _oracle(fields))
    want, wpoint, wpe, wqe, _ = orc.frac_sum_prove(p, q, fields)
    assert proof.data == want and (pe, qe) == (wpe, wqe)
    assert L.FracSum.verify(proof, _oracle(fields)) is not None
