"""The batched/served engine: jobs of mixed shapes in flight together give exactly the roots and
proofs of the one-at-a-time path (and of the CPU oracle), admission holds jobs back when the
HBM budget is exhausted, and a failing job reports its status without stopping the others."""
from __future__ import annotations

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import rng
from ligesis_b200.engine import ProverEngine
from ligesis_b200.workloads import gpt2_layer_witness, shape_for_mu

pytestmark = pytest.mark.gpu

SHAPES = [(3, 10), (4, 11), (5, 13), (3, 10), (4, 12), (5, 13)]


@pytest.fixture(scope="module")
def keyed_jobs(lgs):
    ctx = L.Context.default()
    keys, jobs = {}, []
    for i, (lm, ln) in enumerate(SHAPES):
        if (lm, ln) not in keys:
            A = rng.field_elements(70 + lm, 32 * (64 << lm)).reshape(32, 64 << lm)
            keys[(lm, ln)] = L.Ligesis.setup_with_hash(lm, ln, L.SubsetSumHash(64 << lm, a=A), ctx)
        f = rng.field_elements(800 + i, 1 << (lm + ln))
        z = rng.ext_elements(850 + i, lm + ln)
        jobs.append(((lm, ln), f, z, 900 + i))
    return keys, jobs


def _plain(keys, jobs):
    out = []
    for shape, f, z, os_ in jobs:
        pk, _ = keys[shape]
        c, d = L.Ligesis.commit(pk, L.MlPoly(f))
        out.append((c.root, L.Ligesis.prove(pk, d, z, L.RandomOracle(os_, length=1024)).data))
    return out


def test_engine_matches_one_at_a_time_path(keyed_jobs):
    keys, jobs = keyed_jobs
    ref = _plain(keys, jobs)
    with ProverEngine(0, lanes=3) as eng:
        res = eng.run([(keys[s][0], f, z, L.RandomOracle(o, length=1024)) for s, f, z, o in jobs])
    assert [(r.commit.root, r.proof.data) for r in res] == ref
    with ProverEngine(0, lanes=3) as eng:  # prepared lanes replay captured proves
        eng.prepare(pk for pk, _ in keys.values())
        res = eng.run([(keys[s][0], f, z, L.RandomOracle(o, length=1024)) for s, f, z, o in jobs])
        res += eng.run([(keys[s][0], f, z, L.RandomOracle(o, length=1024)) for s, f, z, o in jobs])
    assert [(r.commit.root, r.proof.data) for r in res] == ref + ref
    for (shape, _, z, os_), r in zip(jobs, res):
        o = L.RandomOracle(os_, length=1024)
        assert L.Ligesis.verify(keys[shape][1], r.commit, z, r.proof, o)
        assert r.start_ms >= r.submit_ms and r.done_ms >= r.start_ms


def test_engine_matches_oracle(keyed_jobs, orc):
    keys, jobs = keyed_jobs
    shape, f, z, os_ = jobs[2]
    lm, ln = shape
    A = rng.field_elements(70 + lm, 32 * (64 << lm)).reshape(32, 64 << lm)
    o = L.RandomOracle(os_, length=1024)
    with ProverEngine(0, lanes=2) as eng:
        r = eng.run([(keys[shape][0], f, z, o)])[0]
    key = orc.Key(lm, ln, A)
    cm = orc.Commitment(key, f)
    o2 = L.RandomOracle(os_, length=1024)
    want, cur = orc.prove(key, cm, z, o2.fields, o2.ints)
    assert r.commit.root == cm.root and r.proof.data == want and r.cursors == cur


def test_tiny_budget_serialises_but_completes(keyed_jobs):
    keys, jobs = keyed_jobs
    ref = _plain(keys, jobs[:3])
    with ProverEngine(0, lanes=3, hbm_budget=1) as eng:
        res = eng.run([(keys[s][0], f, z, L.RandomOracle(o, length=1024)) for s, f, z, o in jobs[:3]])
    assert [(r.commit.root, r.proof.data) for r in res] == ref
    starts = sorted((r.start_ms, r.done_ms) for r in res)
    for (s0, d0), (s1, _) in zip(starts, starts[1:]):
        assert s1 >= d0  # one job at a time when nothing fits beside another


def test_failing_job_reports_and_others_finish(keyed_jobs):
    keys, jobs = keyed_jobs
    (shape, f, z, os_) = jobs[0]
    with ProverEngine(0, lanes=2) as eng:
        bad = eng.submit(keys[shape][0], f, z, L.RandomOracle(os_, length=64))  # too few ints
        good = eng.submit(keys[shape][0], f, z, L.RandomOracle(os_, length=1024))
        with pytest.raises(L.OracleExhausted):
            eng.wait(bad)
        assert eng.wait(good).proof.data == _plain(keys, [jobs[0]])[0][1]


def test_gpt2_witness_job(lgs):
    f = gpt2_layer_witness()
    assert f.size == 1 << 21 and int(f.max()) < L.rng.P
    lm, ln = shape_for_mu(21)
    g = rng.SeededRng(11)
    pk, vk = L.Ligesis.setup(lm, ln, g)
    z = g.ext_elements(21)
    with ProverEngine(0, lanes=2) as eng:
        r = eng.run([(pk, f, z, L.RandomOracle(12, length=1024))])[0]
    assert L.Ligesis.verify(vk, r.commit, z, r.proof, L.RandomOracle(12, length=1024))
    assert r.proof.y == L.MlPoly(f).eval(z)
