"""The C-ABI boundary without a GPU: liblgs.so loads, exports every function include/*.h
declares, and host-only entry points behave (shape rules, oracle budgets, error mapping)."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import ligesis_b200 as L
from ligesis_b200 import rng

ROOT = Path(__file__).resolve().parent.parent


def _declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(lgs_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(lgs):
    lib = C.CDLL(str(ROOT / "ligesis_b200" / "liblgs.so"))
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_strings(lgs):
    lib = L.load()
    assert b"sm_100a" in lib.lgs_version()


def test_oracle_need_matches_transcript_plan(lgs):
    # fields: 3 sumchecks over B_I vars, alpha2(5), r2(7), hash/recon (log W), table (log 2n),
    # rslink + a-batch (log n), 2 gammas, 3 coefficients, R batch rounds.
    for log_m, log_n in [(3, 10), (6, 14), (7, 17), (7, 19)]:
        nf, ni = L.oracle_need(log_m, log_n)
        lw, ls = log_m + 6, 7
        nb = lw + ls
        R = max(11 + log_m, nb, log_n) - 6
        assert nf == 3 * nb + 5 + ls + 2 * lw + (log_n + 1) + 2 * log_n + 2 + 3 + R
        assert ni == 4 * 128 + 100


def test_oracle_need_rejects_bad_shapes(lgs):
    with pytest.raises(L.ShapeError):
        L.oracle_need(10, 10)
    assert L.shape_ok(7, 17) and not L.shape_ok(12, 12)


def test_context_without_device_fails_cleanly(lgs):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(L.LgsError):
        L.Context(0)


def test_rng_is_deterministic_and_canonical():
    a = rng.field_elements(5, 1000)
    b = rng.field_elements(5, 1000)
    assert (a == b).all() and (a < np.uint64(rng.P)).all()
    assert (rng.field_elements(5, 10, start=990) == a[990:]).all()
    e = rng.ext_elements(5, 500)
    assert (e.reshape(-1) == a).all()
    g = rng.SeededRng(5)
    assert (g.field_elements(10) == a[:10]).all() and (g.field_elements(10) == a[10:20]).all()


def test_random_oracle_cursors():
    o = L.RandomOracle(3, length=64)
    f0 = o.next_field()
    assert f0 == (int(o.fields[0, 0]), int(o.fields[0, 1]))
    o.next_n_ints(5)
    assert o.drawn() == (1, 5)
    o.restart()
    assert o.drawn() == (0, 0)


def test_mlpoly_split_matches_reference_layout():
    p = L.MlPoly(np.arange(16, dtype=np.uint64))
    parts = p.split(4)  # num_chunks = 4: chunk j = [j, j+4, j+8, j+12]
    assert [q.evals.tolist() for q in parts] == [[0, 4, 8, 12], [1, 5, 9, 13], [2, 6, 10, 14],
                                                 [3, 7, 11, 15]]
