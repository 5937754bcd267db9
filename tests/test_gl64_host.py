"""The host build of the library's Goldilocks arithmetic (ligesis_b200/csrc/gl64.cuh, the code the
host verifiers and planners use) against Python integers: add, sub, mul, the 128-bit reduction,
multiplication by powers of two for every exponent below 192, and the two-adic generator."""
from __future__ import annotations

import random
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
P = 2**64 - 2**32 + 1

PROGRAM = r"""
#include <cstdio>
#include "gl64.cuh"
using namespace lgs;
int main() {
  unsigned long long a, b;
  unsigned s;
  while (std::scanf("%llu %llu %u", &a, &b, &s) == 3) {
    std::printf("%llu %llu %llu %llu %llu\n", (unsigned long long)gl_add(a, b),
                (unsigned long long)gl_sub(a, b), (unsigned long long)gl_mul(a, b),
                (unsigned long long)gl_reduce(a, b), (unsigned long long)gl_mul_pow2(a, s));
  }
  std::printf("%llu\n", (unsigned long long)gl_two_adic_generator(32));
  return 0;
}
"""


@pytest.fixture(scope="module")
def gl_host(tmp_path_factory):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    d = tmp_path_factory.mktemp("gl64")
    src, exe = d / "gl.cpp", d / "gl"
    src.write_text(PROGRAM)
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", str(ROOT / "ligesis_b200" / "csrc"), str(src),
                    "-o", str(exe)], check=True)
    return exe


def test_field_ops_match_python_integers(gl_host):
    g = random.Random(7)
    edge = [0, 1, 2, P - 1, P - 2, 2**32 - 1, 2**32, 2**63, P // 2]
    cases = []
    for s in range(192):
        for _ in range(12):
            cases.append((g.randrange(P), g.randrange(P), s))
        for e in edge:
            cases.append((e, edge[s % len(edge)], s))
    # gl_reduce takes any (lo, hi) pair: include non-canonical words
    cases += [(2**64 - 1, 2**64 - 1, 0), (P, 2**64 - 1, 5), (2**64 - 1, P, 7)]
    inp = "".join(f"{a} {b} {s}\n" for a, b, s in cases)
    out = subprocess.run([str(gl_host)], input=inp, capture_output=True, text=True,
                         check=True).stdout.split("\n")
    for (a, b, s), line in zip(cases, out):
        add, sub, mul, red, pw = map(int, line.split())
        assert red == (a + (b << 64)) % P, (a, b)
        if a < P and b < P:
            assert add == (a + b) % P and sub == (a - b) % P and mul == a * b % P, (a, b)
            assert pw == a * pow(2, s, P) % P, (a, s)
    assert int(out[len(cases)]) == 1753635133440165772
