"""Regenerates tests/golden/ligesis_large.json: digests of the CPU oracle's LigeSIS commitment
and proof at the large reference-valid shapes, mu = 24 as 2^7 x 2^17 (the README's row,
README.md:175) and mu = 26 as 2^7 x 2^19.  The oracle needs minutes for these shapes, so the
GPU tests compare against these digests instead of running it.

Inputs are the ones tests/helpers.ligesis_inputs draws for the shape (f, A, z and the oracle
arrays from ligesis_b200.rng with seed 10*log_m + log_n), so a GPU run on the same seed must
reproduce every digest byte for byte.  Recorded per shape: the Merkle root, SHA-256 of the
codeword digest H (C x 2n canonical u64 LE), SHA-256 and length of the proof bytes, and the
oracle cursors after the proof.

Run:  python tests/golden/make_ligesis_golden.py [--threads N]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import orc  # noqa: E402
from tests.helpers import ligesis_inputs  # noqa: E402

SHAPES = [(7, 17), (7, 19)]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=None)
    args = ap.parse_args()
    threads = orc.set_threads(args.threads)
    out = []
    for log_m, log_n in SHAPES:
        seed = 10 * log_m + log_n
        f, A, z, fields, ints = ligesis_inputs(log_m, log_n, seed=seed)
        t0 = time.time()
        key = orc.Key(log_m, log_n, A)
        cm = orc.Commitment(key, f)
        proof, cursors = orc.prove(key, cm, z, fields, ints)
        ok = orc.verify(key.com_a, log_m, log_n, cm.root, z, proof, fields, ints)
        if not ok:
            raise SystemExit(f"oracle proof at {log_m}x{log_n} does not verify")
        out.append({"log_m": log_m, "log_n": log_n, "seed": seed,
                    "com_a": key.com_a.hex(), "root": cm.root.hex(),
                    "digest_sha256": hashlib.sha256(cm.digest().tobytes()).hexdigest(),
                    "proof_sha256": hashlib.sha256(proof).hexdigest(),
                    "proof_len": len(proof), "cursors": list(cursors)})
        print(f"{log_m}x{log_n}: {time.time() - t0:.1f} s", flush=True)
        del cm, key
    path = Path(__file__).with_name("ligesis_large.json")
    path.write_text(json.dumps({"generator": "oracle/ (C++ restatement), "
                                f"{threads} threads; tests/golden/make_ligesis_golden.py",
                                "inputs": "tests.helpers.ligesis_inputs(log_m, log_n, seed)",
                                "shapes": out}, indent=1) + "\n")
    print(f"wrote {path}")


if __name__ == "__main__":
    main()
