"""Regenerates tests/golden/blake3_kat.json: BLAKE3 known answers from the `blake3` Python
package (a third-party implementation of the same published function the reference calls via
the blake3 crate, utils/src/merkle.rs:10-12).  Input i of length L is bytes(j % 251 for j < L),
the input pattern of the official BLAKE3 test vectors.

Run:  python tests/golden/make_golden.py
"""
import json
from pathlib import Path

import blake3

LENGTHS = [0, 1, 7, 8, 16, 31, 32, 63, 64, 65, 96, 127, 128, 129, 255, 256, 257, 511, 512, 513,
           1023, 1024, 1025, 2047, 2048, 2049, 3072, 3073, 4096, 4097, 5120, 8192, 31744, 102400]


def main() -> None:
    out = []
    for n in LENGTHS:
        data = bytes(j % 251 for j in range(n))
        out.append({"len": n, "hash": blake3.blake3(data).hexdigest()})
    path = Path(__file__).with_name("blake3_kat.json")
    path.write_text(json.dumps({"generator": "blake3 (Python package) " + blake3.__version__,
                                "input": "bytes(j % 251 for j in range(len))",
                                "vectors": out}, indent=1) + "\n")
    print(f"wrote {path} ({len(out)} vectors)")


if __name__ == "__main__":
    main()
