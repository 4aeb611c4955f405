"""Generates tests/golden/blake3_vectors.json: BLAKE3 known answers for the
tree mode (inputs of 0 bytes to 100 chunks, crossing every chunk and parent
boundary the oracle's and the device's chunk trees handle) and derive-key
mode, the two modes the proving path uses.

The values come from the `blake3` Python package (bindings of the BLAKE3
team's Rust crate, the implementation the reference depends on at 1.8.7:
Cargo.lock) when it is importable; the fixture is committed so the tests need
nothing but the file. Inputs follow the BLAKE3 test-vector convention: byte i
of an input is i mod 251.

    python tests/golden/make_blake3_fixture.py
"""
import json
import os

import blake3

LENGTHS = [0, 1, 63, 64, 65, 127, 128, 1023, 1024, 1025, 2048, 2049, 3072, 3073, 4096, 4097,
           5120, 5121, 6144, 6145, 7168, 7169, 8192, 8193, 16384, 31744, 65536, 102400]
CONTEXTS = ["bitz/pcs/bit-inner-product-weights/v1",
            "BLAKE3 2019-12-27 16:29:52 test vectors context"]


def data(n):
    return bytes(i % 251 for i in range(n))


def main():
    cases = []
    for n in LENGTHS:
        x = data(n)
        cases.append({
            "len": n,
            "hash": blake3.blake3(x).hexdigest(),
            "derive_key": {c: blake3.blake3(x, derive_key_context=c).hexdigest() for c in CONTEXTS},
        })
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "blake3_vectors.json"), "w") as f:
        json.dump({"source": "blake3 Python package %s" % blake3.__version__,
                   "input": "byte i = i mod 251", "contexts": CONTEXTS,
                   "cases": cases}, f, indent=0)


if __name__ == "__main__":
    main()
