"""Generates tests/golden/ghash_nist.json from the reference's NIST GCM vectors.

The reference pins its GF(2^128) arithmetic with NIST CAVP GCM encryption
vectors (crates/field/tests/ghash_vectors.rs over
crates/field/tests/vectors/gcm_encrypt_128.rsp). The tag of a 96-bit-IV case is
GHASH_H(A, C) xor E_K(IV || 0^31 || 1) with H = E_K(0^128). AES is run here, at
fixture time, so the committed fixture holds only field data: H, the AAD, the
ciphertext and the expected GHASH prefix (tag xor mask, truncated to the tag
length). Run in a container where the reference tree is mounted:

    python tests/golden/make_ghash_fixture.py /path/to/reference
"""
import json
import os
import sys

from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes


def parse(text):
    cases, cur, tag_bytes, in_rec = [], {}, 0, False
    for line in text.splitlines():
        line = line.strip()
        if not line or line.startswith("#"):
            if in_rec:
                cases.append(cur)
                in_rec = False
            continue
        if line.startswith("[") and line.endswith("]"):
            p = line[1:-1]
            if p.startswith("Taglen = "):
                tag_bytes = int(p.split(" = ")[1]) // 8
            continue
        name, _, value = line.partition("=")
        name = name.strip()
        value = value.strip()
        if name == "Count":
            cur = {"tag_bytes": tag_bytes}
            in_rec = True
        elif name in ("Key", "IV", "AAD", "CT", "Tag"):
            cur[name] = value
    if in_rec:
        cases.append(cur)
    return cases


def aes_block(key, block):
    enc = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    return enc.update(block) + enc.finalize()


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_ghash_fixture.py <path to the reference tree>")
    ref = sys.argv[1]
    path = os.path.join(ref, "crates/field/tests/vectors/gcm_encrypt_128.rsp")
    cases = parse(open(path).read())
    assert len(cases) == 525, len(cases)
    out = []
    for c in cases:
        key = bytes.fromhex(c["Key"])
        iv = bytes.fromhex(c["IV"])
        h = aes_block(key, bytes(16))
        mask = aes_block(key, iv + b"\x00\x00\x00\x01")
        tag = bytes.fromhex(c["Tag"])
        ghash_prefix = bytes(a ^ b for a, b in zip(tag, mask[: len(tag)]))
        out.append({"h": h.hex(), "aad": c["AAD"], "ct": c["CT"], "ghash_prefix": ghash_prefix.hex()})
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "ghash_nist.json"), "w") as f:
        json.dump({"source": "crates/field/tests/vectors/gcm_encrypt_128.rsp", "cases": out}, f, indent=0)


if __name__ == "__main__":
    main()
