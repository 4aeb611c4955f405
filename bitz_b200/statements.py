"""Statement inputs for the SHA-256 circuits, as tooling/cli/src/circuits.rs:67-139
builds them, from a seeded SplitMix64 byte stream instead of OS entropy."""
import hashlib
import struct

import numpy as np

IV = [0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a, 0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19]
KINDS = {"sha256-compression": 0, "sha256-chain": 1, "sha256-block-aligned": 2, "sha256-2kb": 3}


def splitmix64_bytes(seed: int, n: int) -> bytes:
    out = bytearray()
    x = seed & (2**64 - 1)
    while len(out) < n:
        x = (x + 0x9E3779B97F4A7C15) & (2**64 - 1)
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
        z ^= z >> 31
        out += z.to_bytes(8, "little")
    return bytes(out[:n])


def _sha256_compress(state, block):
    K = [
        0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
        0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
        0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
        0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
        0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
        0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
        0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
        0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2]
    M = 0xffffffff
    rr = lambda x, n: ((x >> n) | (x << (32 - n))) & M
    w = list(struct.unpack(">16I", block))
    for i in range(16, 64):
        s0 = rr(w[i - 15], 7) ^ rr(w[i - 15], 18) ^ (w[i - 15] >> 3)
        s1 = rr(w[i - 2], 17) ^ rr(w[i - 2], 19) ^ (w[i - 2] >> 10)
        w.append((w[i - 16] + s0 + w[i - 7] + s1) & M)
    a, b, c, d, e, f, g, h = state
    for i in range(64):
        t1 = (h + (rr(e, 6) ^ rr(e, 11) ^ rr(e, 25)) + ((e & f) ^ (~e & g)) + K[i] + w[i]) & M
        t2 = ((rr(a, 2) ^ rr(a, 13) ^ rr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c))) & M
        h, g, f, e, d, c, b, a = g, f, e, (d + t1) & M, c, b, a, (t1 + t2) & M
    return [(x + y) & M for x, y in zip(state, [a, b, c, d, e, f, g, h])]


def word_bits(data: bytes):
    bits = []
    for k in range(0, len(data), 4):
        w = int.from_bytes(data[k:k + 4], "big")
        bits += [(w >> i) & 1 for i in range(32)]
    return bits


def stream_bits(data: bytes):
    return [(byte >> i) & 1 for byte in data for i in range(7, -1, -1)]


def instance(kind: str, blocks: int, seed: int, initial_state=None):
    """(input bits, output bits, message bytes) in the circuit's bit order."""
    if kind == "sha256-2kb":
        blocks = 32
    data = splitmix64_bytes(seed, 64 * blocks)
    if kind in ("sha256-compression", "sha256-chain"):
        state = list(initial_state or IV)
        start = list(state)
        for k in range(blocks):
            state = _sha256_compress(state, data[64 * k:64 * k + 64])
        inputs = word_bits(data)
        if kind == "sha256-compression":
            inputs += [(w >> i) & 1 for w in start for i in range(32)]
        outputs = [(w >> i) & 1 for w in state for i in range(32)]
    else:
        inputs = stream_bits(data)
        outputs = stream_bits(hashlib.sha256(data).digest())
    return np.array(inputs, dtype=np.uint8), np.array(outputs, dtype=np.uint8), data


def random_state(seed: int):
    raw = splitmix64_bytes(seed ^ 0x5EED, 32)
    return [int.from_bytes(raw[4 * i:4 * i + 4], "little") for i in range(8)]


def message_instance(kind: str, data: bytes):
    """(input bits, output bits) of a padded-message circuit (block-aligned or
    2kb) for the message ``data`` (tooling/cli/src/circuits.rs:103-139)."""
    return (np.array(stream_bits(data), dtype=np.uint8),
            np.array(stream_bits(hashlib.sha256(data).digest()), dtype=np.uint8))


def blocks_proven(kind: str, n_inputs: int) -> int:
    """Compression blocks a proof covers: message blocks, plus the padding
    block of the padded-message circuits."""
    if kind in ("sha256-block-aligned", "sha256-2kb"):
        return n_inputs // 512 + 1
    return max(n_inputs // 512, 1)


def _u64s(seed: int, n: int):
    raw = splitmix64_bytes(seed, 8 * n)
    return [int.from_bytes(raw[8 * i:8 * i + 8], "little") for i in range(n)]


def batch_mix(seed: int = 3, count: int = 256, max_blocks: int = 32):
    """Independent sha256-block-aligned statements with message lengths
    uniform over 0..max_blocks blocks (empty messages allowed) and uniform
    random bytes: lengths from the SplitMix64 stream of ``seed``, message
    bytes from the stream of ``seed + 1000003``. Returns a list of
    (kind, input bits, output bits)."""
    lengths = [v % (max_blocks + 1) for v in _u64s(seed, count)]
    data = splitmix64_bytes(seed + 1000003, 64 * sum(lengths))
    out, pos = [], 0
    for k in lengths:
        msg = data[pos:pos + 64 * k]
        pos += 64 * k
        out.append(("sha256-block-aligned",) + message_instance("sha256-block-aligned", msg))
    return out


def serve_mix(seed: int = 4, count: int = 64, max_blocks: int = 512):
    """Serving requests: half sha256-2kb (2 KiB random message), half
    sha256-block-aligned with k = floor(2^U(0, log2 max_blocks)) blocks,
    clipped to 1..max_blocks. Kind and length come from the SplitMix64 stream
    of ``seed``, message bytes from the stream of ``seed + 1000003``."""
    import math
    draws = _u64s(seed, 2 * count)
    kinds, lengths = [], []
    for i in range(count):
        if draws[2 * i] & 1:
            kinds.append("sha256-2kb")
            lengths.append(32)
        else:
            u = (draws[2 * i + 1] >> 11) / float(1 << 53) * math.log2(max_blocks)
            kinds.append("sha256-block-aligned")
            lengths.append(min(max(int(2.0 ** u), 1), max_blocks))
    data = splitmix64_bytes(seed + 1000003, 64 * sum(lengths))
    out, pos = [], 0
    for kind, k in zip(kinds, lengths):
        msg = data[pos:pos + 64 * k]
        pos += 64 * k
        out.append((kind,) + message_instance(kind, msg))
    return out
