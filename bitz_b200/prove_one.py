"""Proves one synthetic statement a few times on the default lane and prints
the proof size and each proof's times: a small, fixed workload for timing a
single proof or capturing its kernels under a profiler.

    python -m bitz_b200.prove_one [--kind sha256-block-aligned] [--blocks 16]
                                  [--seed 77] [--security 100] [--proofs 2]

Messages come from the SplitMix64 stream of ``--seed`` (the bench's
generator). With a kernel profiler attached the library runs every sumcheck
round as its own launch by itself; BITZ_RESIDENT_ROUNDS=0 asks for the same
explicitly.
"""
import argparse
import json

from . import CircuitProofSystem, statements


def main():
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--kind", default="sha256-block-aligned",
                   choices=["sha256-block-aligned", "sha256-chain", "sha256-2kb"])
    p.add_argument("--blocks", type=int, default=16)
    p.add_argument("--seed", type=int, default=77)
    p.add_argument("--security", type=int, default=100, choices=[100, 128])
    p.add_argument("--proofs", type=int, default=2)
    a = p.parse_args()
    if a.kind == "sha256-chain":
        inputs, outputs, _ = statements.instance(a.kind, a.blocks, a.seed)
    else:
        blocks = 32 if a.kind == "sha256-2kb" else a.blocks
        msg = statements.splitmix64_bytes(a.seed, 64 * blocks)
        inputs, outputs = statements.message_instance(a.kind, msg)
    ps = CircuitProofSystem(a.kind, inputs, outputs, a.security)
    for i in range(a.proofs):
        proof, times = ps.prove()
        print(json.dumps({"proof": i, "bytes": len(proof), **times}), flush=True)


if __name__ == "__main__":
    main()
