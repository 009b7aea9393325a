"""Finds channel digests whose lowest proof-of-work nonce at 33 and 34 bits is small, for tests of
the grind above 32 bits (where a nonce must zero more than the first hash word).

The grind (src/core/channel/blake2s.zig:135-240) returns the lowest nonce whose
Blake2s(prefix || LE64 nonce) has n_bits trailing zero bits in its first 16 bytes, with
prefix = Blake2s(LE32 0x12345678 || 0^12 || digest || LE32 n_bits). At 33 bits the lowest nonce of
a random digest lies near 2^33, far beyond what the CPU oracle can confirm in a test; this script
grinds the digests sha256(b"pow<bits>-<i>") on the GPU (the library's own grind) and keeps those
whose lowest nonce is below 2^27, which the oracle confirms by scanning every smaller nonce.

Usage (on a machine with the GPU): python tests/golden/make_pow_vectors.py OUT.json
Writes [{"digest": hex, "n_bits": b, "nonce": n}, ...] (two digests per bit count).
"""
from __future__ import annotations

import hashlib
import json
import os
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "stwo-zig_b200"))

LIMIT = 1 << 27
PER_BITS = 2


def prefix_of(digest: bytes, n_bits: int) -> bytes:
    return hashlib.blake2s(struct.pack("<I", 0x12345678) + b"\0" * 12 + digest + struct.pack("<I", n_bits)).digest()


def main(out_path: str) -> None:
    import stwo_b200 as sb
    ctx = sb.Context(0)
    vectors = []
    for n_bits in (33, 34):
        kept, i = 0, 0
        while kept < PER_BITS:
            digest = hashlib.sha256(f"pow{n_bits}-{i}".encode()).digest()
            nonce = ctx.pow_grind(prefix_of(digest, n_bits), n_bits)
            if nonce < LIMIT:
                vectors.append({"digest": digest.hex(), "n_bits": n_bits, "nonce": nonce})
                kept += 1
            i += 1
        print(f"{n_bits} bits: {i} digests ground", flush=True)
    ctx.close()
    with open(out_path, "w") as f:
        json.dump(vectors, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
