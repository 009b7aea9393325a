"""Regenerates the golden fixtures in tests/golden/ from the stwo-zig reference tree.

Reads (as data) the proof artifacts the reference stores under
vectors/reports/benchmark_history/runs/*/bundle/tree/row-*-wide_fibonacci-*/cpu.proof-artifact.json
and the known-answer values in the reference's tests, and writes:

  stored_proofs.json   per stored wide-Fibonacci proof: statement, PCS config, byte length and
                       SHA-256 of the JSON wire bytes (plus the full bytes for the 2^10 x 8 proof)
  kats.json            Blake2s / Merkle / proof known answers quoted in the reference's tests

Usage: python tests/golden/make_golden.py /path/to/stwo-zig
"""
from __future__ import annotations

import glob
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root: str) -> None:
    runs = os.path.join(ref_root, "vectors/reports/benchmark_history/runs")
    pattern = os.path.join(runs, "*", "bundle/tree/row-*-wide_fibonacci-*/cpu.proof-artifact.json")
    seen = {}
    for path in sorted(glob.glob(pattern)):
        art = json.load(open(path))
        if art.get("example") != "wide_fibonacci":
            continue
        st = art["wide_fibonacci_statement"]
        pc = art["pcs_config"]
        raw = bytes.fromhex(art["proof_bytes_hex"])
        key = (st["log_n_rows"], st["sequence_len"], pc["pow_bits"], pc["fri_config"]["n_queries"])
        entry = {
            "log_n_rows": st["log_n_rows"],
            "sequence_len": st["sequence_len"],
            "pow_bits": pc["pow_bits"],
            "log_blowup_factor": pc["fri_config"]["log_blowup_factor"],
            "log_last_layer_degree_bound": pc["fri_config"]["log_last_layer_degree_bound"],
            "n_queries": pc["fri_config"]["n_queries"],
            "len": len(raw),
            "sha256": hashlib.sha256(raw).hexdigest(),
            "source": os.path.relpath(path, ref_root),
        }
        if key in seen:
            # Stored runs at different commits must agree byte-for-byte.
            assert seen[key]["sha256"] == entry["sha256"], (seen[key], entry)
            continue
        if st["log_n_rows"] == 10 and st["sequence_len"] == 8:
            entry["proof_hex"] = raw.hex()
        seen[key] = entry
    proofs = sorted(seen.values(), key=lambda e: (e["log_n_rows"], e["sequence_len"]))
    with open(os.path.join(HERE, "stored_proofs.json"), "w") as f:
        json.dump(proofs, f, indent=1)
        f.write("\n")

    kats = {
        # src/core/vcs_lifted/blake2_merkle.zig:339-370
        "prefixed_empty_leaf": "2a133e150238721921d1ea772882979c810f85f2849099b9d3415a8619d85fad",
        "prefixed_parent_01_02": "24c36247c66cc7b145aee79ccff9d5e3e596a8e13e86d13942f61464364fa53c",
        "plain_leaf_1_2_3": "9549ce18083a73c794b0fe338635a4ab0950333ecb2e3f1945adf7db5f0ef4d0",
        "plain_parent_01_02": "280569932378c99f448df37e893f062fab951bea53515634b7875ae51e1954e7",
        # src/examples/wide_fibonacci/session_test.zig:75-96 (2^5 x 16, pow 0, FRI(0,1,3))
        "wf_5x16_commitments": [
            "2a133e150238721921d1ea772882979c810f85f2849099b9d3415a8619d85fad",
            "dfc402b1c9be2a0b32d61bc810f24190b5e549d5d86c41ac2b1b8d01063aeaeb",
            "ee5df2e32512551d63a489914903324afccee9670125e3f8783ce19f495854a2",
        ],
        # src/examples/wide_fibonacci/session_test.zig:63-72 (2^5 x 8, pow 0, FRI(0,1,3))
        "wf_5x8_proof": {"len": 8912,
                          "sha256": "2c90684b49387804fd51bef3e286201e4b0b43a96b42200a7b6812a5a11e317d"},
        # src/core/air/accumulation.zig:30-48 (recurrence of 100 evaluations, alpha (2,3,4,5))
        "point_accumulator_alpha_2345": [475135206, 878218281, 117218720, 1587643918],
    }
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats, f, indent=1)
        f.write("\n")
    print(f"wrote {len(proofs)} stored proofs")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
