"""The library's C++ verifier on the CPU (it uses no device): pinned on the reference's stored
proof, agreeing with the Python verifier, and rejecting tampering."""
import json
import os
import sys

import pytest

import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
STORED = json.load(open(os.path.join(GOLDEN, "stored_proofs.json")))


def _sb():
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "stwo-zig_b200"))
    import stwo_b200
    return stwo_b200


def test_accepts_the_reference_stored_proof():
    sb = _sb()
    entry = next(e for e in STORED if "proof_hex" in e)
    assert sb.verify_wide_fibonacci(bytes.fromhex(entry["proof_hex"]), entry["log_n_rows"], entry["sequence_len"])


@pytest.mark.parametrize("preset,log_n,W,over,seed", [
    ("smoke", 5, 8, {}, None), ("secure", 8, 20, {}, 5), ("functional", 3, 4, {}, None),
    ("functional", 9, 10, dict(log_blowup_factor=2, n_queries=5, log_last_layer_degree_bound=1), 77)])
def test_accepts_oracle_proofs(preset, log_n, W, over, seed):
    sb = _sb()
    p = oracle.prove_wide_fib(log_n, W, oracle.config(preset, **over), trace_kind=1, trace_seed=11, channel_seed=seed)
    assert sb.verify_wide_fibonacci(p, log_n, W, channel_seed=seed)
    with pytest.raises(sb.StwoError) as e:
        sb.verify_wide_fibonacci(p, log_n, W, channel_seed=(seed or 0) + 1)
    assert e.value.status == sb.E_CONSTRAINTS
    with pytest.raises(sb.StwoError):
        sb.verify_wide_fibonacci(p, log_n, W + 1, channel_seed=seed)


@pytest.mark.parametrize("path", [
    ("queried_values", 1, 3, 0), ("queried_values", 2, 7, 1), ("decommitments", 1, "hash_witness", 2, 5),
    ("sampled_values", 1, 4, 0, 2), ("fri_proof", "first_layer", "fri_witness", 0, 1),
    ("fri_proof", "inner_layers", 2, "decommitment", "hash_witness", 0, 0), ("fri_proof", "last_layer_poly", 0, 0),
    ("commitments", 1, 0), ("proof_of_work",)])
def test_rejects_tampering(path):
    sb = _sb()
    entry = next(e for e in STORED if "proof_hex" in e)
    d = json.loads(bytes.fromhex(entry["proof_hex"]))
    node = d
    for k in path[:-1]:
        node = node[k]
    node[path[-1]] = (node[path[-1]] + 1) % (256 if path[0] in ("commitments", "decommitments") or
                                             "hash_witness" in path else 2**31 - 1)
    with pytest.raises(sb.StwoError) as e:
        sb.verify_wide_fibonacci(json.dumps(d, separators=(",", ":")).encode(), entry["log_n_rows"],
                                 entry["sequence_len"])
    assert e.value.status == sb.E_CONSTRAINTS


@pytest.mark.parametrize("bad", [b"", b"{", b"[1,2", b'{"config": 5}', b"null", b"9" * 40])
def test_rejects_malformed_input(bad):
    sb = _sb()
    with pytest.raises(sb.StwoError) as e:
        sb.verify_wide_fibonacci(bad, 5, 8)
    assert e.value.status == sb.E_CONSTRAINTS


@pytest.mark.parametrize("log_n,W,over", [
    (4, 2, dict(n_queries=3)), (7, 9, dict(log_blowup_factor=3, n_queries=9, log_last_layer_degree_bound=2)),
    (8, 5, dict(log_blowup_factor=4, n_queries=4)), (10, 12, dict(n_queries=120, log_last_layer_degree_bound=3)),
    (9, 3, dict(pow_bits=14, n_queries=2))])
def test_protocol_variants_verify_in_both_verifiers(log_n, W, over):
    import verifier
    sb = _sb()
    p = oracle.prove_wide_fib(log_n, W, oracle.config("functional", **over), trace_kind=1, trace_seed=31 * log_n + W,
                              channel_seed=0)
    assert verifier.verify_wide_fib(p, log_n, W, channel_seed=0)
    assert sb.verify_wide_fibonacci(p, log_n, W, channel_seed=0)
