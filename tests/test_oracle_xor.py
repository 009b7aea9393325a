"""The oracle's LogUp XOR-lookup AIR prover (oracle/oracle.cpp prove_logup_xor) on the CPU.

The AIR has no reference counterpart; the oracle builds its proof from the reference's pinned
pieces (the LogUp scan law of src/tests/metal/backend/commitment_test.zig:73-154, the lifted PCS,
FRI and wire layout that reproduce the reference's stored proofs). Its proofs must be accepted by
both independent verifiers (oracle/verifier.py and the library's host verifier) and rejected under a
different channel seed or a flipped byte; the GPU prover is then compared with it byte for byte
(tests/test_gpu_xor.py)."""
import os
import sys

import pytest

import oracle
import verifier

HERE = os.path.dirname(os.path.abspath(__file__))


def _sb():
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "stwo-zig_b200"))
    import stwo_b200
    return stwo_b200


@pytest.mark.parametrize("log_n,log_table,preset,over", [
    (1, 8, "smoke", {}), (6, 8, "functional", {}), (8, 8, "functional", {}), (11, 8, "functional", {}),
    (9, 8, "functional", dict(log_blowup_factor=2, n_queries=5, log_last_layer_degree_bound=1)),
    (4, 8, "functional", dict(log_blowup_factor=3, n_queries=4)), (12, 16, "functional", {}),
    (16, 16, "functional", {}), (17, 16, "smoke", {}),
    # 70 queries on a lifting domain 2^6 times the table's: preprocessed positions repeat and
    # leave sorted order, the witness still covers them sorted and unique
    (14, 8, "secure", {})])
def test_oracle_xor_proofs_verify(log_n, log_table, preset, over):
    cfg = oracle.config(preset, **over)
    p = oracle.prove_logup_xor(log_n, cfg, seed=40 + log_n, log_table=log_table, channel_seed=6)
    assert verifier.verify_logup_xor(p, log_n, log_table, channel_seed=6)
    assert _sb().verify_logup_xor(p, log_n, log_table, channel_seed=6)
    with pytest.raises(verifier.VerificationError):
        verifier.verify_logup_xor(p, log_n, log_table, channel_seed=7)


def test_oracle_xor_proof_is_deterministic_and_tamper_evident():
    cfg = oracle.config("functional")
    p = oracle.prove_logup_xor(10, cfg, seed=3, log_table=8)
    assert p == oracle.prove_logup_xor(10, cfg, seed=3, log_table=8)
    assert p != oracle.prove_logup_xor(10, cfg, seed=4, log_table=8)
    i = p.index(b'"claimed_sums":[[') + len(b'"claimed_sums":[[')
    bad = p[:i] + (b"1" if p[i:i + 1] != b"1" else b"2") + p[i + 1:]
    with pytest.raises(verifier.VerificationError):
        verifier.verify_logup_xor(bad, 10, 8)
