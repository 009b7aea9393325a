"""LogUp XOR-lookup AIR proofs on the GPU, checked by the independent verifier (the AIR has no
reference counterpart, so the verifier's transcript replay, LogUp cancellation, OODS constraint
check and PCS/FRI decommitment checks are the parity gate). The main and table components keep
their own sizes (2^log_n and 2^log_table rows) under the lifted PCS: cases cover the lookups
smaller than, equal to and larger than the table. Every proof is also compared byte for byte with
the oracle's own XOR-lookup prover, which shares no code with the GPU prover."""
import json

import pytest

import oracle
import verifier

pytestmark = pytest.mark.gpu


def _cfg(preset, **over):
    import stwo_b200 as sb
    c = oracle.config(preset, **over)
    return sb.PcsConfig(c.pow_bits, sb.FriConfig(c.log_blowup_factor, c.log_last_layer_degree_bound, c.n_queries))


@pytest.mark.parametrize("log_n,log_table,preset,over", [
    (1, 8, "smoke", {}), (6, 8, "smoke", {}), (9, 8, "functional", {}), (10, 8, "functional", {}),
    (8, 8, "functional", dict(log_blowup_factor=2, n_queries=5, log_last_layer_degree_bound=1)),
    (11, 8, "functional", dict(log_blowup_factor=2, n_queries=5, log_last_layer_degree_bound=1)),
    (5, 8, "functional", dict(log_blowup_factor=3, n_queries=4)),
    (12, 16, "secure", {}), (16, 16, "functional", {}), (18, 16, "secure", {})])
def test_xor_air_proof_verifies(ctx, log_n, log_table, preset, over):
    g = _cfg(preset, **over)
    p = ctx.prove_logup_xor(log_n, g, seed=7 + log_n, log_table=log_table, channel_seed=3)
    assert verifier.verify_logup_xor(p, log_n, log_table, channel_seed=3)
    with pytest.raises(verifier.VerificationError):
        verifier.verify_logup_xor(p, log_n, log_table, channel_seed=4)


_PRESETS = {"functional": ("functional", {}), "secure": ("secure", {}),
            "blowup2": ("functional", dict(log_blowup_factor=2, n_queries=5, log_last_layer_degree_bound=1))}


@pytest.mark.parametrize("preset", sorted(_PRESETS))
@pytest.mark.parametrize("log_table", [8, 16])
@pytest.mark.parametrize("log_n", [6, 12, 16, 20])
def test_xor_air_proof_equals_the_oracle(ctx, log_n, log_table, preset):
    """Byte for byte against the oracle's independent prover (oracle/oracle.cpp prove_logup_xor):
    lookups smaller than, equal to and larger than the table, three protocol variants."""
    name, over = _PRESETS[preset]
    o = oracle.config(name, **over)
    g = _cfg(name, **over)
    seed, chan = 1000 + log_n + log_table, 11 * log_n
    assert ctx.prove_logup_xor(log_n, g, seed=seed, log_table=log_table, channel_seed=chan) == \
        oracle.prove_logup_xor(log_n, o, seed=seed, log_table=log_table, channel_seed=chan)


def test_xor_air_full_size_and_determinism(ctx):
    g = _cfg("secure")
    a = ctx.prove_logup_xor(20, g, seed=99)
    assert verifier.verify_logup_xor(a, 20, 16)
    assert a == ctx.prove_logup_xor(20, g, seed=99)
    assert a != ctx.prove_logup_xor(20, g, seed=100)


@pytest.mark.parametrize("log_n", [12, 6])
@pytest.mark.parametrize("field", ["claimed", "sampled", "queried", "sampled_table", "queried_table",
                                   "preprocessed"])
def test_xor_air_tampering_rejected(ctx, field, log_n):
    # log_n 12 > log_table 8: the table component is the smaller, lifted one; log_n 6: the lookups are.
    p = ctx.prove_logup_xor(log_n, _cfg("functional"), seed=5, log_table=8)
    assert verifier.verify_logup_xor(p, log_n, 8)
    d = json.loads(p)
    if field == "claimed":
        d["claimed_sums"][0][0] = (d["claimed_sums"][0][0] + 1) % (2**31 - 1)
        d["claimed_sums"][1][0] = (d["claimed_sums"][1][0] - 1) % (2**31 - 1)  # still cancelling
    elif field == "sampled":
        d["sampled_values"][2][3][0][1] = (d["sampled_values"][2][3][0][1] + 1) % (2**31 - 1)
    elif field == "queried":
        d["queried_values"][1][2][0] ^= 1
    elif field == "sampled_table":  # S_T, previous row
        d["sampled_values"][2][5][0][2] = (d["sampled_values"][2][5][0][2] + 1) % (2**31 - 1)
    elif field == "queried_table":  # the multiplicity column m
        d["queried_values"][1][3][1] ^= 1
    else:  # the preprocessed table tree
        d["queried_values"][0][1][0] ^= 1
    with pytest.raises(verifier.VerificationError):
        verifier.verify_logup_xor(json.dumps(d, separators=(",", ":")).encode(), log_n, 8)


def test_xor_air_bad_arguments(ctx):
    import stwo_b200 as sb
    with pytest.raises(sb.StwoError) as e:
        ctx.prove_logup_xor(23, _cfg("smoke"), log_table=16)
    assert e.value.status == sb.E_INVALID
    with pytest.raises(sb.StwoError) as e:
        ctx.prove_logup_xor(10, _cfg("smoke"), log_table=12)
    assert e.value.status == sb.E_INVALID


def test_native_verifier_agrees_on_xor_proofs(ctx):
    import stwo_b200 as sb
    for log_n, lt, seed in ((7, 8, None), (14, 16, 12), (12, 8, 3), (16, 16, None)):
        p = ctx.prove_logup_xor(log_n, _cfg("functional"), seed=3, log_table=lt, channel_seed=seed)
        assert sb.verify_logup_xor(p, log_n, lt, channel_seed=seed)
        with pytest.raises(sb.StwoError):
            sb.verify_logup_xor(p, log_n, lt, channel_seed=(seed or 0) + 1)
        d = json.loads(p)
        d["sampled_values"][1][0][0][0] = (d["sampled_values"][1][0][0][0] + 1) % (2**31 - 1)
        with pytest.raises(sb.StwoError):
            sb.verify_logup_xor(json.dumps(d, separators=(",", ":")).encode(), log_n, lt, channel_seed=seed)
