"""End-to-end proofs on the GPU, byte-for-byte against the oracle and the reference's stored proofs."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
import verifier

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
STORED = json.load(open(os.path.join(GOLDEN, "stored_proofs.json")))
KATS = json.load(open(os.path.join(GOLDEN, "kats.json")))


def cfg_pair(preset, **over):
    import stwo_b200 as sb
    c = oracle.config(preset, **over)
    return c, sb.PcsConfig(c.pow_bits, sb.FriConfig(c.log_blowup_factor, c.log_last_layer_degree_bound, c.n_queries))


def test_kat_5x8(ctx):
    import stwo_b200 as sb
    _, g = cfg_pair("smoke")
    p = ctx.prove_wide_fibonacci(sb.Statement(5, 8), g)
    assert len(p) == KATS["wf_5x8_proof"]["len"]
    assert hashlib.sha256(p).hexdigest() == KATS["wf_5x8_proof"]["sha256"]


@pytest.mark.parametrize("entry", STORED, ids=lambda e: f"{e['log_n_rows']}x{e['sequence_len']}")
def test_stored_functional_proofs(ctx, entry):
    import stwo_b200 as sb
    g = sb.PcsConfig(entry["pow_bits"], sb.FriConfig(entry["log_blowup_factor"], entry["log_last_layer_degree_bound"],
                                                     entry["n_queries"]))
    p = ctx.prove_wide_fibonacci(sb.Statement(entry["log_n_rows"], entry["sequence_len"]), g)
    assert len(p) == entry["len"]
    assert hashlib.sha256(p).hexdigest() == entry["sha256"]


@pytest.mark.parametrize("log_n,W,preset", [(1, 2, "smoke"), (2, 3, "smoke"), (3, 4, "functional"),
                                            (6, 17, "functional"), (11, 16, "functional"), (12, 100, "secure"),
                                            (13, 33, "functional")])
def test_seeded_proofs_match_oracle(ctx, log_n, W, preset):
    import stwo_b200 as sb
    o, g = cfg_pair(preset)
    ref = oracle.prove_wide_fib(log_n, W, o, trace_kind=1, trace_seed=99 + log_n)
    got = ctx.prove_wide_fibonacci(sb.Statement(log_n, W), g, trace_kind=sb.TRACE_SEEDED, trace_seed=99 + log_n)
    assert got == ref


def test_host_and_device_traces(ctx):
    import stwo_b200 as sb
    import torch
    o, g = cfg_pair("functional")
    trace = oracle.gen_trace(10, 20, trace_kind=1, seed=5)
    ref = oracle.prove_wide_fib(10, 20, o, trace=trace)
    assert ctx.prove_wide_fibonacci(sb.Statement(10, 20), g, trace=trace) == ref
    dtrace = torch.from_numpy(trace.view(np.int32)).cuda()
    assert ctx.prove_wide_fibonacci(sb.Statement(10, 20), g, trace=dtrace) == ref


def _recurrence_trace(first_two, W):
    P = 2**31 - 1
    full = np.empty((W, first_two.shape[1]), dtype=np.uint32)
    full[:2] = first_two
    for k in range(2, W):
        a, b = full[k - 2].astype(np.uint64), full[k - 1].astype(np.uint64)
        full[k] = ((a * a + b * b) % P).astype(np.uint32)
    return full


def test_first_two_columns_source(ctx):
    """TRACE_FIRST_COLUMNS: only col0/col1 are given (host or device); the device derives the rest."""
    import stwo_b200 as sb
    import torch
    o, g = cfg_pair("functional")
    rng = np.random.default_rng(8)
    two = rng.integers(0, 2**31 - 1, size=(2, 1 << 11), dtype=np.uint32)  # arbitrary canonical values
    full = _recurrence_trace(two, 24)
    ref = oracle.prove_wide_fib(11, 24, o, trace=full)
    st = sb.Statement(11, 24)
    assert ctx.prove_wide_fibonacci(st, g, trace=two, trace_kind=sb.TRACE_FIRST_COLUMNS) == ref
    dtwo = torch.from_numpy(two.view(np.int32)).cuda()
    assert ctx.prove_wide_fibonacci(st, g, trace=dtwo, trace_kind=sb.TRACE_FIRST_COLUMNS) == ref
    # In place: the kernel fills columns 2.. from the two already in the buffer.
    out = torch.zeros(24 << 11, dtype=torch.int32, device="cuda")
    out[: 2 << 11] = dtwo.reshape(-1)
    ctx.wide_fib_trace(out, 11, 24, sb.TRACE_FIRST_COLUMNS)
    assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(24, -1), full)
    # The seeded source and its own first two columns prove the same statement identically.
    o2, g2 = cfg_pair("secure")
    seeded = oracle.gen_trace(12, 100, trace_kind=1, seed=41)
    want = ctx.prove_wide_fibonacci(sb.Statement(12, 100), g2, trace_kind=sb.TRACE_SEEDED, trace_seed=41)
    got = ctx.prove_wide_fibonacci(sb.Statement(12, 100), g2, trace=np.ascontiguousarray(seeded[:2]),
                                   trace_kind=sb.TRACE_FIRST_COLUMNS)
    assert got == want
    for bad in (dict(trace_kind=sb.TRACE_FIRST_COLUMNS), dict(trace_kind=3, trace_seed=1)):
        with pytest.raises(sb.StwoError) as e:
            ctx.prove_wide_fibonacci(st, g, **bad)
        assert e.value.status == sb.E_INVALID


def test_channel_seed_and_blowup(ctx):
    import stwo_b200 as sb
    o, g = cfg_pair("functional", log_blowup_factor=2, n_queries=5, log_last_layer_degree_bound=1)
    ref = oracle.prove_wide_fib(9, 10, o, trace_kind=1, trace_seed=3, channel_seed=77)
    got = ctx.prove_wide_fibonacci(sb.Statement(9, 10), g, trace_kind=1, trace_seed=3, channel_seed=77)
    assert got == ref
    assert got != ctx.prove_wide_fibonacci(sb.Statement(9, 10), g, trace_kind=1, trace_seed=3, channel_seed=78)


def test_corrupted_trace_fails_closed(ctx):
    import stwo_b200 as sb
    _, g = cfg_pair("smoke")
    t = oracle.gen_trace(6, 8, 0)
    t[4, 11] ^= 3
    with pytest.raises(sb.StwoError) as e:
        ctx.prove_wide_fibonacci(sb.Statement(6, 8), g, trace=t)
    assert e.value.status == sb.E_CONSTRAINTS


def test_batch_matches_single(ctx):
    import stwo_b200 as sb
    _, g = cfg_pair("functional")
    reqs = [dict(statement=sb.Statement(8 + (i % 4), 8 + 3 * i), config=g, trace_kind=1, trace_seed=i,
                 channel_seed=1000 + i) for i in range(8)]
    batch = ctx.prove_wide_fibonacci_batch(reqs, max_in_flight=4)
    for r, p in zip(reqs, batch):
        single = ctx.prove_wide_fibonacci(r["statement"], g, trace_kind=1, trace_seed=r["trace_seed"],
                                          channel_seed=r["channel_seed"])
        assert p == single


def test_repeat_determinism(ctx):
    import stwo_b200 as sb
    _, g = cfg_pair("functional")
    a = ctx.prove_wide_fibonacci(sb.Statement(14, 32), g, trace_kind=1, trace_seed=1)
    b = ctx.prove_wide_fibonacci(sb.Statement(14, 32), g, trace_kind=1, trace_seed=1)
    assert a == b


@pytest.mark.parametrize("log_n,W,preset", [(12, 100, "secure"), (16, 64, "functional")])
def test_gpu_proofs_verify(ctx, log_n, W, preset):
    import stwo_b200 as sb
    _, g = cfg_pair(preset)
    p = ctx.prove_wide_fibonacci(sb.Statement(log_n, W), g, trace_kind=sb.TRACE_SEEDED, trace_seed=42,
                                 channel_seed=9)
    assert verifier.verify_wide_fib(p, log_n, W, channel_seed=9)
    assert sb.verify_wide_fibonacci(p, log_n, W, channel_seed=9)  # the library's own verifier


def mixed_requests(master_seed=2026, count=48):
    """48 wide-Fibonacci statements: log_n_rows uniform in 14..20, sequence_len in {16, 32, 100},
    each with its own trace seed and channel seed, all drawn from one master seed."""
    import stwo_b200 as sb
    rng = np.random.default_rng(master_seed)
    _, g = cfg_pair("secure")
    reqs = []
    for i in range(count):
        reqs.append(dict(statement=sb.Statement(int(rng.integers(14, 21)), int(rng.choice([16, 32, 100]))),
                         config=g, trace_kind=sb.TRACE_SEEDED, trace_seed=int(rng.integers(1, 2**63)),
                         channel_seed=int(rng.integers(0, 2**63))))
    return reqs


def test_mixed_batch_of_48_matches_single_runs(ctx):
    reqs = mixed_requests()
    batch = ctx.prove_wide_fibonacci_batch(reqs, max_in_flight=8)
    for r, p in zip(reqs, batch):
        single = ctx.prove_wide_fibonacci(r["statement"], r["config"], trace_kind=r["trace_kind"],
                                          trace_seed=r["trace_seed"], channel_seed=r["channel_seed"])
        assert p == single
    # A few of them independently verified.
    for r, p in list(zip(reqs, batch))[:3]:
        assert verifier.verify_wide_fib(p, r["statement"].log_n_rows, r["statement"].sequence_len,
                                        channel_seed=r["channel_seed"])


@pytest.mark.parametrize("log_n,W,over", [
    (4, 2, dict(log_blowup_factor=1, n_queries=3)),                                   # minimum width
    (7, 9, dict(log_blowup_factor=3, n_queries=9, log_last_layer_degree_bound=2)),   # blowup 8
    (8, 5, dict(log_blowup_factor=4, n_queries=4, log_last_layer_degree_bound=0)),   # blowup 16
    (10, 12, dict(n_queries=120, log_last_layer_degree_bound=3)),                     # many queries
    (9, 3, dict(pow_bits=14, n_queries=2))])
def test_protocol_variants_match_oracle(ctx, log_n, W, over):
    import stwo_b200 as sb
    o, g = cfg_pair("functional", **over)
    ref = oracle.prove_wide_fib(log_n, W, o, trace_kind=1, trace_seed=31 * log_n + W, channel_seed=0)
    got = ctx.prove_wide_fibonacci(sb.Statement(log_n, W), g, trace_kind=sb.TRACE_SEEDED,
                                   trace_seed=31 * log_n + W, channel_seed=0)
    assert got == ref
    assert sb.verify_wide_fibonacci(got, log_n, W, channel_seed=0)


def test_widest_statement_matches_oracle(ctx):
    """sequence_len 1000, the widest statement the prover takes (1008 quotient columns against the
    quotient kernel's 1024 entries); one column more is refused."""
    import stwo_b200 as sb
    o, g = cfg_pair("functional")
    ref = oracle.prove_wide_fib(6, 1000, o, trace_kind=1, trace_seed=1000)
    got = ctx.prove_wide_fibonacci(sb.Statement(6, 1000), g, trace_kind=sb.TRACE_SEEDED, trace_seed=1000)
    assert got == ref
    assert sb.verify_wide_fibonacci(got, 6, 1000)
    with pytest.raises(sb.StwoError) as e:
        ctx.prove_wide_fibonacci(sb.Statement(6, 1001), g, trace_kind=sb.TRACE_SEEDED, trace_seed=1)
    assert e.value.status == sb.E_INVALID


def test_largest_domain_matches_oracle(ctx):
    """log_n_rows 22, the largest the prover takes (LDE of 2^23 rows); 23 is refused."""
    import stwo_b200 as sb
    o, g = cfg_pair("functional")
    ref = oracle.prove_wide_fib(22, 16, o, trace_kind=1, trace_seed=22)
    got = ctx.prove_wide_fibonacci(sb.Statement(22, 16), g, trace_kind=sb.TRACE_SEEDED, trace_seed=22)
    assert got == ref
    with pytest.raises(sb.StwoError) as e:
        ctx.prove_wide_fibonacci(sb.Statement(23, 16), g, trace_kind=sb.TRACE_SEEDED, trace_seed=1)
    assert e.value.status == sb.E_INVALID


def test_headline_shape_secure_matches_oracle_and_verifies(ctx):
    """The benchmark's statement, 2^20 x 100 under the secure preset (PoW 26 bits, 70 queries),
    byte-for-byte against the oracle, then through the Python and the library verifiers."""
    import stwo_b200 as sb
    o, g = cfg_pair("secure")
    ref = oracle.prove_wide_fib(20, 100, o, trace_kind=1, trace_seed=2020, channel_seed=7)
    got = ctx.prove_wide_fibonacci(sb.Statement(20, 100), g, trace_kind=sb.TRACE_SEEDED, trace_seed=2020,
                                   channel_seed=7)
    assert got == ref
    assert verifier.verify_wide_fib(got, 20, 100, channel_seed=7)
    assert sb.verify_wide_fibonacci(got, 20, 100, channel_seed=7)
