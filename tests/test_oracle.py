"""Pins the CPU oracle to the reference's known answers and stored proofs (no GPU)."""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

import oracle
import verifier

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
KATS = json.load(open(os.path.join(GOLDEN, "kats.json")))
STORED = json.load(open(os.path.join(GOLDEN, "stored_proofs.json")))


def test_blake2s_merkle_kats():
    # src/core/vcs_lifted/blake2_merkle.zig:339-370
    assert oracle.merkle_root([]).hex() == KATS["prefixed_empty_leaf"]
    node = b"node" + b"\0" * 60
    assert oracle.blake2s(node + b"\x01" * 32 + b"\x02" * 32).hex() == KATS["prefixed_parent_01_02"]
    assert oracle.blake2s(struct.pack("<3I", 1, 2, 3)).hex() == KATS["plain_leaf_1_2_3"]
    assert oracle.blake2s(b"\x01" * 32 + b"\x02" * 32).hex() == KATS["plain_parent_01_02"]
    assert oracle.blake2s(b"abc") == hashlib.blake2s(b"abc").digest()
    for n in (0, 1, 63, 64, 65, 128, 200):
        data = bytes(range(256))[:n]
        assert oracle.blake2s(data) == hashlib.blake2s(data).digest()


def test_wide_fib_5x16_commitments():
    # src/examples/wide_fibonacci/session_test.zig:75-96
    proof = json.loads(oracle.prove_wide_fib(5, 16, oracle.config("smoke")))
    assert [bytes(c).hex() for c in proof["commitments"]] == KATS["wf_5x16_commitments"]


def test_wide_fib_5x8_proof_kat():
    # src/examples/wide_fibonacci/session_test.zig:63-72
    p = oracle.prove_wide_fib(5, 8, oracle.config("smoke"))
    assert len(p) == KATS["wf_5x8_proof"]["len"]
    assert hashlib.sha256(p).hexdigest() == KATS["wf_5x8_proof"]["sha256"]


@pytest.mark.parametrize("entry", STORED, ids=lambda e: f"{e['log_n_rows']}x{e['sequence_len']}")
def test_stored_functional_proofs(entry):
    cfg = oracle.PcsConfig(entry["pow_bits"], entry["log_blowup_factor"], entry["log_last_layer_degree_bound"],
                           entry["n_queries"])
    p = oracle.prove_wide_fib(entry["log_n_rows"], entry["sequence_len"], cfg)
    assert len(p) == entry["len"]
    assert hashlib.sha256(p).hexdigest() == entry["sha256"]
    if "proof_hex" in entry:
        assert p == bytes.fromhex(entry["proof_hex"])


def test_fft_roundtrip_and_linearity():
    rng = np.random.default_rng(1)
    for log in (1, 2, 3, 5, 10):
        v = rng.integers(0, 2**31 - 1, size=1 << log, dtype=np.uint32)
        c = oracle.interpolate(v)
        assert np.array_equal(oracle.evaluate(c), v)
        w = rng.integers(0, 2**31 - 1, size=1 << log, dtype=np.uint32)
        s = ((v.astype(np.uint64) + w) % (2**31 - 1)).astype(np.uint32)
        cs = ((oracle.interpolate(v).astype(np.uint64) + oracle.interpolate(w)) % (2**31 - 1)).astype(np.uint32)
        assert np.array_equal(oracle.interpolate(s), cs)


def test_extension_agrees_with_evaluation():
    # The blown-up evaluation of a low-degree column restricted back interpolates to
    # the same coefficients zero-padded.
    rng = np.random.default_rng(2)
    c = rng.integers(0, 2**31 - 1, size=1 << 6, dtype=np.uint32)
    e = oracle.extend(c, 1)
    back = oracle.interpolate(e)
    assert np.array_equal(back[: c.size], c) and not back[c.size:].any()


POW_VECTORS = json.load(open(os.path.join(GOLDEN, "pow_vectors.json")))


@pytest.mark.parametrize("vec", POW_VECTORS, ids=lambda v: f"{v['n_bits']}bits-{v['digest'][:8]}")
def test_pow_vectors_above_32_bits(vec):
    """The fixture's lowest nonces at 33 and 34 bits (made on the GPU by
    tests/golden/make_pow_vectors.py), confirmed by the oracle scanning every smaller nonce."""
    assert oracle.pow_grind(bytes.fromhex(vec["digest"]), vec["n_bits"]) == vec["nonce"]


def test_pow_grind_is_lowest_valid_nonce():
    digest = bytes(range(32))
    nonce = oracle.pow_grind(digest, 8, 4)
    prefix = oracle.blake2s(struct.pack("<I", 0x12345678) + b"\0" * 12 + digest + struct.pack("<I", 8))

    def ok(n):
        h = oracle.blake2s(prefix + struct.pack("<Q", n))
        v = int.from_bytes(h[:16], "little")
        return v & 0xFF == 0

    assert ok(nonce)
    assert not any(ok(n) for n in range(nonce))


def test_seeded_trace_recurrence():
    t = oracle.gen_trace(6, 10, trace_kind=1, seed=7).astype(np.uint64)
    p = 2**31 - 1
    assert (t[:2] < p - 1).all()
    for k in range(2, 10):
        assert np.array_equal(t[k], (t[k - 2] ** 2 + t[k - 1] ** 2) % p)
    assert not np.array_equal(oracle.gen_trace(6, 10, 1, 7), oracle.gen_trace(6, 10, 1, 8))


def test_corrupted_trace_is_rejected():
    # src/examples/wide_fibonacci.zig:651-678: corrupting one cell fails the OODS self-check.
    t = oracle.gen_trace(5, 8, 0)
    t[3, 5] ^= 1
    with pytest.raises(RuntimeError):
        oracle.prove_wide_fib(5, 8, oracle.config("smoke"), trace=t)


def test_verifier_accepts_stored_reference_proof():
    # The reference's own 2^10 x 8 functional proof, bytes from its benchmark bundle.
    entry = next(e for e in STORED if "proof_hex" in e)
    assert verifier.verify_wide_fib(bytes.fromhex(entry["proof_hex"]), entry["log_n_rows"], entry["sequence_len"])


@pytest.mark.parametrize("preset,log_n,W,over", [("smoke", 5, 8, {}), ("secure", 8, 20, {}),
                                                 ("functional", 9, 10, dict(log_blowup_factor=2, n_queries=5,
                                                                            log_last_layer_degree_bound=1))])
def test_verifier_accepts_oracle_proofs(preset, log_n, W, over):
    p = oracle.prove_wide_fib(log_n, W, oracle.config(preset, **over), trace_kind=1, trace_seed=11, channel_seed=5)
    assert verifier.verify_wide_fib(p, log_n, W, channel_seed=5)
    with pytest.raises(verifier.VerificationError):
        verifier.verify_wide_fib(p, log_n, W, channel_seed=6)


@pytest.mark.parametrize("path", [
    ("queried_values", 1, 3, 0), ("queried_values", 2, 7, 1), ("decommitments", 1, "hash_witness", 2, 5),
    ("sampled_values", 1, 4, 0, 2), ("fri_proof", "first_layer", "fri_witness", 0, 1),
    ("fri_proof", "inner_layers", 2, "decommitment", "hash_witness", 0, 0), ("fri_proof", "last_layer_poly", 0, 0),
    ("commitments", 1, 0), ("proof_of_work",)])
def test_verifier_rejects_tampering(path):
    entry = next(e for e in STORED if "proof_hex" in e)
    good = bytes.fromhex(entry["proof_hex"])
    d = json.loads(good)
    node = d
    for k in path[:-1]:
        node = node[k]
    node[path[-1]] = (node[path[-1]] + 1) % (256 if path[0] in ("commitments", "decommitments") or
                                             "hash_witness" in path else 2**31 - 1)
    bad = json.dumps(d, separators=(",", ":")).encode()
    with pytest.raises(verifier.VerificationError):
        verifier.verify_wide_fib(bad, entry["log_n_rows"], entry["sequence_len"])


def _py_inverse(x):
    return verifier.qinv(x)


def test_batch_inverse_oracle():
    rng = np.random.default_rng(3)
    for degree in (1, 2, 4):
        for n in (1, 2, 7, 64):
            v = rng.integers(1, 2**31 - 1, size=(degree, n), dtype=np.uint32)
            got = oracle.batch_inverse(v[0] if degree == 1 else v)
            got = got.reshape(degree, n)
            for i in range(n):
                x = verifier.q(*[int(v[k, i]) for k in range(degree)])
                assert verifier.qflat(verifier.qinv(x))[:degree] == [int(got[k, i]) for k in range(degree)]
    with pytest.raises(oracle.DivisionByZero):
        oracle.batch_inverse(np.array([5, 0, 7], dtype=np.uint32))


def test_logup_scan_law_of_the_reference():
    # src/tests/metal/backend/commitment_test.zig:73-154: 256 rows, one use (11, row + 1),
    # alphas (3, 5), z = 7; fraction = 1 / (3*11 + 5*(row+1) - 7); shift = total / 256; scan in
    # coset order (scan index s -> circle index s/2 or 255 - s/2, stored at its bit reverse).
    rows, log = 256, 8
    col = np.arange(1, rows + 1, dtype=np.uint32)
    out, claimed = oracle.logup_interaction(log, [dict(words=[11, col])], [[3, 0, 0, 0], [5, 0, 0, 0]],
                                            [7, 0, 0, 0], batch=1, order=1)
    q = verifier.q
    fr = [verifier.qinv(verifier.qsub(verifier.qadd(verifier.qmulm(q(3), 11), verifier.qmulm(q(5), r + 1)), q(7)))
          for r in range(rows)]
    total = q(0)
    for f in fr:
        total = verifier.qadd(total, f)
    shift = verifier.qmulm(total, pow(rows, 2**31 - 3, 2**31 - 1))
    acc, expected = q(0), [None] * rows
    for s in range(rows):
        ci = s // 2 if s % 2 == 0 else rows - 1 - s // 2
        r = int(f"{ci:08b}"[::-1], 2)
        acc = verifier.qadd(acc, verifier.qsub(fr[r], shift))
        expected[r] = acc
    assert list(claimed) == verifier.qflat(total)
    for r in range(rows):
        assert [int(out[0, k, r]) for k in range(4)] == verifier.qflat(expected[r])


def test_logup_pairs_storage_order_law():
    # cumulativeColumn (src/frontends/riscv/air/logup.zig:83-105): per row
    # (n1 d2 + n2 d1) / (d1 d2), running sum in storage order, claimed = last value.
    rng = np.random.default_rng(4)
    log, rows = 5, 32
    a = rng.integers(0, 256, size=rows, dtype=np.uint32)
    b = rng.integers(0, 256, size=rows, dtype=np.uint32)
    m = rng.integers(0, 9, size=rows, dtype=np.uint32)
    alphas = [[1, 0, 0, 0], [12345, 6, 7, 8], [99, 1, 2, 3]]
    z = [1000003, 5, 11, 2]
    uses = [dict(words=[a, b]), dict(words=[4, a, b], multiplicity=m, negate=True)]
    out, claimed = oracle.logup_interaction(log, uses, alphas, z, batch=2, order=0)
    Q = [verifier.q(*x) for x in alphas]
    zq = verifier.q(*z)

    def den(ws, r):
        acc = verifier.qsub(verifier.q(0), zq)
        for j, w in enumerate(ws):
            acc = verifier.qadd(acc, verifier.qmulm(Q[j], w if isinstance(w, int) else int(w[r])))
        return acc
    acc = verifier.q(0)
    for r in range(rows):
        d1, d2 = den([a, b], r), den([4, a, b], r)
        n1, n2 = 1, (2**31 - 1 - int(m[r])) % (2**31 - 1)
        num = verifier.qadd(verifier.qmulm(d2, n1), verifier.qmulm(d1, n2))
        acc = verifier.qadd(acc, verifier.qmul(num, verifier.qinv(verifier.qmul(d1, d2))))
        assert [int(out[0, k, r]) for k in range(4)] == verifier.qflat(acc)
    assert list(claimed) == verifier.qflat(acc)


def test_logup_zero_denominator():
    col = np.arange(16, dtype=np.uint32)
    with pytest.raises(oracle.DivisionByZero):
        oracle.logup_interaction(4, [dict(words=[col])], [[1, 0, 0, 0]], [5, 0, 0, 0])


def test_xor_lookup_logup_sums_cancel():
    # LogUp identity of the XOR lookup: sum over trace rows of 1/(z - f(a, b, a^b)) equals the sum
    # over table rows of m/(z - f(row)), i.e. the two claimed sums add to zero.
    main, table, mult = oracle.xor_lookup_trace(10, 3)
    assert int(mult.sum()) == 1 << 10
    alphas = [[1, 0, 0, 0], [77, 1, 2, 3], [5, 9, 11, 13]]
    z = [123456, 7, 8, 9]
    _, c_main = oracle.logup_interaction(10, [dict(words=list(main))], alphas, z, batch=1, order=1)
    _, c_table = oracle.logup_interaction(16, [dict(words=list(table), multiplicity=mult, negate=True)], alphas, z,
                                          batch=1, order=1)
    total = verifier.qadd(verifier.qfrom([int(x) for x in c_main]), verifier.qfrom([int(x) for x in c_table]))
    assert total == verifier.q(0)
