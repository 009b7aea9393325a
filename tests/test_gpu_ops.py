"""Op-level parity of the CUDA kernels (through the C ABI) against the CPU oracle."""
import json
import os
import struct

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


def rand_cols(rng, n_cols, log):
    return rng.integers(0, P, size=(n_cols, 1 << log), dtype=np.uint32)


@pytest.mark.parametrize("log", [1, 2, 3, 4, 7, 11, 12, 13, 15, 16, 17, 18, 19, 20, 21, 22])
def test_interpolate_evaluate(ctx, log):
    rng = np.random.default_rng(log)
    n_cols = 3
    cols = rand_cols(rng, n_cols, log)
    d = dev(cols)
    ctx.interpolate(d, log, n_cols, 1 << log)
    got = host(d).reshape(n_cols, -1)
    for c in range(n_cols):
        assert np.array_equal(got[c], oracle.interpolate(cols[c])), c
    ctx.evaluate(d, log, n_cols, 1 << log)
    assert np.array_equal(host(d).reshape(n_cols, -1), cols)


@pytest.mark.parametrize("log", [16, 20])
def test_interpolate_evaluate_padded_columns(ctx, log):
    """Columns `stride` words apart with a gap between them (the forward pass stores its blocks with
    a tensor copy whose map carries the stride): the transforms equal the oracle's and the gap words
    keep their values."""
    import torch
    rng = np.random.default_rng(900 + log)
    n_cols, pad = 3, 256
    stride = (1 << log) + pad
    cols = rand_cols(rng, n_cols, log)
    buf = np.full((n_cols, stride), 0x5A5A5A5A, dtype=np.uint32)
    buf[:, : 1 << log] = cols
    d = torch.from_numpy(buf.reshape(-1).view(np.int32)).cuda()
    ctx.interpolate(d, log, n_cols, stride)
    got = host(d).reshape(n_cols, stride)
    for c in range(n_cols):
        assert np.array_equal(got[c, : 1 << log], oracle.interpolate(cols[c])), c
    ctx.evaluate(d, log, n_cols, stride)
    got = host(d).reshape(n_cols, stride)
    assert np.array_equal(got[:, : 1 << log], cols)
    assert (got[:, 1 << log:] == 0x5A5A5A5A).all()


@pytest.mark.parametrize("log,blowup", [(1, 1), (3, 1), (10, 1), (11, 1), (12, 1), (15, 1), (16, 1), (17, 1),
                                        (18, 1), (19, 1), (20, 1), (21, 1), (22, 1), (12, 2), (16, 2), (18, 3),
                                        (5, 3)])
def test_interpolate_and_extend(ctx, log, blowup):
    import torch
    rng = np.random.default_rng(100 + log)
    n_cols = 4
    cols = rand_cols(rng, n_cols, log)
    ev = dev(cols)
    coeffs = torch.empty_like(ev)
    lde = torch.empty(n_cols << (log + blowup), dtype=torch.int32, device="cuda")
    ctx.interpolate_and_extend(ev, coeffs, lde, log, blowup, n_cols)
    co = host(coeffs).reshape(n_cols, -1)
    le = host(lde).reshape(n_cols, -1)
    for c in range(n_cols):
        ref_c = oracle.interpolate(cols[c])
        assert np.array_equal(co[c], ref_c), c
        assert np.array_equal(le[c], oracle.extend(ref_c, blowup)), c
    # the unmodified input
    assert np.array_equal(host(ev).reshape(n_cols, -1), cols)


@pytest.mark.parametrize("log,n_cols", [(0, 0), (1, 1), (4, 3), (8, 16), (9, 17), (12, 100), (17, 8)])
def test_merkle(ctx, log, n_cols):
    import torch
    rng = np.random.default_rng(7 + log + n_cols)
    cols = rand_cols(rng, max(n_cols, 1), log)[:n_cols]
    d = dev(cols if n_cols else np.zeros(1, np.uint32))
    layers = torch.empty(((2 << log) - 1) * 32, dtype=torch.uint8, device="cuda")
    root = ctx.merkle_commit(d, log, n_cols, layers)
    ref_layers = oracle.merkle_layers(list(cols))
    assert root == ref_layers[-1][0].tobytes()
    got = host(layers).view(np.uint8).reshape(-1, 32)
    at = 0
    for lay in ref_layers:
        assert np.array_equal(got[at:at + lay.shape[0]], lay)
        at += lay.shape[0]


@pytest.mark.parametrize("log", [2, 3, 5, 12, 21])
def test_fold_circle_into_line(ctx, log):
    import torch
    rng = np.random.default_rng(log)
    src = rand_cols(rng, 4, log)
    alpha = rng.integers(0, P, size=4, dtype=np.uint32)
    prev = rand_cols(rng, 4, log - 1)
    for acc in (False, True):
        dst = dev(prev)
        ctx.fold_circle_into_line(dev(src), dst, log, alpha, accumulate=acc)
        ref = oracle.fold_circle_into_line(src, alpha, prev if acc else None)
        assert np.array_equal(host(dst).reshape(4, -1), ref)


@pytest.mark.parametrize("log", [1, 2, 4, 11, 20])
def test_fold_line(ctx, log):
    import torch
    rng = np.random.default_rng(log + 50)
    src = rand_cols(rng, 4, log)
    alpha = rng.integers(0, P, size=4, dtype=np.uint32)
    dst = torch.empty(4 << (log - 1), dtype=torch.int32, device="cuda")
    ctx.fold_line(dev(src), dst, log, alpha)
    assert np.array_equal(host(dst).reshape(4, -1), oracle.fold_line(src, alpha, log))


@pytest.mark.parametrize("log,n_cols", [(0, 5), (1, 5), (3, 5), (12, 5), (13, 5), (20, 5), (22, 1), (16, 64)])
def test_eval_at_point(ctx, log, n_cols):
    """Chunk partials per column: 1 (small columns), 237 (5 columns of 2^20), 1024 (one column of
    2^22, the most), 16 (64 columns of 2^16): the warp-per-column partial sum at every shape."""
    import torch
    rng = np.random.default_rng(log + 9 + 100 * n_cols)
    cols = rand_cols(rng, n_cols, log)
    px = rng.integers(0, P, size=4, dtype=np.uint32)
    py = rng.integers(0, P, size=4, dtype=np.uint32)
    out = torch.empty(4 * n_cols, dtype=torch.int32, device="cuda")
    ctx.eval_at_point(dev(cols), log, n_cols, 1 << log, px, py, out)
    got = host(out).reshape(n_cols, 4)
    for c in range(n_cols):
        assert np.array_equal(got[c], oracle.eval_at_point(cols[c], px, py)), c


@pytest.mark.parametrize("kind", [0, 1])
def test_trace_generation(ctx, kind):
    import torch
    out = torch.empty(12 << 9, dtype=torch.int32, device="cuda")
    ctx.wide_fib_trace(out, 9, 12, kind, seed=1234)
    assert np.array_equal(host(out).reshape(12, -1), oracle.gen_trace(9, 12, kind, 1234))


@pytest.mark.parametrize("bits", [1, 8, 14])
def test_pow_grind(ctx, bits):
    digest = bytes((i * 37 + bits) & 0xFF for i in range(32))
    prefix = oracle.blake2s(struct.pack("<I", 0x12345678) + b"\0" * 12 + digest + struct.pack("<I", bits))
    assert ctx.pow_grind(prefix, bits) == oracle.pow_grind(digest, bits, 8)


def test_pow_grind_lowest_nonce_across_waves_and_rounds(ctx):
    """24-bit grinds: the lowest valid nonces fall in later CTA waves and later bounded rounds
    (a round is 16.97 M nonces on 148 SMs); the device must still return the lowest one."""
    found = []
    for i in range(6):
        digest = bytes((i * 29 + k * 11) & 0xFF for k in range(32))
        prefix = oracle.blake2s(struct.pack("<I", 0x12345678) + b"\0" * 12 + digest + struct.pack("<I", 24))
        got = ctx.pow_grind(prefix, 24)
        assert got == oracle.pow_grind(digest, 24), i
        found.append(got)
    assert max(found) > 4_300_000  # at least one beyond the first wave of CTAs


POW_VECTORS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "pow_vectors.json")))


@pytest.mark.parametrize("vec", POW_VECTORS, ids=lambda v: f"{v['n_bits']}bits-{v['digest'][:8]}")
def test_pow_grind_above_32_bits(ctx, vec):
    """More than 32 bits: a hit must also zero the second hash word (the 128-bit trailing-zero
    path). The fixture's nonces are the oracle's (tests/test_oracle.py pins them on the CPU)."""
    digest = bytes.fromhex(vec["digest"])
    prefix = oracle.blake2s(struct.pack("<I", 0x12345678) + b"\0" * 12 + digest + struct.pack("<I", vec["n_bits"]))
    assert ctx.pow_grind(prefix, vec["n_bits"]) == vec["nonce"]


def test_bad_arguments_raise(ctx):
    import stwo_b200
    import torch
    d = torch.zeros(16, dtype=torch.int32, device="cuda")
    with pytest.raises(stwo_b200.StwoError):
        ctx.interpolate(d, 40, 1, 16)
    with pytest.raises(stwo_b200.StwoError):
        ctx.fold_circle_into_line(d, d, 1, [1, 0, 0, 0])


@pytest.mark.parametrize("logs", [[3], [4, 2, 4, 1, 3], [10, 9, 10, 8, 9, 10, 7, 10, 8, 10, 9, 10, 6, 10, 9, 10, 8],
                                  [16] * 3 + [12] * 4 + [14] * 2, [20, 16, 16, 16], [1, 1, 2]])
def test_lifted_merkle_mixed_sizes(ctx, logs):
    # Mixed log sizes in one tree (the shape of src/tests/metal/backend/commitment_test.zig's
    # lifted-root case), including columns given out of size order.
    import torch
    rng = np.random.default_rng(sum(logs))
    cols = [rng.integers(0, 2**31 - 1, size=1 << lg, dtype=np.uint32) for lg in logs]
    dev = [torch.from_numpy(c.view(np.int32)).cuda() for c in cols]
    max_log = max(logs)
    layers = torch.empty(((2 << max_log) - 1) * 32, dtype=torch.uint8, device="cuda")
    root = ctx.merkle_commit_lifted(dev, layers)
    assert root == oracle.merkle_root(cols)
    ref_layers = oracle.merkle_layers(cols)
    torch.cuda.synchronize()
    got = layers.cpu().numpy()
    at = 0
    for lay in ref_layers:
        n = lay.shape[0]
        assert np.array_equal(got[at * 32:(at + n) * 32].reshape(n, 32), lay)
        at += n


def test_lifted_merkle_equals_uniform_commit(ctx):
    import torch
    rng = np.random.default_rng(77)
    cols = rng.integers(0, 2**31 - 1, size=(7, 1 << 12), dtype=np.uint32)
    dev = torch.from_numpy(cols.reshape(-1).view(np.int32)).cuda()
    layers_a = torch.empty(((2 << 12) - 1) * 32, dtype=torch.uint8, device="cuda")
    layers_b = torch.empty_like(layers_a)
    ra = ctx.merkle_commit(dev, 12, 7, layers_a)
    rb = ctx.merkle_commit_lifted([dev[i << 12:(i + 1) << 12] for i in range(7)], layers_b)
    assert ra == rb
    assert torch.equal(layers_a, layers_b)


def test_misaligned_pointers_are_refused(ctx):
    """The ABI refuses device pointers its kernels cannot read as vectors (Merkle layers: 16 bytes;
    FRI fold sources: 8 bytes and an even stride; OODS coefficients: 16 bytes) before any launch."""
    import stwo_b200 as sb
    import torch
    buf = torch.zeros(1 << 14, dtype=torch.int32, device="cuda")
    off = buf[1:]                                   # 4 bytes past an aligned base
    dst = torch.zeros(1 << 12, dtype=torch.int32, device="cuda")
    layers = torch.zeros(((2 << 10) - 1) * 32 + 64, dtype=torch.uint8, device="cuda")
    layers_off = layers[4:]
    alpha = [3, 0, 0, 0]
    calls = [
        lambda: ctx.merkle_commit(buf, 8, 4, layers_off),
        lambda: ctx.merkle_commit_lifted([buf[:256], buf[256:384]], layers_off),
        lambda: ctx.fold_circle_into_line(off, dst, 8, alpha),
        lambda: ctx.fold_line(off, dst, 8, alpha),
        lambda: ctx.fold_and_commit(buf, dst, 8, alpha, layers=layers_off),
        lambda: ctx.eval_at_point(off, 10, 2, 1 << 10, [1, 0, 0, 0], [2, 0, 0, 0], dst),
        lambda: ctx.eval_at_point_noalloc(off, 10, 2, 1 << 10, [1, 0, 0, 0], [2, 0, 0, 0], dst),
    ]
    for i, call in enumerate(calls):
        with pytest.raises(sb.StwoError) as e:
            call()
        assert e.value.status == sb.E_INVALID, i
    torch.cuda.synchronize()
    ctx.merkle_commit(buf, 8, 4, layers)  # the same call with aligned pointers still runs
