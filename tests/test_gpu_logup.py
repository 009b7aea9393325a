"""Batch inversion and LogUp interaction columns on the GPU, bit-exact against the oracle."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def _host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("degree", [1, 2, 4])
@pytest.mark.parametrize("n", [1, 5, 255, 4096, 4099, 1 << 20])
def test_batch_inverse_matches_oracle(ctx, degree, n):
    rng = np.random.default_rng(n * 7 + degree)
    v = rng.integers(1, P, size=(degree, n), dtype=np.uint32)
    v[0, :: 3] = rng.integers(1, 4, size=v[0, ::3].shape, dtype=np.uint32)  # small values too
    ref = oracle.batch_inverse(v[0] if degree == 1 else v).reshape(degree, n)
    src = _dev(v)
    dst = _dev(np.zeros_like(v))
    ctx.batch_inverse(src, dst, n, degree)
    assert np.array_equal(_host(dst).reshape(degree, n), ref)
    ctx.batch_inverse(src, src, n, degree)  # in place
    assert np.array_equal(_host(src).reshape(degree, n), ref)


def test_batch_inverse_strided_and_zero(ctx):
    import stwo_b200 as sb
    n, stride = 1000, 1024
    rng = np.random.default_rng(9)
    buf = rng.integers(1, P, size=4 * stride, dtype=np.uint32)
    planes = np.stack([buf[k * stride:k * stride + n] for k in range(4)])
    ref = oracle.batch_inverse(planes)
    src = _dev(buf)
    out = _dev(np.zeros(4 * stride, dtype=np.uint32))
    ctx.batch_inverse(src, out, n, 4, src_stride=stride, dst_stride=stride)
    got = _host(out)
    assert np.array_equal(np.stack([got[k * stride:k * stride + n] for k in range(4)]), ref)
    buf[3 * stride + 17] = 0
    buf[17] = 0
    buf[stride + 17] = 0
    buf[2 * stride + 17] = 0
    with pytest.raises(sb.StwoError) as e:
        ctx.batch_inverse(_dev(buf), out, n, 4, src_stride=stride, dst_stride=stride)
    assert e.value.status == sb.E_DIVISION_BY_ZERO


def _run_both(ctx, log_rows, uses_host, alphas, z, batch, order):
    import torch
    ref, ref_claimed = oracle.logup_interaction(log_rows, uses_host, alphas, z, batch=batch, order=order)
    dev_uses = []
    for d in uses_host:
        dev_uses.append(dict(words=[w if isinstance(w, int) else _dev(w) for w in d["words"]],
                             multiplicity=None if d.get("multiplicity") is None else _dev(d["multiplicity"]),
                             negate=d.get("negate", False)))
    n_cols = (len(uses_host) + batch - 1) // batch
    out = torch.zeros(n_cols * 4 << log_rows, dtype=torch.int32, device="cuda")
    claimed = ctx.logup_interaction(log_rows, dev_uses, alphas, z, out, batch=batch, order=order)
    return ref, ref_claimed, _host(out).reshape(n_cols, 4, 1 << log_rows), np.array(claimed, dtype=np.uint32)


def test_logup_reference_scan_case(ctx):
    # The case of src/tests/metal/backend/commitment_test.zig:73-154.
    col = np.arange(1, 257, dtype=np.uint32)
    ref, rc, got, gc = _run_both(ctx, 8, [dict(words=[11, col])], [[3, 0, 0, 0], [5, 0, 0, 0]], [7, 0, 0, 0], 1, 1)
    assert np.array_equal(got, ref) and np.array_equal(gc, rc)


@pytest.mark.parametrize("log_rows", [0, 1, 2, 5, 10, 11, 12, 16, 20])
@pytest.mark.parametrize("batch,order", [(1, 1), (2, 1), (2, 0), (1, 0)])
def test_logup_matches_oracle(ctx, log_rows, batch, order):
    rng = np.random.default_rng(100 * log_rows + 10 * batch + order)
    rows = 1 << log_rows
    a = rng.integers(0, 256, size=rows, dtype=np.uint32)
    b = rng.integers(0, 256, size=rows, dtype=np.uint32)
    c = a ^ b
    mult = rng.integers(0, 1 << 20, size=rows, dtype=np.uint32)
    alphas = [rng.integers(0, P, size=4).tolist() for _ in range(4)]
    z = rng.integers(0, P, size=4).tolist()
    uses = [dict(words=[7, a, b, c]),                                 # lookup of (a, b, a^b), multiplicity 1
            dict(words=[7, b, a, c], multiplicity=mult, negate=True),  # table side, -multiplicity
            dict(words=[3, a]),
            dict(words=[c], multiplicity=mult),
            dict(words=[9, b, 1])]
    ref, rc, got, gc = _run_both(ctx, log_rows, uses, alphas, z, batch, order)
    assert np.array_equal(got, ref)
    assert np.array_equal(gc, rc)


def test_logup_zero_denominator_and_bad_args(ctx):
    import stwo_b200 as sb
    import torch
    col = _dev(np.arange(16, dtype=np.uint32))
    out = torch.zeros(4 * 16, dtype=torch.int32, device="cuda")
    with pytest.raises(sb.StwoError) as e:
        ctx.logup_interaction(4, [dict(words=[col])], [[1, 0, 0, 0]], [5, 0, 0, 0], out)
    assert e.value.status == sb.E_DIVISION_BY_ZERO
    with pytest.raises(sb.StwoError) as e:
        ctx.logup_interaction(4, [dict(words=[col])], [[1, 0, 0, 0]], [5, 0, 0, 0], out, batch=3)
    assert e.value.status == sb.E_INVALID
    with pytest.raises(sb.StwoError) as e:
        ctx.logup_interaction(4, [dict(words=[1] * 9)], [[1, 0, 0, 0]] * 9, [5, 0, 0, 0], out)
    assert e.value.status == sb.E_INVALID


@pytest.mark.parametrize("log_n", [12, 16, 20])
def test_xor_lookup_interaction(ctx, log_n):
    """The XOR-lookup AIR's interaction phase at serving shapes: trace and multiplicities, LogUp
    columns of both components, their lifted commitment; the claimed sums cancel, and everything
    equals the oracle (all of it at 2^12, the trace and multiplicities at every size)."""
    import torch
    seed = 1000 + log_n
    rows = 1 << log_n
    main = torch.empty(3 * rows, dtype=torch.int32, device="cuda")
    table = torch.empty(3 * 65536, dtype=torch.int32, device="cuda")
    mult = torch.empty(65536, dtype=torch.int32, device="cuda")
    ctx.xor_lookup_trace(log_n, seed, main, table, mult)
    o_main, o_table, o_mult = oracle.xor_lookup_trace(log_n, seed)
    assert np.array_equal(_host(main).reshape(3, rows), o_main)
    assert np.array_equal(_host(table).reshape(3, 65536), o_table)
    assert np.array_equal(_host(mult), o_mult)
    rng = np.random.default_rng(log_n)
    alphas = [rng.integers(0, P, size=4).tolist() for _ in range(3)]
    z = rng.integers(0, P, size=4).tolist()
    inter_main = torch.empty(4 * rows, dtype=torch.int32, device="cuda")
    inter_table = torch.empty(4 * 65536, dtype=torch.int32, device="cuda")
    c_main = ctx.logup_interaction(log_n, [dict(words=[main[k * rows:(k + 1) * rows] for k in range(3)])], alphas, z,
                                   inter_main)
    c_table = ctx.logup_interaction(16, [dict(words=[table[k * 65536:(k + 1) * 65536] for k in range(3)],
                                              multiplicity=mult, negate=True)], alphas, z, inter_table)
    import verifier
    assert verifier.qadd(verifier.qfrom(list(c_main)), verifier.qfrom(list(c_table))) == verifier.q(0)
    cols = [inter_main[k * rows:(k + 1) * rows] for k in range(4)] + \
           [inter_table[k * 65536:(k + 1) * 65536] for k in range(4)]
    max_log = max(log_n, 16)
    layers = torch.empty(((2 << max_log) - 1) * 32, dtype=torch.uint8, device="cuda")
    root = ctx.merkle_commit_lifted(cols, layers)
    if log_n == 12:
        ref_m, _ = oracle.logup_interaction(log_n, [dict(words=list(o_main))], alphas, z)
        ref_t, _ = oracle.logup_interaction(16, [dict(words=list(o_table), multiplicity=o_mult, negate=True)], alphas, z)
        assert np.array_equal(_host(inter_main).reshape(1, 4, rows), ref_m)
        assert np.array_equal(_host(inter_table).reshape(1, 4, 65536), ref_t)
        assert root == oracle.merkle_root([*ref_m[0], *ref_t[0]])
