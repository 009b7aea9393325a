"""The DEEP quotient op's launch variants, above all the bulk-staged kernel (the fourth): a CTA streams
512-row chunks of its columns into a shared-memory ring with 1-D bulk async copies completing on
mbarriers. Proofs through it equal the oracle's bytes (one batch of 24 to 1008 entries, entry counts
that are not a multiple of the 8-column group, the XOR-lookup AIR's several batches), the op agrees
with the register kernels, and its bounded waits, made to run out by a test hook (a stage whose
copies are never issued), end the proof or the op with an error while the context stays usable.
No GPU fault is involved: the hook only leaves a barrier phase incomplete."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
P = 2**31 - 1
STAGED = 3


def _cfg(preset, **over):
    import stwo_b200 as sb
    c = oracle.config(preset, **over)
    return c, sb.PcsConfig(c.pow_bits, sb.FriConfig(c.log_blowup_factor, c.log_last_layer_degree_bound, c.n_queries))


@pytest.fixture
def staged():
    import stwo_b200 as sb
    sb.autotune_mode(STAGED)
    yield
    sb.autotune_mode(-1)


@pytest.mark.parametrize("log_n,width,preset", [
    (15, 16, "functional"), (16, 21, "functional"), (17, 100, "functional"), (15, 1000, "functional"),
    (16, 9, "secure")])
def test_wide_fib_proofs_through_the_staged_kernel_equal_the_oracle(ctx, staged, log_n, width, preset):
    import stwo_b200 as sb
    o, g = _cfg(preset)
    seed = 31 * log_n + width
    got = ctx.prove_wide_fibonacci(sb.Statement(log_n, width), g, trace_kind=sb.TRACE_SEEDED, trace_seed=seed)
    assert got == oracle.prove_wide_fib(log_n, width, o, trace_kind=1, trace_seed=seed)


@pytest.mark.parametrize("log_n,log_table", [(16, 16), (18, 8)])
def test_xor_proofs_through_the_staged_kernel_equal_the_oracle(ctx, staged, log_n, log_table):
    o, g = _cfg("functional")
    seed, chan = 500 + log_n, 7 * log_table
    assert ctx.prove_logup_xor(log_n, g, seed=seed, log_table=log_table, channel_seed=chan) == \
        oracle.prove_logup_xor(log_n, o, seed=seed, log_table=log_table, channel_seed=chan)


@pytest.mark.parametrize("variant", [1, 2])
def test_xor_proofs_through_the_other_quotient_variants_equal_the_oracle(ctx, variant):
    """The XOR-lookup AIR's quotients come in several batches: the register variants with 3 and 9
    loads in flight against the oracle's bytes."""
    import stwo_b200 as sb
    o, g = _cfg("functional")
    try:
        sb.autotune_mode(variant)
        got = ctx.prove_logup_xor(16, g, seed=77, log_table=16, channel_seed=5)
    finally:
        sb.autotune_mode(-1)
    assert got == oracle.prove_logup_xor(16, o, seed=77, log_table=16, channel_seed=5)


def _quotient_case(n_cols, log):
    import torch
    rng = np.random.default_rng(4000 + n_cols)
    cols = torch.from_numpy(rng.integers(0, P, size=(n_cols, 1 << log), dtype=np.uint32).view(np.int32)).cuda()
    ptrs = torch.tensor([cols.data_ptr() + 4 * c * (1 << log) for c in range(n_cols)], dtype=torch.int64,
                        device="cuda")
    coeffs = torch.from_numpy(rng.integers(0, P, size=(n_cols * 4,), dtype=np.uint32).view(np.int32)).cuda()
    pt = [[int(x) for x in rng.integers(0, P, size=4)] for _ in range(4)]
    return cols, ptrs, coeffs, pt


@pytest.mark.parametrize("n_cols", [1, 8, 13, 108])
def test_quotient_op_variants_equal_the_register_kernel(ctx, n_cols):
    """Every quotient variant writes the first variant's words at the op level."""
    import stwo_b200 as sb
    import torch
    log = 17
    cols, ptrs, coeffs, (px, py, sa, sbb) = _quotient_case(n_cols, log)
    outs = []
    try:
        for v in (0, 1, 2, STAGED):
            sb.autotune_mode(v)
            out = torch.empty(4 << log, dtype=torch.int32, device="cuda")
            ctx.accumulate_quotients(log, ptrs, coeffs, px, py, sa, sbb, out, n_cols)
            torch.cuda.synchronize()
            outs.append(out.cpu().numpy())
    finally:
        sb.autotune_mode(-1)
    for o in outs[1:]:
        assert np.array_equal(outs[0], o)
    del cols


def test_staged_wait_that_runs_out_fails_the_proof_and_the_context_stays_usable(ctx, staged):
    import stwo_b200 as sb
    o, g = _cfg("functional")
    st = sb.Statement(16, 12)
    sb.arm_quotient_stage_timeout_for_testing()
    with pytest.raises(sb.StwoError) as ei:
        ctx.prove_wide_fibonacci(st, g, trace_kind=sb.TRACE_SEEDED, trace_seed=3)
    assert ei.value.status == sb.E_CUDA and "ran out of time" in str(ei.value)
    got = ctx.prove_wide_fibonacci(st, g, trace_kind=sb.TRACE_SEEDED, trace_seed=3)
    assert got == oracle.prove_wide_fib(16, 12, o, trace_kind=1, trace_seed=3)


def test_staged_wait_that_runs_out_fails_the_op(ctx, staged):
    import stwo_b200 as sb
    import torch
    log, n_cols = 16, 10
    cols, ptrs, coeffs, (px, py, sa, sbb) = _quotient_case(n_cols, log)
    out = torch.empty(4 << log, dtype=torch.int32, device="cuda")
    sb.arm_quotient_stage_timeout_for_testing()
    with pytest.raises(sb.StwoError) as ei:
        ctx.accumulate_quotients(log, ptrs, coeffs, px, py, sa, sbb, out, n_cols)
    assert "ran out of time" in str(ei.value)
    ctx.accumulate_quotients(log, ptrs, coeffs, px, py, sa, sbb, out, n_cols)
    torch.cuda.synchronize()
    del cols
