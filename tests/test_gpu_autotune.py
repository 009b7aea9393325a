"""The launch-shape autotuner: every variant of every tuned op writes the oracle's bits (each forced
in turn), and a key's first call in tuning mode records a timing of each variant and keeps the
fastest."""
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


def _cfg(preset):
    import stwo_b200 as sb
    c = oracle.config(preset)
    return c, sb.PcsConfig(c.pow_bits, sb.FriConfig(c.log_blowup_factor, c.log_last_layer_degree_bound, c.n_queries))


@pytest.fixture
def forced():
    import stwo_b200 as sb
    yield sb.autotune_mode
    sb.autotune_mode(-1)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_every_variant_is_exact(ctx, forced, variant):
    import torch
    forced(variant)
    rng = np.random.default_rng(60 + variant)
    # interpolate + blow-up-2 extension (op 0) at 2^17 and 2^20
    for log in (17, 20):
        cols = rng.integers(0, P, size=(3, 1 << log), dtype=np.uint32)
        ev = _dev(cols)
        coeffs = torch.empty_like(ev)
        lde = torch.empty(3 << (log + 1), dtype=torch.int32, device="cuda")
        ctx.interpolate_and_extend(ev, coeffs, lde, log, 1, 3)
        co, le = _host(coeffs).reshape(3, -1), _host(lde).reshape(3, -1)
        for c in range(3):
            ref = oracle.interpolate(cols[c])
            assert np.array_equal(co[c], ref) and np.array_equal(le[c], oracle.extend(ref, 1)), (log, c)
    # Merkle leaves (op 1): 2^16 rows x 37 columns
    cols = rng.integers(0, P, size=(37, 1 << 16), dtype=np.uint32)
    layers = torch.empty(((2 << 16) - 1) * 32, dtype=torch.uint8, device="cuda")
    assert ctx.merkle_commit(_dev(cols), 16, 37, layers) == oracle.merkle_root(list(cols))
    # DEEP quotients (op 2) inside a proof whose lifting domain is 2^17
    o, g = _cfg("functional")
    import stwo_b200 as sb
    got = ctx.prove_wide_fibonacci(sb.Statement(16, 24), g, trace_kind=sb.TRACE_SEEDED, trace_seed=70 + variant)
    assert got == oracle.prove_wide_fib(16, 24, o, trace_kind=1, trace_seed=70 + variant)


def test_tuning_records_each_variant_and_keeps_the_fastest(ctx, forced):
    import stwo_b200 as sb
    import torch
    forced(-1)
    rng = np.random.default_rng(77)
    log, n = 18, 5  # a shape no other test tunes
    cols = rng.integers(0, P, size=(n, 1 << log), dtype=np.uint32)
    ev = _dev(cols)
    coeffs = torch.empty_like(ev)
    lde = torch.empty(n << (log + 1), dtype=torch.int32, device="cuda")
    for _ in range(2):  # the first call tunes, the second runs the chosen variant
        ctx.interpolate_and_extend(ev, coeffs, lde, log, 1, n)
        le = _host(lde).reshape(n, -1)
        assert np.array_equal(le[2], oracle.extend(oracle.interpolate(cols[2]), 1))
    entries = [e for e in sb.autotune_table() if e["log_size"] == log and e["n_cols"] == n and
               e["op"] == sb.AUTOTUNE_OPS[0]]
    assert len(entries) == 1
    e = entries[0]
    assert e["ms"][0] > 0 and e["ms"][1] > 0
    assert e["ms"][e["variant"]] == min(e["ms"][:2])
