"""Seven-word quadratic-recurrence traces (stwo_b200_quadratic_recurrence_trace, the
fillQuadraticRecurrenceTrace hook and its recipe ABI, src/examples/wide_fibonacci/trace.zig:13-16):
for logical row k (coset order, stored bit-reversed), col0 = r0 + r1 k, col1 = r2 + r3 k,
col_j = r4 col_{j-2}^2 + r5 col_{j-1}^2 + r6 in M31. The wide-Fibonacci recipe must give the
reference trace (the generator the stored reference proofs pin); random recipes are checked against
numpy. Exact integers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _logical_rows(log_n):
    n = 1 << log_n
    s = np.arange(n, dtype=np.uint64)
    ci = np.zeros(n, dtype=np.uint64)
    for b in range(log_n):
        ci |= ((s >> np.uint64(b)) & np.uint64(1)) << np.uint64(log_n - 1 - b)
    return np.where(ci < n // 2, 2 * ci, 2 * (n - 1 - ci) + 1)


def _expected(log_n, W, r):
    r = [int(x) % P for x in r]
    k = _logical_rows(log_n)
    a = (r[0] + r[1] * k) % P
    b = (r[2] + r[3] * k) % P
    out = [a, b]
    for _ in range(2, W):
        c = (r[4] * (a * a % P) + r[5] * (b * b % P) + r[6]) % P
        out.append(c)
        a, b = b, c
    return np.stack(out).astype(np.uint32)


def test_wide_fibonacci_recipe_is_the_reference_trace(ctx):
    import stwo_b200 as sb
    import torch
    for log_n, W in ((5, 8), (12, 100), (16, 33)):
        a = torch.empty(W << log_n, dtype=torch.int32, device="cuda")
        b = torch.empty_like(a)
        ctx.quadratic_recurrence_trace(a, log_n, W, (1, 0, 0, 1, 1, 1, 0))
        ctx.wide_fib_trace(b, log_n, W, sb.TRACE_REFERENCE)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
        assert np.array_equal(a.cpu().numpy().view(np.uint32).reshape(W, -1), _expected(log_n, W, (1, 0, 0, 1, 1, 1, 0)))


@pytest.mark.parametrize("log_n,W", [(1, 2), (6, 9), (13, 40)])
def test_random_recipes_match_numpy(ctx, log_n, W):
    import torch
    rng = np.random.default_rng(17 * log_n + W)
    for _ in range(3):
        recipe = [int(x) for x in rng.integers(0, 2**32, size=7, dtype=np.uint64)]  # words >= p reduce mod p
        out = torch.full((W << log_n,), -1, dtype=torch.int32, device="cuda")
        ctx.quadratic_recurrence_trace(out, log_n, W, recipe)
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(W, -1), _expected(log_n, W, recipe))


def test_bad_arguments(ctx):
    import stwo_b200 as sb
    import torch
    out = torch.zeros(64, dtype=torch.int32, device="cuda")
    for log_n, W in ((5, 1), (0, 4)):
        with pytest.raises(sb.StwoError) as e:
            ctx.quadratic_recurrence_trace(out, log_n, W, (1, 0, 0, 1, 1, 1, 0))
        assert e.value.status == sb.E_INVALID
