"""Wide-Fibonacci composition evaluation (stwo_b200_wide_fib_composition) against a numpy
evaluation of the constraint sum: out_i[row] = (sum_k coeffs[k]_i * (c_k - a_k^2 - b_k^2)) *
den[row >> log_n] mod p for each QM31 coordinate i (src/examples/wide_fibonacci/component.zig:
138-236), on the two-row vectorised kernel (8-byte aligned columns) and the scalar one (an
unaligned base), small and wide traces, two calls in a row. Integer results: compared exactly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _expected(cols, coeffs, den0, den1, log_n):
    c = cols.astype(np.uint64)
    rows = c.shape[1]
    acc = np.zeros((4, rows), dtype=np.uint64)
    sq = (c * c) % P
    for k in range(c.shape[0] - 2):
        cons = (c[k + 2] + 2 * P - sq[k] - sq[k + 1]) % P
        for i in range(4):
            acc[i] = (acc[i] + int(coeffs[k, i]) * cons) % P
    den = np.where(np.arange(rows) >> log_n, den1, den0).astype(np.uint64)
    return ((acc * den) % P).astype(np.uint32)


@pytest.mark.parametrize("log_n,W,offset", [(9, 100, 0), (10, 17, 0), (9, 3, 0), (10, 1002, 0), (8, 100, 0),
                                            (9, 33, 1), (9, 1010, 0)])
def test_composition_matches_numpy(ctx, log_n, W, offset):
    import torch
    rng = np.random.default_rng(1000 * log_n + W + offset)
    rows = 2 << log_n
    for call in range(2):  # two calls in a row on the same context
        cols = rng.integers(0, P, size=(W, rows), dtype=np.uint32)
        coeffs = rng.integers(0, P, size=(W - 2, 4), dtype=np.uint32)
        den0, den1 = (int(x) for x in rng.integers(1, P, size=2))
        flat = np.zeros(W * rows + offset, dtype=np.uint32)
        flat[offset:] = cols.reshape(-1)
        dev = torch.from_numpy(flat.view(np.int32)).cuda()[offset:]
        dco = torch.from_numpy(coeffs.reshape(-1).view(np.int32)).cuda()
        out = torch.full((4 * rows,), -1, dtype=torch.int32, device="cuda")
        ctx.wide_fib_composition(dev, log_n, W, dco, den0, den1, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.uint32).reshape(4, rows)
        np.testing.assert_array_equal(got, _expected(cols, coeffs, den0, den1, log_n), err_msg=f"call {call}")
