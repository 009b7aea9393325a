"""The allocation-free OODS evaluation entry point (stwo_b200_eval_at_point_noalloc).

It exists for callers that cannot allocate device memory when they need the
value (a serving loop bound to an admitted memory budget, an embedder whose
arena owns all device memory, code where CUDA allocation calls are not
allowed); its partial sums live in a fixed device array inside the library.
The test calls it twice in a row through the C ABI, with different inputs, and
checks each result against stwo_b200_eval_at_point; the values are exact field
elements, so the comparison is equality. It also checks that a size beyond the
fixed scratch is refused. This file is collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def test_eval_at_point_noalloc_matches_allocating_entry_point(ctx):
    import stwo_b200
    import torch

    rng = np.random.default_rng(2024)
    for call, (log_size, n_cols) in enumerate([(18, 7), (13, 33)]):
        cols = rng.integers(0, P, size=(n_cols, 1 << log_size), dtype=np.uint32)
        dev = torch.from_numpy(cols.view(np.int32)).cuda()
        px = rng.integers(0, P, size=4, dtype=np.uint32)
        py = rng.integers(0, P, size=4, dtype=np.uint32)
        want = torch.zeros(4 * n_cols, dtype=torch.int32, device="cuda")
        got = torch.full((4 * n_cols,), -1, dtype=torch.int32, device="cuda")
        ctx.eval_at_point(dev, log_size, n_cols, 1 << log_size, px, py, want)
        ctx.eval_at_point_noalloc(dev, log_size, n_cols, 1 << log_size, px, py, got)
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}"
        assert int((got < 0).sum()) == 0

    # 2^(22-12) chunks x 65 columns = 66560 partial sums > 65536: refused, nothing launched.
    big = torch.zeros(1, dtype=torch.int32, device="cuda")
    with pytest.raises(stwo_b200.StwoError) as err:
        ctx.eval_at_point_noalloc(big, 22, 65, 1 << 22, [1, 0, 0, 0], [0, 0, 0, 0], big)
    assert err.value.status == stwo_b200.E_INVALID
