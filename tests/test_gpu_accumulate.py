"""Lifted accumulation of secure columns (stwo_b200_accumulate): the accumulate hook and the
DomainEvaluationAccumulator's accumulateColumn + finalize (src/prover/air/accumulation.zig:256-347).
The reference's own case "lifted combination matches direct formula" (accumulation.zig:379-430) is
the known answer; random cases are checked against Python QM31 arithmetic. Exact integers."""
import numpy as np
import pytest

import verifier as vf

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _cols(values):
    """Secure values -> 4 coordinate columns, flattened (column-major)."""
    return np.array([[vf.qflat(v)[k] for v in values] for k in range(4)], dtype=np.uint32).reshape(-1)


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def _read(t, n):
    out = t.cpu().numpy().view(np.uint32).reshape(4, n)
    return [vf.qfrom([int(out[k][i]) for k in range(4)]) for i in range(n)]


def test_reference_lifted_combination(ctx):
    import torch
    alpha = vf.q(3)
    large = [vf.q(v) for v in range(1, 9)]
    small = [vf.q(v) for v in (10, 20, 30, 40)]
    dst = torch.zeros(4 * 8, dtype=torch.int32, device="cuda")
    ctx.accumulate(dst, 3, _dev(_cols(large)), 3, vf.qflat(alpha))  # alpha^(2-1) for the first column
    ctx.accumulate(dst, 3, _dev(_cols(small)), 2)                    # alpha^0 for the second
    got = _read(dst, 8)
    for pos in range(8):
        idx_small = ((pos >> 2) << 1) + (pos & 1)
        assert got[pos] == vf.qadd(vf.qmul(large[pos], alpha), small[idx_small])


@pytest.mark.parametrize("dst_log,src_log", [(10, 7), (6, 6), (12, 1), (9, 8)])
def test_accumulate_matches_python(ctx, dst_log, src_log):
    rng = np.random.default_rng(100 * dst_log + src_log)
    n, m = 1 << dst_log, 1 << src_log
    d0 = [vf.qfrom([int(x) for x in rng.integers(0, P, 4)]) for _ in range(n)]
    sv = [vf.qfrom([int(x) for x in rng.integers(0, P, 4)]) for _ in range(m)]
    coeff = vf.qfrom([int(x) for x in rng.integers(0, P, 4)])
    dst = _dev(_cols(d0))
    ctx.accumulate(dst, dst_log, _dev(_cols(sv)), src_log, vf.qflat(coeff))
    got = _read(dst, n)
    sh = dst_log - src_log + 1
    for i in range(n):
        j = i if src_log == dst_log else ((i >> sh) << 1) + (i & 1)
        assert got[i] == vf.qadd(d0[i], vf.qmul(coeff, sv[j])), i


def test_accumulate_rejects_larger_source(ctx):
    import stwo_b200
    import torch
    a = torch.zeros(4 * 16, dtype=torch.int32, device="cuda")
    with pytest.raises(stwo_b200.StwoError) as e:
        ctx.accumulate(a, 3, a, 4)
    assert e.value.status == stwo_b200.E_INVALID
