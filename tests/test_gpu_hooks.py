"""Fused backend hooks against the sequences of entry points they replace and against the oracle
directly (exact integers): stwo_b200_fold_and_commit (foldLineAndCommitNext, the first FRI layer's
fold and commit), stwo_b200_commit_columns (prepareAndCommitPolys) and
stwo_b200_interpolate_secure_composition (interpolateSecureComposition)."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
P = 2**31 - 1


def _rand(rng, n):
    import torch
    return torch.from_numpy(rng.integers(0, P, size=n, dtype=np.uint32).view(np.int32)).cuda()


@pytest.mark.parametrize("circle,src_log", [(True, 12), (False, 11), (True, 3), (False, 2), (True, 21)])
def test_fold_and_commit_equals_fold_then_commit(ctx, circle, src_log):
    import torch
    rng = np.random.default_rng(src_log + 100 * circle)
    src = _rand(rng, 4 << src_log)
    alpha = [int(x) for x in rng.integers(0, P, 4)]
    half = 1 << (src_log - 1)
    dst_a = torch.empty(4 * half, dtype=torch.int32, device="cuda")
    dst_b = torch.empty_like(dst_a)
    lay_a = torch.empty(((2 * half) - 1) * 32, dtype=torch.uint8, device="cuda")
    lay_b = torch.empty_like(lay_a)
    root_a = ctx.fold_and_commit(src, dst_a, src_log, alpha, layers=lay_a, circle=circle)
    if circle:
        ctx.fold_circle_into_line(src, dst_b, src_log, alpha)
    else:
        ctx.fold_line(src, dst_b, src_log, alpha)
    root_b = ctx.merkle_commit(dst_b, src_log - 1, 4, lay_b)
    torch.cuda.synchronize()
    assert torch.equal(dst_a, dst_b)
    assert torch.equal(lay_a, lay_b)
    assert root_a == root_b
    # the oracle: the fold, then the lifted tree of its 4 coordinate columns
    src_h = src.cpu().numpy().view(np.uint32).reshape(4, -1)
    want = oracle.fold_circle_into_line(src_h, alpha) if circle else oracle.fold_line(src_h, alpha, src_log)
    assert np.array_equal(dst_a.cpu().numpy().view(np.uint32).reshape(4, -1), want)
    assert root_a == oracle.merkle_root(list(want))
    dst_c = torch.empty_like(dst_a)
    assert ctx.fold_and_commit(src, dst_c, src_log, alpha, circle=circle) is None  # fold only
    torch.cuda.synchronize()
    assert torch.equal(dst_c, dst_b)


@pytest.mark.parametrize("log_size,log_blowup,n_cols", [(16, 1, 7), (12, 2, 3), (20, 1, 4)])
def test_commit_columns_equals_extend_then_commit(ctx, log_size, log_blowup, n_cols):
    import torch
    rng = np.random.default_rng(log_size * 10 + n_cols)
    ev = _rand(rng, n_cols << log_size)
    n, nl = 1 << log_size, 1 << (log_size + log_blowup)
    co_a, co_b = torch.empty(n_cols * n, dtype=torch.int32, device="cuda"), torch.empty(n_cols * n, dtype=torch.int32,
                                                                                       device="cuda")
    lde_a, lde_b = (torch.empty(n_cols * nl, dtype=torch.int32, device="cuda") for _ in range(2))
    lay_a, lay_b = (torch.empty((2 * nl - 1) * 32, dtype=torch.uint8, device="cuda") for _ in range(2))
    root_a = ctx.commit_columns(ev, co_a, lde_a, lay_a, log_size, log_blowup, n_cols)
    ctx.interpolate_and_extend(ev, co_b, lde_b, log_size, log_blowup, n_cols)
    root_b = ctx.merkle_commit(lde_b, log_size + log_blowup, n_cols, lay_b)
    torch.cuda.synchronize()
    assert torch.equal(co_a, co_b) and torch.equal(lde_a, lde_b) and torch.equal(lay_a, lay_b)
    assert root_a == root_b
    ev_h = ev.cpu().numpy().view(np.uint32).reshape(n_cols, -1)
    co_h = co_a.cpu().numpy().view(np.uint32).reshape(n_cols, -1)
    lde_h = lde_a.cpu().numpy().view(np.uint32).reshape(n_cols, -1)
    want_co = [oracle.interpolate(ev_h[c]) for c in range(n_cols)]
    want_lde = [oracle.extend(w, log_blowup) for w in want_co]
    for c in range(n_cols):
        assert np.array_equal(co_h[c], want_co[c]) and np.array_equal(lde_h[c], want_lde[c]), c
    assert root_a == oracle.merkle_root(want_lde)


@pytest.mark.parametrize("comp_log,log_blowup", [(21, 1), (13, 2), (17, 1)])
def test_interpolate_secure_composition_equals_its_steps(ctx, comp_log, log_blowup):
    import torch
    rng = np.random.default_rng(comp_log * 7 + log_blowup)
    evals = _rand(rng, 4 << comp_log)
    half = 1 << (comp_log - 1)
    nl = half << log_blowup
    comp_a = evals.clone()
    lde_a = torch.empty(8 * nl, dtype=torch.int32, device="cuda")
    ctx.interpolate_secure_composition(comp_a, comp_log, log_blowup, lde_a)
    comp_b = evals.clone()
    ctx.interpolate(comp_b, comp_log, 4, 1 << comp_log)
    lde_b = torch.empty(8 * nl, dtype=torch.int32, device="cuda")
    left = torch.stack([comp_b[c << comp_log:(c << comp_log) + half] for c in range(4)]).reshape(-1).contiguous()
    right = torch.stack([comp_b[(c << comp_log) + half:(c + 1) << comp_log] for c in range(4)]).reshape(-1).contiguous()
    ctx.extend(left, lde_b[: 4 * nl], comp_log - 1, log_blowup, 4)
    ctx.extend(right, lde_b[4 * nl:], comp_log - 1, log_blowup, 4)
    torch.cuda.synchronize()
    assert torch.equal(comp_a, comp_b)
    assert torch.equal(lde_a, lde_b)
    ev_h = evals.cpu().numpy().view(np.uint32).reshape(4, -1)
    co_h = comp_a.cpu().numpy().view(np.uint32).reshape(4, -1)
    lde_h = lde_a.cpu().numpy().view(np.uint32).reshape(8, -1)
    for c in range(4):
        want = oracle.interpolate(ev_h[c])
        assert np.array_equal(co_h[c], want), c
        assert np.array_equal(lde_h[c], oracle.extend(want[:half], log_blowup)), c
        assert np.array_equal(lde_h[4 + c], oracle.extend(want[half:], log_blowup)), c


def test_bad_arguments(ctx):
    import stwo_b200 as sb
    import torch
    a = torch.zeros(64, dtype=torch.int32, device="cuda")
    with pytest.raises(sb.StwoError) as e:
        ctx.fold_and_commit(a, a, 1, [1, 0, 0, 0])
    assert e.value.status == sb.E_INVALID
    with pytest.raises(sb.StwoError) as e:
        ctx.interpolate_secure_composition(a, 1, 1, a)
    assert e.value.status == sb.E_INVALID
