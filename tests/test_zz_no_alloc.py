"""The allocation-free OODS evaluation entry point (stwo_b200_eval_at_point_noalloc).

It exists for callers that cannot allocate device memory when they need the
value (a serving loop bound to an admitted memory budget, an embedder whose
arena owns all device memory, code where CUDA allocation calls are not
allowed); its partial sums live in a fixed device array inside the library.
The test calls it twice in a row through the C ABI, with different inputs, and
checks each result against stwo_b200_eval_at_point; the values are exact field
elements, so the comparison is equality. It also checks that a size beyond the
fixed scratch, or more columns than a grid row count, is refused, and that a
call takes nothing from the device's stream-ordered memory pool (where the
allocating entry point takes its scratch) or from torch's allocator. This file
is collected last.
"""
import ctypes

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
    # More columns than grid rows (65535): refused before any launch.
    with pytest.raises(stwo_b200.StwoError) as err:
        ctx.eval_at_point_noalloc(big, 1, 65536, 2, [1, 0, 0, 0], [0, 0, 0, 0], big)
    assert err.value.status == stwo_b200.E_INVALID


class _DefaultPool:
    """Usage counters of device 0's default stream-ordered memory pool (CUDA driver API)."""
    USED_MEM_CURRENT, USED_MEM_HIGH = 7, 8  # CU_MEMPOOL_ATTR_USED_MEM_CURRENT / _HIGH

    def __init__(self):
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int(0)
        assert self.cu.cuDeviceGet(ctypes.byref(dev), 0) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetDefaultMemPool(ctypes.byref(self.pool), dev) == 0

    def get(self, attr):
        v = ctypes.c_uint64(0)
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return v.value

    def reset_high(self):
        zero = ctypes.c_uint64(0)  # resets the high watermark to the current usage
        assert self.cu.cuMemPoolSetAttribute(self.pool, self.USED_MEM_HIGH, ctypes.byref(zero)) == 0


def test_eval_at_point_noalloc_takes_no_device_memory(ctx):
    import torch

    rng = np.random.default_rng(7)
    log_size, n_cols = 17, 9
    dev = torch.from_numpy(rng.integers(0, P, size=(n_cols, 1 << log_size), dtype=np.uint32).view(np.int32)).cuda()
    out = torch.zeros(4 * n_cols, dtype=torch.int32, device="cuda")
    px, py = [3, 1, 4, 1], [5, 9, 2, 6]
    ctx.eval_at_point_noalloc(dev, log_size, n_cols, 1 << log_size, px, py, out)  # first call: address lookup
    torch.cuda.synchronize()
    pool = _DefaultPool()
    for call in range(2):
        used = pool.get(pool.USED_MEM_CURRENT)
        pool.reset_high()
        torch_bytes = torch.cuda.memory_allocated()
        ctx.eval_at_point_noalloc(dev, log_size, n_cols, 1 << log_size, px, py, out)
        torch.cuda.synchronize()
        assert pool.get(pool.USED_MEM_HIGH) <= used, f"call {call} took pool memory"
        assert torch.cuda.memory_allocated() == torch_bytes
    # The counters do see the allocating entry point's scratch.
    used = pool.get(pool.USED_MEM_CURRENT)
    pool.reset_high()
    ctx.eval_at_point(dev, log_size, n_cols, 1 << log_size, px, py, out)
    torch.cuda.synchronize()
    assert pool.get(pool.USED_MEM_HIGH) > used
