"""The allocation-free prefix sum (orqcu_prefix_sum_a_noalloc).

It exists for callers that cannot allocate device memory when they call in
(a host program that reserved the GPU's memory for its own pool, or a service
loop that must not take cudaMalloc's device-wide synchronisation). Its output
must equal the pooled prefix sum's (orqcu_prefix_sum_a), bit for bit, on two
calls in a row: the second call reuses the fixed scratch array the first one
left behind, with a different size. Oversized calls must be refused.

This file is collected last so that a failure here stops a `-x` run only
after every other test has run.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _p3(t):
    return (ctypes.c_void_p * 3)(*[t[j].data_ptr() for j in range(3)])


@pytest.mark.parametrize("w", [4, 8])
def test_noalloc_prefix_sum_equals_pooled_on_two_calls(cuda_lib, w):
    import torch

    import orq_b200 as orq

    rt = orq.Runtime(seed=5)
    dt = {4: np.uint32, 8: np.uint64}[w]
    for call, n in enumerate(((1 << 20) + 77, 4096 * 3 + 5)):
        data = (np.arange(n, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15 + call)).astype(dt)
        pooled = rt.secret_share_a(data, 0)
        fixed = pooled.clone()
        orq.prefix_sum(pooled)
        rc = cuda_lib.orqcu_prefix_sum_a_noalloc(rt.h, w, ctypes.c_size_t(n), _p3(fixed.shares))
        assert rc == 0, cuda_lib.orqcu_last_error()
        torch.cuda.synchronize()
        assert torch.equal(pooled.shares, fixed.shares), f"call {call}"
        with np.errstate(over="ignore"):
            want = np.cumsum(data, dtype=dt)
        assert np.array_equal(fixed.open().cpu().numpy().view(dt), want)


@pytest.mark.parametrize("w", [4, 8])
def test_noalloc_prefix_sum_takes_no_device_memory(cuda_lib, w):
    """After one warm-up call (which loads the kernels), a call leaves the
    runtime's pool empty (any pooled scratch would be cached there after its
    release), leaves torch's allocator untouched and does not change the
    device's free memory."""
    import torch

    import orq_b200 as orq

    rt = orq.Runtime(seed=6)
    n = (1 << 22) + 9
    dt = {4: np.uint32, 8: np.uint64}[w]
    v = rt.secret_share_a(np.arange(n, dtype=dt), 0)
    ptrs = _p3(v.shares)
    assert cuda_lib.orqcu_prefix_sum_a_noalloc(rt.h, w, ctypes.c_size_t(n), ptrs) == 0
    torch.cuda.synchronize()
    rt.trim()
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    assert cuda_lib.orqcu_prefix_sum_a_noalloc(rt.h, w, ctypes.c_size_t(n), ptrs) == 0
    torch.cuda.synchronize()
    assert rt.trim() == 0, "the call cached pooled scratch"
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.cuda.mem_get_info()[0] == free0


def test_noalloc_prefix_sum_refuses_oversized(cuda_lib):
    import torch

    import orq_b200 as orq

    rt = orq.Runtime(seed=5)
    small = torch.zeros((3, 16), dtype=torch.int32, device="cuda")
    rc = cuda_lib.orqcu_prefix_sum_a_noalloc(rt.h, 4, ctypes.c_size_t((1 << 26) + 1), _p3(small))
    assert rc == -1
    assert b"2^26" in cuda_lib.orqcu_last_error()
    assert not torch.any(small)
