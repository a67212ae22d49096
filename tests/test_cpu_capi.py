"""The C-ABI library loads on a machine without a GPU, exports every entry
point include/orq_cuda.h declares, and reports errors instead of crashing."""
import ctypes

import pytest


def test_header_declares_the_operator_surface():
    import orq_b200

    syms = orq_b200.header_symbols()
    for s in ("orqcu_and_b", "orqcu_multiply_a", "orqcu_b2a_bit", "orqcu_reshare",
              "orqcu_secret_share", "orqcu_open", "orqcu_radix_sort", "orqcu_shuffle",
              "orqcu_apply_elementwise_perm", "orqcu_reserve_permutations"):
        assert s in syms


def test_library_exports_every_declared_symbol(cuda_lib):
    import orq_b200

    for s in orq_b200.header_symbols():
        assert hasattr(cuda_lib, s), s


def test_errors_are_returned_not_raised(cuda_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("host-only check")
    h = ctypes.c_void_p()
    rc = cuda_lib.orqcu_runtime_create(ctypes.c_uint64(1), 0, ctypes.byref(h))
    assert rc < 0
    assert cuda_lib.orqcu_last_error()
    # null runtime is rejected
    assert cuda_lib.orqcu_synchronize(None) == -1


def test_runtime_refuses_without_cuda():
    import torch

    import orq_b200

    if torch.cuda.is_available():
        pytest.skip("host-only check")
    with pytest.raises(orq_b200.OrqError):
        orq_b200.Runtime(seed=1)
