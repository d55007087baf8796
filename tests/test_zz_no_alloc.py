"""oc_thomas_noalloc: the batched tridiagonal solve for callers that cannot
allocate device memory (its scratch is a fixed array inside the library).

Called through the C ABI and checked against oc_thomas on two calls in a row;
both must agree bit for bit, the tolerance of the other Thomas tests. This file
is collected last so that a run stopping at the first failure has run every
other test before it.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(rng, n, ncols):
    sub = rng.uniform(-1.0, 0.0, (n, ncols))
    sup = rng.uniform(-1.0, 0.0, (n, ncols))
    diag = 2.5 + rng.uniform(0.0, 1.0, (n, ncols))
    rhs = rng.standard_normal((n, ncols))
    return sub, diag, sup, rhs


def test_noalloc_thomas_matches_oc_thomas_on_two_calls():
    import torch

    from hydrostatic_ocean_core_benchmark_b200 import _lib
    assert torch.cuda.is_available()
    torch.cuda.set_device(0)
    lib = _lib.load()
    rng = np.random.default_rng(2026)
    for n, ncols in ((41, 9000), (50, 20000)):
        sub, diag, sup, rhs = (torch.as_tensor(a, device="cuda") for a in _system(rng, n, ncols))
        x_ref = torch.empty_like(rhs)
        x_new = torch.full_like(rhs, np.nan)
        ptrs = [a.data_ptr() for a in (sub, diag, sup, rhs)]
        assert lib.oc_thomas(*ptrs, x_ref.data_ptr(), n, ncols, None) == 0
        assert lib.oc_thomas_noalloc(*ptrs, x_new.data_ptr(), n, ncols, None) == 0
        torch.cuda.synchronize()
        assert torch.equal(x_ref, x_new)


def test_noalloc_thomas_allocates_nothing_after_its_warm_up_call():
    """After the warm-up call that commits the fixed scratch, a call on a
    non-default stream leaves the device's free memory unchanged."""
    import torch

    from hydrostatic_ocean_core_benchmark_b200 import _lib
    torch.cuda.set_device(0)
    lib = _lib.load()
    rng = np.random.default_rng(7)
    n, ncols = 32, 4096
    sub, diag, sup, rhs = (torch.as_tensor(a, device="cuda") for a in _system(rng, n, ncols))
    x_ref = torch.empty_like(rhs)
    x_new = torch.empty_like(rhs)
    ptrs = [a.data_ptr() for a in (sub, diag, sup, rhs)]
    assert lib.oc_thomas(*ptrs, x_ref.data_ptr(), n, ncols, None) == 0
    assert lib.oc_thomas_noalloc(*ptrs, x_new.data_ptr(), n, ncols, None) == 0  # warm-up
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    x_new.fill_(np.nan)
    torch.cuda.synchronize()
    assert lib.oc_thomas_noalloc(*ptrs, x_new.data_ptr(), n, ncols, side.cuda_stream) == 0
    side.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert torch.equal(x_ref, x_new)


def test_noalloc_thomas_rejects_sizes_beyond_its_scratch():
    import torch

    from hydrostatic_ocean_core_benchmark_b200 import _lib
    torch.cuda.set_device(0)
    lib = _lib.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    too_many = 1048576 // 64 + 1
    assert lib.oc_thomas_noalloc(p, p, p, p, p, 64, too_many, None) == 7
