"""fwi_residual_noalloc: the misfit residual for callers that cannot let the
library allocate device memory (a latency-critical loop that cannot absorb
cudaMalloc's device-wide synchronisation, or an application whose own memory
pool owns the GPU).  It keeps its partial sums in a fixed device array instead
of context memory; this test checks it through the C ABI against the existing
context entry point fwi_residual_dev, on two calls in a row.

The file name sorts last so that a run stopping at the first failure has
already run every other test; it also passes alone in a fresh process.
"""
import numpy as np
import pytest

from fwi3d_b200 import lib

pytestmark = pytest.mark.gpu


def _ctx():
    return lib.Context(16, 16, 16, 4, 10.0, 20, 1e-3, 30.0, lib.BOUNDARY_ABC)


def test_noalloc_residual_matches_context_entry_point():
    import torch
    ctx = _ctx()
    g = torch.Generator(device="cuda").manual_seed(17)
    for call, n in enumerate((3_000_017, 1_048_576)):  # ragged last chunk, then an exact multiple
        obs = torch.randn(n, generator=g, device="cuda", dtype=torch.float32)
        cal = torch.randn(n, generator=g, device="cuda", dtype=torch.float32)
        res_ref = torch.empty(n, device="cuda", dtype=torch.float32)
        res = torch.full((n,), float("nan"), device="cuda", dtype=torch.float32)
        out = torch.full((1,), float("nan"), device="cuda", dtype=torch.float64)
        torch.cuda.synchronize()
        want = ctx.residual_dev(obs.data_ptr(), cal.data_ptr(), n, res_ref.data_ptr())
        lib.residual_noalloc(obs.data_ptr(), cal.data_ptr(), n, res.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        got = float(out.item())
        # FP64 sums of the same FP32 residuals in two fixed summation orders
        assert abs(got - want) <= 1e-12 * want, (call, got, want)
        assert torch.equal(res, res_ref), call
        exact = float(((obs - cal).double() ** 2).sum().item())
        assert abs(got - exact) <= 1e-12 * exact
    ctx.close()


def test_noalloc_residual_without_residual_output_and_empty_input():
    import torch
    n = 70_001
    obs = torch.arange(n, device="cuda", dtype=torch.float32) * 1e-3
    cal = torch.zeros(n, device="cuda", dtype=torch.float32)
    out = torch.zeros(1, device="cuda", dtype=torch.float64)
    for _ in range(2):
        lib.residual_noalloc(obs.data_ptr(), cal.data_ptr(), n, 0, out.data_ptr())
        torch.cuda.synchronize()
        want = float((obs.double() ** 2).sum().item())
        assert abs(float(out.item()) - want) <= 1e-12 * want
    lib.residual_noalloc(obs.data_ptr(), cal.data_ptr(), 0, 0, out.data_ptr())
    torch.cuda.synchronize()
    assert float(out.item()) == 0.0


def test_noalloc_residual_rejects_sizes_beyond_its_scratch():
    import torch
    x = torch.zeros(4, device="cuda", dtype=torch.float32)
    out = torch.zeros(1, device="cuda", dtype=torch.float64)
    with pytest.raises(lib.FwiError) as e:
        # the size check runs on the host before any launch, so the short
        # buffers are never read
        lib.residual_noalloc(x.data_ptr(), x.data_ptr(), lib.NOALLOC_MAX_N + 1, 0, out.data_ptr())
    assert e.value.code == 1
    assert lib.NOALLOC_MAX_N == 268435456


def test_noalloc_residual_ignores_an_error_left_by_an_earlier_call():
    """A refused allocation leaves a non-sticky error in the CUDA runtime; the
    next no-alloc call must not report it as its own launch failure."""
    import torch
    ctx = _ctx()
    tiny = np.zeros(4, np.float32)
    # the library's device buffer for 3 x 2^41 samples cannot be allocated;
    # the request is refused before the host arrays are read
    st = ctx.lib.fwi_residual(ctx.h, lib._fptr(tiny), lib._fptr(tiny), 1 << 41, None,
                              lib.C.byref(lib.C.c_double()))
    assert st == 3  # FWI_ERR_ALLOC
    n = 4099
    obs = torch.ones(n, device="cuda", dtype=torch.float32)
    cal = torch.zeros(n, device="cuda", dtype=torch.float32)
    out = torch.zeros(1, device="cuda", dtype=torch.float64)
    lib.residual_noalloc(obs.data_ptr(), cal.data_ptr(), n, 0, out.data_ptr())
    torch.cuda.synchronize()
    assert float(out.item()) == float(n)
    ctx.close()
