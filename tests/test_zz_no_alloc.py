"""The allocation-free DNS right-hand side (psb_rhs_dns_noalloc).

It exists for callers that cannot call cudaMalloc when they evaluate the RHS
(inside a CUDA stream capture, under a host pool allocator that owns the
device memory, in loops that cannot take cudaMalloc's synchronisation).  It
keeps its scratch in a fixed device array inside the library.  This test calls
it through the C ABI twice in a row and checks each result against the regular
entry point psb_rhs (which allocates its own scratch) at the FP64 parity bar;
it also checks that a grid beyond the array's limit is rejected.  The file is
named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_rhs_matches_regular_rhs_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import spectral_oracle as orc
    from pyspectral_b200 import _capi
    N = 32
    ctx = _capi.Context(N, N, N, precision=64)
    lib = ctx.lib
    p = _capi.make_params(nu=0.01, rotate=1, Om=(0.1, -0.3, 0.2))
    for seed in (3, 4):
        st = torch.as_tensor(orc.isotropic_state(N, seed, k0=3.0), device="cuda").contiguous()
        ref = torch.empty_like(st)
        ctx.rhs(_capi.DNS, st, ref, p)
        out = torch.full_like(st, float("nan"))
        ctx.bind_stream()
        rc = lib.psb_rhs_dns_noalloc(ctx.h, ctypes.c_void_p(st.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     ctypes.byref(p))
        assert rc == 0, lib.psb_last_error(ctx.h)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_noalloc_rejects_grids_beyond_its_array():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import _capi
    N = 48
    ctx = _capi.Context(N, N, N, precision=64)
    st = torch.zeros((3, N, N, N // 2 + 1), dtype=torch.complex128, device="cuda")
    out = torch.empty_like(st)
    p = _capi.make_params(nu=0.01)
    rc = ctx.lib.psb_rhs_dns_noalloc(ctx.h, ctypes.c_void_p(st.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     ctypes.byref(p))
    assert rc == 2
    assert b"32^3" in ctx.lib.psb_last_error(ctx.h)
