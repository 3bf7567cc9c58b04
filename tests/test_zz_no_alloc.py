"""The allocation-free DNS right-hand side (psb_rhs_dns_noalloc).

It exists for callers that cannot call cudaMalloc when they evaluate the RHS
(a host pool allocator that owns the device memory, so a library cudaMalloc
fails; loops that cannot take cudaMalloc's synchronisation).  It keeps its
scratch in a fixed device array inside the library.  These tests call it
through the C ABI twice in a row and check each result against the regular
entry point psb_rhs (which allocates its own scratch): FP64 at the 1e-12
parity bar, FP32 at the 2e-5 bar of the FP32 tests.  They also check that a
second call changes nothing in the device's free memory, that the caller's
current device is left alone, and that a grid beyond the array's limit is
rejected.  The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _noalloc(ctx, st, out, p):
    ctx.bind_stream()
    rc = ctx.lib.psb_rhs_dns_noalloc(ctx.h, ctypes.c_void_p(st.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     ctypes.byref(p))
    assert rc == 0, ctx.lib.psb_last_error(ctx.h)


def _state(torch, shape, seed, precision):
    N1, N2, N3 = shape
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((3, N1, N2, N3))
    k = np.sqrt(np.add.outer(np.add.outer(np.fft.fftfreq(N1, 1 / N1) ** 2, np.fft.fftfreq(N2, 1 / N2) ** 2),
                             np.fft.rfftfreq(N3, 1 / N3) ** 2))
    st = np.stack([np.fft.rfftn(a) for a in x]) * np.exp(-0.3 * k) / np.sqrt(N1 * N2 * N3)
    cd = torch.complex128 if precision == 64 else torch.complex64
    return torch.as_tensor(st, device="cuda").to(cd).contiguous()


@pytest.mark.parametrize("precision,shape,tol", [(64, (32, 32, 32), 1e-12), (32, (32, 32, 32), 2e-5),
                                                 (32, (32, 32, 64), 2e-5)])
def test_noalloc_rhs_matches_regular_rhs_twice(precision, shape, tol):
    torch = _torch()
    from pyspectral_b200 import _capi
    ctx = _capi.Context(*shape, precision=precision)
    p = _capi.make_params(nu=0.01, rotate=1, Om=(0.1, -0.3, 0.2))
    for seed in (3, 4):
        st = _state(torch, shape, seed, precision)
        ref = torch.empty_like(st)
        ctx.rhs(_capi.DNS, st, ref, p)
        out = torch.full_like(st, float("nan"))
        _noalloc(ctx, st, out, p)
        torch.cuda.synchronize()
        a, b = out.cpu().numpy(), ref.cpu().numpy()
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= tol * np.abs(b).max()


def test_noalloc_leaves_free_memory_and_current_device_alone():
    """On a context that never ran psb_rhs: after one warm call (which looks up
    the array's address and loads the kernels), a second call leaves the
    device's free memory exactly as it was, and neither call changes the
    caller's current device."""
    torch = _torch()
    from pyspectral_b200 import _capi
    N = 32
    dev = torch.cuda.current_device()
    ctx = _capi.Context(N, N, N, precision=64, device=dev)
    p = _capi.make_params(nu=0.01)
    st = _state(torch, (N, N, N), 5, 64)
    out1 = torch.empty_like(st)
    out2 = torch.empty_like(st)
    torch.cuda.synchronize()
    _noalloc(ctx, st, out1, p)
    torch.cuda.synchronize()
    assert torch.cuda.current_device() == dev
    free0, _ = torch.cuda.mem_get_info(dev)
    _noalloc(ctx, st, out2, p)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    assert torch.cuda.current_device() == dev
    assert torch.equal(out1, out2)


@pytest.mark.parametrize("precision,shape", [(64, (48, 48, 48)), (64, (32, 32, 64)), (32, (48, 48, 48))])
def test_noalloc_rejects_grids_beyond_its_array(precision, shape):
    torch = _torch()
    from pyspectral_b200 import _capi
    N1, N2, N3 = shape
    ctx = _capi.Context(N1, N2, N3, precision=precision)
    cd = torch.complex128 if precision == 64 else torch.complex64
    st = torch.zeros((3, N1, N2, N3 // 2 + 1), dtype=cd, device="cuda")
    out = torch.empty_like(st)
    p = _capi.make_params(nu=0.01)
    rc = ctx.lib.psb_rhs_dns_noalloc(ctx.h, ctypes.c_void_p(st.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                     ctypes.byref(p))
    assert rc == 2
    assert b"32^3" in ctx.lib.psb_last_error(ctx.h)
