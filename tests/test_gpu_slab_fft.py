"""Device halves of the slab-decomposed transforms (psb_slab_ifft_y,
psb_slab_ifft_xz, psb_slab_fft_xz, psb_slab_fft_y) on one GPU, the ranks run
one after another and the Alltoall between the halves emulated by copying
blocks on the device (block r of every rank's send buffer, in rank order,
into rank r's receive buffer): each half against the oracle's half, and each
rank's result against what the reference's own FFTclass (src_MPI/Classes.py:
238-258) computed with 2 and 4 ranks (tests/golden/slab_fft.npz), and on a
larger grid against numpy's irfftn / rfftn.  Bars: FP64 1e-12, FP32 1e-5.
"""
import numpy as np
import pytest

from oracle import spectral_oracle as orc
from tests.helpers import golden, rel

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _run(torch, shape, P, precision, u, uhat):
    """Every rank's inverse and forward slab transform; returns the per-rank
    physical y slabs, spectral x slabs and, for the checks of the halves, the
    first-half send buffers of both directions."""
    from pyspectral_b200 import _capi
    N1, N2, N3 = shape
    K = N3 // 2 + 1
    Npx, Npy = N1 // P, N2 // P
    cd = torch.complex128 if precision == 64 else torch.complex64
    rd = torch.float64 if precision == 64 else torch.float32
    ctx = _capi.Context(N1, N2, N3, precision=precision)
    dev = "cuda"
    sends = []
    for r in range(P):
        s = torch.empty((P, Npx, Npy, K), dtype=cd, device=dev)
        ctx.slab_ifft_y(P, torch.as_tensor(uhat[r * Npx:(r + 1) * Npx], device=dev).to(cd).contiguous(), s)
        sends.append(s)
    us = []
    for r in range(P):
        recv = torch.stack([sends[p][r] for p in range(P)]).contiguous()
        ur = torch.empty((N1, Npy, N3), dtype=rd, device=dev)
        ctx.slab_ifft_xz(P, recv, ur)
        us.append(ur)
    fsends = []
    for r in range(P):
        s = torch.empty((P, Npx, Npy, K), dtype=cd, device=dev)
        ctx.slab_fft_xz(P, torch.as_tensor(u[:, r * Npy:(r + 1) * Npy], device=dev).to(rd).contiguous(), s)
        fsends.append(s)
    uhs = []
    for r in range(P):
        recv = torch.stack([fsends[p][r] for p in range(P)]).contiguous()
        uh = torch.empty((Npx, N2, K), dtype=cd, device=dev)
        ctx.slab_fft_y(P, recv, uh)
        uhs.append(uh)
    torch.cuda.synchronize()
    assert ctx.device_status() == 0
    np_ = lambda ts: [t.cpu().numpy().astype(np.complex128 if t.is_complex() else np.float64) for t in ts]
    return np_(us), np_(uhs), np_(sends), np_(fsends)


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("P", [2, 4])
def test_slab_transforms_match_reference_ranks(P, precision):
    torch = _torch()
    d = golden("slab_fft.npz")
    shape = (16, 24, 12)
    N1, N2, N3 = shape
    Npx, Npy = N1 // P, N2 // P
    u, uhat = d["u"], d["uhat"]
    tol = 1e-12 if precision == 64 else 1e-5
    us, uhs, sends, fsends = _run(torch, shape, P, precision, u, uhat)
    for r in range(P):
        assert rel(us[r], d[f"P{P}_r{r}_u"]) < tol, r
        assert rel(uhs[r], d[f"P{P}_r{r}_uhat"]) < tol, r
        # the halves on their own, against the oracle's
        assert rel(sends[r], orc.slab_ifft_y(uhat[r * Npx:(r + 1) * Npx], P)) < tol
        assert rel(fsends[r].reshape(N1, Npy, -1), orc.slab_fft_xz(u[:, r * Npy:(r + 1) * Npy])) < tol


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("shape,P", [((64, 48, 32), 1), ((64, 48, 32), 8), ((96, 96, 64), 4)])
def test_slab_transforms_assemble_numpy_transforms(shape, P, precision):
    torch = _torch()
    rng = np.random.default_rng(17)
    u = rng.standard_normal(shape)
    uhat = np.fft.rfftn(u)
    us, uhs, _, _ = _run(torch, shape, P, precision, u, uhat)
    tol = 1e-12 if precision == 64 else 1e-5
    assert rel(np.concatenate(us, axis=1), u) < tol
    assert rel(np.concatenate(uhs, axis=0), uhat) < tol
