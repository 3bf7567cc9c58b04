"""Slab-decomposed 3-D transforms of the MPI solver (FFTclass.myifft3D /
myfft3D, PySpectral/src_MPI/Classes.py:238-258), no GPU needed:

* the oracle's two local halves of each transform, joined by its Alltoall,
  reproduce what the reference's own FFTclass computed when run by 2 and 4
  ranks (tests/golden/slab_fft.npz, made by tests/golden/make_golden.py with
  the ranks as threads sharing a stand-in communicator);
* pyspectral_b200.mpi.FFTclass with num_processes = 2 over gloo: its buffer
  layout and its all_to_all_single exchange, with the library's four local
  halves replaced by the oracle's (the device halves are held to the same
  oracle in tests/test_gpu_slab_fft.py), reproduce numpy's irfftn / rfftn.
"""
import os
import socket

import numpy as np
import pytest

from oracle import spectral_oracle as orc
from tests.helpers import golden, rel

SHAPE = (16, 24, 12)


@pytest.mark.parametrize("P", [2, 4])
def test_oracle_slab_halves_match_reference_fixture(P):
    d = golden("slab_fft.npz")
    u, uhat = d["u"], d["uhat"]
    N1, N2, N3 = SHAPE
    Npx, Npy = N1 // P, N2 // P
    recv = orc.slab_alltoall([orc.slab_ifft_y(uhat[r * Npx:(r + 1) * Npx], P) for r in range(P)])
    for r in range(P):
        assert rel(orc.slab_ifft_xz(recv[r], N2, N3), d[f"P{P}_r{r}_u"]) < 1e-13
    recv = orc.slab_alltoall([orc.slab_fft_xz(u[:, r * Npy:(r + 1) * Npy]).reshape(P, Npx, Npy, -1)
                              for r in range(P)])
    for r in range(P):
        assert rel(orc.slab_fft_y(recv[r]), d[f"P{P}_r{r}_uhat"]) < 1e-13


def _t(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a))


class _HostHalves:
    """The four local halves of the library's slab transforms (psb_slab_*), on
    host tensors, restated by the oracle: the layouts the C ABI declares."""

    def __init__(self, N2, N3):
        self.N2, self.N3 = N2, N3

    def slab_ifft_y(self, P, uhat, send):
        send.copy_(_t(orc.slab_ifft_y(uhat.numpy(), P)))

    def slab_ifft_xz(self, P, recv, u):
        u.copy_(_t(orc.slab_ifft_xz(recv.numpy(), self.N2, self.N3)))

    def slab_fft_xz(self, P, u, send):
        send.copy_(_t(orc.slab_fft_xz(u.numpy()).reshape(send.shape)))

    def slab_fft_y(self, P, recv, uhat):
        uhat.copy_(_t(orc.slab_fft_y(recv.numpy())))


def _rank(r, P, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=r, world_size=P)
    try:
        from pyspectral_b200.mpi import FFTclass
        N1, N2, N3 = SHAPE
        Npx, Npy = N1 // P, N2 // P
        rng = np.random.default_rng(5)
        u = rng.standard_normal(SHAPE)
        uhat = np.fft.rfftn(u)
        fft = FFTclass(N1, N2, N3, 1, "cuda", Npx, Npy, P, None, r)
        fft._ctx = lambda: _HostHalves(N2, N3)
        ur = torch.zeros((N1, Npy, N3), dtype=torch.float64)
        fft.myifft3D(torch.from_numpy(uhat[r * Npx:(r + 1) * Npx].copy()), ur)
        uh = torch.zeros((Npx, N2, N3 // 2 + 1), dtype=torch.complex128)
        fft.myfft3D(torch.from_numpy(u[:, r * Npy:(r + 1) * Npy].copy()), uh)
        # every rank's slabs, gathered for the check
        got = [None] * P
        dist.all_gather_object(got, (ur.numpy(), uh.numpy()))
        if r == 0:
            np.savez(out, u=np.concatenate([g[0] for g in got], axis=1),
                     uhat=np.concatenate([g[1] for g in got], axis=0), ref_u=u, ref_uhat=uhat)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_fftclass_slab_exchange_over_gloo_world_size_2(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "slab.npz")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
    d = np.load(out)
    assert rel(d["u"], d["ref_u"]) < 1e-13
    assert rel(d["uhat"], d["ref_uhat"]) < 1e-13


def test_fftclass_rejects_a_grid_the_ranks_do_not_divide():
    from pyspectral_b200.mpi import FFTclass
    with pytest.raises(ValueError):
        FFTclass(16, 24, 12, 1, "cuda", None, None, 5, None, 0)
