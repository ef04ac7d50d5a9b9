"""One grid over several ranks as z-slabs (wildfires_b200/domain.py), on the
CPU with gloo at world size 2 and 3: the halo exchange of the RK stages and
the projection, the all-to-all between plane slabs and spectral columns of
the Poisson solve, and the distributed spectral solve against the same solve
on one rank."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from wildfires_b200 import domain


def test_bounds_cover_and_balance():
    assert domain.bounds(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert domain.bounds(8, 1) == [(0, 8)]
    with pytest.raises(ValueError):
        domain.bounds(2, 3)
    with pytest.raises(ValueError):
        domain.ZSlabs(8, 8, 6, 2)       # slabs of 3 planes: the walls' stencils need 4


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _problem(Nx=9, Ny=11, Nz=17, seed=0):
    g = torch.Generator().manual_seed(seed)
    field = torch.randn((Nz, Nx, Ny), generator=g, dtype=torch.float64)
    nk = Nz - 1
    f = torch.randn((nk, Nx - 1, Ny - 1), generator=g, dtype=torch.float64)
    # wavenumbers of the periodic planes (symmetric in r: the spectrum of a real field stays Hermitian)
    kx2 = (2 * np.pi * torch.fft.fftfreq(Nx - 1, dtype=torch.float64)) ** 2
    ky2 = (2 * np.pi * torch.fft.rfftfreq(Ny - 1, dtype=torch.float64)) ** 2
    lo = torch.ones(nk, dtype=torch.float64)
    up = torch.ones(nk, dtype=torch.float64)
    di = -3.0 - torch.rand(nk, generator=g, dtype=torch.float64)
    return field, f, kx2, ky2, (lo, di, up)


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        field, f, kx2, ky2, zd = _problem()
        Nz, Nx, Ny = field.shape
        z = domain.ZSlabs(Nx, Ny, Nz, world)
        slab = z.exchange_halos(z.split(field, rank), rank)
        cols = domain.SpectralColumns(Nz - 1, Nx - 1, (Ny - 1) // 2 + 1, world)
        k0, k1 = cols.kb[rank]
        G = torch.fft.fft(torch.fft.rfft(f[k0:k1], dim=2), dim=1)
        C = cols.to_columns(G, rank)
        back = cols.to_slabs(C, rank)
        p = domain.poisson_spectral(f[k0:k1], kx2, ky2, zd, cols, rank)
        torch.save({"slab": slab, "C": C, "back": back, "G": G, "p": p}, os.path.join(out_dir, "rank%d.pt" % rank))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halos_transposes_and_distributed_solve(world, tmp_path):
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    field, f, kx2, ky2, zd = _problem()
    Nz, Nx, Ny = field.shape
    z = domain.ZSlabs(Nx, Ny, Nz, world)
    h = z.halo
    F = torch.fft.fft(torch.fft.rfft(f, dim=2), dim=1)
    cols = domain.SpectralColumns(Nz - 1, Nx - 1, (Ny - 1) // 2 + 1, world)
    p_serial = domain.poisson_spectral(f, kx2, ky2, zd)
    p_parts = []
    for rank in range(world):
        out = torch.load(tmp_path / ("rank%d.pt" % rank))
        s, e = z.local_planes(rank)
        slab = out["slab"]
        # interior planes, and halo planes equal to the neighbours' (zero beyond the walls)
        for q in range(-h, e - s + h):
            k = s + q
            want = field[k] if 0 <= k < Nz else torch.zeros_like(field[0])
            assert torch.equal(slab[q + h], want), (rank, q)
        a, b = cols.rb[rank]
        assert torch.equal(out["C"], F[:, a:b])          # whole columns of this rank's wavenumber block
        assert torch.equal(out["back"], out["G"])        # the transpose round trip
        p_parts.append(out["p"])
    p = torch.cat(p_parts, dim=0)
    assert torch.allclose(p, p_serial, rtol=0, atol=1e-12 * float(p_serial.abs().max()))
    # and the serial reference solves the system it states
    Ps = torch.fft.fft(torch.fft.rfft(p_serial, dim=2), dim=1)
    lo, di, up = zd
    k2 = kx2[:, None] + ky2[None, :]
    r = (di[:, None, None] - k2[None]) * Ps
    r[1:] += lo[1:, None, None] * Ps[:-1]
    r[:-1] += up[:-1, None, None] * Ps[1:]
    assert torch.allclose(r, F, atol=1e-10 * float(F.abs().max()))
    assert np.isfinite(p.numpy()).all()
