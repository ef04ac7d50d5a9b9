"""One grid across several GPUs: z-slabs.

The time step couples every cell to its neighbours (stencils of +-2 cells in
x, y and z, reference src/cu/pde.cu:139-787, turbulence.cu:255-454) and,
through the pressure Poisson solve, globally: FFTs along x and y and a
tridiagonal solve along z per wavenumber pair (src/cu/pressure.cu:506-549).
Split the grid into slabs of whole x-y planes, one per rank:

* each RK stage needs the stage input on 2 planes below and above the slab:
  one halo exchange with the neighbouring ranks per stage (the walls k = 0
  and k = Nz-1 belong to the first and the last slab; their one-sided
  stencils reach 3 planes into the slab, so every slab holds at least 4);
* the pressure source and the FFTs along x and y are plane-local;
* the tridiagonal solve along z needs whole columns of the half spectrum:
  one all-to-all re-distributes it from plane slabs to blocks of spectral
  columns (x wavenumbers r), the solve runs, a second all-to-all brings the
  result back to the slabs;
* the projection needs p on 2 planes around the slab: one more exchange.

Per step (RK4): 4 state exchanges of 2 x 2 x Nx Ny x 4 values, 2 all-to-alls
of the (Nz-1) (Nx-1) ((Ny-1)/2+1) complex spectrum, 1 exchange of p.  The
collectives go through torch.distributed: NCCL over NVLink on GPUs, gloo on
the CPU; no rank reads another GPU's memory with tensor-memory loads.

This module holds the decomposition and its data movement (usable on CUDA or
CPU tensors) and a reference spectral solve built on it.  A multi-GPU step
would run this package's single-GPU kernels on each slab between these
exchanges; that assembly is not built: every run of this build has one GPU,
and one grid of the benchmark size fits one B200's memory many times over.
Slab arrays are laid out [z][x][y] (planes outermost) so that planes move as
contiguous blocks.
"""
from typing import List, Tuple

import numpy as np
import torch

HALO = 2


def bounds(n: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous [start, stop) ranges of n items over `world` ranks, sizes
    differing by at most one (the first n % world ranks take one more)."""
    if world < 1 or n < world:
        raise ValueError("need 1 <= world <= n (got world=%d, n=%d)" % (world, n))
    q, r = divmod(n, world)
    out, s = [], 0
    for i in range(world):
        e = s + q + (1 if i < r else 0)
        out.append((s, e))
        s = e
    return out


class ZSlabs:
    """Planes k of an Nx x Ny x Nz grid distributed over `world` ranks."""

    def __init__(self, Nx: int, Ny: int, Nz: int, world: int, halo: int = HALO):
        self.Nx, self.Ny, self.Nz, self.world, self.halo = Nx, Ny, Nz, world, halo
        self.planes = bounds(Nz, world)
        if min(e - s for s, e in self.planes) < max(halo, 4):
            raise ValueError("every slab needs at least %d planes" % max(halo, 4))

    def local_planes(self, rank: int) -> Tuple[int, int]:
        return self.planes[rank]

    def split(self, field: torch.Tensor, rank: int) -> torch.Tensor:
        """The rank's slab of a global [z][x][y] field with `halo` empty planes on
        each side (filled by exchange_halos)."""
        s, e = self.planes[rank]
        h = self.halo
        out = field.new_zeros((e - s + 2 * h,) + tuple(field.shape[1:]))
        out[h:h + e - s] = field[s:e]
        return out

    def exchange_halos(self, slab: torch.Tensor, rank: int, group=None) -> torch.Tensor:
        """Fill the halo planes of `slab` (shape [nz_local + 2 halo][...]) from
        the neighbouring ranks; planes beyond the walls stay zero (the stage
        kernel's zero halo in z).  Every rank calls it (one exchange per
        neighbour pair, in a fixed order: deadlock-free)."""
        import torch.distributed as dist
        h = self.halo
        n = slab.shape[0] - 2 * h
        ops = []
        recv_lo = recv_hi = None
        if rank > 0:
            recv_lo = torch.empty_like(slab[:h])
            ops.append(dist.P2POp(dist.isend, slab[h:2 * h].contiguous(), rank - 1, group))
            ops.append(dist.P2POp(dist.irecv, recv_lo, rank - 1, group))
        if rank < self.world - 1:
            recv_hi = torch.empty_like(slab[:h])
            ops.append(dist.P2POp(dist.isend, slab[n:n + h].contiguous(), rank + 1, group))
            ops.append(dist.P2POp(dist.irecv, recv_hi, rank + 1, group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if recv_lo is not None:
            slab[:h] = recv_lo
        if recv_hi is not None:
            slab[n + h:] = recv_hi
        return slab


class SpectralColumns:
    """The half spectrum [k][r][s] (nk planes, n_r x wavenumbers, n_s y
    wavenumbers) in two distributions: plane slabs (k split evenly) and
    column blocks (r split evenly).  The all-to-all between them is the one
    data exchange of the distributed Poisson solve."""

    def __init__(self, nk: int, n_r: int, n_s: int, world: int):
        self.nk, self.n_r, self.n_s, self.world = nk, n_r, n_s, world
        self.kb = bounds(nk, world)
        self.rb = bounds(n_r, world)

    def _exchange(self, send: List[torch.Tensor], recv_shapes: List[Tuple[int, ...]], group) -> List[torch.Tensor]:
        """all_to_all of one block per rank through all_to_all_single (gloo and
        NCCL both provide it); complex blocks travel as pairs of reals."""
        import torch.distributed as dist
        cplx = send[0].is_complex()
        flat = [torch.view_as_real(b).reshape(-1) if cplx else b.reshape(-1) for b in send]
        out_sizes = [int(np.prod(sh)) * (2 if cplx else 1) for sh in recv_shapes]
        sbuf = torch.cat(flat)
        rbuf = sbuf.new_empty(sum(out_sizes))
        dist.all_to_all_single(rbuf, sbuf, out_sizes, [f.numel() for f in flat], group=group)
        out, o = [], 0
        for sh, n in zip(recv_shapes, out_sizes):
            piece = rbuf[o:o + n]
            o += n
            out.append(torch.view_as_complex(piece.reshape(tuple(sh) + (2,))) if cplx else piece.reshape(sh))
        return out

    def to_columns(self, G: torch.Tensor, rank: int, group=None) -> torch.Tensor:
        """[k_local][n_r][n_s] on every rank -> [nk][r_local][n_s]."""
        k0, k1 = self.kb[rank]
        assert G.shape[0] == k1 - k0
        a, b = self.rb[rank]
        send = [G[:, p:q].contiguous() for p, q in self.rb]
        recv = self._exchange(send, [(e - s, b - a, self.n_s) for s, e in self.kb], group)
        return torch.cat(recv, dim=0)

    def to_slabs(self, C: torch.Tensor, rank: int, group=None) -> torch.Tensor:
        """[nk][r_local][n_s] -> [k_local][n_r][n_s] (inverse of to_columns)."""
        k0, k1 = self.kb[rank]
        send = [C[s:e].contiguous() for s, e in self.kb]
        recv = self._exchange(send, [(k1 - k0, q - p, self.n_s) for p, q in self.rb], group)
        return torch.cat(recv, dim=1)


def thomas(a: torch.Tensor, b: torch.Tensor, c: torch.Tensor, d: torch.Tensor) -> torch.Tensor:
    """Batched tridiagonal solve along dim 0 (sub-diagonal a[1:], diagonal b,
    super-diagonal c[:-1]; batch dims broadcast)."""
    n = b.shape[0]
    cp = torch.empty_like(d)
    dp = torch.empty_like(d)
    cp[0] = c[0] / b[0]
    dp[0] = d[0] / b[0]
    for k in range(1, n):
        m = b[k] - a[k] * cp[k - 1]
        cp[k] = c[k] / m
        dp[k] = (d[k] - a[k] * dp[k - 1]) / m
    x = torch.empty_like(d)
    x[n - 1] = dp[n - 1]
    for k in range(n - 2, -1, -1):
        x[k] = dp[k] - cp[k] * x[k + 1]
    return x


def poisson_spectral(f_slab: torch.Tensor, kx2: torch.Tensor, ky2: torch.Tensor, zdiag: Tuple[torch.Tensor, ...],
                     cols: SpectralColumns = None, rank: int = 0, group=None) -> torch.Tensor:
    """Reference distributed solve of  d2p/dz2 - (kx^2 + ky^2) p = f  on a plane
    slab f_slab [k_local][Nx-1][Ny-1] (real, periodic planes): FFT along x and
    real FFT along y per plane, all-to-all to spectral columns, the z solve
    per (r, s) with the second-difference coefficients zdiag = (lower, diag,
    upper) of length nk, all-to-all back, inverse FFTs.  With cols = None it
    runs on one rank (the serial reference the distributed run must equal)."""
    F = torch.fft.fft(torch.fft.rfft(f_slab, dim=2), dim=1)          # [k][r][s]
    if cols is not None:
        F = cols.to_columns(F, rank, group)
        a0, a1 = cols.rb[rank]
    else:
        a0, a1 = 0, F.shape[1]
    lo, di, up = zdiag
    k2 = kx2[a0:a1, None] + ky2[None, :]                                # [r_local][s]
    diag = di[:, None, None] - k2[None]
    P = thomas(lo[:, None, None].to(F.dtype), diag.to(F.dtype), up[:, None, None].to(F.dtype), F)
    if cols is not None:
        P = cols.to_slabs(P, rank, group)
    return torch.fft.irfft(torch.fft.ifft(P, dim=1), n=f_slab.shape[2], dim=2)
