"""Channel-box discretisation with the reference's Domain interface
(jax_spectral_dns/domain.py in dakling/jax-spectral-dns).

Supported: three dimensions, periodic x and z, Chebyshev-Gauss-Lobatto y,
3/2 dealiasing. Grids, wavenumbers and the Chebyshev matrix are built exactly
as the reference builds them (domain.py:130-317, 791-848). The physical <->
spectral transforms here (``field_hat`` / ``field_no_hat``) are host-facing
utilities for building and inspecting fields; the time step never calls them.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Tuple

import numpy as np
import torch

from .seeds import cheb_diff_matrix, cheb_points


def get_cheb_grid(n: int, scale_factor: float = 1.0) -> np.ndarray:
    """Gauss-Lobatto points cos(pi i / (n-1)) (domain.py:130-140)."""
    if scale_factor != 1.0:
        raise NotImplementedError("different scaling of Chebyshev direction not implemented")
    return cheb_points(int(n))


def get_fourier_grid(n: int, scale_factor: float = 2 * np.pi) -> np.ndarray:
    """Equidistant periodic grid (domain.py:143-152)."""
    m = int(n - 1) if n % 2 != 0 else int(n)
    if m % 2 != 0:
        raise Exception("Fourier discretization points must be even!")
    return np.linspace(start=0.0, stop=scale_factor, num=int(m + 1))[:-1]


def assemble_cheb_diff_mat(xs: np.ndarray, order: int = 1) -> np.ndarray:
    """Chebyshev collocation derivative matrix (domain.py:155-163)."""
    return np.linalg.matrix_power(cheb_diff_matrix(np.asarray(xs)), order)


def _default_device():
    return torch.device("cuda") if torch.cuda.is_available() else torch.device("cpu")


@dataclasses.dataclass(frozen=True)
class Domain:
    number_of_dimensions: int
    periodic_directions: Tuple[bool, ...]
    scale_factors: Tuple[float, ...]
    shape: Tuple[int, ...]
    grid: Tuple[np.ndarray, ...]
    diff_mats: Tuple[np.ndarray, ...]
    mgrid: Tuple[np.ndarray, ...]
    aliasing: float = 3 / 2
    dealias_nonperiodic: bool = False

    def number_of_cells(self, direction: int) -> int:
        return len(self.grid[direction])

    def all_dimensions(self):
        return range(self.number_of_dimensions)

    def is_periodic(self, direction: int) -> bool:
        return self.periodic_directions[direction]

    def all_periodic_dimensions(self):
        return [d for d in self.all_dimensions() if self.is_periodic(d)]

    def all_nonperiodic_dimensions(self):
        return [d for d in self.all_dimensions() if not self.is_periodic(d)]

    def get_shape(self):
        return self.shape

    def s(self) -> float:
        """Coefficient scale s = prod over periodic axes of L / (2 pi)."""
        out = 1.0
        for i in self.all_periodic_dimensions():
            out *= self.scale_factors[i] / (2 * np.pi)
        return out


@dataclasses.dataclass(frozen=True)
class PhysicalDomain(Domain):
    """Physical-space description (grids of collocation points)."""

    @classmethod
    def create(cls, shape, periodic_directions, scale_factors: Optional[Tuple[float, ...]] = None,
               aliasing: float = 3 / 2, dealias_nonperiodic: bool = False,
               physical_shape_passed: bool = False) -> "PhysicalDomain":
        """Mode counts and physical grids as in Domain.create (domain.py:201-317)."""
        if len(shape) != 3 or tuple(periodic_directions) != (True, False, True):
            raise NotImplementedError("only 3-D channel boxes (periodic x, Chebyshev y, periodic z) are supported")
        if dealias_nonperiodic:
            raise NotImplementedError("dealias_nonperiodic is not supported")
        if physical_shape_passed:
            raise NotImplementedError("physical_shape_passed is not supported")
        if abs(aliasing - 1.5) > 1e-12:
            raise NotImplementedError("only the 3/2 dealiasing rule is supported")
        sf = list(scale_factors) if scale_factors is not None else []
        modes = []
        phys = []
        for i, n in enumerate(shape):
            n = int(n)
            if periodic_directions[i]:
                m = n if n % 2 != 0 else n + 1
                p = math.ceil(m * aliasing)
                p = p if p % 2 != 0 else p + 1
                modes.append(m)
                phys.append(p)
            else:
                modes.append(n)
                phys.append(n)
        grid, diff_mats = [], []
        for d in range(3):
            if periodic_directions[d]:
                if scale_factors is None:
                    sf.append(2.0 * np.pi)
                grid.append(get_fourier_grid(phys[d], sf[d]))
                diff_mats.append(None)
            else:
                if scale_factors is None:
                    sf.append(1.0)
                grid.append(get_cheb_grid(phys[d], sf[d]))
                diff_mats.append(assemble_cheb_diff_mat(grid[d]))
        for d in (0, 2):
            m = modes[d]
            if m % 4 != 1:
                raise NotImplementedError(
                    f"{m} Fourier modes: the reference's padded transform length and its physical grid "
                    "disagree when the mode count is 3 mod 4 (N = 2 mod 4); use N divisible by 4")
        mgrid = tuple(np.meshgrid(*grid, indexing="ij"))
        return cls(3, tuple(periodic_directions), tuple(sf), tuple(modes), tuple(grid), tuple(diff_mats),
                   mgrid, aliasing, dealias_nonperiodic)

    def get_shape_aliasing(self):
        return tuple(len(g) for g in self.grid)

    def get_extent(self, i: int) -> float:
        return self.scale_factors[i] if self.is_periodic(i) else 2.0

    def hat(self) -> "FourierDomain":
        return FourierDomain.FromPhysicalDomain(self)

    def field_hat(self, field) -> torch.Tensor:
        """Spectral coefficients of a physical field: fftn(ortho)/s over x and z,
        truncated per axis to [0..K-1], K, conj(K), [-K+1..-1]
        (PhysicalDomain.field_hat, domain.py:716-764)."""
        f = torch.as_tensor(field, dtype=torch.float64)
        out = torch.fft.fftn(f.to(torch.complex128), dim=(0, 2), norm="ortho") / self.s()
        for ax, p in ((0, self.number_of_cells(0)), (2, self.number_of_cells(2))):
            ks = int((p - p * (1 - 1 / self.aliasing)) / 2)
            idx1 = torch.arange(0, ks, device=out.device)
            idx2 = torch.tensor([ks], device=out.device)
            idx3 = torch.arange(p - ks + 1, p, device=out.device)
            o1 = out.index_select(ax, idx1)
            o2 = out.index_select(ax, idx2)
            o3 = out.index_select(ax, idx3)
            out = torch.cat([o1, o2, o2.conj(), o3], dim=ax)
        return out.contiguous()

    def diff(self, field, direction: int, order: int = 1):
        """Physical derivative along y with the collocation matrix (domain.py:355-373)."""
        if direction != 1:
            raise NotImplementedError("physical derivatives along periodic directions go through hat()")
        f = torch.as_tensor(field, dtype=torch.float64)
        m = torch.as_tensor(np.linalg.matrix_power(self.diff_mats[1], order), dtype=torch.float64, device=f.device)
        return torch.einsum("ijk,lj->ilk", f, m)

    def y_weights(self) -> np.ndarray:
        from ._ops import operator_tables
        return operator_tables(self.shape[1]).y_weights


@dataclasses.dataclass(frozen=True)
class FourierDomain(Domain):
    physical_domain: Optional[PhysicalDomain] = None

    @classmethod
    def FromPhysicalDomain(cls, physical_domain: PhysicalDomain) -> "FourierDomain":
        """Wavenumber grids in FFT order (domain.py:791-848)."""
        grid = []
        for i in range(3):
            if physical_domain.periodic_directions[i]:
                n = physical_domain.shape[i]
                inp = np.linspace(0, n - 1, int(n))
                grid.append((np.block([inp[n // 2:], inp[: n // 2]]) - n // 2) * (2 * np.pi)
                            / physical_domain.scale_factors[i])
            else:
                grid.append(physical_domain.grid[i])
        mgrid = tuple(np.meshgrid(*grid, indexing="ij"))
        diff_mats = (None, assemble_cheb_diff_mat(grid[1]), None)
        return cls(3, physical_domain.periodic_directions, physical_domain.scale_factors, physical_domain.shape,
                   tuple(grid), diff_mats, mgrid, physical_domain.aliasing, physical_domain.dealias_nonperiodic,
                   physical_domain)

    def get_shape_aliasing(self):
        return self.physical_domain.get_shape_aliasing()

    def diff(self, field_hat, direction: int, order: int = 1) -> torch.Tensor:
        """(i k)^order f along x/z, D^order along y (domain.py:891-918)."""
        f = torch.as_tensor(field_hat)
        if direction in (0, 2):
            k = torch.as_tensor(self.grid[direction], dtype=torch.float64, device=f.device)
            shape = [1, 1, 1]
            shape[direction] = -1
            return (1j * k.reshape(shape)) ** order * f
        m = torch.as_tensor(np.linalg.matrix_power(self.diff_mats[1], order), dtype=torch.float64,
                            device=f.device).to(f.dtype)
        return torch.einsum("ijk,lj->ilk", f, m)

    def curl(self, field_hat) -> torch.Tensor:
        f = torch.as_tensor(field_hat)
        return torch.stack([
            self.diff(f[2], 1) - self.diff(f[1], 2),
            self.diff(f[0], 2) - self.diff(f[2], 0),
            self.diff(f[1], 0) - self.diff(f[0], 1),
        ])

    def field_no_hat(self, field_hat) -> torch.Tensor:
        """Physical values: zero-pad [0..K] + zeros + [-K..-1] along x and z,
        ifftn(ortho), real part, times s (domain.py:1167-1242)."""
        f = torch.as_tensor(field_hat).to(torch.complex128)
        for ax in (0, 2):
            m = self.shape[ax]
            k = m // 2
            nz = math.ceil(m * (self.aliasing - 1))
            f1 = f.narrow(ax, 0, k + 1)
            f2 = f.narrow(ax, m - k, k)
            zshape = list(f.shape)
            zshape[ax] = nz
            f = torch.cat([f1, torch.zeros(zshape, dtype=f.dtype, device=f.device), f2], dim=ax)
        return torch.fft.ifftn(f, dim=(0, 2), norm="ortho").real * self.s()
