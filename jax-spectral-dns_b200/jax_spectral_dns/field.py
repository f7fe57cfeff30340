"""Field containers with the reference's interface (jax_spectral_dns/field.py).

Data live in torch tensors (on the GPU when one is present). PhysicalField
holds (Px, Ny, Pz) float64 values on the reference physical grid; FourierField
holds (Mx, Ny, Mz) complex128 coefficients in the reference layout and
normalisation. Integrals follow the reference (field.py:1456-1481,
2618-2710): periodic directions by the rectangle rule, y by the Chebyshev
integration weights.
"""
from __future__ import annotations

from typing import Callable, List, Optional

import numpy as np
import torch

from .domain import FourierDomain, PhysicalDomain, _default_device


def _as_tensor(x, dtype, device=None):
    t = torch.as_tensor(x)
    return t.to(device=device or (t.device if isinstance(x, torch.Tensor) else _default_device()), dtype=dtype)


class Field:
    activate_jit_ = False

    def __init__(self, name: str = "field"):
        self.name = name
        self.time_step = 0

    def get_name(self) -> str:
        return self.name

    def set_name(self, name: str) -> None:
        self.name = name

    def set_time_step(self, t: int) -> None:
        self.time_step = t

    def get_time_step(self) -> int:
        return self.time_step

    @classmethod
    def initialize(cls, cleanup: bool = True) -> None:
        pass


class PhysicalField(Field):
    def __init__(self, physical_domain: PhysicalDomain, data, name: str = "field"):
        super().__init__(name)
        self.physical_domain = physical_domain
        self.data = _as_tensor(data, torch.float64)

    @classmethod
    def FromFunc(cls, domain: PhysicalDomain, func: Optional[Callable] = None, name: str = "field"):
        """Evaluate func(X) on the grid (field.py:1265-1279); func receives the
        three meshgrid arrays."""
        X = tuple(np.asarray(m) for m in domain.mgrid)
        if func is None:
            data = np.zeros(domain.get_shape_aliasing())
        else:
            data = np.asarray(func(X), dtype=np.float64) * np.ones(domain.get_shape_aliasing())
        return cls(domain, data, name)

    @classmethod
    def Zeros(cls, domain: PhysicalDomain, name: str = "field"):
        return cls(domain, np.zeros(domain.get_shape_aliasing()), name)

    @classmethod
    def FromRandom(cls, domain: PhysicalDomain, seed: int = 0, energy_norm: float = 1.0, name: str = "field"):
        """Uniform random values in [-1, 1] on the physical grid, walls set to
        zero, scaled to energy `energy_norm` (field.py:1281-1310). The values
        come from NumPy's PCG64 seeded with `seed` (the reference draws them
        with jax.random, which is not available here)."""
        rng = np.random.default_rng(int(seed))
        out = cls(domain, rng.uniform(-1.0, 1.0, size=domain.get_shape_aliasing()), name)
        out.update_boundary_conditions()
        out.normalize_by_energy()
        out.data = out.data * float(np.sqrt(energy_norm))
        return out

    def normalize_by_energy(self) -> "PhysicalField":
        self.data = self.data / float(np.sqrt(self.energy()))
        return self

    def get_domain(self):
        return self.physical_domain

    def get_data(self):
        return self.data

    def hat(self) -> "FourierField":
        out = FourierField(self.physical_domain, self.physical_domain.field_hat(self.data), self.name + "_hat")
        out.time_step = self.time_step
        return out

    def diff(self, direction: int, order: int = 1) -> "PhysicalField":
        if direction == 1:
            return PhysicalField(self.physical_domain, self.physical_domain.diff(self.data, 1, order))
        return self.hat().diff(direction, order).no_hat()

    def update_boundary_conditions(self) -> None:
        self.data = self.data.clone()
        self.data[:, 0, :] = 0.0
        self.data[:, -1, :] = 0.0

    def volume_integral(self) -> float:
        d = self.physical_domain
        px, _, pz = d.get_shape_aliasing()
        w = torch.as_tensor(d.y_weights(), dtype=torch.float64, device=self.data.device)
        iz = d.scale_factors[2] / pz * self.data.sum(dim=2)
        iy = iz @ w
        return float(d.scale_factors[0] / px * iy.sum())

    def definite_integral(self, direction: int):
        """y: sum_y w_y f (a (Px, Pz) tensor); x/z: rectangle rule."""
        d = self.physical_domain
        if direction == 1:
            w = torch.as_tensor(d.y_weights(), dtype=torch.float64, device=self.data.device)
            return torch.einsum("ijk,j->ik", self.data, w)
        p = d.get_shape_aliasing()[direction]
        return d.scale_factors[direction] / p * self.data.sum(dim=direction)

    def energy(self) -> float:
        vol = 2.0 * float(np.prod(self.physical_domain.scale_factors))
        return PhysicalField(self.physical_domain, 0.5 * self.data * self.data).volume_integral() / vol

    def energy_with_other(self, other: "PhysicalField") -> float:
        vol = 2.0 * float(np.prod(self.physical_domain.scale_factors))
        return PhysicalField(self.physical_domain, 0.5 * self.data * other.data).volume_integral() / vol

    def max(self) -> float:
        return float(self.data.max())

    def absmax(self) -> float:
        return float(self.data.abs().max())

    def _wrap(self, data):
        return PhysicalField(self.physical_domain, data, self.name)

    def __add__(self, o):
        return self._wrap(self.data + (o.data if isinstance(o, PhysicalField) else o))

    def __sub__(self, o):
        return self._wrap(self.data - (o.data if isinstance(o, PhysicalField) else o))

    def __mul__(self, o):
        return self._wrap(self.data * (o.data if isinstance(o, PhysicalField) else o))

    __rmul__ = __mul__

    def __truediv__(self, o):
        return self._wrap(self.data / o)

    def __neg__(self):
        return self._wrap(-self.data)

    def __abs__(self):
        return float(torch.linalg.norm(self.data))

    def __getitem__(self, idx):
        return self.data[idx]


class FourierField(Field):
    def __init__(self, physical_domain: PhysicalDomain, data, name: str = "field_hat"):
        super().__init__(name)
        self.physical_domain = physical_domain
        self.fourier_domain: FourierDomain = physical_domain.hat()
        self.data = _as_tensor(data, torch.complex128)

    @classmethod
    def FromField(cls, field: PhysicalField) -> "FourierField":
        return field.hat()

    @classmethod
    def Zeros(cls, physical_domain: PhysicalDomain, name: str = "field_hat"):
        return cls(physical_domain, np.zeros(physical_domain.get_shape(), dtype=np.complex128), name)

    def get_domain(self):
        return self.fourier_domain

    def get_data(self):
        return self.data

    def no_hat(self) -> PhysicalField:
        out = PhysicalField(self.physical_domain, self.fourier_domain.field_no_hat(self.data), self.name)
        out.time_step = self.time_step
        return out

    def diff(self, direction: int, order: int = 1) -> "FourierField":
        return FourierField(self.physical_domain, self.fourier_domain.diff(self.data, direction, order), self.name)

    def field_2d(self, direction: int) -> "FourierField":
        """Keep only the zero wavenumber along `direction` (field.py:2912)."""
        out = torch.zeros_like(self.data)
        sl = [slice(None)] * 3
        sl[direction] = slice(0, 1)
        out[tuple(sl)] = self.data[tuple(sl)]
        return FourierField(self.physical_domain, out, self.name)

    def energy(self) -> float:
        return self.no_hat().energy()

    def solve_poisson(self, mat=None) -> "FourierField":
        """Per-wavenumber Poisson solve with homogeneous Dirichlet rows
        (field.py:3059-3083, matrix of domain.py:857-889): the reference's
        inv(-k^2 eye_bc + BC(D2)) is the identity on the wall rows and
        (D2_int - k^2)^-1 on the interior, applied here in the eigenbasis
        D2_int = V diag(lam) V^-1 (or with `mat`, (Mx, Mz, Ny, Ny), when given)."""
        from ._ops import operator_tables

        f = self.data
        if mat is not None:
            m = torch.as_tensor(mat, device=f.device).to(torch.complex128)
            out = torch.einsum("ijkl,ilj->ikj", m, f)
            return FourierField(self.physical_domain, out, self.name + "_poisson")
        ny = f.shape[1]
        t = operator_tables(ny)
        dev = f.device
        V = torch.as_tensor(t.V, device=dev).to(torch.complex128)
        Vinv = torch.as_tensor(t.Vinv, device=dev).to(torch.complex128)
        lam = torch.as_tensor(t.lam, device=dev)
        kx = torch.as_tensor(self.fourier_domain.grid[0], device=dev, dtype=torch.float64)
        kz = torch.as_tensor(self.fourier_domain.grid[2], device=dev, dtype=torch.float64)
        k2 = kx[:, None] ** 2 + kz[None, :] ** 2                      # (Mx, Mz)
        inner = torch.einsum("ab,ibj->iaj", Vinv, f[:, 1:-1, :])        # V^-1 rhs_int
        inner = inner / (lam[None, :, None] - k2[:, None, :])
        out = f.clone()
        out[:, 1:-1, :] = torch.einsum("ab,ibj->iaj", V, inner)
        return FourierField(self.physical_domain, out, self.name + "_poisson")

    def _wrap(self, data):
        return FourierField(self.physical_domain, data, self.name)

    def __add__(self, o):
        return self._wrap(self.data + (o.data if isinstance(o, FourierField) else o))

    def __sub__(self, o):
        return self._wrap(self.data - (o.data if isinstance(o, FourierField) else o))

    def __mul__(self, o):
        return self._wrap(self.data * (o.data if isinstance(o, FourierField) else o))

    __rmul__ = __mul__

    def __truediv__(self, o):
        return self._wrap(self.data / o)

    def __neg__(self):
        return self._wrap(-self.data)

    def __getitem__(self, idx):
        return self.data[idx]


class VectorField:
    def __init__(self, fields: List, name: Optional[str] = None):
        self.fields = list(fields)
        self.name = name or (self.fields[0].name if self.fields else "vector")

    @classmethod
    def FromData(cls, field_cls, physical_domain: PhysicalDomain, data, name: str = "field") -> "VectorField":
        t = torch.as_tensor(data)
        return cls([field_cls(physical_domain, t[i], name + "_" + "xyz"[i]) for i in range(t.shape[0])], name)

    @classmethod
    def Zeros(cls, field_cls, physical_domain: PhysicalDomain, name: str = "field") -> "VectorField":
        return cls([field_cls.Zeros(physical_domain) for _ in range(3)], name)

    def __getitem__(self, i):
        return self.fields[i]

    def __len__(self):
        return len(self.fields)

    def __iter__(self):
        return iter(self.fields)

    def get_name(self) -> str:
        return self.name

    def set_name(self, name: str) -> None:
        self.name = name
        for i, f in enumerate(self.fields):
            f.name = name + "_" + "xyz"[i]

    def set_time_step(self, t: int) -> None:
        for f in self.fields:
            f.time_step = t

    def get_time_step(self) -> int:
        return self.fields[0].time_step

    def get_physical_domain(self) -> PhysicalDomain:
        return self.fields[0].physical_domain

    def get_data(self) -> torch.Tensor:
        return torch.stack([f.data for f in self.fields])

    def hat(self) -> "VectorField":
        return VectorField([f.hat() for f in self.fields], self.name + "_hat")

    def no_hat(self) -> "VectorField":
        return VectorField([f.no_hat() for f in self.fields], self.name)

    def energy(self) -> float:
        return float(sum(f.energy() for f in self.fields))

    def energy_with_other(self, other: "VectorField") -> float:
        return float(sum(f.energy_with_other(other[i]) for i, f in enumerate(self.fields)))

    def field_2d(self, direction: int) -> "VectorField":
        return VectorField([f.field_2d(direction) for f in self.fields], self.name)

    def all_dimensions(self):
        return range(len(self.fields))

    def curl(self) -> "VectorField":
        """(w_y - v_z, u_z - w_x, v_x - u_y) (field.py:917-939); physical or
        spectral fields alike."""
        assert len(self) == 3, "rotation only defined in 3 dimensions"
        u, v, w = self.fields
        out = [w.diff(1) - v.diff(2), u.diff(2) - w.diff(0), v.diff(0) - u.diff(1)]
        for f in out:
            f.time_step = self.get_time_step()
        return VectorField(out, "curl_" + (self.name or "field"))

    def div(self):
        """u_x + v_y + w_z (field.py:941-948)."""
        out = self.fields[0].diff(0)
        for d in list(self.all_dimensions())[1:]:
            out = out + self.fields[d].diff(d)
        out.name = "div_" + self.name if self.name is not None else "div_field"
        return out

    def normalize_by_energy(self) -> "VectorField":
        """Divide each component by the square root of the vector field's energy (field.py:666-673)."""
        en = self.energy()
        for f in self.fields:
            f.data = f.data / float(np.sqrt(en))
        return self

    def _map(self, fn) -> "VectorField":
        return VectorField([fn(i, f) for i, f in enumerate(self.fields)], self.name)

    def __add__(self, o):
        return self._map(lambda i, f: f + (o[i] if isinstance(o, VectorField) else o))

    def __sub__(self, o):
        return self._map(lambda i, f: f - (o[i] if isinstance(o, VectorField) else o))

    def __mul__(self, o):
        return self._map(lambda i, f: f * o)

    __rmul__ = __mul__

    def __truediv__(self, o):
        return self._map(lambda i, f: f / o)

    def __neg__(self):
        return self._map(lambda i, f: -f)
