"""The discrete adjoint of the linearised perturbation step (jsd_step_adjoint)
and the exact gain gradient behind torch.autograd.Function.

1. Transpose: for random (non-Hermitian, walls included) states x, y,
   <S^n x, y> = <x, (S^T)^n y> in the real inner product of the real and
   imaginary parts, S being n native forward steps, to round-off.
2. Energy gradient: jsd_energy_grad against central differences of jsd_energy.
3. Gain gradient at the size of BASELINE config 2 (33x65x33 modes, Re = 3000,
   Lx = 2 pi, Lz = pi, dt = 0.01, T = 0.5): the autograd gradient against
   central finite differences of the native gain along 8 seeded solenoidal
   directions with every wavenumber up to |k| = K populated, to 1e-6
   relative. The reference's continuous dual (gradient="dual") is compared on
   the same directions and its gap reported: it is not the derivative of the
   discrete gain (jax.grad of the reference would be; JAX is not installed).
"""
import numpy as np
import pytest
import torch

from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.adjoint import GainProblem, gain
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu


def _plan(shape, lx, lz, re=3000.0, dt=0.01):
    modes, phys = mode_counts(shape)
    return StepPlan(modes, phys, lx, lz, _native.JSD_KIND_PERTURBATION, re, dt, linearise=True,
                    base_u=1 - cheb_points(modes[1]) ** 2)


def _rdot(a, b):
    return float(torch.sum(a.real * b.real + a.imag * b.imag).item())


@pytest.mark.parametrize("shape,n", [((8, 33, 8), 1), ((8, 24, 12), 3), ((32, 65, 32), 2)])
def test_step_adjoint_is_the_transpose(cuda, shape, n):
    lx, lz = 2 * np.pi, np.pi
    plan = _plan(shape, lx, lz)
    mx, ny, mz = plan.modes
    gen = torch.Generator(device="cpu").manual_seed(7)
    x = torch.randn((3, ny, mx, mz), dtype=torch.complex128, generator=gen).cuda()
    y = torch.randn((3, ny, mx, mz), dtype=torch.complex128, generator=gen).cuda()
    sx = x.clone()
    plan.step(sx, torch.zeros(1, dtype=torch.float64, device="cuda"), 0, n)
    sty = y.clone()
    plan.step_adjoint(sty, n)
    plan.check_device_errors()
    lhs, rhs = _rdot(sx, y), _rdot(x, sty)
    assert abs(lhs - rhs) < 1e-12 * (sx.abs().norm() * y.abs().norm()).item(), (lhs, rhs)


def test_energy_gradient(cuda):
    lx, lz = 2 * np.pi, np.pi
    shape = (8, 33, 8)
    plan = _plan(shape, lx, lz)
    u = to_device_layout(seeded_velocity_hat(shape, (lx, lz), (4, 4), 1e-3, seed=3))
    gen = torch.Generator(device="cpu").manual_seed(8)
    d = torch.randn(u.shape, dtype=torch.complex128, generator=gen).cuda() * u.abs().max()
    h = 1e-4
    fd = (plan.energy(u + h * d) - plan.energy(u - h * d)).item() / (2 * h)
    ad = _rdot(plan.energy_grad(u), d)
    assert abs(ad / fd - 1) < 1e-9, (ad, fd)


def test_gain_gradient_matches_finite_differences_config2(cuda):
    shape, lx, lz, re, dt, T = (32, 65, 32), 2 * np.pi, np.pi, 3000.0, 0.01, 0.5
    modes, phys = mode_counts(shape)
    K = (modes[0] // 2, modes[2] // 2)  # every wavenumber up to the maximum modes
    u0 = torch.as_tensor(seeded_velocity_hat(shape, (lx, lz), K, 1e-6, seed=2), device="cuda")
    p = GainProblem(modes, phys, lx, lz, re, dt, T, True, checkpoint_every=25)
    assert p.gradient == "discrete"
    x = u0.clone().requires_grad_(True)
    G = gain(x, p)
    G.backward()
    grad = x.grad.clone()
    pd = GainProblem(modes, phys, lx, lz, re, dt, T, True, checkpoint_every=25, gradient="dual")
    xd = u0.clone().requires_grad_(True)
    gain(xd, pd).backward()
    worst, worst_dual = 0.0, 0.0
    for seed in range(100, 108):
        dvec = torch.as_tensor(seeded_velocity_hat(shape, (lx, lz), K, 1e-6, seed=seed), device="cuda")
        h = 1e-4
        fd = (gain(u0 + h * dvec, p) - gain(u0 - h * dvec, p)).item() / (2 * h)
        ad = torch.sum((grad.conj() * dvec).real).item()
        adual = torch.sum((xd.grad.conj() * dvec).real).item()
        worst = max(worst, abs(ad / fd - 1))
        worst_dual = max(worst_dual, abs(adual / fd - 1))
    print(f"discrete adjoint vs FD: max rel err {worst:.2e}; continuous dual vs FD: {worst_dual:.2e}")
    assert worst < 1e-6, worst


def test_discrete_gradient_graphs_and_segments_agree(cuda):
    """The adjoint replayed from captured graphs in segments of K steps equals
    one eager call over all steps, bitwise."""
    shape, lx, lz = (8, 33, 8), 2 * np.pi, np.pi
    modes, phys = mode_counts(shape)
    u0 = to_device_layout(seeded_velocity_hat(shape, (lx, lz), (4, 4), 1e-6, seed=5))
    out = []
    for graphs, K in ((False, 30), (True, 7), (True, 7)):
        p = GainProblem(modes, phys, lx, lz, 3000.0, 0.01, 0.3, True, checkpoint_every=K, use_graphs=graphs)
        out.append(p.discrete_gradient(u0)[1])
    assert torch.equal(out[1], out[2])
    assert torch.allclose(out[0], out[1], rtol=1e-13, atol=1e-13 * out[0].abs().max().item())
