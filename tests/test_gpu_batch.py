"""Batches of independent runs stepped by one plan (n_batch > 1).

A batch of perturbation runs with different Reynolds numbers and initial
fields must step exactly as the same runs one plan each (the batch changes
only the column count of each y-product and the number of transform planes,
not the arithmetic of any one run); shrinking the batch keeps the remaining
runs on track; the batched ensemble reproduces the one-plan-per-run ensemble.
"""
import numpy as np
import pytest
import torch

from conftest import rel
from jax_spectral_dns import _native
from jax_spectral_dns._plan import StepPlan, pack_runs, to_device_layout, to_reference_layout, unpack_runs
from jax_spectral_dns.ensemble import BatchedEnsemble, Ensemble, RunSpec
from jax_spectral_dns.seeds import cheb_points, mode_counts, seeded_velocity_hat

pytestmark = pytest.mark.gpu
SHAPE, LX, LZ, DT = (16, 33, 16), 2 * np.pi, np.pi, 0.01
RES = [2000.0, 3500.0, 5200.0]


def _plan(re, precision="fp64", linearise=False):
    modes, phys = mode_counts(SHAPE)
    return StepPlan(modes, phys, LX, LZ, _native.JSD_KIND_PERTURBATION, re, DT, linearise=linearise,
                    base_u=1 - cheb_points(modes[1]) ** 2, precision=precision)


def _seeds():
    return [seeded_velocity_hat(SHAPE, (LX, LZ), (6, 6), e0, seed=40 + i) for i, e0 in enumerate((1e-4, 3e-3, 1e-2))]


@pytest.mark.parametrize("precision,linearise", [("fp64", False), ("mixed", False), ("fp64", True)])
def test_batch_steps_like_separate_runs(cuda, precision, linearise):
    u0 = _seeds()
    batch = _plan(RES, precision, linearise)
    assert batch.n_batch == 3 and batch.batch_active() == 3
    st = pack_runs(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    batch.step(st, dp, 0, 10)
    e_batch = batch.energy_runs(st).cpu().numpy()
    got = unpack_runs(st)
    for r, re in enumerate(RES):
        single = _plan(re, precision, linearise)
        s1 = to_device_layout(u0[r])
        d1 = torch.zeros(1, dtype=torch.float64, device="cuda")
        single.step(s1, d1, 0, 10)
        assert rel(got[r].cpu().numpy(), to_reference_layout(s1).cpu().numpy()) < 1e-12
        assert abs(e_batch[r] / single.energy(s1).item() - 1) < 1e-12


def test_shrinking_the_batch(cuda):
    u0 = _seeds()
    batch = _plan(RES)
    st = pack_runs(u0)
    dp = torch.zeros(1, dtype=torch.float64, device="cuda")
    batch.step(st, dp, 0, 5)
    # drop the last run: repack the first two runs and step on
    keep = st[:, :, :2].contiguous()
    batch.set_batch_active(2)
    batch.step(keep, dp, 5, 5)
    got = unpack_runs(keep)
    for r in range(2):
        single = _plan(RES[r])
        s1 = to_device_layout(u0[r])
        d1 = torch.zeros(1, dtype=torch.float64, device="cuda")
        single.step(s1, d1, 0, 10)
        assert rel(got[r].cpu().numpy(), to_reference_layout(s1).cpu().numpy()) < 1e-12
    with pytest.raises(_native.NativeError):
        batch.set_batch_active(4)
    with pytest.raises(_native.NativeError):
        batch.energy(keep)  # single-run entry point on a batch plan


def test_batched_ensemble_matches_one_plan_per_run(cuda):
    specs = []
    for i, (n, ny) in enumerate([(16, 33), (16, 33), (16, 33), (16, 49), (32, 33), (16, 49), (16, 33)]):
        specs.append(RunSpec(n, ny, 2000.0 + 500 * i, 10 ** (-5 + 0.4 * i), horizon=[0.3, 0.2, 0.5, 0.3, 0.2, 0.1, 0.5][i],
                             seed=100 + i))
    ref = Ensemble(specs, streams=2, chunk=7)
    ref.run()
    bat = BatchedEnsemble(specs, streams=2, chunk=7)
    bat.run()
    e_ref, e_bat = ref.energies(), bat.energies()
    assert np.abs(e_bat / e_ref - 1).max() < 1e-11
    # a second run from the reset state gives the same result
    bat.reset()
    bat.run()
    assert np.abs(bat.energies() / e_ref - 1).max() < 1e-11
