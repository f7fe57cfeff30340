"""Ensembles: overlapped replay on a stream pool equals one-after-another replay."""
import numpy as np
import pytest
import torch

from jax_spectral_dns.ensemble import Ensemble, draw_ensemble

pytestmark = pytest.mark.gpu


def test_ensemble_concurrent_equals_sequential(cuda):
    specs = draw_ensemble(12, seed=3, horizon_scale=0.01)
    ens = Ensemble(specs, streams=4, chunk=20)
    ens.run()
    a = ens.energies()
    ens.reset()
    ens.run_sequential()
    b = ens.energies()
    assert np.all(np.isfinite(a)) and np.array_equal(a, b)
    assert ens.total_steps == sum(s.steps for s in specs)

