"""CUDA-graph replay of the step loop gives bit-identical results to direct
launches of the same calls (forward with constant mass flux, and the graphed
adjoint segments)."""
import numpy as np
import pytest
import torch

from conftest import golden, rel
from jax_spectral_dns._plan import GraphedSteps, StepPlan, to_device_layout, to_reference_layout
from jax_spectral_dns.adjoint import GainProblem, dual_gradient
from jax_spectral_dns.seeds import mode_counts

pytestmark = pytest.mark.gpu


def test_graph_replay_matches_direct_steps(cuda):
    d = golden("ns_cmf_9x33x9")
    modes, phys = mode_counts(tuple(d["shape"]))
    probe = StepPlan(modes, phys, *d["lengths"], 0, float(d["re_tau"]), float(d["dt"]))
    q0 = probe.flow_rate(to_device_layout(d["u0"])[0]).item()
    p = StepPlan(modes, phys, *d["lengths"], 0, float(d["re_tau"]), float(d["dt"]), constant_mass_flux=True,
                 flow_rate_target=q0)
    a = to_device_layout(d["u0"])
    da = torch.tensor([float(d["dpdx"][0])], dtype=torch.float64, device="cuda")
    # two calls of 5 steps, as the graph below: each call derives the carried
    # eigen-space state from its input, so the chunking is part of the rounding
    p.step(a, da, 0, 5)
    p.step(a, da, 0, 5)
    b = to_device_layout(d["u0"])
    db = torch.tensor([float(d["dpdx"][0])], dtype=torch.float64, device="cuda")
    g = GraphedSteps(p, b, db, 0, 5)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(a, b) and torch.equal(da, db)
    assert rel(to_reference_layout(b).cpu().numpy(), d["u10"]) < 1e-10


@pytest.mark.parametrize("name,lin", [("dual_lin_5x33x5", True), ("dual_nonlin_9x33x9", False)])
def test_graphed_adjoint_matches_eager(cuda, name, lin):
    d = golden(name)
    modes, phys = mode_counts(tuple(d["shape"]))
    n, dt = int(d["n_steps"]), float(d["dt"])
    out = []
    for graphs in (False, True):
        p = GainProblem(modes, phys, *d["lengths"], float(d["re"]), dt, n * dt, lin, checkpoint_every=2,
                        use_graphs=graphs)
        out.append(dual_gradient(torch.as_tensor(d["u0"]), p)[1])
        if graphs:  # second gradient replays the captured graphs
            out.append(dual_gradient(torch.as_tensor(d["u0"]), p)[1])
    assert torch.equal(out[0], out[1]) and torch.equal(out[1], out[2])
    assert rel(out[2].cpu().numpy(), d["grad"]) < 1e-10
