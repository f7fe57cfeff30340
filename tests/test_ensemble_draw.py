"""The ensemble draw follows the benchmark ensemble definition (host only)."""
from jax_spectral_dns.ensemble import draw_ensemble


def test_ensemble_draw_matches_configuration():
    specs = draw_ensemble(256, seed=0)
    assert len(specs) == 256
    assert {s.n for s in specs} <= {16, 32, 48, 64} and {s.ny for s in specs} <= {49, 65, 97}
    assert all(2000 <= s.re <= 6000 and 1e-6 <= s.e0 <= 1e-2 for s in specs)
    assert {s.horizon for s in specs} <= {5.0, 10.0, 15.0, 20.0}
    assert all(s.dt == 0.01 for s in specs)
