"""The spectral reductions (shell spectra per component, E, Omega, band
energy) are compensated and run in a fixed order: two runs give bit-identical
results, and they agree with the float64 oracle on the same state."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,dtype", [(128, torch.float32), (64, torch.float64)])
def test_spectrum_and_budget_bit_identical_and_match_oracle(h3, orc, N, dtype):
    g = h3.make_grid(N, dtype=dtype)
    u = h3.hit_initial_field(5, g)
    f = h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0)
    runs = []
    for _ in range(2):
        _, e11, e22, e33 = h3.component_spectra(u, g)
        b = {k: float(v) for k, v in h3.energy_budget(u, g, 6e-4, f).items()}
        runs.append((np.stack([e11, e22, e33]), b))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]
    og = orc.make_grid(N, dtype=np.float32 if dtype == torch.float32 else np.float64)
    uh = u.cpu().numpy()
    _, E, comp = orc.energy_spectrum_f64(uh, og)
    np.testing.assert_allclose(runs[0][0], np.stack(comp), rtol=1e-12, atol=1e-30)
    bo = orc.energy_budget_f64(uh, og, 6e-4, orc.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    for k in ("E", "eps", "P"):
        assert runs[0][1][k] == pytest.approx(bo[k], rel=1e-12)
