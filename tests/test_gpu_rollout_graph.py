"""The rollout as one CUDA graph with a device-side while loop
(`hit_rollout`, reference `rollout`, src/hit3d/integrators.py:41-53): one
instantiated graph serves every step count, the loop count living in device
memory (a single step is enqueued without the graph, whose conditional node
would hide its kernels from per-kernel profilers).  Rollouts of 1, 4, 2 and
7 steps on the same plan, one after the other, must equal the same number
of one-step rollouts (to float32 rounding:
a one-step rollout starts from the state's own x-inverse and forcing sums,
a longer one from those its previous step fused; a step too many or too few
moves the state by ~1e-3), and a 6-step rollout must match the oracle."""

import numpy as np
import pytest
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dealiased", [True, False])
def test_rollout_graph_reuse_matches_single_steps(h3, dealiased):
    g = h3.make_grid(32)
    u0 = h3.hit_initial_field(0, g)
    p = h3.NSParams(nu=0.01, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    rhs = h3.make_ns_rhs(g)
    dt = 2e-3
    u = u0
    for n in (1, 4, 2, 7):
        got = h3.rollout(rhs, u, p, dt, n, assume_dealiased=dealiased)
        ref = u
        for _ in range(n):
            ref = h3.rollout(rhs, ref, p, dt, 1, assume_dealiased=dealiased)
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < 2e-6, n
        u = got
    h3.check_device("rollout graph")


def test_rollout_graph_matches_oracle(h3, orc):
    og = orc.make_grid(32, dtype=np.float32)
    u0 = orc.hit_initial_field(1, og)
    g = h3.make_grid(32)
    p = h3.NSParams(nu=0.02, forcing=h3.LinearForcing(0.1))
    po = orc.NSParams(nu=0.02, forcing=orc.LinearForcing(0.1))
    got = h3.rollout(h3.make_ns_rhs(g), u0, p, 2e-3, 6).cpu().numpy()
    ref = orc.rollout(orc.make_ns_rhs(og), u0, po, 2e-3, 6)
    assert rel_l2(got, ref) < 1e-5
