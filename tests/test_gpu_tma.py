"""The TMA-staged transform passes report no timed-out wait after a run (the
bounded mbarrier waits set a device flag when they give up, read and cleared
by ``hit_device_status``).  Correctness of those passes is covered by the
parity tests, which run through them."""

import ctypes

import pytest

pytestmark = pytest.mark.gpu


def test_transform_waits_never_gave_up(h3):
    nat = h3._native
    for n, dealiased in ((64, True), (32, False)):
        g = h3.make_grid(n)
        u0 = h3.hit_initial_field(0, g)
        p = h3.NSParams(nu=0.01, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
        h3.rollout(h3.make_ns_rhs(g), u0, p, 1e-3, 3, assume_dealiased=dealiased)
        h3.to_spectral(h3.to_physical(u0, g), g)
    st = ctypes.c_int(-1)
    nat.call("hit_device_status", ctypes.byref(st))
    assert st.value == 0
