"""The TMA-staged transform passes report no timed-out wait after a run (the
bounded mbarrier waits set a device flag when they give up, read and cleared
by ``hit_device_status``).  Correctness of those passes is covered by the
parity tests, which run through them."""

import ctypes

import pytest
import torch

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


@pytest.mark.parametrize("dims", [(32, 32, 32), (16, 16, 512)])
def test_wait_give_up_is_reported_and_raised(h3, dims):
    """With the wait limit at 0 polls every TMA tile wait gives up at once (the
    CTA drains its copies with the default limit and ends; the 16 x 16 x 512
    grid takes the warp-resident z pass of the 512^3 rows): the device flag is
    raised, `check_device` raises, and with the default limit restored the
    same RHS is bit-identical to the one computed before."""
    nat = h3._native
    g = h3.make_grid(*dims)
    u0 = h3.hit_initial_field(0, g)
    p = h3.NSParams(nu=0.01, forcing=h3.BandForcing(eps=0.1, kmin=1.0, kmax=2.0))
    rhs = h3.make_ns_rhs(g)
    ref = rhs(u0, p, 0.0, assume_dealiased=True)
    h3.check_device()  # starts clear
    nat.call("hit_set_wait_limit", 0)
    try:
        rhs(u0, p, 0.0, assume_dealiased=True)
        with pytest.raises(h3.DeviceWaitError):
            h3.check_device("give-up test")
    finally:
        nat.call("hit_set_wait_limit", -1)
    h3.check_device()  # read and cleared
    again = rhs(u0, p, 0.0, assume_dealiased=True)
    assert torch.equal(again, ref)
    h3.check_device()
