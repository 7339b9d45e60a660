"""Failure detection without a GPU fault: every device-side wait in the
library is bounded.  Each probe waits on a condition nothing satisfies; the
wait must give up, the host must read ASD_ERR_TIMEOUT, and the device and the
library must stay usable afterwards."""
from __future__ import annotations

import pytest

import asd_b200 as asd

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_reports_timeout_and_recovers(which):
    lib = asd.load()
    rc = lib.asd_check_bounded_wait(which, 1 << 14, None)
    assert rc == asd.ASD_ERR_TIMEOUT, asd.last_error()
    # the context is intact: a normal S(q,t) evaluation works afterwards
    N, nf = 16, 4
    with asd.Context(asd.Params.make(N, nf)) as ctx:
        ctx.set_spins(asd.random_spins(N, nf, seed=1), as_origin=True)
        ctx.step(2)
        v = ctx.sqt("bf16x3")
        ctx.check_device_status()
    assert abs(v) > 0


def test_status_word_is_clear_after_normal_work():
    N, nf = 32, 8
    with asd.Context(asd.Params.make(N, nf)) as ctx:
        ctx.set_spins(asd.random_spins(N, nf, seed=2), as_origin=True)
        for mode in ("tf32x3", "bf16x3", "fp64"):
            ctx.sqt(mode)
        ctx.check_device_status()  # raises on a recorded timeout
