"""Bounded device waits of the row-pipelined step kernel.

Every mbarrier wait of the bulk-copy kernel gives up after a limit on the
GPU's global timer.  The test hook dnslbm_test_withhold_load makes one block
withhold the load of its first row group, so its consumers wait for data that
never comes; with a 1 ms limit the step call must come back promptly with
DNSLBM_ERR_TIMEOUT (no fault, no hang, no copy left in flight), refuse to step
the invalid state, and step a reloaded state exactly as before.  The failure
is made on the host side of the kernel (a load that is never issued), never by
a fault of the GPU.
"""
import time

import numpy as np
import pytest

import dnslbm
import inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [64, 32, 16])
def test_withheld_load_times_out_and_context_recovers(oracle_mod, prec):
    nx, ny, nz, omega, gx = 40, 16, 10, 1.7, 2e-5
    fl = inputs.flags_smooth(nx, ny, nz)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 31)
    with dnslbm.Channel(nx, ny, nz, omega, gx=gx, force_mode=dnslbm.CONST_G, precision=prec) as ch:
        assert "bulk-copy" in ch.kernel
        ch.set_flags(fl)
        ch.load_state(s0)
        ch.step(2)
        ch.set_wait_limit(1.0)
        ch.test_withhold_load()
        t0 = time.perf_counter()
        with pytest.raises(dnslbm.DnsLbmError) as e:
            ch.step(1)
        elapsed = time.perf_counter() - t0
        assert e.value.code == dnslbm.ERR_TIMEOUT, str(e.value)
        assert elapsed < 5.0, elapsed
        with pytest.raises(dnslbm.DnsLbmError) as e:
            ch.step(1)  # the state is invalid until it is reloaded
        assert e.value.code == dnslbm.ERR_STATE
        ch.set_wait_limit(1000.0)
        ch.load_state(s0)
        ch.step(6)
        got = ch.store_state()
    ref = s0.copy()
    oracle_mod.run(ref, fl, omega, gx=gx, const_g=True, nsteps=6)
    if prec == 64:
        np.testing.assert_array_equal(got, ref)
    else:
        np.testing.assert_allclose(got, ref, rtol=0, atol={32: 1e-6, 16: 2e-4}[prec])


def test_wait_limit_is_validated():
    with dnslbm.Channel(16, 8, 6, 1.5, gx=1e-5, force_mode=dnslbm.CONST_G) as ch:
        for bad in (0.0, -1.0, 1e9):
            with pytest.raises(dnslbm.DnsLbmError) as e:
                ch.set_wait_limit(bad)
            assert e.value.code == dnslbm.ERR_ARG
