"""State loading in x-slabs (dnslbm_load_state_slab), the per-rank lbf read
of the reference (dns-const-q-xycut.c:405-416): uneven slabs give the same
state as one dnslbm_load_state, slabs out of order are refused, and a
partly loaded state cannot be stepped.  Also the slab generator of large
synthetic fields against the whole-field one."""
import numpy as np
import pytest

import dnslbm
import inputs


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [64, 16])
def test_slabs_equal_whole_load(prec):
    nx, ny, nz = 23, 9, 7
    s0 = inputs.laminar_state(nx, ny, nz, 0.07, 0.1, 4)
    out = []
    for slabs in (None, [(0, 5), (5, 1), (6, 17)]):
        with dnslbm.Channel(nx, ny, nz, 1.7, gx=1e-5, precision=prec) as ch:
            ch.set_flags(inputs.flags_posts(nx, ny, nz))
            if slabs is None:
                ch.load_state(s0)
            else:
                ch.load_state_slabs((x0, s0[x0:x0 + n]) for x0, n in slabs)
            ch.step(3)
            out.append((ch.store_state(), ch.logs()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


@pytest.mark.gpu
def test_slab_order_and_partial_state_are_checked():
    nx, ny, nz = 12, 6, 5
    s0 = inputs.laminar_state(nx, ny, nz, 0.07, 0.1, 5)
    with dnslbm.Channel(nx, ny, nz, 1.7) as ch:
        ch.load_state_slab(0, s0[:4])
        with pytest.raises(dnslbm.DnsLbmError) as e:
            ch.load_state_slab(6, s0[6:8])  # a gap
        assert e.value.code == dnslbm.ERR_STATE
        with pytest.raises(dnslbm.DnsLbmError) as e:
            ch.step(1)  # partial state
        assert e.value.code == dnslbm.ERR_STATE
        with pytest.raises(dnslbm.DnsLbmError) as e:
            ch.load_state_slab(10, s0[:4])  # beyond the grid
        assert e.value.code == dnslbm.ERR_ARG
        ch.load_state_slab(4, s0[4:])
        ch.step(1)


def test_turbulent_slabs_match_whole_field():
    nx, ny, nz = 30, 14, 10
    whole = inputs.turbulent_state(nx, ny, nz, 0.07, 0.1, 8)
    parts = np.concatenate([s for _, s in inputs.turbulent_slabs(nx, ny, nz, 0.07, 0.1, 8, slab=7)])
    np.testing.assert_allclose(parts, whole, rtol=1e-13, atol=1e-16)
