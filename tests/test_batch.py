"""Batched channels: one launch per step for channels of uneven size, wall
texture and force mode, time loop replayed from a CUDA graph (chunks of 32
steps).  Each channel must evolve exactly as the same channel stepped alone
(FP64 and FP32: identical populations; per-row partial sums make the plane
sums independent of which block owns a row)."""
import numpy as np
import pytest

import dnslbm
import inputs

pytestmark = pytest.mark.gpu

SPECS = [  # (nx, ny, nz, omega, texture, const_g)
    (40, 24, 10, 1.8, "smooth", True),
    (63, 31, 16, 1.9, "longitudinal", True),
    (26, 12, 7, 1.6, "transverse", False),
    (48, 20, 12, 1.75, "posts", True),
]


def flags_for(tex, nx, ny, nz):
    if tex == "smooth":
        return inputs.flags_smooth(nx, ny, nz)
    if tex == "longitudinal":
        return inputs.flags_longitudinal(nx, ny, nz, 3, 5)
    if tex == "transverse":
        return inputs.flags_transverse(nx, ny, nz, 2, 2)
    return inputs.flags_posts(nx, ny, nz)


def decks(prec):
    return [dnslbm.deck(nx, ny, nz, om, ubulk=0.06, gx=2e-5, force_mode=dnslbm.CONST_G if cg else dnslbm.CONST_Q,
                        precision=prec) for nx, ny, nz, om, _, cg in SPECS]


@pytest.mark.parametrize("prec", [64, 32])
def test_batch_matches_channels_stepped_alone(prec):
    states = [inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 30 + i) for i, (nx, ny, nz, *_r) in enumerate(SPECS)]
    chunks = (1, 70, 33)  # odd start, graph chunks of 32 from both parities, remainders
    with dnslbm.Batch(decks(prec)) as b:
        assert "CUDA graph" in b.kernel
        for ch, st, (nx, ny, nz, om, tex, cg) in zip(b.channels, states, SPECS):
            ch.set_flags(flags_for(tex, nx, ny, nz))
            ch.load_state(st)
        for n in chunks:
            b.step(n)
        got = [ch.store_state() for ch in b.channels]
        got_logs = [ch.logs() for ch in b.channels]
    for i, (d, st, (nx, ny, nz, om, tex, cg)) in enumerate(zip(decks(prec), states, SPECS)):
        with dnslbm.Channel(nx, ny, nz, om, ubulk=0.06, gx=2e-5, force_mode=d.force_mode, precision=prec) as ch:
            ch.set_flags(flags_for(tex, nx, ny, nz))
            ch.load_state(st)
            for n in chunks:
                ch.step(n)
            want = ch.store_state()
            want_logs = ch.logs()
        if cg:
            np.testing.assert_array_equal(got[i], want, err_msg=f"channel {i}")
        else:  # constant Q: the force may come from a differently partitioned sum
            np.testing.assert_allclose(got[i], want, rtol=1e-11 if prec == 64 else 1e-5, atol=1e-14)
        np.testing.assert_allclose(got_logs[i], want_logs, rtol=1e-9 if prec == 64 else 1e-5, atol=1e-14)


def test_batch_autotune_keeps_results():
    states = [inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 50 + i) for i, (nx, ny, nz, *_r) in enumerate(SPECS)]
    out = []
    for tune in (False, True):
        with dnslbm.Batch(decks(64)) as b:
            if tune:
                rep = b.autotune(4)
                assert "best of" in rep
            for ch, st, (nx, ny, nz, om, tex, cg) in zip(b.channels, states, SPECS):
                ch.set_flags(flags_for(tex, nx, ny, nz))
                ch.load_state(st)
            b.step(40)
            out.append([ch.store_state() for ch in b.channels])
    for i, (*_r, cg) in enumerate(SPECS):
        if cg:
            np.testing.assert_array_equal(out[0][i], out[1][i])
        else:
            np.testing.assert_allclose(out[0][i], out[1][i], rtol=1e-11, atol=1e-14)


def test_batch_refuses_mixed_precision_and_unsynchronised_channels():
    ds = decks(64)
    ds[1].precision = 32
    with pytest.raises(dnslbm.DnsLbmError):
        dnslbm.Batch(ds)
    with dnslbm.Batch(decks(64)[:2]) as b:
        for ch, (nx, ny, nz, *_r) in zip(b.channels, SPECS):
            ch.load_state(inputs.laminar_state(nx, ny, nz, 0.05, 0.1, 1))
        b.channels[0].step(1)  # channel 0 ahead by one step
        with pytest.raises(dnslbm.DnsLbmError) as e:
            b.step(2)
        assert e.value.code == dnslbm.ERR_STATE
        with pytest.raises(dnslbm.DnsLbmError) as e:
            b.autotune()  # states are loaded
        assert e.value.code == dnslbm.ERR_STATE
