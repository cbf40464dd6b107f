"""Batched channels of uneven size, wall texture and force mode, advanced by
the persistent kernel (one cooperative launch per 32 steps, replayed from a
CUDA graph; blocks take items of work from a per-step counter) or by one
launch per step (DNSLBM_BATCH=launch).  Each channel must evolve exactly as
the same channel stepped alone (FP64 and FP32 with a constant force:
identical populations; each item sums into its own slot of its plane, so the
plane sums do not depend on which block took it)."""
import os

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


@pytest.fixture(params=["persistent", "launch"])
def batch_mode(request):
    old = os.environ.get("DNSLBM_BATCH")
    if request.param == "launch":
        os.environ["DNSLBM_BATCH"] = "launch"
    else:
        os.environ.pop("DNSLBM_BATCH", None)
    yield request.param
    if old is None:
        os.environ.pop("DNSLBM_BATCH", None)
    else:
        os.environ["DNSLBM_BATCH"] = old


@pytest.mark.parametrize("prec", [64, 32])
def test_batch_matches_channels_stepped_alone(prec, batch_mode):
    states = [inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 30 + i) for i, (nx, ny, nz, *_r) in enumerate(SPECS)]
    chunks = (1, 70, 33)  # odd start, graph chunks of 32 from both parities, remainders
    with dnslbm.Batch(decks(prec)) as b:
        assert "CUDA graph" in b.kernel
        assert ("persist_batch_kernel" in b.kernel) == (batch_mode == "persistent"), b.kernel
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


@pytest.mark.parametrize("prec", [64, 16])
def test_batch_with_riblets_matches_channels_stepped_alone(prec, batch_mode):
    """Channels with solids inside the flow (planes stepped per cell) beside
    smooth and grooved ones; constant force: identical populations."""
    specs = [(40, 24, 12, 1.8, "riblets"), (33, 16, 10, 1.7, "longitudinal"), (26, 12, 7, 1.6, "smooth")]

    def fl(tex, nx, ny, nz):
        return inputs.flags_riblets(nx, ny, nz, 3, 6) if tex == "riblets" else flags_for(tex, nx, ny, nz)

    ds = [dnslbm.deck(nx, ny, nz, om, gx=2e-5, force_mode=dnslbm.CONST_G, precision=prec,
                      bc_mode=dnslbm.BC_GENERAL if tex == "riblets" else dnslbm.BC_REFERENCE)
          for nx, ny, nz, om, tex in specs]
    states = [inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 60 + i) for i, (nx, ny, nz, *_r) in enumerate(specs)]
    states = [inputs.rest_solids(st, fl(sp[4], *sp[:3])) for st, sp in zip(states, specs)]
    with dnslbm.Batch(ds) as b:
        for ch, st, (nx, ny, nz, om, tex) in zip(b.channels, states, specs):
            ch.set_flags(fl(tex, nx, ny, nz))
            ch.load_state(st)
        b.step(37)
        got = [ch.store_state() for ch in b.channels]
    for i, (d, st, (nx, ny, nz, om, tex)) in enumerate(zip(ds, states, specs)):
        with dnslbm.Channel(nx, ny, nz, om, gx=2e-5, force_mode=dnslbm.CONST_G, precision=prec,
                            bc_mode=d.bc_mode) as ch:
            ch.set_flags(fl(tex, nx, ny, nz))
            ch.load_state(st)
            ch.step(37)
            np.testing.assert_array_equal(got[i], ch.store_state(), err_msg=f"channel {i} ({tex})")


def test_persistent_batch_wait_runs_out_and_recovers():
    """A withheld load in the persistent kernel: the bounded wait gives up,
    the batch reports ERR_TIMEOUT without hanging, and a reloaded batch steps
    as before."""
    os.environ.pop("DNSLBM_BATCH", None)
    states = [inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 70 + i) for i, (nx, ny, nz, *_r) in enumerate(SPECS)]
    with dnslbm.Batch(decks(64)) as b:
        for ch, st, (nx, ny, nz, om, tex, cg) in zip(b.channels, states, SPECS):
            ch.set_flags(flags_for(tex, nx, ny, nz))
            ch.load_state(st)
        b.step(3)
        b.test_withhold_load(1.0)
        with pytest.raises(dnslbm.DnsLbmError) as e:
            b.step(5)
        assert e.value.code == dnslbm.ERR_TIMEOUT, str(e.value)
        with pytest.raises(dnslbm.DnsLbmError) as e:
            b.step(1)  # the states are invalid until reloaded
        assert e.value.code == dnslbm.ERR_STATE
        for ch, st in zip(b.channels, states):
            ch.load_state(st)
        b.step(40)
        got = [ch.store_state() for ch in b.channels]
    for i, (d, st, (nx, ny, nz, om, tex, cg)) in enumerate(zip(decks(64), states, SPECS)):
        if not cg:
            continue
        with dnslbm.Channel(nx, ny, nz, om, gx=2e-5, force_mode=d.force_mode) as ch:
            ch.set_flags(flags_for(tex, nx, ny, nz))
            ch.load_state(st)
            ch.step(40)
            np.testing.assert_array_equal(got[i], ch.store_state(), err_msg=f"channel {i}")
