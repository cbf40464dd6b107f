"""Solids inside the flow (boundary mode DNSLBM_BC_GENERAL): riblets cut into
the walls, solid blocks on slip (grooved) walls and blocks floating in the
channel, against the oracle's general rule (bc_mode=1, lbm_oracle.c
orc_step_ab): bounce-back on every link into a solid, the reference's wall
rule otherwise, and bounce-back where a specular reflection would land on a
solid cell.

The reference itself cannot express a solid inside the flow; its own wall
rule is pinned by the reference-mode tests, and on flags without interior
solids the general mode gives the reference mode's populations bit for bit
(test_general_mode_without_solids_is_reference_mode).

FP64 populations must equal the oracle's bit for bit after odd and even step
counts (both AA parities, read back through store_state); per-step logs to
1e-9 relative (plane sums in a different order).  Solid cells hold the rest
state f = w in both codes.
"""
import numpy as np
import pytest

import dnslbm
import inputs

pytestmark = pytest.mark.gpu

OMEGA, GX = 1.85, 3e-5


def blocks_on_grooves(nx, ny, nz, seed):
    """Longitudinal slip grooves on both walls plus seeded solid blocks: some
    standing on a wall (next to slip cells), some floating."""
    rng = np.random.default_rng(seed)
    f = inputs.flags_longitudinal(nx, ny, nz, 3, 3)
    for _ in range(6):
        bx, by, bz = (int(rng.integers(1, 4)) for _ in range(3))
        x0, y0 = int(rng.integers(nx)), int(rng.integers(ny))
        z0 = int(rng.choice([1, nz + 1 - bz, int(rng.integers(2, nz - bz))]))
        for i in range(bx):
            for j in range(by):
                f[(x0 + i) % nx, (y0 + j) % ny, z0:z0 + bz] = -1
    return f


CASES = {
    "riblets": (24, 16, 14, lambda nx, ny, nz: inputs.flags_riblets(nx, ny, nz, 4, 8)),
    "riblets_cut_at_seam": (20, 18, 16, lambda nx, ny, nz: inputs.flags_riblets(nx, ny, nz, 5, 10)),
    "blocks_on_grooves": (22, 15, 12, lambda nx, ny, nz: blocks_on_grooves(nx, ny, nz, 7)),
}


def case_state(name, seed=11):
    nx, ny, nz, mk = CASES[name]
    flags = mk(nx, ny, nz)
    s0 = inputs.rest_solids(inputs.laminar_state(nx, ny, nz, 0.08, 0.1, seed), flags)
    return nx, ny, nz, flags, s0


def solid_cells(state, flags):
    nz = flags.shape[2] - 2
    return state[:, :, 1:nz + 1][flags[:, :, 1:nz + 1] == -1]


def channel(nx, ny, nz, prec=64, const_q=False):
    return dnslbm.Channel(nx, ny, nz, OMEGA, ubulk=0.05, gx=GX,
                          force_mode=dnslbm.CONST_Q if const_q else dnslbm.CONST_G, precision=prec,
                          bc_mode=dnslbm.BC_GENERAL)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("nsteps", [1, 6, 9])
def test_fp64_matches_oracle(oracle_mod, name, nsteps):
    nx, ny, nz, flags, s0 = case_state(name)
    want = s0.copy()
    want_logs = oracle_mod.run(want, flags, OMEGA, gx=GX, const_g=True, nsteps=nsteps, bc_mode=1)
    with channel(nx, ny, nz) as ch:
        ch.set_flags(flags)
        ch.load_state(s0)
        ch.step(nsteps)
        got = ch.store_state()
        logs = ch.logs()
        stats = ch.statistics()
        vel, den = ch.moments()
    np.testing.assert_array_equal(got, want)
    np.testing.assert_allclose(logs, want_logs, rtol=1e-9, atol=1e-13)
    np.testing.assert_allclose(stats, oracle_mod.statistics(want), rtol=1e-9, atol=1e-13)
    rvel, rden = oracle_mod.moments(want)
    np.testing.assert_array_equal(vel, rvel)
    np.testing.assert_array_equal(den, rden)


def test_solid_cells_stay_at_rest_and_mass_is_conserved():
    nx, ny, nz, flags, s0 = case_state("riblets")
    with channel(nx, ny, nz) as ch:
        ch.set_flags(flags)
        noisy = s0.copy()
        noisy[:, :, 1:nz + 1][flags[:, :, 1:nz + 1] == -1] += 0.01  # solids are reset to rest on load
        ch.load_state(noisy)
        m0 = ch.store_state()[:, :, 1:nz + 1].sum()
        ch.step(25)
        got = ch.store_state()
    assert np.all(solid_cells(got, flags) == inputs.W)
    assert abs(got[:, :, 1:nz + 1].sum() - m0) < 1e-9 * m0


def test_const_q_with_riblets(oracle_mod):
    nx, ny, nz, flags, s0 = case_state("riblets", seed=4)
    want = s0.copy()
    want_logs = oracle_mod.run(want, flags, OMEGA, ubulk=0.05, const_g=False, nsteps=8, bc_mode=1)
    with channel(nx, ny, nz, const_q=True) as ch:
        ch.set_flags(flags)
        ch.load_state(s0)
        ch.step(8)
        got = ch.store_state()
        logs = ch.logs()
    # the force is a sum over the grid taken in another order
    np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(logs, want_logs, rtol=1e-8, atol=1e-13)


def test_general_mode_without_solids_is_reference_mode(oracle_mod):
    nx, ny, nz = 20, 12, 10
    flags = inputs.flags_posts(nx, ny, nz)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 3)
    want = s0.copy()
    oracle_mod.run(want, flags, OMEGA, gx=GX, const_g=True, nsteps=7, bc_mode=0)
    with channel(nx, ny, nz) as ch:
        ch.set_flags(flags)
        ch.load_state(s0)
        ch.step(7)
        np.testing.assert_array_equal(ch.store_state(), want)


@pytest.mark.parametrize("prec,bound", [(32, 5e-7), (16, 2e-4)])
def test_low_precision_error_vs_oracle(oracle_mod, prec, bound):
    """Per-population error after 10 steps, relative to the largest
    population (the bounds of the smooth-wall precision tests)."""
    nx, ny, nz, flags, s0 = case_state("blocks_on_grooves")
    want = s0.copy()
    oracle_mod.run(want, flags, OMEGA, gx=GX, const_g=True, nsteps=10, bc_mode=1)
    with channel(nx, ny, nz, prec=prec) as ch:
        ch.set_flags(flags)
        ch.load_state(s0)
        ch.step(10)
        got = ch.store_state()
    err = np.max(np.abs(got - want)) / np.max(np.abs(want))
    assert err < bound, err
    assert np.all(solid_cells(got, flags) == inputs.W)


def test_scalar_and_row_pipelined_paths_agree(monkeypatch):
    nx, ny, nz, flags, s0 = case_state("riblets_cut_at_seam")
    out = []
    for path in ("scalar", None):
        if path:
            monkeypatch.setenv("DNSLBM_PATH", path)
        else:
            monkeypatch.delenv("DNSLBM_PATH", raising=False)
        with channel(nx, ny, nz) as ch:
            ch.set_flags(flags)
            ch.load_state(s0)
            ch.step(5)
            out.append(ch.store_state())
    np.testing.assert_array_equal(out[0], out[1])


def test_interior_solids_need_general_mode():
    nx, ny, nz, flags, s0 = case_state("riblets")
    with dnslbm.Channel(nx, ny, nz, OMEGA, gx=GX) as ch:
        with pytest.raises(dnslbm.DnsLbmError) as e:
            ch.set_flags(flags)
        assert e.value.code == dnslbm.ERR_ARG and "DNSLBM_BC_GENERAL" in str(e.value)
    bad = flags.copy()
    bad[3, 3, 5] = -2  # a slip cell inside the flow has no meaning
    with channel(nx, ny, nz) as ch:
        with pytest.raises(dnslbm.DnsLbmError):
            ch.set_flags(bad)


def test_batch_with_riblet_channel():
    nx, ny, nz, flags, s0 = case_state("riblets")
    nx2, ny2, nz2, flags2, s2 = case_state("blocks_on_grooves")
    fl3, s3 = inputs.flags_smooth(30, 12, 10), inputs.laminar_state(30, 12, 10, 0.08, 0.1, 9)
    ds = [dnslbm.deck(nx, ny, nz, OMEGA, gx=GX, bc_mode=dnslbm.BC_GENERAL),
          dnslbm.deck(nx2, ny2, nz2, OMEGA, gx=GX, bc_mode=dnslbm.BC_GENERAL),
          dnslbm.deck(30, 12, 10, OMEGA, gx=GX)]
    fls, sts = (flags, flags2, fl3), (s0, s2, s3)
    with dnslbm.Batch(ds) as b:
        for ch, fl, st in zip(b.channels, fls, sts):
            ch.set_flags(fl)
            ch.load_state(st)
        b.step(37)
        got = [ch.store_state() for ch in b.channels]
    for i, (fl, st, d) in enumerate(zip(fls, sts, ds)):
        with dnslbm.Channel(d.xdv, d.ydv, d.zdv, OMEGA, gx=GX, bc_mode=d.bc_mode) as ch:
            ch.set_flags(fl)
            ch.load_state(st)
            ch.step(37)
            np.testing.assert_array_equal(got[i], ch.store_state(), err_msg=f"channel {i}")
