"""The oracle's general boundary rule (bc_mode=1, lbm_oracle.c orc_step_ab)
on the CPU: solids inside the flow are beyond the reference, so besides the
GPU-vs-oracle parity tests the rule itself is checked here.
  * With no interior solid it is the reference rule (bc_mode=0) bit for bit.
  * With omega = 0 and no force a step is pure streaming: every population
    of a fluid cell lands in exactly one fluid slot, so the multiset of
    fluid populations is unchanged (no population lost or duplicated), for
    riblets and for blocks standing on slip-grooved walls.
  * Mass is conserved over many collide-and-stream steps, and solid cells
    keep their rest populations.
  * The per-cell link masks the library builds on the host
    (dnslbm_link_masks, used by dnslbm_set_flags) follow the same rule,
    written once more in numpy here."""
import numpy as np
import pytest

import inputs


def blocks_on_grooves(nx, ny, nz, seed):
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


def fluid(flags):
    return flags[:, :, 1:-1] != -1


def test_general_rule_without_solids_is_reference_rule(oracle_mod):
    nx, ny, nz = 18, 11, 9
    for fl in (inputs.flags_posts(nx, ny, nz), inputs.flags_transverse(nx, ny, nz, 2, 3)):
        s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 2)
        a, b = s0.copy(), s0.copy()
        oracle_mod.run(a, fl, 1.7, gx=3e-5, const_g=True, nsteps=5, bc_mode=0)
        oracle_mod.run(b, fl, 1.7, gx=3e-5, const_g=True, nsteps=5, bc_mode=1)
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("kind", ["riblets", "blocks"])
def test_streaming_is_a_permutation(oracle_mod, kind):
    nx, ny, nz = 20, 16, 12
    fl = inputs.flags_riblets(nx, ny, nz, 4, 8) if kind == "riblets" else blocks_on_grooves(nx, ny, nz, 5)
    rng = np.random.default_rng(9)
    st = np.zeros((nx, ny, nz + 2, 19))
    st[:, :, 1:-1] = rng.random((nx, ny, nz, 19))  # distinct values everywhere
    st = inputs.rest_solids(st, fl)
    before = np.sort(st[:, :, 1:-1][fluid(fl)].ravel())
    oracle_mod.step(st, fl, 0.0, 0.0, bc_mode=1)  # omega 0, no force: streaming only
    after = np.sort(st[:, :, 1:-1][fluid(fl)].ravel())
    np.testing.assert_array_equal(before, after)


@pytest.mark.parametrize("kind", ["riblets", "blocks"])
def test_mass_conserved_and_solids_at_rest(oracle_mod, kind):
    nx, ny, nz = 20, 16, 12
    fl = inputs.flags_riblets(nx, ny, nz, 4, 8) if kind == "riblets" else blocks_on_grooves(nx, ny, nz, 6)
    st = inputs.rest_solids(inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 4), fl)
    m0 = st[:, :, 1:-1].sum()
    oracle_mod.run(st, fl, 1.8, gx=3e-5, const_g=True, nsteps=30, bc_mode=1)
    assert abs(st[:, :, 1:-1].sum() - m0) < 1e-11 * m0
    assert np.all(st[:, :, 1:-1][~fluid(fl)] == inputs.W)


def link_masks_restated(flags):
    """The general wall rule, written once more in numpy: for every fluid
    cell of a plane within one plane of a solid, bit A set when the link in
    direction A bounces back (lbm_oracle.c orc_step_ab, bc_mode 1)."""
    nx, ny, zd = flags.shape
    nz = zd - 2
    solid = (flags[:, :, 1:-1] == -1).any(axis=(0, 1))
    band = -np.ones(nz, int)
    nb = 0
    for z in range(nz):
        if solid[max(z - 1, 0):z + 2].any():
            band[z] = nb
            nb += 1
    E = inputs.E.astype(int)
    out = np.zeros((nb, ny, nx), np.uint32)
    X, Y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    for z in range(nz):
        if band[z] < 0:
            continue
        k = z + 1
        v = np.zeros((nx, ny), np.uint32)
        for a in range(1, 19):
            xt, yt, kt = (X + E[a, 0]) % nx, (Y + E[a, 1]) % ny, k + E[a, 2]
            sld, sld1, sdest = flags[xt, yt, kt], flags[X, Y, kt], flags[xt, yt, k]
            spec = ((sld == -1) & (sld1 == -2)) | (sld == -2)
            bounce = np.where(sld > -1, False, np.where((sld == -1) & (sld1 == -1), True,
                                                         np.where(spec, sdest == -1, True)))
            v |= (bounce.astype(np.uint32) << a)
        v[flags[:, :, k] == -1] = 1
        out[band[z]] = v.T
    return band, out


@pytest.mark.parametrize("kind", ["riblets", "blocks", "grooves only"])
def test_library_link_masks_follow_the_rule(kind):
    import dnslbm
    nx, ny, nz = 20, 16, 12
    fl = {"riblets": lambda: inputs.flags_riblets(nx, ny, nz, 4, 8),
          "blocks": lambda: blocks_on_grooves(nx, ny, nz, 5),
          "grooves only": lambda: inputs.flags_longitudinal(nx, ny, nz, 3, 3)}[kind]()
    band, links = dnslbm.link_masks(fl)
    rband, rlinks = link_masks_restated(fl)
    np.testing.assert_array_equal(band, rband)
    np.testing.assert_array_equal(links, rlinks)
    if kind == "grooves only":
        assert links.size == 0
    else:
        with pytest.raises(dnslbm.DnsLbmError) as e:
            dnslbm.link_masks(fl, bc_mode=dnslbm.BC_REFERENCE)
        assert "DNSLBM_BC_GENERAL" in str(e.value)
