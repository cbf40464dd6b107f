"""Pin the CPU oracle (oracle/lbm_oracle.c) to the reference.

The goldens in tests/golden/ were produced by the reference's own step
functions (tests/golden/make_golden.py).  The restatement must reproduce the
reference's populations, force and density bit for bit, its statistics
(turb-fld) and vel/den outputs bit for bit, and its text logs to their print
precision (%.12f / %.14f, i.e. 5e-13 absolute).
"""
import glob
import os

import numpy as np
import pytest

import inputs

# step goldens (the quadrant-analysis fixtures are tests/test_quadrant.py's)
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("quadrant_", "correl_")))
LOG_COLS = ("energy", "flowrate", "massrate", "stup", "stdown", "stress", "pgrad")


def golden_case(path):
    g = np.load(path)
    nx, ny, nz = (int(v) for v in g["dims"])
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, int(g["seed"]))
    return g, (nx, ny, nz), s0


def oracle_flags(oracle, tex, nx, ny, nz):
    return oracle.flags(tex, nx, ny, nz)  # reference rules: ridges gap=width=2, posts 2x2 period 4


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_matches_reference_golden(oracle_mod, path):
    g, (nx, ny, nz), s0 = golden_case(path)
    steps = int(g["steps"])
    fl = oracle_flags(oracle_mod, str(g["texture"]), nx, ny, nz)
    st = s0.copy()
    # run steps-1 steps, check stats/vel/den there (the reference writes them
    # before the last step), then the last step
    logs = oracle_mod.run(st, fl, float(g["omega"]), float(g["ubulk"]), float(g["gx"]), bool(g["const_g"]), steps - 1)
    np.testing.assert_array_equal(oracle_mod.statistics(st), g["stats_last"])
    vel, den = oracle_mod.moments(st)
    np.testing.assert_array_equal(vel, g["vel_last"])
    np.testing.assert_array_equal(den, g["den_last"])
    last = oracle_mod.run(st, fl, float(g["omega"]), float(g["ubulk"]), float(g["gx"]), bool(g["const_g"]), 1)
    logs = np.concatenate([logs, last])
    np.testing.assert_array_equal(st, g["state"])  # bit-exact populations
    np.testing.assert_array_equal(logs[:, 0], g["force"])
    np.testing.assert_array_equal(logs[:, 1], g["rho"])
    np.testing.assert_allclose(logs[:, 2:], g["logs"], rtol=0, atol=5.1e-13)


def test_oracle_initial_statistics_golden(oracle_mod):
    g, (nx, ny, nz), s0 = golden_case(GOLDEN[0])
    np.testing.assert_array_equal(oracle_mod.statistics(s0), g["stats_first"])


@pytest.mark.parametrize("kind,kw", [("ridges", dict(gap=2, width=2)), ("transverse", dict(gap=3, width=5)),
                                     ("posts", dict(gx=2, wx=2, gy=2, wy=2))])
def test_product_flags_match_oracle_flags(oracle_mod, kind, kw):
    nx, ny, nz = 16, 12, 5
    ref = oracle_mod.flags(kind, nx, ny, nz, **kw)
    if kind == "ridges":
        mine = inputs.flags_longitudinal(nx, ny, nz, kw["gap"], kw["width"])
    elif kind == "transverse":
        mine = inputs.flags_transverse(nx, ny, nz, kw["gap"], kw["width"])
    else:
        mine = inputs.flags_posts(nx, ny, nz, **kw)
    np.testing.assert_array_equal(mine, ref)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref", "dnsref")),
                    reason="reference build not present")
@pytest.mark.parametrize("tex,cg,dims", [("file", True, (10, 9, 7)), ("file", False, (7, 11, 6))])
def test_oracle_matches_reference_transverse_and_odd_sizes(oracle_mod, tex, cg, dims):
    """Grids and textures the goldens do not cover (odd sizes, transverse
    grooves given to the reference as an explicit flag array)."""
    nx, ny, nz = dims
    fl = inputs.flags_transverse(nx, ny, nz, 2, 3)
    s0 = inputs.laminar_state(nx, ny, nz, 0.07, 0.05, 11)
    r = oracle_mod.run_reference(s0, 1.6, ubulk=0.05, gx=1e-5, const_g=cg, nsteps=13, flags_periodic=fl)
    st = s0.copy()
    logs = oracle_mod.run(st, fl, 1.6, 0.05, 1e-5, cg, 13)
    np.testing.assert_array_equal(st, r["state"])
    np.testing.assert_array_equal(logs[:, 0], r["force"])


def test_oracle_invariants(oracle_mod):
    """Mass is conserved exactly in exact arithmetic by collision and by every
    wall rule; the per-cell momentum gain of the forcing is g."""
    nx, ny, nz = 8, 8, 6
    fl = inputs.flags_posts(nx, ny, nz)
    s = inputs.laminar_state(nx, ny, nz, 0.05, 0.05, 3)
    m0 = s.sum()
    oracle_mod.run(s, fl, 1.3, 0.0, 1e-4, True, 10)
    assert abs(s.sum() - m0) < 1e-12 * m0
