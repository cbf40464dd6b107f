"""Quadrant analysis (quadrant-analysis/src/qUADrantA.c) on the GPU.

The golden fixtures hold the reference's own qUADrantA run on the velocity
field of a stepped channel (tests/golden/make_golden.py, oracle/_ref/quadref);
the field itself is regenerated from its seed with the oracle (which
reproduces the reference's step bit for bit).  The numpy restatement is
pinned to the fixtures on the CPU; the GPU kernels are checked against them
on the live state of a channel stepped on the GPU, on an uploaded vel field,
and through run-dns (QUADRANT 1).  The GPU sums run in a different order
from the reference's sequential loops: plane sums and means agree to
rounding (1e-10 relative), and the conditional means also to 1e-9, as no
fluctuation of these fields lies within rounding of zero.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

import inputs

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CASES = sorted(glob.glob(os.path.join(HERE, "golden", "quadrant_*.npz")))
RUN_DNS = os.path.join(ROOT, "dns-solvers_b200", "run-dns")


def field(oracle_mod, g):
    nx, ny, nz = (int(v) for v in g["dims"])
    st = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, int(g["seed"]))
    s0 = st.copy()
    oracle_mod.run(st, inputs.flags_smooth(nx, ny, nz), 1.7, gx=2e-5, const_g=True, nsteps=int(g["steps"]))
    return s0, st, oracle_mod.moments(st)[0]


def check(got, g, rtol_q=1e-9):
    q, dq, uw = got
    np.testing.assert_allclose(q, g["quadrant"], rtol=rtol_q, atol=1e-20)
    np.testing.assert_allclose(dq, g["dquadrant"], rtol=1e-10, atol=1e-20)
    np.testing.assert_allclose(uw, g["uw"], rtol=1e-10, atol=1e-20)


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_restatement_matches_reference_golden(oracle_mod, path):
    g = np.load(path)
    _, _, vel = field(oracle_mod, g)
    check(oracle_mod.quadrant(vel), g, rtol_q=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_gpu_quadrant_of_the_live_state(oracle_mod, path):
    import dnslbm
    g = np.load(path)
    nx, ny, nz = (int(v) for v in g["dims"])
    s0, _, vel = field(oracle_mod, g)
    with dnslbm.Channel(nx, ny, nz, 1.7, gx=2e-5, force_mode=dnslbm.CONST_G) as ch:
        ch.load_state(s0)
        ch.step(int(g["steps"]))
        check(ch.quadrant(), g)
    check(dnslbm.quadrant_vel(vel), g)


@pytest.mark.gpu
def test_run_dns_writes_quadrant_files(oracle_mod, tmp_path):
    """run-dns -p from a perturbed field with QUADRANT 1: the quadrant files
    of every output event against the restatement on that event's vel file."""
    d = str(tmp_path)
    nx, ny, nz = 16, 8, 6
    with open(os.path.join(d, "deck.txt"), "w") as f:
        f.write(f"xdv {nx}\nydv {ny}\nzdv {nz}\nRebs 100\nub 0.1\nCFL 0.1\nTSTR 4\nTEND 9\nITER 61\n"
                "QUADRANT 1\nFORCE g\nGX 2e-5\n")
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, 9)
    np.concatenate([s0.ravel(), s0.ravel()]).tofile(os.path.join(d, "lbf.0004"))
    subprocess.run([RUN_DNS, "-p", "deck.txt"], cwd=d, check=True, timeout=120, capture_output=True)
    zd = nz + 2
    for label in (4, 5, 6):
        vel = np.fromfile(os.path.join(d, f"vel.{label:04d}")).reshape(nx, ny, zd, 3)
        q, dq, uw = oracle_mod.quadrant(vel)
        a = np.fromfile(os.path.join(d, f"quadrant.000.{label:04d}"))
        b = np.fromfile(os.path.join(d, f"dquadrant.000.{label:04d}"))
        np.testing.assert_allclose(a[:4 * zd].reshape(4, zd), q, rtol=1e-9, atol=1e-20)
        np.testing.assert_allclose(b[:4 * zd].reshape(4, zd), dq, rtol=1e-10, atol=1e-20)
        np.testing.assert_allclose(a[4 * zd:], uw, rtol=1e-10, atol=1e-20)
        np.testing.assert_array_equal(a[4 * zd:], b[4 * zd:])
