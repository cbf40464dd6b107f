"""run-dns, the C host driver over the C ABI (dns-solvers_b200/host), against
the oracle: every output file of the reference's main loop
(dns-const-q-xycut.c:485-519) in the reference's format.

Deck: 16 x 8 x 4 fluid cells, Rebs 100, ub 0.1, CFL 0.1 -> utime = 20,
ITER 45 -> 46 steps; vel/den/turb-fld at steps 0, 20, 40, lbf/force at 0.
Text logs are compared to their printed precision; binary outputs to 1e-10
relative (constant Q: the force comes from a differently ordered sum), with
an absolute floor of 1e-13 for statistics entries that are round-off (plane
means of v and w of order 1e-17).
"""
import os
import subprocess

import numpy as np
import pytest

import inputs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUN_DNS = os.path.join(ROOT, "dns-solvers_b200", "run-dns")
NX, NY, NZ = 16, 8, 4
REBS, UB, CFL, ITER = 100.0, 0.1, 0.1, 45
UTIME = int(0.5 * NZ / CFL)
OMEGA = 1.0 / ((3.0 / REBS) * UB * NZ + 0.5)
DT = 1.0 / (0.5 * NZ / CFL)
LOGS = (("energy.txt", 2), ("flowrate.txt", 3), ("massrate.txt", 4), ("str-up.txt", 5), ("str-do.txt", 6),
        ("w-str.txt", 7), ("p-grad.txt", 8))


def write_deck(d, tstr, extra=""):
    with open(os.path.join(d, "deck.txt"), "w") as f:
        f.write(f"# test deck\nxdv {NX}\nydv {NY}\nzdv {NZ}\nRebs {REBS}\nub {UB}\nCFL {CFL}\n"
                f"TSTR {tstr}\nTEND {tstr + 5}\nITER {ITER}\n{extra}")


def oracle_run(oracle_mod, s0, flags, bc_mode=0):
    """Logs of steps 0..ITER and the states at the output steps."""
    st = s0.copy()
    logs, snaps = [], {}
    for ss in range(ITER + 1):
        if ss % UTIME == 0:
            snaps[ss] = st.copy()
        logs.append(oracle_mod.run(st, flags, OMEGA, ubulk=UB, const_g=False, nsteps=1, bc_mode=bc_mode)[0])
    return np.array(logs), snaps


def check_outputs(d, oracle_mod, logs, snaps, tm):
    for fn, col in LOGS:
        got = np.loadtxt(os.path.join(d, fn), ndmin=2)
        assert got.shape == (ITER + 1, 2), fn
        np.testing.assert_allclose(got[:, 0], tm + DT * np.arange(ITER + 1), atol=5e-7)  # printed %f
        np.testing.assert_allclose(got[:, 1], logs[:, col], rtol=1e-9, atol=6e-13, err_msg=fn)
    for ss, st in snaps.items():
        label = tm + ss // UTIME
        stats = np.fromfile(os.path.join(d, f"turb-fld.000.{label:03d}")).reshape(9, NZ + 2)
        np.testing.assert_allclose(stats, oracle_mod.statistics(st), rtol=1e-10, atol=1e-13)
        vel = np.fromfile(os.path.join(d, f"vel.{label:04d}")).reshape(NX, NY, NZ + 2, 3)
        den = np.fromfile(os.path.join(d, f"den.{label:04d}")).reshape(NX, NY, NZ + 2)
        rvel, rden = oracle_mod.moments(st)
        np.testing.assert_allclose(vel, rvel, rtol=1e-10, atol=1e-15)
        np.testing.assert_allclose(den, rden, rtol=1e-12)
    lbf = np.fromfile(os.path.join(d, f"lbf.{tm:04d}")).reshape(2, NX, NY, NZ + 2, 19)
    np.testing.assert_array_equal(lbf[0], snaps[0])
    np.testing.assert_array_equal(lbf[1], snaps[0])
    force = np.fromfile(os.path.join(d, f"force.{tm:04d}"))
    np.testing.assert_allclose(force, [logs[0, 0]], rtol=1e-9, atol=1e-16)
    assert "Total computational time" in open(os.path.join(d, "report.code")).read()


def test_fresh_start_matches_oracle(oracle_mod, tmp_path):
    d = str(tmp_path)
    write_deck(d, 0)
    subprocess.run([RUN_DNS, "-s", "deck.txt"], cwd=d, check=True, timeout=120, capture_output=True)
    s0 = np.zeros((NX, NY, NZ + 2, 19))
    s0[:, :, 1:NZ + 1] = inputs.W
    logs, snaps = oracle_run(oracle_mod, s0, inputs.flags_smooth(NX, NY, NZ))
    check_outputs(d, oracle_mod, logs, snaps, 0)


def test_fresh_start_with_riblets(oracle_mod, tmp_path):
    """TEXTURE riblets (RIBH, RIBS): solids inside the flow, general wall rule."""
    d = str(tmp_path)
    write_deck(d, 0, "TEXTURE riblets\nRIBH 2\nRIBS 4\n")
    subprocess.run([RUN_DNS, "-s", "deck.txt"], cwd=d, check=True, timeout=120, capture_output=True)
    s0 = np.zeros((NX, NY, NZ + 2, 19))
    s0[:, :, 1:NZ + 1] = inputs.W
    flags = inputs.flags_riblets(NX, NY, NZ, 2, 4)
    assert (flags[:, :, 1:-1] == -1).any()
    logs, snaps = oracle_run(oracle_mod, s0, flags, bc_mode=1)
    check_outputs(d, oracle_mod, logs, snaps, 0)


def test_restart_from_lbf_with_posts(oracle_mod, tmp_path):
    d = str(tmp_path)
    write_deck(d, 7, "PSLIP 1\n")
    s0 = inputs.laminar_state(NX, NY, NZ, 0.08, 0.1, 5)
    np.concatenate([s0.ravel(), s0.ravel()]).tofile(os.path.join(d, "lbf.0007"))
    np.array([1.0e-6]).tofile(os.path.join(d, "force.0007"))
    subprocess.run([RUN_DNS, "-p", "deck.txt"], cwd=d, check=True, timeout=120, capture_output=True)
    logs, snaps = oracle_run(oracle_mod, s0, inputs.flags_posts(NX, NY, NZ))
    check_outputs(d, oracle_mod, logs, snaps, 7)


def test_bad_arguments_fail_cleanly(tmp_path):
    d = str(tmp_path)
    r = subprocess.run([RUN_DNS], cwd=d, capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
    write_deck(d, 3)
    r = subprocess.run([RUN_DNS, "-p", "deck.txt"], cwd=d, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "lbf.0003" in r.stderr  # restart file missing: a message, no abort
