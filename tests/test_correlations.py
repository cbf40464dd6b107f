"""Two-point velocity correlations (2pt-correlations/src) on the GPU.

The golden fixtures hold the reference's own ycorrel and xcorrel
(oracle/_ref/corref) run on the velocity fluctuations of a channel stepped by
the oracle, at the program's compile-time streamwise size (512 cells: its
xcorrel wraps the lags with it); the field is regenerated from its seed.  The
program's mean subtraction divides by the period of a stripe texture, 0 in its
shipped settings, so it cannot run: the restatement (oracle.mean_subtract)
takes the plane means, made symmetric about the centre, which is its value
for any period that divides the span.  The numpy restatement is pinned to the
fixtures on the CPU; the GPU kernels are checked against the fixtures and the
restatement, on an uploaded vel field and on the live state, and run-dns
(CORREL 1) writes the program's files.  The GPU sums run in another order
than the reference's sequential loops: agreement to rounding, relative to
the zero-lag value of each plane and component.
"""
import glob
import os
import subprocess

import numpy as np
import pytest

import inputs

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CASES = sorted(glob.glob(os.path.join(HERE, "golden", "correl_*.npz")))
RUN_DNS = os.path.join(ROOT, "dns-solvers_b200", "run-dns")


def field(oracle_mod, dims, steps, seed):
    nx, ny, nz = dims
    st = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, seed)
    s0 = st.copy()
    oracle_mod.run(st, inputs.flags_smooth(nx, ny, nz), 1.7, gx=2e-5, const_g=True, nsteps=steps)
    return s0, oracle_mod.moments(st)[0]


def close(got, want, rtol):
    """Per plane and component, relative to the zero-lag sum (the largest)."""
    scale = np.maximum(np.abs(want[:, :1, :]), 1e-300)
    err = np.abs(got - want) / scale
    assert err.max() <= rtol, err.max()


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_restatement_matches_reference_golden(oracle_mod, path):
    g = np.load(path)
    _, vel = field(oracle_mod, tuple(int(v) for v in g["dims"]), int(g["steps"]), int(g["seed"]))
    xc, yc, _ = oracle_mod.correlations(vel)
    close(xc, g["xcorl"], 1e-12)
    close(yc, g["ycorl"], 1e-12)


def test_mean_subtraction_is_symmetric(oracle_mod):
    rng = np.random.default_rng(4)
    for nz in (6, 7):  # an even and an odd number of fluid planes
        vel = rng.standard_normal((10, 6, nz + 2, 3))
        fl, ua = oracle_mod.mean_subtract(vel)
        zd = nz + 2
        np.testing.assert_array_equal(ua[0], 0.0)
        np.testing.assert_array_equal(ua[-1], 0.0)
        for k in range(1, zd - 1):
            assert ua[k, 0] == ua[zd - 1 - k, 0] and ua[k, 1] == ua[zd - 1 - k, 1]
            assert ua[k, 2] == -ua[zd - 1 - k, 2]
        np.testing.assert_array_equal(fl[:, :, 0], vel[:, :, 0])
        # the planes' mean fluctuation is the antisymmetric (u, v) or
        # symmetric (w) part of the plane means
        m = vel[:, :, 1:-1].mean(axis=(0, 1))
        np.testing.assert_allclose(fl[:, :, 1:-1, 0].mean(axis=(0, 1)), 0.5 * (m[:, 0] - m[::-1, 0]), atol=1e-14)
        np.testing.assert_allclose(fl[:, :, 1:-1, 2].mean(axis=(0, 1)), 0.5 * (m[:, 2] + m[::-1, 2]), atol=1e-14)


def test_restatement_matches_reference_live(oracle_mod):
    """Another seed through the reference's own functions, where they are
    built (oracle/_ref/corref)."""
    if not oracle_mod.have_correlation_reference():
        pytest.skip("oracle/_ref/corref not built")
    _, vel = field(oracle_mod, (oracle_mod.CORR_REF_NX, 7, 5), 3, 31)
    fl, _ = oracle_mod.mean_subtract(vel)
    rx, ry = oracle_mod.correlations_reference(fl)
    xc, yc, _ = oracle_mod.correlations(vel)
    close(xc, rx, 1e-12)
    close(yc, ry, 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_gpu_correlations_match_reference_golden(oracle_mod, path):
    import dnslbm
    g = np.load(path)
    dims = tuple(int(v) for v in g["dims"])
    s0, vel = field(oracle_mod, dims, int(g["steps"]), int(g["seed"]))
    xc, yc, ua = dnslbm.correlations_vel(vel)
    close(xc, g["xcorl"], 1e-10)
    close(yc, g["ycorl"], 1e-10)
    _, ua_ref = oracle_mod.mean_subtract(vel)
    np.testing.assert_allclose(ua, ua_ref[:, 0], rtol=1e-12, atol=1e-17)
    nx, ny, nz = dims
    with dnslbm.Channel(nx, ny, nz, 1.7, gx=2e-5, force_mode=dnslbm.CONST_G) as ch:
        ch.load_state(s0)
        ch.step(int(g["steps"]))
        lx, ly, lu = ch.correlations()
    close(lx, g["xcorl"], 1e-10)
    close(ly, g["ycorl"], 1e-10)
    np.testing.assert_allclose(lu, ua_ref[:, 0], rtol=1e-12, atol=1e-17)


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(40, 24, 12), (37, 21, 11), (1256, 6, 4)])
def test_gpu_correlations_match_restatement(oracle_mod, dims):
    import dnslbm
    nx, ny, nz = dims
    rng = np.random.default_rng(nx + ny)
    vel = rng.standard_normal((nx, ny, nz + 2, 3))
    vel[..., 0] += np.linspace(0.0, 1.0, nz + 2)[None, None, :]
    xc, yc, ua = dnslbm.correlations_vel(vel)
    rx, ry, ru = oracle_mod.correlations(vel)
    close(xc, rx, 1e-11)
    close(yc, ry, 1e-11)
    np.testing.assert_allclose(ua, ru, rtol=1e-12, atol=1e-15)


@pytest.mark.gpu
def test_run_dns_writes_correlation_files(oracle_mod, tmp_path):
    """run-dns -p from a perturbed field with CORREL 1: the correlation files
    of every output event against the restatement on that event's vel file."""
    d = str(tmp_path)
    nx, ny, nz = 24, 12, 8
    with open(os.path.join(d, "deck.txt"), "w") as f:
        f.write(f"xdv {nx}\nydv {ny}\nzdv {nz}\nRebs 100\nub 0.1\nCFL 0.1\nTSTR 4\nTEND 9\nITER 61\n"
                "CORREL 1\nFORCE g\nGX 2e-5\n")
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, 19)
    np.concatenate([s0.ravel(), s0.ravel()]).tofile(os.path.join(d, "lbf.0004"))
    subprocess.run([RUN_DNS, "-p", "deck.txt"], cwd=d, check=True, timeout=120, capture_output=True)
    zd = nz + 2
    labels = sorted(int(n[4:]) for n in os.listdir(d) if n.startswith("vel."))
    assert len(labels) >= 2 and labels[0] == 4, labels
    for label in labels:
        vel = np.fromfile(os.path.join(d, f"vel.{label:04d}")).reshape(nx, ny, zd, 3)
        rx, ry, ru = oracle_mod.correlations(vel)
        close(np.fromfile(os.path.join(d, f"xcorl.{label:04d}")).reshape(zd, nx, 3), rx, 1e-11)
        close(np.fromfile(os.path.join(d, f"ycorl.{label:04d}")).reshape(zd, ny, 3), ry, 1e-11)
        np.testing.assert_allclose(np.fromfile(os.path.join(d, f"uavg.{label:03d}")), ru, rtol=1e-12, atol=1e-17)
