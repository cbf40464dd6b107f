"""One-dimensional energy spectra (e-spectra/src/1d-spectra.c) on the GPU.

The reference program calls FFTW 3's MPI real-to-complex 2-D transform,
which is neither vendored nor installed, so it cannot be built here; its own
code around the transform (scaling, removal of the mean mode, the half-plane
weights, the sums into Euux..Ewwy) is restated in oracle.spectra on numpy's
DFT.  The restatement is checked against the DFT's definition (a direct sum)
and Parseval's relation on the CPU; the GPU kernels (direct FP64 DFTs)
against the restatement on uploaded fields, the live state and run-dns
(SPECTRA 1) files, to rounding relative to each plane's largest mode.
"""
import os
import subprocess

import numpy as np
import pytest

import inputs

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
RUN_DNS = os.path.join(ROOT, "dns-solvers_b200", "run-dns")


def close(got, want, rtol):
    """Per component and plane, relative to the largest mode."""
    scale = np.maximum(np.abs(want).max(axis=1, keepdims=True), 1e-300)
    err = np.abs(got - want) / scale
    assert err.max() <= rtol, err.max()


def _field(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    vel = rng.standard_normal((nx, ny, nz + 2, 3))
    vel[..., 0] += np.linspace(0.0, 1.0, nz + 2)[None, None, :]
    vel[:, :, 0] = vel[:, :, -1] = 0.0
    return vel


def test_restatement_is_the_dft(oracle_mod):
    nx, ny, nz = 9, 6, 3
    vel = _field(nx, ny, nz, 1)
    ex, ey = oracle_mod.spectra(vel)
    xs, ys = np.arange(nx), np.arange(ny)
    nj = ny // 2 + 1
    for k in range(1, nz + 1):
        for c in range(3):
            u = vel[:, :, k, c]
            C = np.array([[np.sum(u * np.exp(-2j * np.pi * (i * xs[:, None] / nx + j * ys[None, :] / ny)))
                           for j in range(nj)] for i in range(nx)]) / (nx * ny)
            C[0, 0] = 0.0
            p = 0.5 * np.abs(C) ** 2 * np.where(np.arange(nj) == 0, 1.0, 2.0)[None, :]
            np.testing.assert_allclose(ex[c, :, k], p.sum(axis=1), rtol=1e-12, atol=1e-18)
            np.testing.assert_allclose(ey[c, :, k], p.sum(axis=0), rtol=1e-12, atol=1e-18)
    assert np.all(ex[:, :, 0] == 0.0) and np.all(ey[:, :, -1] == 0.0)


def test_parseval(oracle_mod):
    """Odd ny: the half plane with weights 2 covers every mode once, so the
    spectra sum to half the plane variance."""
    vel = _field(12, 7, 4, 2)
    ex, ey = oracle_mod.spectra(vel)
    var = vel[:, :, 1:-1, :].var(axis=(0, 1))  # [zdv][3]
    np.testing.assert_allclose(ex[:, :, 1:-1].sum(axis=1), 0.5 * var.T, rtol=1e-12)
    np.testing.assert_allclose(ey[:, :, 1:-1].sum(axis=1), 0.5 * var.T, rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(40, 24, 6), (37, 21, 5), (628, 31, 3), (1256, 10, 2)])
def test_gpu_spectra_match_restatement(oracle_mod, dims):
    import dnslbm
    vel = _field(*dims, seed=sum(dims))
    ex, ey = dnslbm.spectra_vel(vel)
    rx, ry = oracle_mod.spectra(vel)
    close(ex, rx, 1e-10)
    close(ey, ry, 1e-10)


@pytest.mark.gpu
def test_gpu_spectra_of_the_live_state(oracle_mod):
    import dnslbm
    nx, ny, nz = 48, 20, 10
    st = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, 5)
    s0 = st.copy()
    oracle_mod.run(st, inputs.flags_smooth(nx, ny, nz), 1.7, gx=2e-5, const_g=True, nsteps=7)
    vel = oracle_mod.moments(st)[0]
    rx, ry = oracle_mod.spectra(vel)
    with dnslbm.Channel(nx, ny, nz, 1.7, gx=2e-5, force_mode=dnslbm.CONST_G) as ch:
        ch.load_state(s0)
        ch.step(7)
        ex, ey = ch.spectra()
    close(ex, rx, 1e-10)
    close(ey, ry, 1e-10)


@pytest.mark.gpu
def test_run_dns_writes_spectra_files(oracle_mod, tmp_path):
    d = str(tmp_path)
    nx, ny, nz = 24, 12, 8
    with open(os.path.join(d, "deck.txt"), "w") as f:
        f.write(f"xdv {nx}\nydv {ny}\nzdv {nz}\nRebs 100\nub 0.1\nCFL 0.1\nTSTR 4\nTEND 9\nITER 61\n"
                "SPECTRA 1\nFORCE g\nGX 2e-5\n")
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.3, 29)
    np.concatenate([s0.ravel(), s0.ravel()]).tofile(os.path.join(d, "lbf.0004"))
    subprocess.run([RUN_DNS, "-p", "deck.txt"], cwd=d, check=True, timeout=120, capture_output=True)
    zd, nj = nz + 2, ny // 2 + 1
    labels = sorted(int(n[4:]) for n in os.listdir(d) if n.startswith("vel."))
    assert len(labels) >= 2 and labels[0] == 4, labels
    for label in labels:
        vel = np.fromfile(os.path.join(d, f"vel.{label:04d}")).reshape(nx, ny, zd, 3)
        rx, ry = oracle_mod.spectra(vel)
        got_x = np.stack([np.fromfile(os.path.join(d, f"E{c}x.{label:04d}")).reshape(nx, zd) for c in ("uu", "vv", "ww")])
        got_y = np.stack([np.fromfile(os.path.join(d, f"E{c}y.{label:04d}")).reshape(nj, zd) for c in ("uu", "vv", "ww")])
        close(got_x, rx, 1e-10)
        close(got_y, ry, 1e-10)
