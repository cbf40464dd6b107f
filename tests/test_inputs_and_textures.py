"""CPU checks of the synthetic inputs and wall textures: the three texture
generators (Python inputs.py, the C host driver's host/textures.c, the
oracle's lbm_oracle.c) agree flag for flag; the riblet profile; the seeded
24-channel batch draws its parameters inside the stated ranges,
reproducibly; solid cells are put at rest without touching the wall planes."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "dns-solvers_b200", "host")


@pytest.fixture(scope="module")
def textures_lib(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("tex") / "libtextures.so")
    subprocess.run(["/usr/bin/gcc", "-O2", "-shared", "-fPIC", "-o", so, os.path.join(HOST, "textures.c"), "-lm"],
                   check=True)
    L = ctypes.CDLL(so)
    return L


def c_flags(L, fn, nx, ny, nz, *args):
    f = np.zeros((nx, ny, nz + 2), np.int8)
    getattr(L, fn)(nx, ny, nz, *args, f.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)))
    return f


@pytest.mark.parametrize("nx,ny,nz", [(16, 8, 6), (21, 19, 14), (40, 33, 20)])
def test_host_driver_textures_match_inputs(textures_lib, nx, ny, nz):
    L = textures_lib
    np.testing.assert_array_equal(c_flags(L, "tex_smooth", nx, ny, nz), inputs.flags_smooth(nx, ny, nz))
    np.testing.assert_array_equal(c_flags(L, "tex_longitudinal", nx, ny, nz, 3, 2),
                                  inputs.flags_longitudinal(nx, ny, nz, 3, 2))
    np.testing.assert_array_equal(c_flags(L, "tex_transverse", nx, ny, nz, 2, 3),
                                  inputs.flags_transverse(nx, ny, nz, 2, 3))
    np.testing.assert_array_equal(c_flags(L, "tex_posts", nx, ny, nz, 2, 2, 3, 1),
                                  inputs.flags_posts(nx, ny, nz, 2, 2, 3, 1))
    for h, s in ((2, 4), (3, 6), (4, 8)):
        np.testing.assert_array_equal(c_flags(L, "tex_riblets", nx, ny, nz, h, s), inputs.flags_riblets(nx, ny, nz, h, s))


def test_inputs_textures_match_oracle(oracle_mod):
    nx, ny, nz = 24, 17, 10
    np.testing.assert_array_equal(oracle_mod.flags("smooth", nx, ny, nz), inputs.flags_smooth(nx, ny, nz))
    np.testing.assert_array_equal(oracle_mod.flags("ridges", nx, ny, nz, gap=3, width=2),
                                  inputs.flags_longitudinal(nx, ny, nz, 3, 2))
    np.testing.assert_array_equal(oracle_mod.flags("transverse", nx, ny, nz, gap=2, width=3),
                                  inputs.flags_transverse(nx, ny, nz, 2, 3))


def test_riblet_profile():
    h, s = 8, 16
    nk = inputs.riblet_profile(64, h, s)
    assert nk.max() == h - 1 and nk.min() == 0
    assert np.array_equal(nk[:s], nk[s:2 * s])                 # periodic in the spacing
    assert np.array_equal(nk[:s], nk[:s][::-1])                # symmetric triangle
    yc = np.arange(s) + 0.5
    top = h * (1 - np.abs(2 * yc / s - 1))
    assert np.all(nk[:s] - 0.5 < top) and np.all(nk[:s] + 0.5 >= top)  # k - 1/2 < h(y) for every solid k
    f = inputs.flags_riblets(10, 64, 20, h, s)
    assert np.array_equal((f[0, :, 1:-1] == -1).sum(-1), 2 * nk)
    assert np.all(f[:, :, 0] == -1) and np.all(f[:, :, -1] == -1)


def test_batch_channels_are_seeded_and_in_range():
    a, b = inputs.batch_channels(24, seed=0), inputs.batch_channels(24, seed=0)
    assert [w.name for w in a] == [w.name for w in b]
    assert [w.name for w in a] != [w.name for w in inputs.batch_channels(24, seed=1)]
    hs = [w.nz // 2 for w in a]
    assert sorted(set(hs)) == [20, 32, 48, 64] and all(hs.count(h) == 6 for h in (20, 32, 48, 64))
    kinds = {w.texture for w in a}
    assert kinds <= {"smooth", "longitudinal", "transverse", "riblets"} and len(kinds) >= 3
    for w in a:
        h = w.nz // 2
        assert (w.nx, w.ny) == (round(2 * np.pi * h), round(np.pi * h))
        nu = (2 / w.omega - 1) / 6
        assert 120 - 1e-9 <= 0.005 * h / nu <= 180 + 1e-9          # Re_tau in [120, 180]
        if w.texture == "longitudinal":
            pitch = w.tex["gap"] + w.tex["width"]
            assert 8 <= pitch <= 32 and 0.45 <= w.tex["gap"] / pitch <= 0.95
        if w.texture == "transverse":
            assert w.tex["gap"] + w.tex["width"] == 16
        if w.texture == "riblets":
            assert 4 <= w.tex["height"] <= 8 and w.tex["spacing"] == 2 * w.tex["height"]


def test_rest_solids_leaves_walls_and_fluid():
    nx, ny, nz = 12, 16, 10
    f = inputs.flags_riblets(nx, ny, nz, 4, 8)
    s = inputs.laminar_state(nx, ny, nz, 0.05, 0.1, 3)
    s[:, :, 0] = 7.0  # wall planes are not populations: left alone
    r = inputs.rest_solids(s, f)
    inner = f[:, :, 1:-1] == -1
    assert np.all(r[:, :, 1:-1][inner] == inputs.W)
    assert np.array_equal(r[:, :, 1:-1][~inner], s[:, :, 1:-1][~inner])
    assert np.all(r[:, :, 0] == 7.0)


def test_laminar_and_turbulent_fields_are_near_equilibrium():
    nx, ny, nz = 20, 12, 16
    for st in (inputs.laminar_state(nx, ny, nz, 0.05, 0.1, 0), inputs.turbulent_state(nx, ny, nz, 0.06, 0.1, 0)):
        f = st[:, :, 1:-1]
        rho = f.sum(-1)
        assert np.allclose(rho, 1.0, atol=1e-12)
        u = (f @ inputs.E) / rho[..., None]
        np.testing.assert_allclose(inputs.equilibrium(rho, u), f, atol=1e-12)
        assert 0.0 < u[..., 0].mean() < 0.2
