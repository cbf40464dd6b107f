"""GPU parity: the sm_100a kernels through the C ABI against the oracle.

Tolerances (written here):
  * FP64, constant g: bit-identical populations to the reference (goldens)
    and to the oracle, for every texture, grid and step count (either AA
    parity).  Logs: force exact; reductions within 1e-12 relative (only the
    summation order differs from the reference's sequential sums).
  * FP64, constant Q: the force of each step comes from a differently ordered
    FP64 sum, so populations agree to <= 1e-12 relative.
  * FP32 / FP16 storage: errors against the FP64 oracle are measured and
    bounded in test_lowp_precision.py.
"""
import glob
import os

import numpy as np
import pytest

import dnslbm
import inputs

pytestmark = pytest.mark.gpu

# step goldens (the quadrant-analysis fixtures are tests/test_quadrant.py's)
GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("quadrant_", "correl_")))


def gpu_run(s0, flags, omega, steps, gx=0.0, ubulk=0.0, const_g=True, precision=64, chunks=None):
    nx, ny, zd, _ = s0.shape
    ch = dnslbm.Channel(nx, ny, zd - 2, omega, ubulk=ubulk, gx=gx,
                        force_mode=dnslbm.CONST_G if const_g else dnslbm.CONST_Q, precision=precision)
    ch.set_flags(flags)
    ch.load_state(s0)
    for n in (chunks or [steps]):
        ch.step(n)
    return ch


def ref_flags(oracle, tex, nx, ny, nz):
    return oracle.flags(tex, nx, ny, nz)


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_f64_matches_reference_golden(oracle_mod, path):
    g = np.load(path)
    nx, ny, nz = (int(v) for v in g["dims"])
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, int(g["seed"]))
    steps, cg = int(g["steps"]), bool(g["const_g"])
    fl = ref_flags(oracle_mod, str(g["texture"]), nx, ny, nz)
    ch = gpu_run(s0, fl, float(g["omega"]), steps, gx=float(g["gx"]), ubulk=float(g["ubulk"]), const_g=cg,
                 chunks=[steps - 1, 1])
    st = ch.store_state()
    logs = ch.logs()
    if cg:
        np.testing.assert_array_equal(st, g["state"])
        np.testing.assert_array_equal(logs[:, 0], g["force"])
    else:
        np.testing.assert_allclose(st, g["state"], rtol=1e-12, atol=0)
        np.testing.assert_allclose(logs[:, 0], g["force"], rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(logs[:, 1], g["rho"], rtol=1e-13)
    # text logs are printed with 12-14 decimals by the reference
    np.testing.assert_allclose(logs[:, 2:], g["logs"], rtol=0, atol=6e-13)


@pytest.mark.parametrize("steps", [1, 2, 5, 8])
@pytest.mark.parametrize("tex", ["smooth", "ridges", "posts"])
def test_f64_bitexact_any_parity(oracle_mod, tex, steps):
    nx, ny, nz = 16, 12, 7
    fl = ref_flags(oracle_mod, tex, nx, ny, nz)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 7)
    ref = s0.copy()
    rlogs = oracle_mod.run(ref, fl, 1.85, gx=3e-5, const_g=True, nsteps=steps)
    ch = gpu_run(s0, fl, 1.85, steps, gx=3e-5)
    np.testing.assert_array_equal(ch.store_state(), ref)
    logs = ch.logs()
    np.testing.assert_array_equal(logs[:, 0], rlogs[:, 0])
    np.testing.assert_allclose(logs[:, 1:], rlogs[:, 1:], rtol=1e-11, atol=1e-15)


@pytest.mark.parametrize("dims", [(9, 5, 3), (13, 7, 4), (33, 17, 9), (130, 3, 5)])
def test_f64_bitexact_ragged_grids_transverse(oracle_mod, dims):
    """Odd sizes, rows narrower and wider than a block, transverse grooves."""
    nx, ny, nz = dims
    fl = inputs.flags_transverse(nx, ny, nz, 2, 3)
    s0 = inputs.laminar_state(nx, ny, nz, 0.06, 0.1, 3)
    ref = s0.copy()
    oracle_mod.run(ref, fl, 1.7, gx=1e-5, const_g=True, nsteps=11)
    ch = gpu_run(s0, fl, 1.7, 11, gx=1e-5)
    np.testing.assert_array_equal(ch.store_state(), ref)


@pytest.mark.parametrize("tex", ["smooth", "posts"])
def test_f64_constant_q(oracle_mod, tex):
    nx, ny, nz = 24, 16, 10
    fl = ref_flags(oracle_mod, tex, nx, ny, nz)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 5)
    ref = s0.copy()
    rlogs = oracle_mod.run(ref, fl, 1.6, ubulk=0.07, const_g=False, nsteps=20)
    ch = gpu_run(s0, fl, 1.6, 20, ubulk=0.07, const_g=False)
    st = ch.store_state()
    np.testing.assert_allclose(st, ref, rtol=1e-12, atol=0)
    logs = ch.logs()
    np.testing.assert_allclose(logs[:, 0], rlogs[:, 0], rtol=1e-9, atol=1e-16)
    np.testing.assert_allclose(ch.force(), oracle_mod.encalc(ref, 0.07)[0], rtol=1e-9, atol=1e-16)


@pytest.mark.parametrize("steps", [4, 5])
def test_statistics_and_moments(oracle_mod, steps):
    nx, ny, nz = 20, 12, 8
    fl = inputs.flags_longitudinal(nx, ny, nz, 2, 2)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 9)
    ref = s0.copy()
    oracle_mod.run(ref, fl, 1.5, gx=2e-5, const_g=True, nsteps=steps)
    ch = gpu_run(s0, fl, 1.5, steps, gx=2e-5)
    vel, den = ch.moments()
    rvel, rden = oracle_mod.moments(ref)
    np.testing.assert_array_equal(vel, rvel)
    np.testing.assert_array_equal(den, rden)
    np.testing.assert_allclose(ch.statistics(), oracle_mod.statistics(ref), rtol=1e-11, atol=1e-15)


def test_laminar64_1000_steps_bitexact(oracle_mod):
    """The first workload: 64 x 66 x 32, tau 0.52, g 1e-6, 1000 steps."""
    wl = inputs.workload("laminar64")
    s0 = inputs.make_state(wl, seed=0)
    fl = inputs.make_flags(wl)
    ref = s0.copy()
    rlogs = oracle_mod.run(ref, fl, wl.omega, gx=wl.gx, const_g=True, nsteps=wl.steps)
    ch = gpu_run(s0, fl, wl.omega, wl.steps, gx=wl.gx)
    np.testing.assert_array_equal(ch.store_state(), ref)
    np.testing.assert_allclose(ch.logs()[:, 1:], rlogs[:, 1:], rtol=1e-10, atol=1e-15)


def test_rest_start_matches_reference_init(oracle_mod):
    """init.c rest state, constant Q: the flow accelerates from rest."""
    nx, ny, nz = 12, 8, 6
    ch = dnslbm.Channel(nx, ny, nz, 1.4, ubulk=0.05, force_mode=dnslbm.CONST_Q)
    ch.init_rest()
    ch.step(9)
    s0 = np.zeros((nx, ny, nz + 2, 19))
    s0[:, :, 1:nz + 1] = inputs.W
    ref = s0.copy()
    oracle_mod.run(ref, oracle_mod.flags("smooth", nx, ny, nz), 1.4, ubulk=0.05, const_g=False, nsteps=9)
    np.testing.assert_allclose(ch.store_state(), ref, rtol=1e-12, atol=1e-18)


def test_load_store_roundtrip_and_wall_zeros():
    nx, ny, nz = 10, 6, 5
    s0 = inputs.laminar_state(nx, ny, nz, 0.05, 0.1, 1)
    ch = dnslbm.Channel(nx, ny, nz, 1.2)
    ch.load_state(s0)
    out = ch.store_state()
    np.testing.assert_array_equal(out, s0)
    assert not out[:, :, 0].any() and not out[:, :, -1].any()


def test_nan_is_reported_not_aborted():
    nx, ny, nz = 8, 6, 5
    s0 = inputs.laminar_state(nx, ny, nz, 0.05, 0.1, 1)
    s0[3, 2, 1, 4] = np.nan  # a NaN in the wall-adjacent plane reaches the wall stress
    ch = dnslbm.Channel(nx, ny, nz, 1.2, gx=1e-6)
    ch.load_state(s0)
    with pytest.raises(dnslbm.DnsLbmError) as e:
        ch.step(3)
    assert e.value.code == dnslbm.ERR_NAN
    # the context stays usable: a clean state steps again
    ch.load_state(inputs.laminar_state(nx, ny, nz, 0.05, 0.1, 2))
    ch.step(2)


def test_flag_validation():
    nx, ny, nz = 8, 6, 5
    ch = dnslbm.Channel(nx, ny, nz, 1.2)
    fl = inputs.flags_smooth(nx, ny, nz)
    fl[2, 2, 3] = -1  # a solid inside the flow
    with pytest.raises(dnslbm.DnsLbmError) as e:
        ch.set_flags(fl)
    assert e.value.code == dnslbm.ERR_ARG
    fl = inputs.flags_smooth(nx, ny, nz)
    fl[1, 1, 0] = 0  # a fluid cell in the wall plane
    with pytest.raises(dnslbm.DnsLbmError):
        ch.set_flags(fl)


def test_reference_ghost_flag_array(oracle_mod):
    """dnslbm_set_flags takes the reference's V.s array with ghost planes."""
    nx, ny, nz = 12, 8, 6
    fl = oracle_mod.flags("posts", nx, ny, nz)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 4)
    ch = dnslbm.Channel(nx, ny, nz, 1.3, gx=1e-5)
    ch.set_flags(oracle_mod.ghost_flags(fl))
    ch.load_state(s0)
    ch.step(6)
    ref = s0.copy()
    oracle_mod.run(ref, fl, 1.3, gx=1e-5, const_g=True, nsteps=6)
    np.testing.assert_array_equal(ch.store_state(), ref)


@pytest.mark.parametrize("name", ["channel180", "grooves180"])
def test_full_size_20_steps_bitexact(oracle_mod, name):
    """The 20-step field check at full size: 628 x 202 x 314 (39.4M fluid
    cells), Re_tau ~ 180, FP64, constant g, smooth walls and pitch-32 /
    gas-fraction-0.5 longitudinal grooves; bit-identical to the oracle."""
    wl = inputs.workload(name)
    s0 = inputs.make_state(wl, seed=0)
    fl = inputs.make_flags(wl)
    with dnslbm.Channel(wl.nx, wl.ny, wl.nz, wl.omega, gx=wl.gx, force_mode=dnslbm.CONST_G) as ch:
        ch.set_flags(fl)
        ch.load_state(s0)
        ch.step(20)
        got = ch.store_state()
        logs = ch.logs()
    assert np.isfinite(logs).all()
    oracle_mod.steps(s0, fl, wl.omega, wl.gx, 20)  # in place
    np.testing.assert_array_equal(got, s0)


def _with_path(path, fn):
    old = os.environ.get("DNSLBM_PATH")
    os.environ["DNSLBM_PATH"] = path
    try:
        return fn()
    finally:
        if old is None:
            del os.environ["DNSLBM_PATH"]
        else:
            os.environ["DNSLBM_PATH"] = old


@pytest.mark.parametrize("prec", [64, 32, 16])
@pytest.mark.parametrize("tex", ["smooth", "ridges"])
@pytest.mark.parametrize("const_g", [True, False])
@pytest.mark.parametrize("nx", [44, 45])
def test_row_pipelined_and_per_thread_paths_agree(oracle_mod, prec, tex, const_g, nx):
    """The bulk-copy kernel and the per-thread kernel run the same step.
    With a constant force the populations are bit-identical at every
    precision: the FP32/FP16 bulk-copy kernel collides two cells at once on
    the packed FP32 pipe with the same explicitly rounded operations as the
    per-thread kernel's one cell (an odd nx leaves a one-cell pair at the end
    of each row).  Constant-Q forces come from differently ordered sums."""
    ny, nz = 18, 9
    fl = ref_flags(oracle_mod, tex, nx, ny, nz)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 13)

    def run():
        ch = gpu_run(s0, fl, 1.7, 7, gx=2e-5, ubulk=0.07, const_g=const_g, precision=prec)
        return ch.kernel, ch.store_state(), ch.logs()

    kt, st_t, lg_t = run()
    ks, st_s, lg_s = _with_path("scalar", run)
    assert "bulk-copy" in kt and "per-thread" in ks
    if const_g:
        np.testing.assert_array_equal(st_t, st_s)
    else:
        tol = {64: 1e-13, 32: 1e-6, 16: 2e-3}[prec]
        np.testing.assert_allclose(st_t, st_s, rtol=0, atol=tol)
    # FP16 keeps 11 bits of each deviation: with constant Q, forces that
    # differ in their last bits flip roundings of stored values, which moves
    # the logs by ~1e-5 relative
    rtol = 1e-4 if (prec == 16 and not const_g) else (1e-5 if prec < 64 else 1e-11)
    np.testing.assert_allclose(lg_t, lg_s, rtol=rtol, atol=1e-12)


@pytest.mark.parametrize("prec", [64, 16])
def test_autotuned_kernel_is_exact_and_tuning_needs_no_state(oracle_mod, prec):
    """dnslbm_autotune picks a launch shape by timing; whatever it picks
    computes the same step (FP64 bit-exact), and it refuses to run once a
    state is loaded (it would overwrite it)."""
    nx, ny, nz = 40, 20, 10
    fl = inputs.flags_longitudinal(nx, ny, nz, 3, 3)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 17)
    ch = dnslbm.Channel(nx, ny, nz, 1.8, gx=2e-5, force_mode=dnslbm.CONST_G, precision=prec)
    report = ch.autotune(steps=3)
    assert "ms/step" in report and ch.kernel in report
    ch.set_flags(fl)
    ch.load_state(s0)
    ch.step(9)
    ref = s0.copy()
    oracle_mod.run(ref, fl, 1.8, gx=2e-5, const_g=True, nsteps=9)
    if prec == 64:
        np.testing.assert_array_equal(ch.store_state(), ref)
    else:
        np.testing.assert_allclose(ch.store_state(), ref, rtol=0, atol=2e-4)
    with pytest.raises(dnslbm.DnsLbmError) as e:
        ch.autotune()
    assert e.value.code == dnslbm.ERR_STATE
