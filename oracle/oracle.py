"""CPU oracle bindings -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.  It exposes

* the C restatement ``liblbmoracle.so`` (lbm_oracle.c) through ctypes, and
* ``run_reference``: the reference's own unmodified step functions, compiled
  into ``oracle/_ref/dnsref`` (ref_harness.c), run as a subprocess in a
  scratch directory, with the log files they write parsed back.

State layout everywhere: the reference's lbf/ftemp layout without ghosts,
``state[x, y, z, a]`` float64 with shape (nx, ny, nz+2, 19); z=0 and z=nz+1 are
the wall planes.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblbmoracle.so")
REF_BIN = os.path.join(HERE, "_ref", "dnsref")
QUAD_BIN = os.path.join(HERE, "_ref", "quadref")
# the reference's DNS-solver/src directory (the one place it is named; the
# Makefile's REF_SRC gets the same value)
REF_SRC = os.environ.get("REF_SRC", "/root/reference/DNS-solver/src")

LOG_NAMES = ("force", "rho", "energy", "flowrate", "massrate", "stup", "stdown", "stress", "pgrad")
NLOG = len(LOG_NAMES)

_lib = None


def build(quiet: bool = True) -> None:
    """Compile the restatement (always) and the reference harness (when the
    reference sources are present on this machine)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "all"], check=True, stdout=out)
    if have_reference_sources():
        subprocess.run(["make", "-C", HERE, "ref", f"REF_SRC={REF_SRC}"], check=True, stdout=out)


def have_reference_sources() -> bool:
    return os.path.isdir(REF_SRC)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        i8p = ctypes.POINTER(ctypes.c_int8)
        ci, cd, cl = ctypes.c_int, ctypes.c_double, ctypes.c_long
        L.orc_step.argtypes = [ci, ci, ci, dp, dp, i8p, cd, cd, ci]
        L.orc_steps.argtypes = [ci, ci, ci, dp, dp, i8p, cd, cd, ci, cl]
        L.orc_encalc.argtypes = [ci, ci, ci, dp, cd, dp]
        L.orc_encalc.restype = cd
        L.orc_wshearstr.argtypes = [ci, ci, ci, dp, cd, cd, dp]
        L.orc_statistics.argtypes = [ci, ci, ci, dp, dp]
        L.orc_moments.argtypes = [ci, ci, ci, dp, dp, dp]
        L.orc_run.argtypes = [ci, ci, ci, dp, i8p, cd, cd, cd, ci, cl, dp, ci]
        L.orc_run.restype = cl
        L.orc_flags_smooth.argtypes = [ci, ci, ci, i8p]
        L.orc_flags_ridges.argtypes = [ci, ci, ci, ci, ci, i8p]
        L.orc_flags_transverse.argtypes = [ci, ci, ci, ci, ci, i8p]
        L.orc_flags_posts.argtypes = [ci, ci, ci, ci, ci, ci, ci, i8p]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i8(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))


def _dims(state):
    nx, ny, zd, q = state.shape
    assert q == 19 and state.dtype == np.float64 and state.flags.c_contiguous
    return nx, ny, zd - 2


# ---------------------------------------------------------------- flags
def flags(kind: str, nx: int, ny: int, nz: int, **kw) -> np.ndarray:
    """Periodic-grid flags (nx, ny, nz+2) int8: 0 fluid, -1 no-slip, -2 slip."""
    f = np.zeros((nx, ny, nz + 2), np.int8)
    L = lib()
    if kind == "smooth":
        L.orc_flags_smooth(nx, ny, nz, _i8(f))
    elif kind == "ridges":
        L.orc_flags_ridges(nx, ny, nz, kw.get("gap", 2), kw.get("width", 2), _i8(f))
    elif kind == "transverse":
        L.orc_flags_transverse(nx, ny, nz, kw.get("gap", 2), kw.get("width", 2), _i8(f))
    elif kind == "posts":
        L.orc_flags_posts(nx, ny, nz, kw.get("gx", 2), kw.get("wx", 2), kw.get("gy", 2), kw.get("wy", 2), _i8(f))
    else:
        raise ValueError(kind)
    return f


# ---------------------------------------------------------------- restatement
def run(state, flg, omega, ubulk=0.0, gx=0.0, const_g=True, nsteps=1, bc_mode=0):
    """Advance ``state`` (modified in place) nsteps; returns logs (nsteps, 9)."""
    nx, ny, nz = _dims(state)
    flg = np.ascontiguousarray(flg, np.int8)
    logs = np.zeros((nsteps, NLOG), np.float64)
    done = lib().orc_run(nx, ny, nz, _dp(state), _i8(flg), omega, ubulk, gx, int(const_g), nsteps, _dp(logs), bc_mode)
    if done != nsteps:
        raise FloatingPointError(f"oracle stopped after {done} of {nsteps} steps (NaN wall stress)")
    return logs


def step(state, flg, omega, force, bc_mode=0):
    nx, ny, nz = _dims(state)
    scratch = state.copy()
    lib().orc_step(nx, ny, nz, _dp(state), _dp(scratch), _i8(np.ascontiguousarray(flg, np.int8)), omega, force, bc_mode)


def steps(state, flg, omega, force, nsteps, bc_mode=0):
    """nsteps steps at a fixed force, populations only (no per-step logs)."""
    nx, ny, nz = _dims(state)
    scratch = np.empty_like(state)
    lib().orc_steps(nx, ny, nz, _dp(state), _dp(scratch), _i8(np.ascontiguousarray(flg, np.int8)), omega, force,
                    bc_mode, nsteps)


def encalc(state, ubulk):
    nx, ny, nz = _dims(state)
    out = np.zeros(NLOG)
    force = lib().orc_encalc(nx, ny, nz, _dp(state), ubulk, _dp(out))
    out[0] = force
    return out


def wshearstr(state, omega, force):
    nx, ny, nz = _dims(state)
    out = np.zeros(NLOG)
    lib().orc_wshearstr(nx, ny, nz, _dp(state), omega, force, _dp(out))
    return out


def statistics(state):
    nx, ny, nz = _dims(state)
    out = np.zeros(9 * (nz + 2))
    lib().orc_statistics(nx, ny, nz, _dp(state), _dp(out))
    return out.reshape(9, nz + 2)


def moments(state):
    nx, ny, nz = _dims(state)
    vel = np.zeros((nx, ny, nz + 2, 3))
    den = np.zeros((nx, ny, nz + 2))
    lib().orc_moments(nx, ny, nz, _dp(state), _dp(vel), _dp(den))
    return vel, den


# ---------------------------------------------------------------- reference
def have_reference() -> bool:
    return os.path.exists(REF_BIN)


def ghost_flags(flg: np.ndarray) -> np.ndarray:
    """Periodic-grid flags -> the reference's int32 s-array [xd][yd][zd] with
    ghost planes (flag 1 on the fluid part of the i/j edge planes, exactly as
    solid_init.c:30-45 sets them; wall planes copied periodically)."""
    nx, ny, zd = flg.shape
    s = np.zeros((nx + 1, ny + 1, zd), np.int32)
    s[:nx, :ny] = flg
    s[nx, :ny] = flg[0]
    s[:nx, ny] = flg[:, 0]
    s[nx, ny] = flg[0, 0]
    fluid = s[:, :, 1:zd - 1] >= 0
    edge = np.zeros_like(fluid)
    edge[0], edge[nx] = True, True
    edge[:, 0], edge[:, ny] = True, True
    s[:, :, 1:zd - 1][fluid & edge] = 1
    return s


def _parse_log(path):
    if not os.path.exists(path):
        return None
    return np.loadtxt(path, ndmin=2)[:, 1]


def run_reference(state, omega, ubulk=0.0, gx=0.0, const_g=True, nsteps=1, texture="smooth",
                  flags_periodic=None, stats_every=0, vel_every=0, timeout=600):
    """Run the reference's own step functions.  Returns dict with 'state',
    'force'/'rho' (full precision, per step), the parsed text logs, and
    statistics / vel / den arrays when requested."""
    if not have_reference():
        raise FileNotFoundError(REF_BIN)
    nx, ny, nz = _dims(state)
    with tempfile.TemporaryDirectory() as td:
        inp = os.path.join(td, "in.bin")
        state.tofile(inp)
        args = [REF_BIN, f"xdv={nx}", f"ydv={ny}", f"zdv={nz}", f"omega={omega!r}", f"ubulk={ubulk!r}",
                f"mode={'g' if const_g else 'q'}", f"gx={gx!r}", f"steps={nsteps}", "in=in.bin",
                "out=out.bin", "force_out=force.bin", f"stats_every={stats_every}", f"vel_every={vel_every}"]
        if flags_periodic is not None:
            ghost_flags(flags_periodic).tofile(os.path.join(td, "flags.bin"))
            args += ["texture=file", "flags=flags.bin"]
        else:
            args += [f"texture={texture}"]
        subprocess.run(args, cwd=td, check=True, timeout=timeout, stdout=subprocess.DEVNULL)
        res = {"state": np.fromfile(os.path.join(td, "out.bin")).reshape(state.shape)}
        fr = np.fromfile(os.path.join(td, "force.bin")).reshape(-1, 2)
        res["force"], res["rho"] = fr[:, 0], fr[:, 1]
        for name, fn in (("energy", "energy.txt"), ("flowrate", "flowrate.txt"), ("massrate", "massrate.txt"),
                         ("stup", "str-up.txt"), ("stdown", "str-do.txt"), ("stress", "w-str.txt"),
                         ("pgrad", "p-grad.txt")):
            res[name] = _parse_log(os.path.join(td, fn))
        if stats_every:
            res["stats"] = [np.fromfile(os.path.join(td, f"turb-fld.000.{t:03d}")).reshape(9, nz + 2)
                            for t in range((nsteps - 1) // stats_every + 1)]
        if vel_every:
            res["vel"] = [np.fromfile(os.path.join(td, f"vel.{t:04d}")).reshape(nx, ny, nz + 2, 3)
                          for t in range((nsteps - 1) // vel_every + 1)]
            res["den"] = [np.fromfile(os.path.join(td, f"den.{t:04d}")).reshape(nx, ny, nz + 2)
                          for t in range((nsteps - 1) // vel_every + 1)]
        return res


def time_reference(nx, ny, nz, nsteps, warmup=0, omega=1.9, ubulk=0.05, procs=None, slab=None, timeout=900,
                   only_step=False):
    """CPU baseline: ``procs`` independent single-rank reference processes,
    each advancing its own x-slab (``slab`` cells of x, default nx//procs)
    of the workload as its own periodic box from the reference's rest state
    (the reference's multi-rank halo path is not usable, its neighbours are
    all itself).  Each process does ``warmup`` untimed then ``nsteps`` timed
    full reference steps (encalc + wshearstr + xcomputations), or
    xcomputations alone with ``only_step``.  Returns (aggregate MLUPS,
    slowest process seconds, procs, slab)."""
    procs = procs or max(1, min(os.cpu_count() or 1, nx))
    slab = slab or max(nx // procs, 2)
    with tempfile.TemporaryDirectory() as td:
        ps = []
        for p in range(procs):
            d = os.path.join(td, str(p))
            os.makedirs(d)
            ps.append(subprocess.Popen([REF_BIN, f"xdv={slab}", f"ydv={ny}", f"zdv={nz}", f"omega={omega!r}",
                                        f"ubulk={ubulk!r}", "mode=q", f"steps={nsteps}", f"warmup={warmup}",
                                        "time=1", f"only_step={int(only_step)}"], cwd=d, stdout=subprocess.PIPE,
                                       text=True))
        outs = [p.communicate(timeout=timeout)[0] for p in ps]
    if any(p.returncode for p in ps):
        raise RuntimeError("reference process failed")
    secs = [float(o.split()[2]) for o in outs if o.startswith("MLUPS_STEP")]
    slowest = max(secs)
    cells = float(slab) * ny * nz * nsteps * procs
    return cells / slowest / 1e6, slowest, procs, slab


# ---------------------------------------------------------------- quadrant analysis
def quadrant(vel):
    """quadrant-analysis/src/qUADrantA.c:40-170 restated (numpy, FP64): per
    wall-normal plane k = 1..zd-2 the plane means of u, w over (x, y); the
    fluctuations u' = u - <u>, w' = w - <w>; the four quadrants Q1 (u'>0,
    w'>0), Q2 (u'<0, w'>0), Q3 (u'<0, w'<0), Q4 (u'>0, w'<0) (a zero u' or
    w' falls in none).  Returns quadrant[4][zd] (conditional means of u'w'),
    dquadrant[4][zd] (sums / cells of the plane) and uw[zd] (plane mean of
    u'w'); wall planes 0.  vel: [nx][ny][zd][3] (vel_print.c layout)."""
    nx, ny, zd, _ = vel.shape
    n = nx * ny
    q = np.zeros((4, zd))
    dq = np.zeros((4, zd))
    uw = np.zeros(zd)
    for k in range(1, zd - 1):
        u = vel[:, :, k, 0]
        w = vel[:, :, k, 2]
        up = u - u.sum() / n
        wp = w - w.sum() / n
        p = up * wp
        uw[k] = p.sum() / n
        masks = ((up > 0) & (wp > 0), (up < 0) & (wp > 0), (up < 0) & (wp < 0), (up > 0) & (wp < 0))
        for a, m in enumerate(masks):
            s_ = p[m].sum()
            with np.errstate(invalid="ignore", divide="ignore"):
                q[a, k] = s_ / m.sum()
            dq[a, k] = s_ / n
    return q, dq, uw


def have_quadrant_reference() -> bool:
    return os.path.exists(QUAD_BIN)


def quadrant_reference(vel, label=0, timeout=300):
    """The reference's own qUADrantA (oracle/_ref/quadref) on one velocity
    field; returns (quadrant[4][zd], dquadrant[4][zd], uw[zd]) as it writes
    them (quadrant.000.TTTT: [4][zd] then [zd])."""
    if not have_quadrant_reference():
        raise FileNotFoundError(QUAD_BIN)
    nx, ny, zd, _ = vel.shape
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(vel, np.float64).tofile(os.path.join(td, "vel.bin"))
        subprocess.run([QUAD_BIN, str(nx), str(ny), str(zd - 2), "vel.bin", str(label)], cwd=td, check=True,
                       timeout=timeout, stdout=subprocess.DEVNULL)
        a = np.fromfile(os.path.join(td, f"quadrant.000.{label:04d}"))
        b = np.fromfile(os.path.join(td, f"dquadrant.000.{label:04d}"))
    return a[:4 * zd].reshape(4, zd), b[:4 * zd].reshape(4, zd), a[4 * zd:]


CORR_BIN = os.path.join(HERE, "_ref", "corref")
# the streamwise size the reference's 2pt-correlations program is compiled
# for (its definitions.h xdv): xcorrel.c wraps its lags with it
CORR_REF_NX = 512


def mean_subtract(vel):
    """2pt-correlations/src/mean_subtract.c restated (numpy, FP64): per plane
    k = 1..zd-2 the means of u, v, w over (x, y) (mean_subtract.c:28-60 then
    the average over the span, :197-213), made symmetric about the channel
    centre -- u, v even, w odd (:178-196) -- and subtracted from the fluid
    planes (:214-224); the wall planes keep their velocities.  The program
    averages over the period (gplus + wplus) of a stripe texture first
    (:80-177); its shipped setting, a period of 0, divides by zero, and for
    any period that divides the span the span average of the phase averages
    is the plane mean used here.  Returns (fluct, ua[zd][3]); ua[:, 0] is what
    the program writes to uavg.TTT."""
    vel = np.asarray(vel, np.float64)
    nx, ny, zd, _ = vel.shape
    m = np.zeros((zd, 3))
    m[1:zd - 1] = vel[:, :, 1:zd - 1, :].sum(axis=(0, 1)) / (nx * ny)
    ua = np.zeros((zd, 3))
    k = np.arange(1, zd - 1)
    kk = zd - 1 - k
    ua[k, 0] = 0.5 * (m[k, 0] + m[kk, 0])
    ua[k, 1] = 0.5 * (m[k, 1] + m[kk, 1])
    ua[k, 2] = 0.5 * (m[k, 2] - m[kk, 2])
    fl = vel.copy()
    fl[:, :, 1:zd - 1, :] -= ua[None, None, 1:zd - 1, :]
    return fl, ua


def correlations(vel):
    """The program's correlations of one velocity field (correlations.c:124-
    128): mean_subtract, then ycorrel.c and xcorrel.c restated:
    xcorl[k][d][c] = sum over (x, y) of u'_c(x, y, k) u'_c(x+d, y, k) and
    ycorl[k][d][c] = sum over (x, y) of u'_c(x, y, k) u'_c(x, y+d, k), lags
    periodic, every plane k = 0..zd-1, unnormalised.  Returns (xcorl
    [zd][nx][3], ycorl [zd][ny][3], uavg [zd])."""
    fl, ua = mean_subtract(vel)
    nx, ny, zd, _ = fl.shape
    xc = np.zeros((zd, nx, 3))
    yc = np.zeros((zd, ny, 3))
    for d in range(nx):
        xc[:, d, :] = (fl * np.roll(fl, -d, axis=0)).sum(axis=(0, 1))
    for d in range(ny):
        yc[:, d, :] = (fl * np.roll(fl, -d, axis=1)).sum(axis=(0, 1))
    return xc, yc, ua[:, 0].copy()


def have_correlation_reference() -> bool:
    return os.path.exists(CORR_BIN)


def correlations_reference(fluct, label=0, timeout=600):
    """The reference's own ycorrel and xcorrel (oracle/_ref/corref) on a
    fluctuation field [nx][ny][zd][3] with nx = CORR_REF_NX; returns (xcorl
    [zd][nx][3], ycorl [zd][ny][3]) as the program writes them."""
    if not have_correlation_reference():
        raise FileNotFoundError(CORR_BIN)
    nx, ny, zd, _ = fluct.shape
    if nx != CORR_REF_NX:
        raise ValueError(f"the reference's xcorrel is compiled for nx = {CORR_REF_NX}")
    with tempfile.TemporaryDirectory() as td:
        np.ascontiguousarray(fluct, np.float64).tofile(os.path.join(td, "fluct.bin"))
        subprocess.run([CORR_BIN, str(nx), str(ny), str(zd - 2), "fluct.bin", str(label)], cwd=td, check=True,
                       timeout=timeout, stdout=subprocess.DEVNULL)
        xc = np.fromfile(os.path.join(td, f"xcorl.{label:04d}")).reshape(zd, nx, 3)
        yc = np.fromfile(os.path.join(td, f"ycorl.{label:04d}")).reshape(zd, ny, 3)
    return xc, yc


def spectra(vel):
    """e-spectra/src/1d-spectra.c restated (numpy, FP64).  The program calls
    FFTW 3 (fftw_mpi_plan_dft_r2c_2d, version not pinned by the reference,
    not vendored); r2c_2d computes the unnormalised 2-D DFT C[i][j] =
    sum_{x,y} u(x,y) exp(-2 pi i (i x / nx + j y / ny)) for i < nx, j <=
    ny/2, which numpy's rfft2 computes too.  Per fluid plane k (:116-128):
    the DFT of u, v, w; scaled by 2 / (2 nx ny) (:131-143); the (0, 0) mode
    set to 0 (:146-151); p = fac_j 0.5 |C|^2, fac_0 = 1 and fac_j = 2 for
    j > 0 (:156-172), summed over j into Euux[i][k] and over i into
    Euuy[j][k].  Returns (ex[3][nx][zd], ey[3][ny//2+1][zd]); wall planes
    0."""
    vel = np.asarray(vel, np.float64)
    nx, ny, zd, _ = vel.shape
    nj = ny // 2 + 1
    ex = np.zeros((3, nx, zd))
    ey = np.zeros((3, nj, zd))
    fac = np.full(nj, 2.0)
    fac[0] = 1.0
    scale = 2.0 * (1.0 / (2.0 * nx * ny))
    for k in range(1, zd - 1):
        for c in range(3):
            C = np.fft.rfft2(vel[:, :, k, c]) * scale
            C[0, 0] = 0.0
            p = 0.5 * fac[None, :] * (C.real ** 2 + C.imag ** 2)
            ex[c, :, k] = p.sum(axis=1)
            ey[c, :, k] = p.sum(axis=0)
    return ex, ey
