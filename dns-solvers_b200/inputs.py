"""Seeded synthetic inputs and the channel workloads.

The reference reads its initial populations from an ``lbf.NNNN`` file and
publishes no input data set; these generators stand in for it with seeded
fields of the configured shapes.  States use the lbf/ftemp layout
(x, y, z incl. walls, 19) float64; flags use the periodic grid (x, y, z) int8
with the reference's values (DNS-solver/src/solid_init.c:3-8).

Axis convention: the reference's i (x, streamwise), j (y, spanwise),
k (z, wall-normal).  A workload written as Nx x Ny_wall x Nz_span maps to
xdv = Nx, zdv = Ny_wall - 2, ydv = Nz_span.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
E = np.array([[0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, 1, -1, -1, 0, 0, 0, 0],
              [0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, 1, -1, -1],
              [0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1]], dtype=np.float64).T


def equilibrium(rho, u):
    """feq of DNS-solver/src/xcomputations.c:330-331 for arrays rho (...),
    u (..., 3) -> (..., 19)."""
    eu = u @ E.T
    uu = (u * u).sum(-1)[..., None]
    return W * rho[..., None] * (1 + 3 * eu + 4.5 * eu ** 2 - 1.5 * uu)


def zeta(nz):
    """Wall-normal coordinate of the fluid planes, (k - 1/2)/nz for k=1..nz
    (output_twoD.c:14-17)."""
    return (np.arange(1, nz + 1) - 0.5) / nz


def laminar_state(nx, ny, nz, umax, amp, seed):
    """rho = 1, Poiseuille u_x = umax 4 zeta (1 - zeta) plus uniform
    perturbations of +-amp*umax on all three components, at equilibrium."""
    rng = np.random.default_rng(seed)
    s = np.zeros((nx, ny, nz + 2, 19))
    u = np.zeros((nx, ny, nz, 3))
    u[..., 0] = umax * 4 * zeta(nz) * (1 - zeta(nz))
    u += rng.uniform(-1.0, 1.0, u.shape) * amp * umax
    s[:, :, 1:nz + 1] = equilibrium(np.ones((nx, ny, nz)), u)
    return s


def turbulent_state(nx, ny, nz, ubulk, amp, seed, modes=4, kmax=6):
    """Laminar profile of bulk velocity `ubulk` plus a divergence-free
    perturbation of rms amp*ubulk: the curl of a seeded, low-pass vector
    potential A whose wall-normal profile sin(pi z) sin(m pi z) vanishes with
    its derivative at both walls, so the perturbation is zero there."""
    rng = np.random.default_rng(seed)
    z = zeta(nz)
    H = float(nz)
    # low-pass random 2-D fields B[c][m](x, y) and their x/y derivatives
    kx = np.fft.fftfreq(nx, 1.0 / nx)[:, None]
    ky = np.fft.rfftfreq(ny, 1.0 / ny)[None, :]
    mask = (np.abs(kx) <= kmax) & (np.abs(ky) <= kmax) & ((kx != 0) | (ky != 0))
    B, Bx, By = (np.zeros((3, modes, nx, ny)) for _ in range(3))
    for c in range(3):
        for m in range(modes):
            spec = (rng.standard_normal((nx, ny // 2 + 1)) + 1j * rng.standard_normal((nx, ny // 2 + 1))) * mask
            B[c, m] = np.fft.irfft2(spec, s=(nx, ny))
            Bx[c, m] = np.fft.irfft2(spec * (2j * np.pi * kx / nx), s=(nx, ny))
            By[c, m] = np.fft.irfft2(spec * (2j * np.pi * ky / ny), s=(nx, ny))
    m = np.arange(1, modes + 1)[:, None]
    pz = np.sin(np.pi * z)[None] * np.sin(m * np.pi * z[None])  # (modes, nz)
    dpz = (np.pi / H) * (np.cos(np.pi * z)[None] * np.sin(m * np.pi * z[None])
                         + m * np.sin(np.pi * z)[None] * np.cos(m * np.pi * z[None]))
    # u' = curl A, A_c = sum_m pz_m(z) B[c,m](x,y)
    up = np.empty((nx, ny, nz, 3), np.float64)
    up[..., 0] = np.einsum("mxy,mz->xyz", By[2], pz) - np.einsum("mxy,mz->xyz", B[1], dpz)
    up[..., 1] = np.einsum("mxy,mz->xyz", B[0], dpz) - np.einsum("mxy,mz->xyz", Bx[2], pz)
    up[..., 2] = np.einsum("mxy,mz->xyz", Bx[1], pz) - np.einsum("mxy,mz->xyz", By[0], pz)
    up *= amp * ubulk / max(np.sqrt((up ** 2).sum(-1).mean()), 1e-300)
    up[..., 0] += 1.5 * ubulk * 4 * z * (1 - z)
    s = np.zeros((nx, ny, nz + 2, 19))
    one = np.ones((ny, nz))
    for x in range(nx):  # plane by plane keeps temporaries small
        s[x, :, 1:nz + 1] = equilibrium(one, up[x])
    return s


def turbulent_slabs(nx, ny, nz, ubulk, amp, seed, slab=16, flags=None, workers=None, modes=4, kmax=6):
    """The field of turbulent_state (same construction and seed; the rms
    normalisation is summed slab by slab) as x-slabs (x0, state[x0:x0+n]) in
    order, for grids whose whole state does not fit host memory comfortably.
    Slabs are made by a thread pool (numpy releases the GIL), `workers` at a
    time; solid cells of `flags` (-1 inside the flow) are set to rest."""
    from concurrent.futures import ThreadPoolExecutor
    import os
    rng = np.random.default_rng(seed)
    z = zeta(nz)
    H = float(nz)
    kx = np.fft.fftfreq(nx, 1.0 / nx)[:, None]
    ky = np.fft.rfftfreq(ny, 1.0 / ny)[None, :]
    mask = (np.abs(kx) <= kmax) & (np.abs(ky) <= kmax) & ((kx != 0) | (ky != 0))
    B, Bx, By = (np.zeros((3, modes, nx, ny)) for _ in range(3))
    for c in range(3):
        for m in range(modes):
            spec = (rng.standard_normal((nx, ny // 2 + 1)) + 1j * rng.standard_normal((nx, ny // 2 + 1))) * mask
            B[c, m] = np.fft.irfft2(spec, s=(nx, ny))
            Bx[c, m] = np.fft.irfft2(spec * (2j * np.pi * kx / nx), s=(nx, ny))
            By[c, m] = np.fft.irfft2(spec * (2j * np.pi * ky / ny), s=(nx, ny))
    m = np.arange(1, modes + 1)[:, None]
    pz = np.sin(np.pi * z)[None] * np.sin(m * np.pi * z[None])
    dpz = (np.pi / H) * (np.cos(np.pi * z)[None] * np.sin(m * np.pi * z[None])
                         + m * np.sin(np.pi * z)[None] * np.cos(m * np.pi * z[None]))

    def perturbation(x0, x1):
        sl = slice(x0, x1)
        up = np.empty((x1 - x0, ny, nz, 3), np.float64)
        up[..., 0] = np.einsum("mxy,mz->xyz", By[2][:, sl], pz) - np.einsum("mxy,mz->xyz", B[1][:, sl], dpz)
        up[..., 1] = np.einsum("mxy,mz->xyz", B[0][:, sl], dpz) - np.einsum("mxy,mz->xyz", Bx[2][:, sl], pz)
        up[..., 2] = np.einsum("mxy,mz->xyz", Bx[1][:, sl], pz) - np.einsum("mxy,mz->xyz", By[0][:, sl], pz)
        return up

    bounds = [(x0, min(x0 + slab, nx)) for x0 in range(0, nx, slab)]
    workers = workers or min(16, os.cpu_count() or 1)
    with ThreadPoolExecutor(workers) as ex:
        ss = sum(ex.map(lambda b: float((perturbation(*b) ** 2).sum()), bounds))
        scale = amp * ubulk / max(np.sqrt(ss / (nx * ny * nz)), 1e-300)
        lam = 1.5 * ubulk * 4 * z * (1 - z)
        one = np.ones((ny, nz))

        def make(b):
            up = perturbation(*b)
            up *= scale
            up[..., 0] += lam
            st = np.zeros((b[1] - b[0], ny, nz + 2, 19))
            for i in range(b[1] - b[0]):
                st[i, :, 1:nz + 1] = equilibrium(one, up[i])
            if flags is not None:
                st = rest_solids(st, flags[b[0]:b[1]])
            return st

        pending = []
        for b in bounds:
            pending.append((b[0], ex.submit(make, b)))
            if len(pending) > workers:
                x0, f = pending.pop(0)
                yield x0, f.result()
        for x0, f in pending:
            yield x0, f.result()


# ------------------------------------------------------------------ textures
def flags_smooth(nx, ny, nz):
    """solid_init.c:18-45 on the periodic grid: no-slip walls, fluid inside."""
    f = np.zeros((nx, ny, nz + 2), np.int8)
    f[:, :, 0] = -1
    f[:, :, -1] = -1
    return f


def flags_longitudinal(nx, ny, nz, gap, width):
    """Streamwise slip stripes on both walls: slip_ridges_init.c:11-40 with
    its hard-coded gap (slip cells) and width (no-slip cells) as parameters;
    first stripe at y = width/2, period gap + width."""
    f = flags_smooth(nx, ny, nz)
    for j in range(width // 2, ny, gap + width):
        f[:, j:min(j + gap, ny), 0] = -2
        f[:, j:min(j + gap, ny), -1] = -2
    return f


def flags_transverse(nx, ny, nz, gap, width):
    """The same stripe rule across the flow (spanwise slip stripes)."""
    f = flags_smooth(nx, ny, nz)
    for i in range(width // 2, nx, gap + width):
        f[i:min(i + gap, nx), :, 0] = -2
        f[i:min(i + gap, nx), :, -1] = -2
    return f


def flags_posts(nx, ny, nz, gx=2, wx=2, gy=2, wy=2):
    """slip_posts_init.c:14-70 parameterised: gx x gy slip squares with
    periods gx+wx and gy+wy, first at (1, 1), both walls."""
    f = flags_smooth(nx, ny, nz)
    for j in range(1, ny, gy + wy):
        for i in range(1, nx, gx + wx):
            f[i:min(i + gx, nx), j:min(j + gy, ny), 0] = -2
            f[i:min(i + gx, nx), j:min(j + gy, ny), -1] = -2
    return f


def riblet_profile(ny, height, spacing):
    """Solid cells per spanwise index of triangular streamwise riblets: a cell
    of wall distance k - 1/2 (k = 1 the first fluid plane; the halfway wall
    sits at 0) is solid when it lies below the triangle of the given height
    whose base spans one spacing, h(y) = height (1 - |2 y_c / spacing - 1|)
    with y_c = (y mod spacing) + 1/2."""
    yc = (np.arange(ny) % spacing) + 0.5
    h = height * (1.0 - np.abs(2.0 * yc / spacing - 1.0))
    return (np.ceil(h + 0.5) - 1).astype(int)  # number of planes k >= 1 with k - 1/2 < h


def flags_riblets(nx, ny, nz, height, spacing):
    """Triangular riblets aligned with the flow cut into both no-slip walls
    (solid cells -1 inside the flow; boundary mode DNSLBM_BC_GENERAL)."""
    f = flags_smooth(nx, ny, nz)
    nk = riblet_profile(ny, height, spacing)
    for y in range(ny):
        if nk[y] > 0:
            f[:, y, 1:1 + nk[y]] = -1
            f[:, y, nz + 1 - nk[y]:nz + 1] = -1
    return f


def grooves_pitch(pitch, gas_fraction):
    """(gap, width) of a groove texture of the given pitch and gas fraction."""
    gap = int(round(pitch * gas_fraction))
    return gap, pitch - gap


# ------------------------------------------------------------------ workloads
@dataclass
class Workload:
    name: str
    nx: int   # xdv, streamwise
    ny: int   # ydv, spanwise
    nz: int   # zdv, wall-normal fluid planes
    omega: float
    gx: float
    ubulk: float
    steps: int
    texture: str = "smooth"
    tex: dict = field(default_factory=dict)

    @property
    def cells(self):
        return self.nx * self.ny * self.nz


def channel(h=100, re_tau=180.0, texture="smooth", name=None, **tex):
    """Channel of half-height h at friction Reynolds number re_tau:
    (2 pi h) x (2h + 2) x (pi h), u_tau = 0.005, nu = u_tau h / re_tau,
    tau = 0.5 + 3 nu, g = u_tau^2 / h."""
    utau = 0.005
    nu = utau * h / re_tau
    tau = 0.5 + 3 * nu
    nx, ny, nz = round(2 * math.pi * h), round(math.pi * h), 2 * h
    ub = 15.7 * utau * (re_tau / 180.0) ** (1 / 7)  # bulk velocity, 1/7 power law
    return Workload(name or f"channel_re{re_tau:g}_h{h}", nx, ny, nz, 1.0 / tau, utau ** 2 / h, ub, 20, texture, tex)


def channel_180(h=100, texture="smooth", **tex):
    """Re_tau ~ 180 channel of half-height h."""
    return channel(h, 180.0, texture, name=f"channel_re180_h{h}", **tex)


BATCH_HEIGHTS = (20, 32, 48, 64)


def batch_channels(n=24, seed=0):
    """n independent channels with half-heights cycling through 20, 32, 48,
    64, and per channel (numpy PCG64, seed + index): Re_tau uniform in
    [120, 180] and a wall texture drawn from smooth walls, longitudinal
    grooves (pitch 8-32, gas fraction 0.5-0.9), transverse grooves (pitch 16,
    gas fraction 0.5) and triangular riblets (height 4-8, spacing twice the
    height)."""
    out = []
    for i in range(n):
        rng = np.random.Generator(np.random.PCG64(seed + i))
        h = BATCH_HEIGHTS[i % len(BATCH_HEIGHTS)]
        re = float(rng.uniform(120.0, 180.0))
        kind = ("smooth", "longitudinal", "transverse", "riblets")[int(rng.integers(4))]
        if kind == "longitudinal":
            gap, width = grooves_pitch(int(rng.integers(8, 33)), float(rng.uniform(0.5, 0.9)))
            tex = {"gap": max(gap, 1), "width": max(width, 1)}
        elif kind == "transverse":
            tex = dict(zip(("gap", "width"), grooves_pitch(16, 0.5)))
        elif kind == "riblets":
            height = int(rng.integers(4, 9))
            tex = {"height": height, "spacing": 2 * height}
        else:
            tex = {}
        out.append(channel(h, re, kind, name=f"batch{i:02d}_h{h}_re{re:.0f}_{kind}", **tex))
    return out


def workload(name):
    """The reference-shaped workloads: 'laminar64' (64 x 66 x 32, tau 0.52,
    g 1e-6, 1000 steps), 'channel180' (628 x 202 x 314, Re_tau 180),
    'grooves180' (the same with pitch-32, gas-fraction-0.5 longitudinal
    grooves on both walls), 'riblets180' (the same grid with triangular
    riblets of height 8 and spacing 16 cut into both walls) and 'riblets395'
    (Re_tau 395, h = 200: 1256 x 408 x 628 with the same riblets)."""
    if name == "laminar64":
        return Workload("laminar64", 64, 32, 64, 1.0 / 0.52, 1e-6, 0.0, 1000)
    if name == "channel180":
        return channel_180(100)
    if name.startswith("channel180_h"):  # smaller half-heights, same Re_tau
        return channel_180(int(name[len("channel180_h"):]))
    if name == "grooves180":
        g, w = grooves_pitch(32, 0.5)
        return channel_180(100, "longitudinal", gap=g, width=w)
    if name == "riblets180":  # the Re_tau 180 grid with riblets of height 8, spacing 16
        return channel(100, 180.0, "riblets", name="riblets_re180_h100", height=8, spacing=16)
    if name.startswith("riblets180_h"):  # smaller half-heights, same riblets
        h = int(name[len("riblets180_h"):])
        return channel(h, 180.0, "riblets", name=f"riblets_re180_h{h}", height=8, spacing=16)
    if name == "riblets395":  # 1256 x 408 x 628 incl. walls, riblets of height 8, spacing 16
        w = channel(200, 395.0, "riblets", name="riblets_re395_h200", height=8, spacing=16)
        w.nx, w.nz = 1256, 406  # the riblets take the first planes at each wall
        return w
    raise KeyError(name)


def make_flags(wl: Workload):
    if wl.texture == "smooth":
        return flags_smooth(wl.nx, wl.ny, wl.nz)
    if wl.texture == "longitudinal":
        return flags_longitudinal(wl.nx, wl.ny, wl.nz, wl.tex["gap"], wl.tex["width"])
    if wl.texture == "transverse":
        return flags_transverse(wl.nx, wl.ny, wl.nz, wl.tex["gap"], wl.tex["width"])
    if wl.texture == "posts":
        return flags_posts(wl.nx, wl.ny, wl.nz, **wl.tex)
    if wl.texture == "riblets":
        return flags_riblets(wl.nx, wl.ny, wl.nz, wl.tex["height"], wl.tex["spacing"])
    raise KeyError(wl.texture)


def needs_general(wl: Workload):
    """True when the walls put solid cells inside the flow."""
    return wl.texture == "riblets"


def rest_solids(state, flags):
    """The state with every solid cell inside the flow at rest (f = w); the
    wall planes are left as they are."""
    s = state.copy()
    inner = s[:, :, 1:-1]
    inner[flags[:, :, 1:-1] == -1] = W
    return s


def make_state(wl: Workload, seed=0):
    if wl.name == "laminar64":
        return laminar_state(wl.nx, wl.ny, wl.nz, 0.05, 0.01, seed)
    return turbulent_state(wl.nx, wl.ny, wl.nz, wl.ubulk, 0.1, seed)
