"""A channel split into wall-normal slabs (dnslbm_create_slab, slabs.py).

CPU: the slab ranges, and the halo plumbing of HaloExchange as 2 and 3 gloo
ranks (the same code moves CUDA tensors over NCCL): before an odd step each
rank's ghost planes receive its neighbours' edge planes, after it the
ghosts go back into the neighbours' edge planes, and the plane sums of all
ranks are gathered in plane order.

GPU (one device; the slabs of a SlabGroup sit on it side by side and
exchange by device copies): the slabs advance a channel exactly as one
context does -- FP64 and FP32/FP16 populations bit-identical with constant
g (and to the oracle for FP64), constant-Q within 1e-12 -- across both AA
parities and textured walls; the calls out of order are refused."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "dns-solvers_b200"))

import inputs  # noqa: E402
import slabs  # noqa: E402


def test_slab_ranges():
    assert slabs.slab_ranges(10, 3) == [(0, 4), (4, 3), (7, 3)]
    assert slabs.slab_ranges(200, 8)[-1] == (175, 25)
    for zdv, n in ((7, 3), (200, 8), (406, 4)):
        r = slabs.slab_ranges(zdv, n)
        assert r[0][0] == 0 and sum(c for _, c in r) == zdv and all(c >= 2 for _, c in r)
        assert all(a[0] + a[1] == b[0] for a, b in zip(r, r[1:]))
    with pytest.raises(ValueError):
        slabs.slab_ranges(5, 3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


GLOO_RANK = """
import sys, os
sys.path.insert(0, {pkg!r})
import torch, torch.distributed as dist
import slabs
dist.init_process_group("gloo", init_method="env://", timeout=__import__("datetime").timedelta(seconds=60))
r, n = dist.get_rank(), dist.get_world_size()
counts = {counts!r}
P = 7  # elements per halo plane
def edge_val(rank, side, i): return 1000.0 * rank + 100.0 * side + i
halos = {{}}
for side, peer in ((0, r - 1), (1, r + 1)):
    if 0 <= peer < n:
        halos[side] = ([torch.full((P,), -1.0) for _ in range(5)],
                       [torch.full((P,), edge_val(r, side, i)) for i in range(5)])
sums = torch.arange(counts[r] * slabs.SUM_N, dtype=torch.float64) + 10000.0 * r
sums_all = torch.zeros(sum(counts) * slabs.SUM_N, dtype=torch.float64)
x = slabs.HaloExchange(halos, sums, sums_all, counts)
x.fill()
for side, (ghost, edge) in halos.items():
    peer = r - 1 if side == 0 else r + 1
    for i in range(5):  # my ghost on side s mirrors the neighbour's edge on side 1-s
        assert torch.equal(ghost[i], torch.full((P,), edge_val(peer, 1 - side, i))), (r, side, i)
        ghost[i] += 0.5 + 10 * r  # what this rank's odd step streamed across the face
x.drain()
for side, (ghost, edge) in halos.items():
    peer = r - 1 if side == 0 else r + 1
    for i in range(5):
        want = edge_val(r, side, i) + 0.5 + 10 * peer
        assert torch.equal(edge[i], torch.full((P,), want)), (r, side, i, edge[i][0].item(), want)
x.gather()
want = torch.cat([torch.arange(c * slabs.SUM_N, dtype=torch.float64) + 10000.0 * q for q, c in enumerate(counts)])
assert torch.equal(sums_all, want)
dist.barrier()
dist.destroy_process_group()
print("ok", r)
"""


@pytest.mark.parametrize("counts", [[3, 4], [2, 5, 3]])
def test_halo_exchange_gloo(counts):
    code = GLOO_RANK.format(pkg=os.path.join(ROOT, "dns-solvers_b200"), counts=counts)
    port = _free_port()
    procs = []
    for rank in range(len(counts)):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(len(counts)), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, "-c", code], cwd=ROOT, env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    for rank, p in enumerate(procs):
        try:
            o, e = p.communicate(timeout=180)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, e[-2000:]
        assert o.split() == ["ok", str(rank)]


# ------------------------------------------------------------------ GPU
def _whole(s0, fl, omega, nsteps, precision, **kw):
    import dnslbm
    nx, ny, nz = s0.shape[0], s0.shape[1], s0.shape[2] - 2
    with dnslbm.Channel(nx, ny, nz, omega, precision=precision, device=0, **kw) as ch:
        ch.set_flags(fl)
        ch.load_state(s0)
        ch.step(nsteps)
        return ch.store_state(), ch.logs()


def _sliced(s0, fl, omega, nsteps, precision, ranges, **kw):
    import dnslbm
    nx, ny, nz = s0.shape[0], s0.shape[1], s0.shape[2] - 2
    g = slabs.SlabGroup([dnslbm.Slab(nx, ny, nz, z0, n, omega, precision=precision, device=0, **kw)
                         for z0, n in ranges])
    try:
        g.set_flags(fl)
        g.load_state(s0)
        g.step(nsteps)
        return g.store_state(), g.logs()
    finally:
        g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("tex", ["smooth", "grooves"])
@pytest.mark.parametrize("ranges", [[(0, 5), (5, 4), (9, 5)], [(0, 2), (2, 12)], [(0, 14)]])
def test_slabs_fp64_constant_g_bitexact(oracle_mod, tex, ranges):
    nx, ny, nz, omega, g = 40, 12, 14, 1.7, 2e-5
    fl = inputs.flags_smooth(nx, ny, nz) if tex == "smooth" else inputs.flags_longitudinal(nx, ny, nz, 3, 2)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 5)
    ref = s0.copy()
    oracle_mod.run(ref, fl, omega, gx=g, const_g=True, nsteps=10)
    got, lg = _sliced(s0, fl, omega, 10, 64, ranges, gx=g)
    np.testing.assert_array_equal(got[:, :, 1:-1], ref[:, :, 1:-1])
    whole, lw = _whole(s0, fl, omega, 10, 64, gx=g)
    np.testing.assert_array_equal(got[:, :, 1:-1], whole[:, :, 1:-1])
    np.testing.assert_allclose(lg, lw, rtol=1e-11, atol=1e-14)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [32, 16])
def test_slabs_low_precision_constant_g_bitexact(prec):
    nx, ny, nz, omega, g = 36, 10, 12, 1.8, 2e-5
    fl = inputs.flags_longitudinal(nx, ny, nz, 2, 2)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 9)
    got, lg = _sliced(s0, fl, omega, 8, prec, [(0, 4), (4, 3), (7, 5)], gx=g)
    whole, lw = _whole(s0, fl, omega, 8, prec, gx=g)
    np.testing.assert_array_equal(got[:, :, 1:-1], whole[:, :, 1:-1])
    np.testing.assert_allclose(lg, lw, rtol=1e-5, atol=1e-12)


@pytest.mark.gpu
def test_slabs_constant_q():
    import dnslbm
    nx, ny, nz, omega = 32, 12, 16, 1.6
    fl = inputs.flags_longitudinal(nx, ny, nz, 2, 3)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 21)
    kw = dict(ubulk=0.07, force_mode=dnslbm.CONST_Q)
    got, lg = _sliced(s0, fl, omega, 12, 64, [(0, 6), (6, 5), (11, 5)], **kw)
    whole, lw = _whole(s0, fl, omega, 12, 64, **kw)
    np.testing.assert_allclose(got[:, :, 1:-1], whole[:, :, 1:-1], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(lg, lw, rtol=1e-10, atol=1e-14)


@pytest.mark.gpu
def test_slab_calls_out_of_order_are_refused():
    import dnslbm
    nx, ny, nz = 24, 8, 10
    s = dnslbm.Slab(nx, ny, nz, 3, 4, 1.7, gx=1e-5, device=0)
    try:
        assert s.halo(0) is not None and s.halo(1) is not None
        with pytest.raises(dnslbm.DnsLbmError) as e:
            s.step(1)  # a slab never steps alone
        assert e.value.code == dnslbm.ERR_STATE
        s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 2)
        s.load_state(s.part(s0))
        with pytest.raises(dnslbm.DnsLbmError) as e:
            s.kernel_step()  # the load's tail is owed first
        assert e.value.code == dnslbm.ERR_STATE
    finally:
        s.close()
    w = dnslbm.Slab(nx, ny, nz, 0, 4, 1.7, gx=1e-5, device=0)
    try:
        assert w.halo(0) is None  # the lower face is the bottom wall
        rc = w.L.dnslbm_slab_halo(w.h, 0, (dnslbm.ctypes.c_void_p * 5)(), (dnslbm.ctypes.c_void_p * 5)(),
                                  dnslbm.ctypes.byref(dnslbm.ctypes.c_size_t()))
        assert rc == dnslbm.ERR_ARG
    finally:
        w.close()
    with pytest.raises(dnslbm.DnsLbmError) as e:
        dnslbm.Slab(nx, ny, nz, 9, 2, 1.7, device=0)  # planes beyond the channel
    assert e.value.code == dnslbm.ERR_ARG


@pytest.mark.gpu
def test_slab_state_is_read_between_even_steps():
    import dnslbm
    nx, ny, nz = 24, 8, 10
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 4)
    g = slabs.SlabGroup([dnslbm.Slab(nx, ny, nz, z0, n, 1.7, gx=1e-5, device=0) for z0, n in [(0, 5), (5, 5)]])
    try:
        g.load_state(s0)
        g.step(1)
        with pytest.raises(dnslbm.DnsLbmError) as e:
            g.slabs[0].store_state()
        assert e.value.code == dnslbm.ERR_STATE
        g.step(1)
        g.store_state()
    finally:
        g.close()


@pytest.mark.gpu
def test_slab_readers_match_the_whole_channel():
    """Moments and plane statistics of each slab are the whole channel's
    rows for the slab's planes."""
    import dnslbm
    nx, ny, nz, omega, g = 32, 12, 12, 1.7, 2e-5
    fl = inputs.flags_longitudinal(nx, ny, nz, 2, 2)
    s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 31)
    with dnslbm.Channel(nx, ny, nz, omega, gx=g, device=0) as ch:
        ch.set_flags(fl)
        ch.load_state(s0)
        ch.step(6)
        vel, den = ch.moments()
        stats = ch.statistics()
    grp = slabs.SlabGroup([dnslbm.Slab(nx, ny, nz, z0, n, omega, gx=g, device=0) for z0, n in [(0, 5), (5, 7)]])
    try:
        grp.set_flags(fl)
        grp.load_state(s0)
        grp.step(6)
        for s in grp.slabs:
            v, d = s.moments()
            st = s.statistics()
            k = slice(s.z0 + 1, s.z0 + s.nzs + 1)
            np.testing.assert_array_equal(v[:, :, 1:-1], vel[:, :, k])
            np.testing.assert_array_equal(d[:, :, 1:-1], den[:, :, k])
            np.testing.assert_allclose(st[:, 1:-1], stats[:, k], rtol=1e-12, atol=1e-16)
    finally:
        grp.close()


DIST_ONE_RANK = """
import sys, os, datetime
sys.path.insert(0, {pkg!r})
import numpy as np, torch, torch.distributed as dist
import dnslbm, inputs, slabs
dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=60),
                        device_id=torch.device("cuda:0"))
nx, ny, nz, omega, g = 32, 12, 10, 1.7, 2e-5
fl = inputs.flags_longitudinal(nx, ny, nz, 2, 2)
s0 = inputs.laminar_state(nx, ny, nz, 0.08, 0.1, 17)
with dnslbm.Channel(nx, ny, nz, omega, gx=g, device=0) as ch:
    ch.set_flags(fl); ch.load_state(s0); ch.step(8); want = ch.store_state(); wl = ch.logs()
s = dnslbm.Slab(nx, ny, nz, 0, nz, omega, gx=g, device=0)
s.set_flags(fl)
s.load_state(s.part(s0))
ds = slabs.DistributedSlab(s)
ds.after_load()
ds.step(8)
got = s.store_state()
assert np.array_equal(got[:, :, 1:-1], want[:, :, 1:-1])
assert np.allclose(s.logs(), wl, rtol=1e-11, atol=1e-14)
s.close()
dist.destroy_process_group()
print("ok")
"""


@pytest.mark.gpu
def test_distributed_slab_one_rank_nccl():
    """DistributedSlab on a one-rank NCCL group (this run has one GPU): the
    sums gather and the tail run on the slab's own stream through NCCL, and
    the channel steps bit-identically to one context."""
    code = DIST_ONE_RANK.format(pkg=os.path.join(ROOT, "dns-solvers_b200"))
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()),
               NCCL_NVLS_ENABLE="0")
    p = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    assert p.stdout.split()[-1:] == ["ok"], p.stdout[-500:]  # NCCL may print its version first
