"""A channel split into wall-normal slabs over several GPUs.

The reference splits its domain over MPI ranks (the cartesian grid of
DNS-solver/src/dns-const-q-xycut.c:63-125) and exchanges halo faces every
step through persistent requests (xcomputations.c:222-289,435-555).  Here a
slab is a range of whole wall-normal planes (dnslbm.Slab, one context per
GPU): planes are contiguous in every population array, so the halo is five
whole planes per face, and each plane's statistics belong to one slab.

In the AA scheme only the odd step reads and writes across a face, so the
exchange happens around odd steps only: before it every slab fills its
ghost planes from its neighbours' edge planes, after it the ghosts (now
holding what the slab streamed across the face) go back to the neighbours'
edge planes.  Every step the slabs' plane sums are gathered in plane order
and each slab runs the whole channel's step tail on them (logs, constant-Q
force, plane means: the same on every slab).

Two ways to move the data:
  * SlabGroup: all slabs in this process (on one GPU or several), device
    copies between them;
  * HaloExchange / DistributedSlab: one slab per rank of a torch.distributed
    group (NCCL over NVLink on GPUs; the same code moves CPU tensors under
    gloo), point-to-point sends of the halo planes and an all-gather of the
    sums.
"""
from __future__ import annotations

import numpy as np

import dnslbm

SUM_N = dnslbm.Slab.SUM_N
_TORCH_DTYPE = {64: "float64", 32: "float32", 16: "float16"}


def slab_ranges(zdv, n):
    """Split zdv planes into n contiguous slabs (z0, nzs), as even as
    possible, bottom first; every slab gets at least 2 planes."""
    if n < 1 or zdv < 2 * n:
        raise ValueError(f"{zdv} planes cannot make {n} slabs of at least 2 planes")
    base, extra = divmod(zdv, n)
    out, z0 = [], 0
    for r in range(n):
        nzs = base + (1 if r < extra else 0)
        out.append((z0, nzs))
        z0 += nzs
    return out


class _DeviceArray:
    """A raw device pointer seen through the CUDA array interface."""

    def __init__(self, ptr, count, typestr):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def device_tensor(ptr, nbytes, precision, device):
    """A torch tensor over `nbytes` of device memory at `ptr` (no copy)."""
    import torch
    esize = precision // 8
    typestr = {8: "<f8", 4: "<f4", 2: "<f2"}[esize]
    t = torch.as_tensor(_DeviceArray(ptr, nbytes // esize, typestr), device=f"cuda:{device}")
    assert t.dtype == getattr(torch, _TORCH_DTYPE[precision])
    return t


def _halo_tensors(slab):
    """{side: (ghost tensors[5], edge tensors[5])} of a slab's non-wall faces."""
    out = {}
    for side in (0, 1):
        h = slab.halo(side)
        if h is None:
            continue
        ghost, edge, nbytes = h
        prec = slab.deck.precision
        out[side] = ([device_tensor(p, nbytes, prec, slab.device) for p in ghost],
                     [device_tensor(p, nbytes, prec, slab.device) for p in edge])
    return out


class SlabGroup:
    """All slabs of one channel in this process, ordered bottom to top (they
    may sit on different GPUs).  Ghost planes and plane sums move by device
    copies; the host waits for every slab's stream around each copy."""

    def __init__(self, slabs):
        import torch
        self.slabs = list(slabs)
        z = 0
        for s in self.slabs:
            assert s.z0 == z, "slabs must cover the channel bottom to top"
            z += s.nzs
        assert z == self.slabs[0].channel_shape[2]
        self.halos = [_halo_tensors(s) for s in self.slabs]
        self.sums = [device_tensor(s.sums_ptr(), s.nzs * SUM_N * 8, 64, s.device) for s in self.slabs]
        self.sums_all = {}
        for s in self.slabs:
            if s.device not in self.sums_all:
                self.sums_all[s.device] = torch.zeros(z * SUM_N, dtype=torch.float64, device=f"cuda:{s.device}")

    def _wait(self):
        import torch
        for s in self.slabs:
            s.sync()
        for d in self.sums_all:
            torch.cuda.synchronize(d)

    def _exchange(self, fill):
        # the ghost of slab r on side 1 mirrors the edge of slab r+1 on side 0,
        # and the ghost of slab r+1 on side 0 the edge of slab r on side 1
        for r in range(len(self.slabs) - 1):
            lo_g, lo_e = self.halos[r][1]
            hi_g, hi_e = self.halos[r + 1][0]
            for i in range(5):
                if fill:
                    lo_g[i].copy_(hi_e[i])
                    hi_g[i].copy_(lo_e[i])
                else:
                    hi_e[i].copy_(lo_g[i])
                    lo_e[i].copy_(hi_g[i])

    def _tail(self):
        import torch
        self._wait()
        for d, buf in self.sums_all.items():
            buf.copy_(torch.cat([t.to(buf.device) for t in self.sums]))
        self._wait()
        for s in self.slabs:
            s.tail(self.sums_all[s.device].data_ptr())

    def set_flags(self, flags):
        for s in self.slabs:
            s.set_flags(flags)

    def load_state(self, state):
        """Whole-channel state (xdv, ydv, zdv+2, 19)."""
        for s in self.slabs:
            s.load_state(s.part(state))
        self._tail()  # the initial reduction's tail
        self._wait()

    def init_rest(self):
        for s in self.slabs:
            s.init_rest()
        self._tail()
        self._wait()

    def step(self, n=1):
        for _ in range(n):
            odd = self.slabs[0].steps_done % 2 == 1
            if odd:
                self._wait()
                self._exchange(fill=True)
                self._wait()
            for s in self.slabs:
                s.kernel_step()
            if odd:
                self._wait()
                self._exchange(fill=False)
            self._tail()
        for s in self.slabs:
            s.status()

    def store_state(self):
        """Whole-channel state assembled from the slabs (after an even number
        of steps)."""
        x, y, zdv = self.slabs[0].channel_shape
        out = np.zeros((x, y, zdv + 2, 19))
        for s in self.slabs:
            out[:, :, s.z0 + 1:s.z0 + s.nzs + 1] = s.store_state()[:, :, 1:s.nzs + 1]
        return out

    def logs(self, first=0, count=None):
        return self.slabs[0].logs(first, count)

    @property
    def steps_done(self):
        return self.slabs[0].steps_done

    def close(self):
        for s in self.slabs:
            s.close()


class HaloExchange:
    """The ghost-plane exchange and the sums gather of one slab per rank of a
    torch.distributed group: rank r holds slab r, rank r-1 the slab below,
    rank r+1 the one above.  `halos` is {side: (ghost[5], edge[5])} for the
    faces that meet a neighbour, `sums` the slab's plane sums (counts[rank] *
    SUM_N values), `sums_all` receives every rank's sums in plane order.
    The tensors may be CUDA tensors (NCCL) or CPU tensors (gloo)."""

    def __init__(self, halos, sums, sums_all, counts, group=None):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        assert len(counts) == self.world and sum(counts) * SUM_N == sums_all.numel()
        assert sums.numel() == counts[self.rank] * SUM_N
        for side, peer in ((0, self.rank - 1), (1, self.rank + 1)):
            assert (side in halos) == (0 <= peer < self.world), f"face {side} of rank {self.rank}"
        self.halos, self.sums, self.sums_all, self.counts = halos, sums, sums_all, list(counts)
        self.width = max(counts) * SUM_N
        self.pad = torch.zeros(self.width, dtype=sums.dtype, device=sums.device)
        self.gathered = torch.zeros(self.world * self.width, dtype=sums.dtype, device=sums.device)

    def _peer(self, side):
        r = self.rank - 1 if side == 0 else self.rank + 1
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def _p2p(self, send_ghosts):
        ops = []
        for side in sorted(self.halos):
            ghost, edge = self.halos[side]
            peer = self._peer(side)
            for i in range(5):
                # edges travel into the neighbour's ghosts (fill); ghosts
                # travel back into the neighbour's edges (drain)
                send, recv = (ghost[i], edge[i]) if send_ghosts else (edge[i], ghost[i])
                ops.append(self.dist.P2POp(self.dist.isend, send, peer, self.group))
                ops.append(self.dist.P2POp(self.dist.irecv, recv, peer, self.group))
        if ops:
            for w in self.dist.batch_isend_irecv(ops):
                w.wait()

    def fill(self):
        """Before an odd step: ghost <- neighbour's edge."""
        self._p2p(send_ghosts=False)

    def drain(self):
        """After an odd step: neighbour's edge <- ghost."""
        self._p2p(send_ghosts=True)

    def gather(self):
        """sums_all <- every rank's sums, in plane order."""
        n = self.sums.numel()
        self.pad[:n].copy_(self.sums)
        self.dist.all_gather_into_tensor(self.gathered, self.pad, group=self.group)
        o = 0
        for r, c in enumerate(self.counts):
            m = c * SUM_N
            self.sums_all[o:o + m].copy_(self.gathered[r * self.width:r * self.width + m])
            o += m


class DistributedSlab:
    """One slab per rank (one process per GPU) of a channel split over a
    torch.distributed group, the exchange on the slab's own CUDA stream."""

    def __init__(self, slab, group=None):
        import torch
        import torch.distributed as dist
        self.slab = slab
        world = dist.get_world_size(group)
        n = torch.tensor([slab.nzs], dtype=torch.int64, device=f"cuda:{slab.device}")
        counts = torch.zeros(world, dtype=torch.int64, device=n.device)
        dist.all_gather_into_tensor(counts, n, group=group)
        counts = [int(c) for c in counts.cpu()]
        zdv = slab.channel_shape[2]
        assert sum(counts) == zdv
        self.sums_all = torch.zeros(zdv * SUM_N, dtype=torch.float64, device=n.device)
        sums = device_tensor(slab.sums_ptr(), slab.nzs * SUM_N * 8, 64, slab.device)
        self.x = HaloExchange(_halo_tensors(slab), sums, self.sums_all, counts, group)
        self.stream = torch.cuda.ExternalStream(slab.stream, device=n.device)

    def _tail(self):
        self.x.gather()
        self.slab.tail(self.sums_all.data_ptr())

    def after_load(self):
        """The tail a load or init_rest owes."""
        import torch
        with torch.cuda.stream(self.stream):
            self._tail()

    def step(self, n=1):
        import torch
        with torch.cuda.stream(self.stream):
            for _ in range(n):
                odd = self.slab.steps_done % 2 == 1
                if odd:
                    self.x.fill()
                self.slab.kernel_step()
                if odd:
                    self.x.drain()
                self._tail()
        self.slab.status()
