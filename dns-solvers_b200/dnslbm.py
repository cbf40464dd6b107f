"""Python binding of the dnslbm C ABI (include/dnslbm.h) over ctypes.

The product is ``libdnslbm.so`` (sm_100a kernels + C ABI); this module only
marshals numpy arrays to it.  There is no fallback: if the library or a CUDA
device is missing, every call raises.

Array layouts are the reference's (see include/dnslbm.h):
  state  float64 (xdv, ydv, zdv+2, 19)   lbf/ftemp layout without ghosts
  flags  int8    (xdv, ydv, zdv+2)       0 fluid, -1 no-slip, -2 slip
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdnslbm.so")

OK, ERR_ARG, ERR_CUDA, ERR_NAN, ERR_TIMEOUT, ERR_NOMEM, ERR_IO, ERR_STATE = range(8)
F64, F32, F16 = 64, 32, 16
CONST_Q, CONST_G = 0, 1
BC_REFERENCE, BC_GENERAL = 0, 1
LOG_NAMES = ("force", "rho", "energy", "flowrate", "massrate", "stup", "stdown", "stress", "pgrad")


class DnsLbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"dnslbm error {code}: {msg}")
        self.code = code


class Deck(ctypes.Structure):
    """The reference's parameter deck (definitions.h:30-59), at run time."""
    _fields_ = [("xdv", ctypes.c_int), ("ydv", ctypes.c_int), ("zdv", ctypes.c_int),
                ("omega", ctypes.c_double), ("ubulk", ctypes.c_double), ("gx", ctypes.c_double),
                ("force_mode", ctypes.c_int), ("precision", ctypes.c_int), ("bc_mode", ctypes.c_int),
                ("log_capacity", ctypes.c_int), ("device", ctypes.c_int)]


_lib = None


def lib():
    """Load libdnslbm.so (raises if it is missing: there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not built (run __graft_entry__.build())")
    L = ctypes.CDLL(LIB_PATH)
    vp, dp, ip, i8p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int), \
        ctypes.POINTER(ctypes.c_int8)
    L.dnslbm_create.argtypes = [ctypes.POINTER(Deck), ctypes.POINTER(vp)]
    L.dnslbm_destroy.argtypes = [vp]
    L.dnslbm_destroy.restype = None
    L.dnslbm_last_error.argtypes = [vp]
    L.dnslbm_last_error.restype = ctypes.c_char_p
    L.dnslbm_set_flags.argtypes = [vp, ip]
    L.dnslbm_set_flags_periodic.argtypes = [vp, i8p]
    L.dnslbm_link_masks.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, i8p, ip,
                                    ctypes.POINTER(ctypes.c_uint), ctypes.c_size_t, ip]
    L.dnslbm_init_rest.argtypes = [vp]
    L.dnslbm_load_state.argtypes = [vp, dp]
    L.dnslbm_store_state.argtypes = [vp, dp]
    L.dnslbm_load_state_slab.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
    L.dnslbm_step.argtypes = [vp, ctypes.c_long]
    L.dnslbm_steps_done.argtypes = [vp]
    L.dnslbm_steps_done.restype = ctypes.c_long
    L.dnslbm_logs.argtypes = [vp, ctypes.c_long, ctypes.c_long, dp]
    L.dnslbm_get_force.argtypes = [vp, dp]
    L.dnslbm_statistics.argtypes = [vp, dp]
    L.dnslbm_stats_accumulate.argtypes = [vp]
    L.dnslbm_stats_average.argtypes = [vp, dp, ctypes.POINTER(ctypes.c_long)]
    L.dnslbm_stats_reset.argtypes = [vp]
    L.dnslbm_moments.argtypes = [vp, dp, dp]
    L.dnslbm_step_timed.argtypes = [vp, ctypes.c_long, dp, dp, dp]
    L.dnslbm_autotune.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    L.dnslbm_quadrant.argtypes = [vp, dp, dp, dp]
    L.dnslbm_quadrant_vel.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.dnslbm_correlations.argtypes = [vp, dp, dp, dp]
    L.dnslbm_spectra.argtypes = [vp, dp, dp]
    L.dnslbm_spectra_vel.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp]
    L.dnslbm_correlations_vel.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, dp]
    L.dnslbm_output_begin.argtypes = [vp, dp, dp, dp, dp]
    L.dnslbm_output_wait.argtypes = [vp]
    L.dnslbm_set_wait_limit.argtypes = [vp, ctypes.c_double]
    L.dnslbm_test_withhold_load.argtypes = [vp]
    L.dnslbm_step_kernel.argtypes = [vp]
    L.dnslbm_step_kernel.restype = ctypes.c_char_p
    L.dnslbm_bytes_per_cell.argtypes = [vp]
    L.dnslbm_bytes_per_cell.restype = ctypes.c_double
    L.dnslbm_sync.argtypes = [vp]
    L.dnslbm_batch_create.argtypes = [ctypes.POINTER(Deck), ctypes.c_int, ctypes.POINTER(vp)]
    L.dnslbm_batch_destroy.argtypes = [vp]
    L.dnslbm_batch_destroy.restype = None
    L.dnslbm_batch_last_error.argtypes = [vp]
    L.dnslbm_batch_last_error.restype = ctypes.c_char_p
    L.dnslbm_batch_size.argtypes = [vp]
    L.dnslbm_batch_channel.argtypes = [vp, ctypes.c_int]
    L.dnslbm_batch_channel.restype = vp
    L.dnslbm_batch_step.argtypes = [vp, ctypes.c_long]
    L.dnslbm_batch_step_timed.argtypes = [vp, ctypes.c_long, dp]
    L.dnslbm_batch_kernel.argtypes = [vp]
    L.dnslbm_batch_kernel.restype = ctypes.c_char_p
    L.dnslbm_batch_autotune.argtypes = [vp, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t]
    L.dnslbm_batch_test_withhold_load.argtypes = [vp, ctypes.c_double]
    L.dnslbm_create_slab.argtypes = [ctypes.POINTER(Deck), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]
    L.dnslbm_slab_step.argtypes = [vp]
    L.dnslbm_slab_sums.argtypes = [vp, ctypes.POINTER(ctypes.c_void_p)]
    L.dnslbm_slab_tail.argtypes = [vp, vp]
    L.dnslbm_slab_status.argtypes = [vp]
    L.dnslbm_slab_halo.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                   ctypes.POINTER(ctypes.c_size_t)]
    L.dnslbm_stream.argtypes = [vp]
    L.dnslbm_stream.restype = vp
    L.dnslbm_host_alloc.argtypes = [ctypes.c_size_t]
    L.dnslbm_host_alloc.restype = vp
    L.dnslbm_host_free.argtypes = [vp]
    L.dnslbm_host_free.restype = None
    _lib = L
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Channel:
    """One channel on one GPU: a dnslbm context."""

    def __init__(self, xdv, ydv, zdv, omega, ubulk=0.0, gx=0.0, force_mode=CONST_G, precision=F64,
                 bc_mode=BC_REFERENCE, log_capacity=0, device=0):
        self.L = lib()
        self.shape = (xdv, ydv, zdv)
        d = Deck(xdv, ydv, zdv, omega, ubulk, gx, force_mode, precision, bc_mode, log_capacity, device)
        h = ctypes.c_void_p()
        rc = self.L.dnslbm_create(ctypes.byref(d), ctypes.byref(h))
        if rc:
            raise DnsLbmError(rc, self.L.dnslbm_last_error(None).decode())
        self.h = h
        self.deck = d

    def _ck(self, rc):
        if rc:
            raise DnsLbmError(rc, self.L.dnslbm_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.dnslbm_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def state_shape(self):
        x, y, z = self.shape
        return (x, y, z + 2, 19)

    def set_flags(self, flags):
        """flags: int8 (xdv, ydv, zdv+2) periodic grid, or int32 reference
        V.s array (xdv+1, ydv+1, zdv+2) with ghost planes."""
        if flags.dtype == np.int8:
            f = np.ascontiguousarray(flags)
            assert f.shape == self.state_shape[:3]
            self._ck(self.L.dnslbm_set_flags_periodic(self.h, f.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))))
        else:
            f = np.ascontiguousarray(flags, np.int32)
            x, y, z = self.shape
            assert f.shape == (x + 1, y + 1, z + 2)
            self._ck(self.L.dnslbm_set_flags(self.h, f.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    def init_rest(self):
        self._ck(self.L.dnslbm_init_rest(self.h))

    def load_state(self, state):
        s = np.ascontiguousarray(state, np.float64)
        assert s.shape == self.state_shape, (s.shape, self.state_shape)
        self._ck(self.L.dnslbm_load_state(self.h, _dp(s)))

    def load_state_slab(self, x0, slab):
        """Part of a state: x in [x0, x0 + len(slab)) (dnslbm_load_state_slab)."""
        s = np.ascontiguousarray(slab, np.float64)
        assert s.shape[1:] == self.state_shape[1:], (s.shape, self.state_shape)
        self._ck(self.L.dnslbm_load_state_slab(self.h, x0, s.shape[0], _dp(s)))

    def load_state_slabs(self, slabs):
        """A whole state from (x0, slab) pairs in order of x."""
        for x0, slab in slabs:
            self.load_state_slab(x0, slab)

    def store_state(self, out=None):
        if out is None:
            out = np.empty(self.state_shape, np.float64)
        self._ck(self.L.dnslbm_store_state(self.h, _dp(out)))
        return out

    def step(self, n=1):
        self._ck(self.L.dnslbm_step(self.h, n))

    def step_timed(self, n, per_launch=True):
        """(total ms, even-launch ms, odd-launch ms) of n steps; per_launch
        False times the whole run only (even/odd None)."""
        t, e, o = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        if not per_launch:
            self._ck(self.L.dnslbm_step_timed(self.h, n, ctypes.byref(t), None, None))
            return t.value, None, None
        self._ck(self.L.dnslbm_step_timed(self.h, n, ctypes.byref(t), ctypes.byref(e), ctypes.byref(o)))
        return t.value, e.value, o.value

    def correlations(self):
        """Two-point correlations of the current state: (xcorl[zd][nx][3],
        ycorl[zd][ny][3], uavg[zd]) as the reference's 2pt-correlations
        program writes them."""
        zd = self.shape[2] + 2
        xc, yc, ua = np.zeros((zd, self.shape[0], 3)), np.zeros((zd, self.shape[1], 3)), np.zeros(zd)
        self._ck(self.L.dnslbm_correlations(self.h, _dp(xc), _dp(yc), _dp(ua)))
        return xc, yc, ua

    def spectra(self):
        """One-dimensional energy spectra of the current state: (ex[3][nx][zd],
        ey[3][ny//2+1][zd]) as the reference's e-spectra program writes
        Euux/Evvx/Ewwx and Euuy/Evvy/Ewwy."""
        nx, ny, nz = self.shape
        ex, ey = np.zeros((3, nx, nz + 2)), np.zeros((3, ny // 2 + 1, nz + 2))
        self._ck(self.L.dnslbm_spectra(self.h, _dp(ex), _dp(ey)))
        return ex, ey

    def quadrant(self):
        """Quadrant analysis of the current state: (quadrant[4][zd],
        dquadrant[4][zd], uw[zd]) as the reference's quadrant files."""
        zd = self.shape[2] + 2
        q, dq, uw = np.zeros((4, zd)), np.zeros((4, zd)), np.zeros(zd)
        self._ck(self.L.dnslbm_quadrant(self.h, _dp(q), _dp(dq), _dp(uw)))
        return q, dq, uw

    def output_begin(self, state=None, vel=None, den=None, stats=None):
        """Start the asynchronous output of the current state into the given
        host arrays (page-locked for overlap: PinnedArray); they are valid
        after output_wait()."""
        shapes = {"state": self.state_shape, "vel": self.state_shape[:3] + (3,), "den": self.state_shape[:3],
                  "stats": (9, self.shape[2] + 2)}
        ptrs = []
        for name, a in (("state", state), ("vel", vel), ("den", den), ("stats", stats)):
            if a is None:
                ptrs.append(None)
                continue
            assert a.shape == shapes[name] and a.dtype == np.float64 and a.flags.c_contiguous, name
            ptrs.append(_dp(a))
        self._ck(self.L.dnslbm_output_begin(self.h, *ptrs))

    def output_wait(self):
        self._ck(self.L.dnslbm_output_wait(self.h))

    def set_wait_limit(self, ms):
        """Limit (ms) of the row-pipelined kernel's bounded device waits."""
        self._ck(self.L.dnslbm_set_wait_limit(self.h, ms))

    def test_withhold_load(self):
        """Test hook: the next bulk-copy launch withholds one load, so a
        bounded wait runs out and that step call raises ERR_TIMEOUT."""
        self._ck(self.L.dnslbm_test_withhold_load(self.h))

    @property
    def steps_done(self):
        return self.L.dnslbm_steps_done(self.h)

    def logs(self, first=0, count=None):
        if count is None:
            count = self.steps_done - first
        out = np.zeros((count, 9), np.float64)
        self._ck(self.L.dnslbm_logs(self.h, first, count, _dp(out)))
        return out

    def force(self):
        v = ctypes.c_double()
        self._ck(self.L.dnslbm_get_force(self.h, ctypes.byref(v)))
        return v.value

    def statistics(self):
        zd = self.shape[2] + 2
        out = np.zeros(9 * zd)
        self._ck(self.L.dnslbm_statistics(self.h, _dp(out)))
        return out.reshape(9, zd)

    def stats_accumulate(self):
        """Add a sample of the current plane statistics to the device average."""
        self._ck(self.L.dnslbm_stats_accumulate(self.h))

    def stats_average(self):
        """(averages [9, zd], number of samples) of the device time average."""
        out = np.zeros((9, self.shape[2] + 2), np.float64)
        n = ctypes.c_long()
        self._ck(self.L.dnslbm_stats_average(self.h, _dp(out), ctypes.byref(n)))
        return out, n.value

    def stats_reset(self):
        self._ck(self.L.dnslbm_stats_reset(self.h))
    def moments(self, vel=None, den=None):
        x, y, z = self.shape
        if vel is None:
            vel = np.zeros((x, y, z + 2, 3))
        if den is None:
            den = np.zeros((x, y, z + 2))
        assert vel.shape == (x, y, z + 2, 3) and den.shape == (x, y, z + 2)
        self._ck(self.L.dnslbm_moments(self.h, _dp(vel), _dp(den)))
        return vel, den

    def autotune(self, steps=6):
        """Time the candidate launch shapes on this grid and keep the fastest
        (call before loading a state).  Returns the tuner's one-line report."""
        buf = ctypes.create_string_buffer(512)
        self._ck(self.L.dnslbm_autotune(self.h, steps, buf, len(buf)))
        return buf.value.decode()

    @property
    def kernel(self):
        """Description of the step kernel this context launches."""
        return self.L.dnslbm_step_kernel(self.h).decode()

    @property
    def bytes_per_cell(self):
        return self.L.dnslbm_bytes_per_cell(self.h)

    def sync(self):
        self._ck(self.L.dnslbm_sync(self.h))


class Slab(Channel):
    """Wall-normal planes [z0, z0 + nzs) of a channel of zdv planes, on one
    GPU (dnslbm_create_slab).  States (load/store, moments, statistics) are
    the slab's planes, arrays of shape (xdv, ydv, nzs + 2, 19); flags are the
    whole channel's.  It steps with its neighbours through a SlabGroup or a
    HaloExchange (slabs.py), never alone with step()."""

    SUM_N = 8  # doubles per plane of the slab sums (DNSLBM_SUM_N)

    def __init__(self, xdv, ydv, zdv, z0, nzs, omega, ubulk=0.0, gx=0.0, force_mode=CONST_G, precision=F64,
                 log_capacity=0, device=0):
        self.L = lib()
        self.channel_shape = (xdv, ydv, zdv)
        self.shape = (xdv, ydv, nzs)
        self.z0, self.nzs, self.device = z0, nzs, device
        d = Deck(xdv, ydv, zdv, omega, ubulk, gx, force_mode, precision, BC_REFERENCE, log_capacity, device)
        h = ctypes.c_void_p()
        rc = self.L.dnslbm_create_slab(ctypes.byref(d), z0, nzs, ctypes.byref(h))
        if rc:
            raise DnsLbmError(rc, self.L.dnslbm_last_error(None).decode())
        self.h = h
        self.deck = d
        self.walls = (z0 == 0, z0 + nzs == zdv)

    def set_flags(self, flags):
        """The whole channel's flags: int8 (xdv, ydv, zdv+2) or the
        reference's V.s (xdv+1, ydv+1, zdv+2)."""
        x, y, z = self.channel_shape
        if flags.dtype == np.int8:
            f = np.ascontiguousarray(flags)
            assert f.shape == (x, y, z + 2)
            self._ck(self.L.dnslbm_set_flags_periodic(self.h, f.ctypes.data_as(ctypes.POINTER(ctypes.c_int8))))
        else:
            f = np.ascontiguousarray(flags, np.int32)
            assert f.shape == (x + 1, y + 1, z + 2)
            self._ck(self.L.dnslbm_set_flags(self.h, f.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    def part(self, whole):
        """The slab's planes k = z0 .. z0+nzs+1 of a whole-channel array
        (state, vel, den: axis 2 is k)."""
        return np.ascontiguousarray(whole[:, :, self.z0:self.z0 + self.nzs + 2])

    def kernel_step(self):
        self._ck(self.L.dnslbm_slab_step(self.h))

    def sums_ptr(self):
        p = ctypes.c_void_p()
        self._ck(self.L.dnslbm_slab_sums(self.h, ctypes.byref(p)))
        return p.value

    def tail(self, sums_all_ptr):
        self._ck(self.L.dnslbm_slab_tail(self.h, ctypes.c_void_p(sums_all_ptr)))

    def status(self):
        self._ck(self.L.dnslbm_slab_status(self.h))

    def halo(self, side):
        """(ghost pointers[5], edge pointers[5], bytes per plane) of face
        `side` (0 lower, 1 upper), or None on a wall face."""
        if self.walls[side]:
            return None
        g, e, n = (ctypes.c_void_p * 5)(), (ctypes.c_void_p * 5)(), ctypes.c_size_t()
        self._ck(self.L.dnslbm_slab_halo(self.h, side, g, e, ctypes.byref(n)))
        return [v for v in g], [v for v in e], n.value

    @property
    def stream(self):
        return self.L.dnslbm_stream(self.h)


class _Borrowed(Channel):
    """A channel owned by a Batch (destroyed with the batch, not alone)."""

    def __init__(self, L, h, shape, deck):
        self.L, self.h, self.shape, self.deck = L, h, shape, deck

    def close(self):
        self.h = None

    __del__ = close


def deck(xdv, ydv, zdv, omega, ubulk=0.0, gx=0.0, force_mode=CONST_G, precision=F64, bc_mode=BC_REFERENCE,
         log_capacity=0, device=0):
    return Deck(xdv, ydv, zdv, omega, ubulk, gx, force_mode, precision, bc_mode, log_capacity, device)


class Batch:
    """Many independent channels stepped together by the persistent batch
    kernel, the time loop replayed from a CUDA graph (dnslbm_batch_*)."""

    def __init__(self, decks):
        self.L = lib()
        arr = (Deck * len(decks))(*decks)
        h = ctypes.c_void_p()
        rc = self.L.dnslbm_batch_create(arr, len(decks), ctypes.byref(h))
        if rc:
            raise DnsLbmError(rc, self.L.dnslbm_batch_last_error(None).decode())
        self.h = h
        self.channels = [_Borrowed(self.L, ctypes.c_void_p(self.L.dnslbm_batch_channel(h, i)),
                                   (d.xdv, d.ydv, d.zdv), d) for i, d in enumerate(decks)]

    def _ck(self, rc):
        if rc:
            raise DnsLbmError(rc, self.L.dnslbm_batch_last_error(self.h).decode())

    def step(self, n=1):
        self._ck(self.L.dnslbm_batch_step(self.h, n))

    def step_timed(self, n):
        ms = ctypes.c_double()
        self._ck(self.L.dnslbm_batch_step_timed(self.h, n, ctypes.byref(ms)))
        return ms.value

    @property
    def kernel(self):
        return self.L.dnslbm_batch_kernel(self.h).decode()

    def test_withhold_load(self, wait_ms=1.0):
        """Test hook: the next step call withholds one load (ERR_TIMEOUT)."""
        self._ck(self.L.dnslbm_batch_test_withhold_load(self.h, wait_ms))

    def autotune(self, steps=8):
        """Pick the fastest launch shape on rest states; before any load."""
        buf = ctypes.create_string_buffer(512)
        self._ck(self.L.dnslbm_batch_autotune(self.h, steps, buf, 512))
        return buf.value.decode()

    def close(self):
        if getattr(self, "h", None):
            for c in self.channels:
                c.close()
            self.L.dnslbm_batch_destroy(self.h)
            self.h = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def link_masks(flags, bc_mode=BC_GENERAL):
    """(band_of [zdv], links [nband, ydv, xdv]) the library builds from an
    int8 (xdv, ydv, zdv+2) flag array (host only, dnslbm_link_masks)."""
    L = lib()
    f = np.ascontiguousarray(flags, np.int8)
    nx, ny, zd = f.shape
    band = np.zeros(zd - 2, np.int32)
    links = np.zeros((zd - 2) * ny * nx, np.uint32)
    nb = ctypes.c_int()
    rc = L.dnslbm_link_masks(nx, ny, zd - 2, bc_mode, f.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)),
                             band.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             links.ctypes.data_as(ctypes.POINTER(ctypes.c_uint)), links.size, ctypes.byref(nb))
    if rc:
        raise DnsLbmError(rc, L.dnslbm_last_error(None).decode())
    return band, links[:nb.value * ny * nx].reshape(nb.value, ny, nx)


class PinnedArray:
    """A numpy view of page-locked host memory from dnslbm_host_alloc."""

    def __init__(self, shape, dtype=np.float64):
        self.L = lib()
        n = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = self.L.dnslbm_host_alloc(n)
        if not self.ptr:
            raise MemoryError(f"dnslbm_host_alloc({n}) failed")
        buf = (ctypes.c_char * n).from_address(self.ptr)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self.ptr:
            self.array = None
            self.L.dnslbm_host_free(self.ptr)
            self.ptr = None

    __del__ = free


def quadrant_vel(vel, device=0):
    """Quadrant analysis of a velocity field [xdv][ydv][zd][3] on the GPU."""
    L = lib()
    v = np.ascontiguousarray(vel, np.float64)
    nx, ny, zd, three = v.shape
    assert three == 3
    q, dq, uw = np.zeros((4, zd)), np.zeros((4, zd)), np.zeros(zd)
    rc = L.dnslbm_quadrant_vel(_dp(v), nx, ny, zd - 2, device, _dp(q), _dp(dq), _dp(uw))
    if rc:
        raise DnsLbmError(rc, L.dnslbm_last_error(None).decode())
    return q, dq, uw


def correlations_vel(vel, device=0):
    """Two-point correlations of a velocity field [xdv][ydv][zd][3] on the
    GPU: (xcorl[zd][xdv][3], ycorl[zd][ydv][3], uavg[zd])."""
    L = lib()
    v = np.ascontiguousarray(vel, np.float64)
    nx, ny, zd, three = v.shape
    assert three == 3
    xc, yc, ua = np.zeros((zd, nx, 3)), np.zeros((zd, ny, 3)), np.zeros(zd)
    rc = L.dnslbm_correlations_vel(_dp(v), nx, ny, zd - 2, device, _dp(xc), _dp(yc), _dp(ua))
    if rc:
        raise DnsLbmError(rc, L.dnslbm_last_error(None).decode())
    return xc, yc, ua


def spectra_vel(vel, device=0):
    """One-dimensional energy spectra of a velocity field [xdv][ydv][zd][3]
    on the GPU: (ex[3][xdv][zd], ey[3][ydv//2+1][zd])."""
    L = lib()
    v = np.ascontiguousarray(vel, np.float64)
    nx, ny, zd, three = v.shape
    assert three == 3
    ex, ey = np.zeros((3, nx, zd)), np.zeros((3, ny // 2 + 1, zd))
    rc = L.dnslbm_spectra_vel(_dp(v), nx, ny, zd - 2, device, _dp(ex), _dp(ey))
    if rc:
        raise DnsLbmError(rc, L.dnslbm_last_error(None).decode())
    return ex, ey
